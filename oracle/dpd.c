/*
 * CPU ORACLE (test infrastructure only): DPD size math, element addressing
 * and the layout transforms iexpso / icompso / isymtrso.
 */
#include "cpsd_oracle.h"
#include <stdlib.h>
#include <string.h>

static i64 g_nirrep = 1;
static i64 g_dirprd[8][8]; /* [i-1][j-1] */

int o_set_symmetry(i64 nirrep, const i64 *dirprd)
{
    if (nirrep < 1 || nirrep > 8) return O_EARG;
    g_nirrep = nirrep;
    for (int j = 0; j < 8; j++)
        for (int i = 0; i < 8; i++) g_dirprd[i][j] = dirprd[j * 8 + i];
    return O_OK;
}

i64 o_nirrep(void) { return g_nirrep; }
i64 o_dirprd(i64 i, i64 j) { return g_dirprd[i - 1][j - 1]; }

/* irpdso (src/libsrint/irpdso.f:1-52): number of (p,q) pairs of irrep sym */
i64 o_irpdso(i64 sym, const i64 *popp, const i64 *popq, i64 ioppq)
{
    i64 n = 0;
    if (ioppq == 1) {
        for (i64 r = 1; r <= g_nirrep; r++) {
            i64 l = o_dirprd(r, sym);
            n += popp[l - 1] * popq[r - 1];
        }
    } else if (ioppq == 0 || ioppq == 2) {
        for (i64 r = 1; r <= g_nirrep; r++) {
            i64 l = o_dirprd(r, sym);
            if (l > r) continue;
            if (l < r) n += popp[l - 1] * popq[r - 1];
            else if (ioppq == 0) n += popp[l - 1] * (popq[r - 1] - 1) / 2;
            else n += popp[l - 1] * (popq[r - 1] + 1) / 2;
        }
    } else if (ioppq == -1) {
        n = popp[sym - 1];
    }
    return n;
}

/* idsymsoc (src/libsrint/idsymsoc.f:1-30) */
i64 o_idsymsoc(i64 irrepx, const i64 *popp, const i64 *popq, i64 ioppq,
               const i64 *popr, const i64 *pops, i64 ioprs)
{
    i64 n = 0;
    for (i64 r = 1; r <= g_nirrep; r++) {
        i64 l = o_dirprd(r, irrepx);
        n += o_irpdso(l, popp, popq, ioppq) * o_irpdso(r, popr, pops, ioprs);
    }
    return n;
}

/* isymoffso (src/libsrint/isymoffso.f:1-54): 1-based start of the q-irrep
 * sub-block inside the pair space of irrep `irrep` */
i64 o_isymoffso(i64 irrepq1, i64 irrep, const i64 *popp, const i64 *popq, i64 iop)
{
    i64 off = 1;
    for (i64 q = 1; q <= irrepq1 - 1; q++) {
        i64 p = o_dirprd(q, irrep);
        if (iop == 1) {
            off += popp[p - 1] * popq[q - 1];
        } else if (iop == 0) {
            if (p < q) off += popp[p - 1] * popq[q - 1];
            else if (p == q) off += popp[p - 1] * (popp[q - 1] - 1) / 2;
        } else if (iop == 2) {
            if (p < q) off += popp[p - 1] * popq[q - 1];
            else if (p == q) off += popp[p - 1] * (popp[q - 1] + 1) / 2;
        }
    }
    return off;
}

void o_desc_init(o_desc *d, const i64 *popp, const i64 *popq, const i64 *popr,
                 const i64 *pops, i64 ioppq, i64 ioprs, i64 sym)
{
    memcpy(d->pop[0], popp, 8 * sizeof(i64));
    memcpy(d->pop[1], popq, 8 * sizeof(i64));
    memcpy(d->pop[2], popr, 8 * sizeof(i64));
    memcpy(d->pop[3], pops, 8 * sizeof(i64));
    d->iop[0] = ioppq;
    d->iop[1] = ioprs;
    d->sym = sym;
}

i64 o_desc_len(const o_desc *d)
{
    return o_idsymsoc(d->sym, d->pop[0], d->pop[1], d->iop[0], d->pop[2], d->pop[3], d->iop[1]);
}

/* offset of the pair (ip,p),(iq,q) inside the pair space of irrep ip x iq;
 * 0-based, -1 if not stored; may swap (sign) for packed pairs */
static i64 pair_offset(const i64 *popp, const i64 *popq, i64 iop, i64 ip, i64 p,
                       i64 iq, i64 q, int *sign)
{
    i64 irr = o_dirprd(ip, iq);
    if (p < 0 || q < 0 || p >= popp[ip - 1] || q >= popq[iq - 1]) return -1;
    if (iop == 1) {
        return o_isymoffso(iq, irr, popp, popq, 1) - 1 + q * popp[ip - 1] + p;
    }
    /* packed: stored only for irrep(p) < irrep(q), or same irrep p<q (p<=q) */
    if (ip > iq || (ip == iq && p > q)) {
        i64 t = ip; ip = iq; iq = t;
        t = p; p = q; q = t;
        *sign *= (iop == 0) ? -1 : 1;
    }
    if (ip < iq) return o_isymoffso(iq, irr, popp, popq, iop) - 1 + q * popp[ip - 1] + p;
    /* same irrep */
    if (iop == 0) {
        if (p == q) return -1;
        return o_isymoffso(iq, irr, popp, popq, 0) - 1 + q * (q - 1) / 2 + p;
    }
    return o_isymoffso(iq, irr, popp, popq, 2) - 1 + q * (q + 1) / 2 + p;
}

i64 o_elem_offset(const o_desc *d, const i64 irr[4], const i64 idx[4], int *sign)
{
    *sign = 1;
    i64 L = o_dirprd(irr[0], irr[1]);
    i64 R = o_dirprd(irr[2], irr[3]);
    if (o_dirprd(L, R) != d->sym) return -1;
    if (d->iop[0] != 1 && d->iop[0] != 0 && d->iop[0] != 2) return -1;
    i64 pl = pair_offset(d->pop[0], d->pop[1], d->iop[0], irr[0], idx[0], irr[1], idx[1], sign);
    if (pl < 0) return -1;
    i64 pr = pair_offset(d->pop[2], d->pop[3], d->iop[1], irr[2], idx[2], irr[3], idx[3], sign);
    if (pr < 0) return -1;
    i64 base = 0;
    for (i64 r = 1; r < R; r++) {
        i64 l = o_dirprd(r, d->sym);
        base += o_irpdso(l, d->pop[0], d->pop[1], d->iop[0]) * o_irpdso(r, d->pop[2], d->pop[3], d->iop[1]);
    }
    i64 nleft = o_irpdso(L, d->pop[0], d->pop[1], d->iop[0]);
    return base + pr * nleft + pl;
}

/* Generic element loop over every (irreps, indices) of the FULL index space
 * of descriptor `dout` (iop ignored: all p,q / r,s), calling f for each
 * element that dout stores in canonical order. */
typedef void (*elem_fn)(const i64 irr[4], const i64 idx[4], i64 off_out, void *ctx);

static void foreach_stored(const o_desc *dout, elem_fn f, void *ctx)
{
    i64 n = g_nirrep;
    i64 irr[4], idx[4];
    for (irr[0] = 1; irr[0] <= n; irr[0]++)
        for (irr[1] = 1; irr[1] <= n; irr[1]++)
            for (irr[2] = 1; irr[2] <= n; irr[2]++) {
                irr[3] = o_dirprd(o_dirprd(o_dirprd(irr[0], irr[1]), irr[2]), dout->sym);
                if (dout->iop[0] != 1 && irr[0] > irr[1]) continue;
                if (dout->iop[1] != 1 && irr[2] > irr[3]) continue;
                for (idx[3] = 0; idx[3] < dout->pop[3][irr[3] - 1]; idx[3]++)
                    for (idx[2] = 0; idx[2] < dout->pop[2][irr[2] - 1]; idx[2]++) {
                        if (dout->iop[1] == 0 && irr[2] == irr[3] && idx[2] >= idx[3]) continue;
                        if (dout->iop[1] == 2 && irr[2] == irr[3] && idx[2] > idx[3]) continue;
                        for (idx[1] = 0; idx[1] < dout->pop[1][irr[1] - 1]; idx[1]++)
                            for (idx[0] = 0; idx[0] < dout->pop[0][irr[0] - 1]; idx[0]++) {
                                if (dout->iop[0] == 0 && irr[0] == irr[1] && idx[0] >= idx[1]) continue;
                                if (dout->iop[0] == 2 && irr[0] == irr[1] && idx[0] > idx[1]) continue;
                                int s;
                                i64 o = o_elem_offset(dout, irr, idx, &s);
                                if (o >= 0) f(irr, idx, o, ctx);
                            }
                    }
            }
}

typedef struct {
    const double *in;
    double *out;
    const o_desc *din;
    int swpq, swrs;
} xform_ctx;

/* out(element) = in(same element, maybe pair-swapped) with the packed sign */
static void copy_elem(const i64 irr[4], const i64 idx[4], i64 off_out, void *vctx)
{
    xform_ctx *c = (xform_ctx *)vctx;
    i64 ir[4] = {irr[0], irr[1], irr[2], irr[3]};
    i64 ix[4] = {idx[0], idx[1], idx[2], idx[3]};
    if (c->swpq) { i64 t = ir[0]; ir[0] = ir[1]; ir[1] = t; t = ix[0]; ix[0] = ix[1]; ix[1] = t; }
    if (c->swrs) { i64 t = ir[2]; ir[2] = ir[3]; ir[3] = t; t = ix[2]; ix[2] = ix[3]; ix[3] = t; }
    int s;
    i64 o = o_elem_offset(c->din, ir, ix, &s);
    c->out[off_out] = (o < 0) ? 0.0 : s * c->in[o];
}

/* iexpso (src/libsrint/iexpso.f90:24-120, exp_pq: out(q,p) = -in(p<q),
 * out(p,p) = 0) */
int o_iexpso(const double *in, double *out, const o_desc *din, i64 exppq, i64 exprs)
{
    o_desc dout = *din;
    if (exppq) dout.iop[0] = 1;
    if (exprs) dout.iop[1] = 1;
    xform_ctx c = {in, out, din, 0, 0};
    foreach_stored(&dout, copy_elem, &c);
    return O_OK;
}

/* icompso (src/libsrint/icompso.f:1-80, sqsymso.f): take the stored-order
 * elements of a full pair.  As in the reference, cpq/crs = 1 means "leave
 * that pair as it is", 0 / 2 compress a full pair to p<q / p<=q. */
int o_icompso(const double *in, double *out, const o_desc *din, i64 cpq, i64 crs)
{
    if ((cpq != 1 && din->iop[0] != 1) || (crs != 1 && din->iop[1] != 1)) return O_EARG;
    o_desc dout = *din;
    if (cpq != 1) dout.iop[0] = cpq;
    if (crs != 1) dout.iop[1] = crs;
    xform_ctx c = {in, out, din, 0, 0};
    foreach_stored(&dout, copy_elem, &c);
    return O_OK;
}

/* isymtrso (src/libsrint/isymtrso.f, symtr1so.f:80-132): pure index swap,
 * the output pair takes the swapped populations (no sign) */
int o_isymtrso(const double *in, double *out, const o_desc *din, i64 swpq, i64 swrs)
{
    o_desc dout = *din;
    if (swpq) {
        if (din->iop[0] != 1) return O_EARG;
        memcpy(dout.pop[0], din->pop[1], sizeof(dout.pop[0]));
        memcpy(dout.pop[1], din->pop[0], sizeof(dout.pop[0]));
    }
    if (swrs) {
        if (din->iop[1] != 1) return O_EARG;
        memcpy(dout.pop[2], din->pop[3], sizeof(dout.pop[0]));
        memcpy(dout.pop[3], din->pop[2], sizeof(dout.pop[0]));
    }
    xform_ctx c = {in, out, din, (int)swpq, (int)swrs};
    foreach_stored(&dout, copy_elem, &c);
    return O_OK;
}
