/*
 * CPU ORACLE (test infrastructure only): DPD size math, element addressing
 * and the layout transforms iexpso / icompso / isymtrso.
 */
#include "cpsd_oracle.h"
#include "oracle_internal.h"
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

static i64 block_base(const o_desc *d, i64 R)
{
    i64 b = 0;
    for (i64 r = 1; r < R; r++)
        b += o_irpdso(o_dirprd(r, d->sym), d->pop[0], d->pop[1], d->iop[0]) *
             o_irpdso(r, d->pop[2], d->pop[3], d->iop[1]);
    return b;
}

/* For every stored pair of `dout`'s pair k in the pair space of irrep X:
 * the offset of the same (possibly swapped) pair in `din` and its sign. */
static void pair_map(const o_desc *din, const o_desc *dout, int k, i64 X, int swap, o_pairs *pl,
                     i64 **off, double **sgn)
{
    o_pairs_build(pl, dout->pop[2 * k], dout->pop[2 * k + 1], dout->iop[k], X);
    *off = (i64 *)malloc(sizeof(i64) * (size_t)(pl->n + 1));
    *sgn = (double *)malloc(sizeof(double) * (size_t)(pl->n + 1));
    for (i64 e = 0; e < pl->n; e++) {
        i64 ip = pl->ip[e], p = pl->p[e], iq = pl->iq[e], q = pl->q[e];
        if (swap) { i64 t = ip; ip = iq; iq = t; t = p; p = q; q = t; }
        int s = 1;
        (*off)[e] = pair_offset(din->pop[2 * k], din->pop[2 * k + 1], din->iop[k], ip, p, iq, q, &s);
        (*sgn)[e] = s;
    }
}

/* out(element) = sign * in(same element, pairs possibly swapped); zero for
 * structurally vanishing elements (p == q of a p<q pair).  Works block by
 * block on separable per-pair maps. */
static void xform(const double *in, double *out, const o_desc *din, const o_desc *dout, int swpq, int swrs)
{
    for (i64 R = 1; R <= g_nirrep; R++) {
        i64 L = o_dirprd(R, dout->sym);
        o_pairs pl, pr;
        i64 *lo, *ro;
        double *ls, *rs;
        pair_map(din, dout, 0, L, swpq, &pl, &lo, &ls);
        pair_map(din, dout, 1, R, swrs, &pr, &ro, &rs);
        i64 ob = block_base(dout, R), ib = block_base(din, R);
        i64 nlo = pl.n, nli = o_irpdso(L, din->pop[0], din->pop[1], din->iop[0]);
#pragma omp parallel for schedule(static)
        for (i64 r = 0; r < pr.n; r++) {
            double *o = out + ob + r * nlo;
            if (ro[r] < 0) {
                for (i64 l = 0; l < nlo; l++) o[l] = 0.0;
                continue;
            }
            const double *x = in + ib + ro[r] * nli;
            for (i64 l = 0; l < nlo; l++) o[l] = (lo[l] < 0) ? 0.0 : rs[r] * ls[l] * x[lo[l]];
        }
        free(lo); free(ls); free(ro); free(rs);
        o_pairs_free(&pl);
        o_pairs_free(&pr);
    }
}

/* iexpso (src/libsrint/iexpso.f90:24-120, exp_pq: out(q,p) = -in(p<q),
 * out(p,p) = 0) */
int o_iexpso(const double *in, double *out, const o_desc *din, i64 exppq, i64 exprs)
{
    o_desc dout = *din;
    if (exppq) dout.iop[0] = 1;
    if (exprs) dout.iop[1] = 1;
    xform(in, out, din, &dout, 0, 0);
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
    xform(in, out, din, &dout, 0, 0);
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
    xform(in, out, din, &dout, (int)swpq, (int)swrs);
    return O_OK;
}
