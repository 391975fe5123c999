/*
 * CPU ORACLE (test infrastructure only): orbital-energy differences,
 * denominators, initial guesses, the non-symmetric Davidson solver and DIIS.
 */
#include "cpsd_oracle.h"
#include "oracle_internal.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

extern void scipy_dgeev_64_(const char *jobvl, const char *jobvr, const i64 *n, double *a,
                            const i64 *lda, double *wr, double *wi, double *vl, const i64 *ldvl,
                            double *vr, const i64 *ldvr, double *work, const i64 *lwork, i64 *info,
                            i64 l1, i64 l2);

/* ---------- small BLAS-1 in the reference's summation order ---------- */
double o_ddot(i64 n, const double *x, const double *y)
{
    double s = 0.0;
    for (i64 i = 0; i < n; i++) s += x[i] * y[i];
    return s;
}
double o_dnrm2(i64 n, const double *x)
{
    double s = 0.0;
    for (i64 i = 0; i < n; i++) s += x[i] * x[i];
    return sqrt(s);
}
void o_daxpy(i64 n, double a, const double *x, double *y)
{
    for (i64 i = 0; i < n; i++) y[i] += a * x[i];
}
/* idamax: first index of the largest |x| (0-based) */
i64 o_idamax(i64 n, const double *x)
{
    i64 k = 0;
    double m = -1.0;
    for (i64 i = 0; i < n; i++)
        if (fabs(x[i]) > m) { m = fabs(x[i]); k = i; }
    return k;
}

/* ---------- pair lists in storage order ---------- */
void o_pairs_build(o_pairs *pl, const i64 *popp, const i64 *popq, i64 iop, i64 irr)
{
    i64 n = o_irpdso(irr, popp, popq, iop);
    pl->n = n;
    pl->ip = (i64 *)malloc(sizeof(i64) * (size_t)(n > 0 ? n : 1) * 4);
    pl->p = pl->ip + n; pl->iq = pl->p + n; pl->q = pl->iq + n;
    i64 k = 0;
    for (i64 iq = 1; iq <= o_nirrep(); iq++) {
        i64 ip = o_dirprd(iq, irr);
        if (iop != 1 && ip > iq) continue;
        for (i64 q = 0; q < popq[iq - 1]; q++) {
            i64 pmax = popp[ip - 1];
            if (iop == 0 && ip == iq) pmax = q;
            if (iop == 2 && ip == iq) pmax = q + 1;
            for (i64 p = 0; p < pmax; p++) {
                pl->ip[k] = ip; pl->p[k] = p; pl->iq[k] = iq; pl->q[k] = q;
                k++;
            }
        }
    }
}
void o_pairs_free(o_pairs *pl) { free(pl->ip); pl->ip = NULL; }

/* offsets of orbital irrep blocks inside the spin-free Eorb array
 * (occupied irreps first, then virtual irreps; resortEorb / seperateEorb) */
static void eorb_offsets(const i64 *pop_a, const i64 *pop_i, i64 *ioff_a, i64 *ioff_i)
{
    i64 n = o_nirrep();
    ioff_i[0] = 0;
    for (i64 r = 1; r < n; r++) ioff_i[r] = ioff_i[r - 1] + pop_i[r - 1];
    ioff_a[0] = ioff_i[n - 1] + pop_i[n - 1];
    for (i64 r = 1; r < n; r++) ioff_a[r] = ioff_a[r - 1] + pop_a[r - 1];
}

/* Eorb_diff1 (src/lib_cc/Eorb_diff.f90:6-64): e(a,i) = e(a) - e(i) */
void o_eorb_diff1(double *oed1, const double *eorb, const i64 *pop_a, const i64 *pop_i, i64 sym)
{
    i64 oa[8], oi[8];
    eorb_offsets(pop_a, pop_i, oa, oi);
    for (i64 ii = 1; ii <= o_nirrep(); ii++) {
        i64 ia = o_dirprd(ii, sym);
        i64 base = o_isymoffso(ii, sym, pop_a, pop_i, 1) - 1;
        for (i64 i = 0; i < pop_i[ii - 1]; i++)
            for (i64 a = 0; a < pop_a[ia - 1]; a++)
                oed1[base + i * pop_a[ia - 1] + a] = eorb[oa[ia - 1] + a] - eorb[oi[ii - 1] + i];
    }
}

/* iterate the stored (ab,ij) elements of a (v,v,o,o) tensor */
typedef void (*abij_fn)(i64 off, double ea, double eb, double ei, double ej, void *ctx);
static void foreach_abij(const double *eorb, const i64 *pop_a, const i64 *pop_i, i64 sym, i64 iop,
                         abij_fn fn, void *ctx)
{
    i64 oa[8], oi[8];
    eorb_offsets(pop_a, pop_i, oa, oi);
    i64 off = 0;
    for (i64 R = 1; R <= o_nirrep(); R++) {
        i64 L = o_dirprd(R, sym);
        o_pairs pr, pl;
        o_pairs_build(&pr, pop_i, pop_i, iop, R);
        o_pairs_build(&pl, pop_a, pop_a, iop, L);
        for (i64 r = 0; r < pr.n; r++) {
            double ei = eorb[oi[pr.ip[r] - 1] + pr.p[r]];
            double ej = eorb[oi[pr.iq[r] - 1] + pr.q[r]];
            for (i64 l = 0; l < pl.n; l++) {
                double ea = eorb[oa[pl.ip[l] - 1] + pl.p[l]];
                double eb = eorb[oa[pl.iq[l] - 1] + pl.q[l]];
                fn(off + r * pl.n + l, ea, eb, ei, ej, ctx);
            }
        }
        off += pr.n * pl.n;
        o_pairs_free(&pr);
        o_pairs_free(&pl);
    }
}

static void oed2_fn(i64 off, double ea, double eb, double ei, double ej, void *ctx)
{
    ((double *)ctx)[off] = ea + eb - ei - ej;
}
/* Eorb_diff2 (src/lib_cc/Eorb_diff.f90:68-220): e(ab,ij) = e(a)+e(b)-e(i)-e(j) */
void o_eorb_diff2(double *oed2, const double *eorb, const i64 *pop_a, const i64 *pop_i, i64 sym, i64 iop)
{
    foreach_abij(eorb, pop_a, pop_i, sym, iop, oed2_fn, oed2);
}

/* denomT1 (src/lib_cc/denomT.f90:25-91): t(a,i) = r(a,i)/(e(i)-e(a)) */
void o_denomT1(double *t1, const double *r1, const double *eorb, const i64 *pop_a, const i64 *pop_i, i64 sym)
{
    i64 oa[8], oi[8];
    eorb_offsets(pop_a, pop_i, oa, oi);
    for (i64 ii = 1; ii <= o_nirrep(); ii++) {
        i64 ia = o_dirprd(ii, sym);
        i64 base = o_isymoffso(ii, sym, pop_a, pop_i, 1) - 1;
        for (i64 i = 0; i < pop_i[ii - 1]; i++)
            for (i64 a = 0; a < pop_a[ia - 1]; a++) {
                i64 k = base + i * pop_a[ia - 1] + a;
                double d = eorb[oi[ii - 1] + i] - eorb[oa[ia - 1] + a];
                t1[k] = r1[k] / d;
            }
    }
}

typedef struct { double *t; const double *r; } dt2_ctx;
static void dt2_fn(i64 off, double ea, double eb, double ei, double ej, void *vctx)
{
    dt2_ctx *c = (dt2_ctx *)vctx;
    double d = ei + ej - ea - eb;
    c->t[off] = c->r[off] / d;
}
/* denomT2 (src/lib_cc/denomT.f90:93-249): t(ab,ij) = r/(e(i)+e(j)-e(a)-e(b)) */
void o_denomT2(double *t2, const double *r2, const double *eorb, const i64 *pop_a, const i64 *pop_i, i64 sym, i64 iop)
{
    dt2_ctx c = {t2, r2};
    foreach_abij(eorb, pop_a, pop_i, sym, iop, dt2_fn, &c);
}

/* ---------- initial guesses (src/lib_cc/preDavidson.f90) ---------- */

/* getLowest (src/lib_cc/get_n_idx.f90:7-63), 1-based positions */
static void get_lowest(const double *v, i64 n, i64 nl, i64 *low)
{
    for (i64 i = 0; i < nl; i++) low[i] = i + 1;
    for (i64 i = 0; i < nl - 1; i++)
        for (i64 j = i + 1; j < nl; j++)
            if (v[low[i] - 1] > v[low[j] - 1]) { i64 t = low[i]; low[i] = low[j]; low[j] = t; }
    for (i64 i = nl + 1; i <= n; i++) {
        if (v[i - 1] < v[low[nl - 1] - 1]) {
            i64 s = 1, e = nl;
            for (;;) {
                i64 mid = s + (e - s) / 2;
                if (v[low[mid - 1] - 1] > v[i - 1]) e = mid;
                else s = mid + 1;
                if (s == e) break;
            }
            i64 idx = e;
            for (i64 j = 0; j <= nl - idx - 1; j++) low[nl - j - 1] = low[nl - j - 2];
            low[idx - 1] = i;
        }
    }
}

/* seperateEorb (src/lib_cc/seperateEorb.f90): spin-free -> alpha / beta
 * arrays laid out (occ irreps, vir irreps) */
static void separate_eorb(const o_system *s, const double *eorb, double *Ea, double *Eb)
{
    i64 n = s->nirrep;
    i64 oa[8], ob[8], o[8], va[8], vb[8], v[8];
    oa[0] = ob[0] = o[0] = 0;
    for (i64 r = 1; r < n; r++) {
        oa[r] = oa[r - 1] + s->popa[r - 1];
        ob[r] = ob[r - 1] + s->popb[r - 1];
        o[r] = o[r - 1] + s->popo[r - 1];
    }
    va[0] = oa[n - 1] + s->popa[n - 1];
    vb[0] = ob[n - 1] + s->popb[n - 1];
    v[0] = o[n - 1] + s->popo[n - 1];
    for (i64 r = 1; r < n; r++) {
        va[r] = va[r - 1] + s->vrta[r - 1];
        vb[r] = vb[r - 1] + s->vrtb[r - 1];
        v[r] = v[r - 1] + s->popv[r - 1];
    }
    for (i64 r = 1; r <= n; r++) {
        i64 rb = o_dirprd(r, s->symry);
        memcpy(Ea + oa[r - 1], eorb + o[r - 1], sizeof(double) * (size_t)s->popa[r - 1]);
        memcpy(Eb + ob[rb - 1], eorb + o[r - 1] + s->popa[r - 1], sizeof(double) * (size_t)s->popb[rb - 1]);
        memcpy(Ea + va[r - 1], eorb + v[r - 1], sizeof(double) * (size_t)s->vrta[r - 1]);
        memcpy(Eb + vb[rb - 1], eorb + v[r - 1] + s->vrta[r - 1], sizeof(double) * (size_t)s->vrtb[rb - 1]);
    }
}

/* Eorb_diff_ab (src/lib_cc/Eorb_diff.f90:222-276): e(a,i) = E1(a) - E2(i)
 * with a over pop_a1 (E1 layout: pop_i1 occupied then pop_a1 virtual) and
 * i over pop_i2 (E2 layout). */
static void eorb_diff_ab(double *oed, const double *E1, const i64 *pop_a1, const i64 *pop_i1,
                         const double *E2, const i64 *pop_i2, i64 sym)
{
    i64 n = o_nirrep(), oi2[8], oa1[8];
    oi2[0] = 0;
    for (i64 r = 1; r < n; r++) oi2[r] = oi2[r - 1] + pop_i2[r - 1];
    i64 t = 0;
    for (i64 r = 0; r < n; r++) t += pop_i1[r];
    oa1[0] = t;
    for (i64 r = 1; r < n; r++) oa1[r] = oa1[r - 1] + pop_a1[r - 1];
    for (i64 ii = 1; ii <= n; ii++) {
        i64 ia = o_dirprd(ii, sym);
        i64 base = o_isymoffso(ii, sym, pop_a1, pop_i2, 1) - 1;
        for (i64 i = 0; i < pop_i2[ii - 1]; i++)
            for (i64 a = 0; a < pop_a1[ia - 1]; a++)
                oed[base + i * pop_a1[ia - 1] + a] = E1[oa1[ia - 1] + a] - E2[oi2[ii - 1] + i];
    }
}

/* getidx for a 2-index (p,q) iop=1 tensor of irrep sym: 1-based idx ->
 * (irrep p, irrep q, p, q) with 1-based p,q */
static void getidx2(i64 idx, const i64 *popp, const i64 *popq, i64 sym, i64 *ip, i64 *iq, i64 *p, i64 *q)
{
    o_pairs pl;
    o_pairs_build(&pl, popp, popq, 1, sym);
    i64 k = idx - 1;
    *ip = pl.ip[k]; *iq = pl.iq[k]; *p = pl.p[k] + 1; *q = pl.q[k] + 1;
    o_pairs_free(&pl);
}

/* 0-based offset of (a,i) in an R1 vector of irrep sym (putidx) */
static i64 putidx2(i64 ia, i64 ii, i64 a1, i64 i1, const i64 *popp, const i64 *popq, i64 sym)
{
    (void)sym;
    i64 irr = o_dirprd(ia, ii);
    return o_isymoffso(ii, irr, popp, popq, 1) - 1 + (i1 - 1) * popp[ia - 1] + (a1 - 1);
}

/* preDavidson1_ns (src/lib_cc/preDavidson.f90:6-117) for irrep irrepex:
 * writes nroot records (exE, R1) into guess[(1+len)*k] */
int o_guess(const o_system *s, const double *eorb, const o_params *p, i64 irrepex, i64 nroot, double *guess)
{
    i64 n = s->nirrep;
    i64 na = 0, nb = 0;
    for (i64 r = 0; r < n; r++) {
        na += s->popa[r] + s->vrta[r];
        nb += s->popb[r] + s->vrtb[r];
    }
    double *Ea = (double *)calloc((size_t)na + 1, sizeof(double));
    double *Eb = (double *)calloc((size_t)nb + 1, sizeof(double));
    separate_eorb(s, eorb, Ea, Eb);
    i64 vlen = o_irpdso(irrepex, s->popv, s->popo, 1);
    i64 *low = (i64 *)malloc(sizeof(i64) * (size_t)nroot);
    int rc = O_OK;
    if (p->spin_flip == 1 || p->spin_flip == 2) {
        /* p_pre_spin_flip_ns (preDavidson.f90:120-223) */
        int ab = (p->spin_flip == 1);
        i64 ssym = o_dirprd(irrepex, s->symry);
        i64 nsz = ab ? o_irpdso(ssym, s->vrtb, s->popa, 1) : o_irpdso(ssym, s->vrta, s->popb, 1);
        double *oed = (double *)calloc((size_t)nsz + 1, sizeof(double));
        if (ab) eorb_diff_ab(oed, Eb, s->vrtb, s->popb, Ea, s->popa, ssym);
        else eorb_diff_ab(oed, Ea, s->vrta, s->popa, Eb, s->popb, ssym);
        if (nsz < nroot) { free(oed); rc = O_EARG; goto out; }
        get_lowest(oed, nsz, nroot, low);
        for (i64 k = 0; k < nroot; k++) {
            double *rec = guess + (1 + vlen) * k;
            rec[0] = oed[low[k] - 1];
            memset(rec + 1, 0, sizeof(double) * (size_t)vlen);
            i64 ia, ii, a, i;
            if (ab) {
                getidx2(low[k], s->vrtb, s->popa, ssym, &ia, &ii, &a, &i);
                ia = o_dirprd(ia, s->symry);
                a = s->vrta[ia - 1] + a;
            } else {
                getidx2(low[k], s->vrta, s->popb, ssym, &ia, &ii, &a, &i);
                ii = o_dirprd(ii, s->symry);
                i = s->popa[ii - 1] + i;
            }
            rec[1 + putidx2(ia, ii, a, i, s->popv, s->popo, irrepex)] = 1.0;
        }
        free(oed);
    } else if (p->open_shell) {
        /* p_pre_open_ns (preDavidson.f90:226-320) */
        i64 n1 = o_irpdso(irrepex, s->vrta, s->popa, 1), n2 = o_irpdso(irrepex, s->vrtb, s->popb, 1);
        double *oed = (double *)calloc((size_t)(n1 + n2) + 1, sizeof(double));
        o_eorb_diff1(oed, Ea, s->vrta, s->popa, irrepex);
        o_eorb_diff1(oed + n1, Eb, s->vrtb, s->popb, irrepex);
        if (n1 + n2 < nroot) { free(oed); rc = O_EARG; goto out; }
        get_lowest(oed, n1 + n2, nroot, low);
        for (i64 k = 0; k < nroot; k++) {
            double *rec = guess + (1 + vlen) * k;
            rec[0] = oed[low[k] - 1];
            memset(rec + 1, 0, sizeof(double) * (size_t)vlen);
            i64 ia, ii, a, i;
            if (low[k] <= n1) {
                getidx2(low[k], s->vrta, s->popa, irrepex, &ia, &ii, &a, &i);
            } else {
                getidx2(low[k] - n1, s->vrtb, s->popb, irrepex, &ia, &ii, &a, &i);
                ia = o_dirprd(ia, s->symry);
                ii = o_dirprd(ii, s->symry);
                a += s->vrta[ia - 1];
                i += s->popa[ii - 1];
            }
            rec[1 + putidx2(ia, ii, a, i, s->popv, s->popo, irrepex)] = 1.0;
        }
        free(oed);
    } else {
        /* p_pre_close_ns (preDavidson.f90:420-515) */
        i64 n1 = o_irpdso(irrepex, s->vrta, s->popa, 1);
        double *oed = (double *)calloc((size_t)n1 + 1, sizeof(double));
        o_eorb_diff1(oed, Ea, s->vrta, s->popa, irrepex);
        if (n1 < nroot) { free(oed); rc = O_EARG; goto out; }
        get_lowest(oed, n1, nroot, low);
        for (i64 k = 0; k < nroot; k++) {
            double *rec = guess + (1 + vlen) * k;
            rec[0] = oed[low[k] - 1];
            memset(rec + 1, 0, sizeof(double) * (size_t)vlen);
            i64 ia, ii, a, i;
            getidx2(low[k], s->vrta, s->popa, irrepex, &ia, &ii, &a, &i);
            rec[1 + putidx2(ia, ii, a, i, s->popv, s->popo, irrepex)] = 1.0 / sqrt(2.0);
            i64 ib = o_dirprd(ia, s->symry), jb = o_dirprd(ii, s->symry);
            double v = (p->ex_mult == 3) ? -1.0 / sqrt(2.0) : 1.0 / sqrt(2.0);
            rec[1 + putidx2(ib, jb, s->vrta[ib - 1] + a, s->popa[jb - 1] + i, s->popv, s->popo, irrepex)] = v;
        }
        free(oed);
    }
out:
    free(low); free(Ea); free(Eb);
    return rc;
}

/* ---------- Davidson (src/lib_cc/mod_davidson.f90:40-728) ---------- */

/* sort (mod_davidson.f90:620-640): selection sort of indices, 1-based */
static void dv_sort(i64 n, const double *v, i64 *idx)
{
    for (i64 i = 0; i < n; i++) idx[i] = i + 1;
    for (i64 i = 0; i < n - 1; i++)
        for (i64 j = i + 1; j < n; j++)
            if (v[idx[j] - 1] < v[idx[i] - 1]) { i64 t = idx[j]; idx[j] = idx[i]; idx[i] = t; }
}

/* Schmidt_2D (mod_davidson.f90:642-680) */
static void schmidt_2d(const double *in, double *out, i64 len, i64 dim)
{
    memcpy(out, in, sizeof(double) * (size_t)(len * dim));
    for (i64 i = 1; i < dim; i++) {
        for (i64 j = 0; j < i; j++) {
            double ov = o_ddot(len, out + j * len, out + i * len);
            o_daxpy(len, -ov, out + j * len, out + i * len);
        }
        double nrm = o_dnrm2(len, out + i * len);
        for (i64 k = 0; k < len; k++) out[i * len + k] *= 1.0 / nrm;
    }
}

int o_davidson(double *fileEV, const double *diagA, i64 dimA, i64 nroot, i64 istate,
               const o_params *p, o_sigma_fn calAR, void *ctx, i64 *iters_out)
{
    i64 dimAbar = p->davidson_dim;
    i64 dimDel = dimAbar - nroot - 5;
    if (nroot >= dimAbar) return O_EARG;
    if (nroot == 0) return O_OK;
    double maxError = pow(10.0, -(double)p->davidson_conv);
    i64 D = dimAbar;
    double *Abar = (double *)calloc((size_t)(D * D), sizeof(double));
    double *tmpAbar = (double *)calloc((size_t)(D * D), sizeof(double));
    double *valR = (double *)calloc((size_t)D, sizeof(double));
    double *valI = (double *)calloc((size_t)D, sizeof(double));
    double *vecR = (double *)calloc((size_t)(D * D), sizeof(double));
    double *vecNeed = (double *)calloc((size_t)(D * nroot), sizeof(double));
    double *eigenVal = (double *)calloc((size_t)nroot, sizeof(double));
    i64 *lowestE = (i64 *)calloc((size_t)D, sizeof(i64));
    i64 *conv = (i64 *)calloc((size_t)nroot, sizeof(i64));
    i64 lwork = 10 * D;
    double *work = (double *)calloc((size_t)lwork, sizeof(double));
    double *fb[2], *fAb[2];
    for (int k = 0; k < 2; k++) {
        fb[k] = (double *)calloc((size_t)(D * dimA), sizeof(double));
        fAb[k] = (double *)calloc((size_t)(D * dimA), sizeof(double));
    }
    double *w0 = (double *)calloc((size_t)dimA, sizeof(double));
    double *w1 = (double *)calloc((size_t)dimA, sizeof(double));
    double *oldE = (double *)calloc((size_t)(D * D), sizeof(double));
    double *newE = (double *)calloc((size_t)(D * D), sizeof(double));
    int cur = 0;
    int rc = O_OK;
    /* initDavidson (mod_davidson.f90:562-615) */
    for (i64 i = 0; i < nroot; i++) {
        const double *rec = fileEV + (istate + i - 1) * (dimA + 1);
        eigenVal[i] = rec[0];
        memcpy(fb[cur] + i * dimA, rec + 1, sizeof(double) * (size_t)dimA);
        calAR(ctx, fb[cur] + i * dimA, fAb[cur] + i * dimA);
        for (i64 j = 0; j < nroot; j++)
            Abar[j + i * D] = o_ddot(dimA, fileEV + (istate + j - 1) * (dimA + 1) + 1, fAb[cur] + i * dimA);
        vecNeed[i + i * D] = 1.0;
    }
    i64 iterations = 1, dimIter = nroot, dimFree = D - dimIter;
    int dim_exceed = 0;
    i64 ndimIter = 0, ndimFree = 0;
    for (;;) {
        if (iterations > p->davidson_cyc) break;
        memcpy(tmpAbar, Abar, sizeof(double) * (size_t)(D * D));
        i64 info = 0;
        scipy_dgeev_64_("N", "V", &dimIter, tmpAbar, &D, valR, valI, vecR, &D, vecR, &D, work, &lwork, &info, 1, 1);
        if (info != 0) { rc = O_ELAPACK; break; }
        for (i64 i = 0; i < dimIter; i++) {
            double t = o_dnrm2(dimIter, vecR + i * D);
            if (fabs(t - 1.0) > 1.0e-10)
                for (i64 k = 0; k < dimIter; k++) vecR[i * D + k] *= 1.0 / t;
        }
        dv_sort(dimIter, valR, lowestE);
        if (!p->lowest) {
            /* largest component over the positions not yet given to a root
             * (the reference searches j = 1..dimIter and can give one
             * eigenvector to two roots, which makes its collapse divide by
             * zero; identical wherever it assigns distinct vectors) */
            for (i64 iroot = 1; iroot <= nroot; iroot++) {
                double t1 = 0.0;
                i64 i = iroot;
                for (i64 j = iroot; j <= dimIter; j++) {
                    double t2 = fabs(vecR[(iroot - 1) + (lowestE[j - 1] - 1) * D]);
                    if (t2 > t1) { t1 = t2; i = j; }
                }
                i64 idx = lowestE[i - 1];
                for (i64 j = 1; j <= i - iroot; j++) lowestE[i - j] = lowestE[i - j - 1];
                lowestE[iroot - 1] = idx;
            }
        }
        for (i64 iroot = 0; iroot < nroot; iroot++) {
            memcpy(vecNeed + iroot * D, vecR + (lowestE[iroot] - 1) * D, sizeof(double) * (size_t)D);
            eigenVal[iroot] = valR[lowestE[iroot] - 1];
        }
        if (dim_exceed) {
            for (i64 i = 0; i < ndimIter; i++)
                memcpy(oldE + i * dimIter, vecR + (lowestE[i] - 1) * D, sizeof(double) * (size_t)dimIter);
            schmidt_2d(oldE, newE, dimIter, ndimIter);
            int nw = 1 - cur;
            for (i64 ir = 0; ir < ndimIter; ir++) {
                memset(w0, 0, sizeof(double) * (size_t)dimA);
                memset(w1, 0, sizeof(double) * (size_t)dimA);
                for (i64 i = 0; i < dimIter; i++) {
                    double t = newE[i + ir * dimIter];
                    o_daxpy(dimA, t, fAb[cur] + i * dimA, w0);
                    o_daxpy(dimA, t, fb[cur] + i * dimA, w1);
                }
                memcpy(fAb[nw] + ir * dimA, w0, sizeof(double) * (size_t)dimA);
                memcpy(fb[nw] + ir * dimA, w1, sizeof(double) * (size_t)dimA);
            }
            cur = nw;
            dimFree = ndimFree;
            dimIter = ndimIter;
            for (i64 i = 0; i < dimIter; i++)
                for (i64 j = 0; j < dimIter; j++)
                    Abar[j + i * D] = o_ddot(dimA, fAb[cur] + i * dimA, fb[cur] + j * dimA);
        }
        i64 nNew = 0;
        for (i64 ir = 0; ir < nroot; ir++) conv[ir] = 0;
        for (i64 ir = 0; ir < nroot; ir++) {
            if (dim_exceed) {
                memcpy(w0, fAb[cur] + ir * dimA, sizeof(double) * (size_t)dimA);
                memcpy(w1, fb[cur] + ir * dimA, sizeof(double) * (size_t)dimA);
            } else {
                memset(w0, 0, sizeof(double) * (size_t)dimA);
                memset(w1, 0, sizeof(double) * (size_t)dimA);
                for (i64 i = 0; i < dimIter; i++) {
                    double t = vecNeed[i + ir * D];
                    o_daxpy(dimA, t, fAb[cur] + i * dimA, w0);
                    o_daxpy(dimA, t, fb[cur] + i * dimA, w1);
                }
            }
            double t = o_dnrm2(dimA, w1);
            if (fabs(t - 1.0) > 1.0e-10)
                for (i64 k = 0; k < dimA; k++) { w1[k] *= 1.0 / t; w0[k] *= 1.0 / t; }
            double *rec = fileEV + (istate + ir - 1) * (dimA + 1);
            rec[0] = eigenVal[ir];
            memcpy(rec + 1, w1, sizeof(double) * (size_t)dimA);
            o_daxpy(dimA, -eigenVal[ir], w1, w0);
            double em = w0[o_idamax(dimA, w0)];
            if (fabs(em) < maxError) { conv[ir] = 1; continue; }
            if (dimFree == 0) continue;
            for (i64 i = 0; i < dimA; i++) {
                double d = eigenVal[ir] - diagA[i];
                if (fabs(d) < 1.0e-4) d = (d < 0.0) ? -1.0e-4 : 1.0e-4;
                w1[i] = w0[i] / d;
            }
            /* SchmidtS (mod_davidson.f90:682-727) */
            double nrm = o_dnrm2(dimA, w1);
            for (i64 k = 0; k < dimA; k++) w1[k] *= 1.0 / nrm;
            for (i64 i = 0; i < dimIter + nNew; i++) {
                double ov = o_ddot(dimA, fb[cur] + i * dimA, w1);
                o_daxpy(dimA, -ov, fb[cur] + i * dimA, w1);
            }
            nrm = o_dnrm2(dimA, w1);
            if (nrm < 1.0e-6) continue;
            for (i64 k = 0; k < dimA; k++) w1[k] *= 1.0 / nrm;
            i64 pos = dimIter + nNew;
            memcpy(fb[cur] + pos * dimA, w1, sizeof(double) * (size_t)dimA);
            calAR(ctx, fb[cur] + pos * dimA, fAb[cur] + pos * dimA);
            dimFree--;
            nNew++;
        }
        i64 nc = 0;
        for (i64 ir = 0; ir < nroot; ir++) nc += conv[ir];
        if (nc == nroot) break;
        if (dim_exceed) dim_exceed = 0;
        if (dimFree == 0) {
            dim_exceed = 1;
            ndimIter = D - dimDel;
            if (ndimIter < nroot) { ndimIter = nroot; ndimFree = D - ndimIter; }
            else ndimFree = dimDel;
        }
        for (i64 j = 0; j < dimIter; j++)
            for (i64 i = dimIter; i < dimIter + nNew; i++)
                Abar[i + j * D] = o_ddot(dimA, fb[cur] + i * dimA, fAb[cur] + j * dimA);
        for (i64 j = dimIter; j < dimIter + nNew; j++)
            for (i64 i = 0; i < dimIter + nNew; i++)
                Abar[i + j * D] = o_ddot(dimA, fb[cur] + i * dimA, fAb[cur] + j * dimA);
        dimIter += nNew;
        iterations++;
    }
    if (iters_out) *iters_out = iterations;
    free(Abar); free(tmpAbar); free(valR); free(valI); free(vecR); free(vecNeed);
    free(eigenVal); free(lowestE); free(conv); free(work);
    for (int k = 0; k < 2; k++) { free(fb[k]); free(fAb[k]); }
    free(w0); free(w1); free(oldE); free(newE);
    return rc;
}

/* ---------- DIIS: dosodiis2_d (src/libsrint/dosodiis2_d.f:1-119) with
 * dodiis (src/libsrint/dodiis.f) solved by LINPACK dgefa/dgesl as MINV
 * (src/libsrint/minv.f) does ---------- */
void o_diis_init(o_diis *st, i64 len, i64 maxdim)
{
    st->len = len; st->maxdim = maxdim; st->ndimr = 1; st->idimr = 1;
    st->prev = (double *)calloc((size_t)len, sizeof(double));
    st->err = (double *)calloc((size_t)(len * maxdim), sizeof(double));
    st->amp = (double *)calloc((size_t)(len * maxdim), sizeof(double));
}
void o_diis_free(o_diis *st) { free(st->prev); free(st->err); free(st->amp); }

/* LINPACK dgefa: LU with partial pivoting, column-major a(lda,n) */
void o_dgefa(double *a, i64 lda, i64 n, i64 *ipvt)
{
    for (i64 k = 0; k < n - 1; k++) {
        i64 l = k + o_idamax(n - k, a + k + k * lda);
        ipvt[k] = l;
        if (a[l + k * lda] == 0.0) continue;
        if (l != k) { double t = a[l + k * lda]; a[l + k * lda] = a[k + k * lda]; a[k + k * lda] = t; }
        double t = -1.0 / a[k + k * lda];
        for (i64 i = k + 1; i < n; i++) a[i + k * lda] *= t;
        for (i64 j = k + 1; j < n; j++) {
            double tj = a[l + j * lda];
            if (l != k) { a[l + j * lda] = a[k + j * lda]; a[k + j * lda] = tj; }
            for (i64 i = k + 1; i < n; i++) a[i + j * lda] += tj * a[i + k * lda];
        }
    }
    ipvt[n - 1] = n - 1;
}
/* LINPACK dgesl, job = 0 */
void o_dgesl(const double *a, i64 lda, i64 n, const i64 *ipvt, double *b)
{
    for (i64 k = 0; k < n - 1; k++) {
        i64 l = ipvt[k];
        double t = b[l];
        if (l != k) { b[l] = b[k]; b[k] = t; }
        for (i64 i = k + 1; i < n; i++) b[i] += t * a[i + k * lda];
    }
    for (i64 kb = 0; kb < n; kb++) {
        i64 k = n - 1 - kb;
        b[k] /= a[k + k * lda];
        double t = -b[k];
        for (i64 i = 0; i < k; i++) b[i] += t * a[i + k * lda];
    }
}

double o_diis_step(o_diis *st, i64 iter, double *vec)
{
    i64 len = st->len, maxdim = st->maxdim;
    if (iter == 1) {
        st->idimr = 1; st->ndimr = 1;
        memcpy(st->prev, vec, sizeof(double) * (size_t)len);
        return 1.0;
    }
    memcpy(st->amp + (st->idimr - 1) * len, st->prev, sizeof(double) * (size_t)len);
    o_daxpy(len, -1.0, st->prev, vec);
    memcpy(st->err + (st->idimr - 1) * len, vec, sizeof(double) * (size_t)len);
    i64 nd = st->ndimr;
    double B[64 * 64];
    for (i64 i = 0; i < nd; i++)
        for (i64 j = 0; j <= i; j++) {
            double x = o_ddot(len, st->err + i * len, st->err + j * len);
            B[i + j * maxdim] = x;
            B[j + i * maxdim] = x;
        }
    /* dodiis: augmented (nd+1) x (nd+1) system with the -1e-4 border */
    i64 n1 = nd + 1;
    double aug[65 * 65], rhs[65];
    i64 ipvt[65];
    memset(aug, 0, sizeof(aug));
    for (i64 j = 0; j < nd; j++)
        for (i64 i = 0; i < nd; i++) aug[(i + 1) + (j + 1) * n1] = B[i + j * maxdim];
    for (i64 i = 1; i <= nd; i++) { aug[i] = -1.0e-4; aug[i * n1] = -1.0e-4; }
    rhs[0] = -1.0e-4;
    for (i64 i = 1; i <= nd; i++) rhs[i] = 0.0;
    o_dgefa(aug, n1, n1, ipvt);
    o_dgesl(aug, n1, n1, ipvt, rhs);
    memset(vec, 0, sizeof(double) * (size_t)len);
    for (i64 i = 0; i < nd; i++) o_daxpy(len, rhs[i + 1], st->err + i * len, vec);
    double res = vec[o_idamax(len, vec)];
    for (i64 i = 0; i < nd; i++) o_daxpy(len, rhs[i + 1], st->amp + i * len, vec);
    memcpy(st->prev, vec, sizeof(double) * (size_t)len);
    st->ndimr = (st->ndimr + 1 < maxdim) ? st->ndimr + 1 : maxdim;
    st->idimr++;
    if (st->idimr > maxdim) st->idimr = 1;
    return res;
}
