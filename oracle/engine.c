/*
 * CPU ORACLE (test infrastructure only): the DPD contraction engine.
 *
 * Restates vv2v_dpd_444_d (src/libsrint/vv2v_dpd_444_d.f90:4-529) and its
 * 424/442 siblings as one general routine: the reference's "fallback" tile
 * assembly (task list over irrep assignments, pack A/B from strided DPD
 * blocks, one DGEMM, unpack with alpha/beta) with intact packed pairs
 * treated as one composite index — which is exactly the reference's fast
 * path ('3412'*'3456'->'1256' etc., src/libsrint/vv2v_dpd_444_d.f90:120-225)
 * when every index is a whole pair.  BLAS is numpy's bundled ILP64 OpenBLAS,
 * the same library family the reference links (src/make.config:99-100).
 */
#include "cpsd_oracle.h"
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

extern void scipy_dgemm_64_(const char *ta, const char *tb, const i64 *m, const i64 *n,
                            const i64 *k, const double *alpha, const double *a, const i64 *lda,
                            const double *b, const i64 *ldb, const double *beta, double *c,
                            const i64 *ldc, i64 lta, i64 ltb);
extern void scipy_openblas_set_num_threads64_(int n);

static i64 g_threads = 1;

void o_set_threads(i64 n)
{
    if (n < 1) n = 1;
    g_threads = n;
#ifdef _OPENMP
    omp_set_num_threads((int)n);
#endif
    scipy_openblas_set_num_threads64_((int)n);
}

#define MAXU 6

typedef struct {
    int nlet;     /* 1 or 2 (packed pair) */
    int let[2];   /* letter ids */
    int iop;      /* pair iop for packed units, 1 for single letters */
    int in[3];    /* present in tensor t */
    int slot[3];  /* slot (single) or pair index 0/1 (packed) in tensor t */
    int cls;      /* 0 = M (v1,v3), 1 = N (v2,v3), 2 = K (v1,v2) */
} unit_t;

typedef struct {
    i64 key;              /* output (M,N) irrep key, for grouping */
    i64 base[3];
    i64 ext[MAXU];
    i64 st[3][MAXU];
} task_t;

static int cmp_task(const void *a, const void *b)
{
    i64 x = ((const task_t *)a)->key, y = ((const task_t *)b)->key;
    return (x > y) - (x < y);
}

static int is_zorb(const i64 *pop)
{
    if (pop[0] != 1) return 0;
    for (int i = 1; i < 8; i++)
        if (pop[i] != 0) return 0;
    return 1;
}

/* base offset and slot strides of a tensor block for slot irreps irr[4] */
static void block_geom(const o_desc *d, const i64 irr[4], i64 *base, i64 st[4], i64 *nleft_out)
{
    i64 L = o_dirprd(irr[0], irr[1]);
    i64 R = o_dirprd(irr[2], irr[3]);
    i64 b = 0;
    for (i64 r = 1; r < R; r++) {
        i64 l = o_dirprd(r, d->sym);
        b += o_irpdso(l, d->pop[0], d->pop[1], d->iop[0]) * o_irpdso(r, d->pop[2], d->pop[3], d->iop[1]);
    }
    i64 nleft = o_irpdso(L, d->pop[0], d->pop[1], d->iop[0]);
    i64 lsub = o_isymoffso(irr[1], L, d->pop[0], d->pop[1], d->iop[0]) - 1;
    i64 rsub = o_isymoffso(irr[3], R, d->pop[2], d->pop[3], d->iop[1]) - 1;
    *base = b + rsub * nleft + lsub;
    st[0] = 1;
    st[1] = d->pop[0][irr[0] - 1];
    st[2] = nleft;
    st[3] = nleft * d->pop[2][irr[2] - 1];
    *nleft_out = nleft;
}

int o_vv2v_dpd(const double *v1, const o_desc *d1, const char *t1,
               const double *v2, const o_desc *d2, const char *t2,
               double *v3, const o_desc *d3, const char *t3,
               double f1, double f2)
{
    const o_desc *D[3] = {d1, d2, d3};
    const char *T[3] = {t1, t2, t3};
    char letters[12];
    int nlet = 0;
    int lslot[3][4]; /* letter id per slot, -1 dummy */
    /* ---- parse letters ---- */
    for (int t = 0; t < 3; t++)
        for (int s = 0; s < 4; s++) {
            char ch = T[t][s];
            if (ch == '.') {
                if (!is_zorb(D[t]->pop[s])) return O_ELAYOUT;
                lslot[t][s] = -1;
                continue;
            }
            int id = -1;
            for (int k = 0; k < nlet; k++)
                if (letters[k] == ch) id = k;
            if (id < 0) {
                if (nlet >= 6) return O_EARG;
                id = nlet;
                letters[nlet++] = ch;
            }
            lslot[t][s] = id;
        }
    /* each letter: exactly two tensors, once each, equal populations */
    int where[6][3];
    for (int k = 0; k < nlet; k++) {
        int cnt = 0;
        for (int t = 0; t < 3; t++) {
            where[k][t] = -1;
            for (int s = 0; s < 4; s++)
                if (lslot[t][s] == k) {
                    if (where[k][t] >= 0) return O_EARG;
                    where[k][t] = s;
                }
            if (where[k][t] >= 0) cnt++;
        }
        if (cnt != 2) return O_EARG;
        int ta = -1, tb = -1;
        for (int t = 0; t < 3; t++)
            if (where[k][t] >= 0) { if (ta < 0) ta = t; else tb = t; }
        if (memcmp(D[ta]->pop[where[k][ta]], D[tb]->pop[where[k][tb]], 8 * sizeof(i64)) != 0)
            return O_ELAYOUT;
    }
    /* ---- units ---- */
    unit_t U[MAXU];
    int nu = 0;
    int lunit[6];
    for (int k = 0; k < nlet; k++) lunit[k] = -1;
    for (int t = 0; t < 3; t++)
        for (int p = 0; p < 2; p++) {
            i64 iop = D[t]->iop[p];
            if (iop == 1) continue;
            int a = lslot[t][2 * p], b = lslot[t][2 * p + 1];
            if (a < 0 || b < 0) return O_ELAYOUT;
            if (lunit[a] >= 0 && lunit[a] == lunit[b] && U[lunit[a]].nlet == 2) continue;
            /* partner tensor must hold (a,b) as an intact pair with equal iop */
            int ok = 0;
            for (int u = 0; u < 3; u++) {
                if (u == t) continue;
                for (int q = 0; q < 2; q++)
                    if (lslot[u][2 * q] == a && lslot[u][2 * q + 1] == b && D[u]->iop[q] == iop) ok = 1;
            }
            if (!ok) return O_ELAYOUT;
            if (nu >= MAXU) return O_EARG;
            U[nu].nlet = 2; U[nu].let[0] = a; U[nu].let[1] = b; U[nu].iop = (int)iop;
            lunit[a] = lunit[b] = nu;
            nu++;
        }
    for (int k = 0; k < nlet; k++) {
        if (lunit[k] >= 0) continue;
        if (nu >= MAXU) return O_EARG;
        U[nu].nlet = 1; U[nu].let[0] = k; U[nu].let[1] = -1; U[nu].iop = 1;
        lunit[k] = nu;
        nu++;
    }
    for (int u = 0; u < nu; u++) {
        int k = U[u].let[0];
        for (int t = 0; t < 3; t++) {
            U[u].in[t] = where[k][t] >= 0;
            U[u].slot[t] = (U[u].nlet == 2) ? where[k][t] / 2 : where[k][t];
        }
        if (U[u].in[0] && U[u].in[2]) U[u].cls = 0;
        else if (U[u].in[1] && U[u].in[2]) U[u].cls = 1;
        else U[u].cls = 2;
    }
    /* packed-unit ordering inside each tensor must be (let0, let1) */
    for (int u = 0; u < nu; u++) {
        if (U[u].nlet != 2) continue;
        for (int t = 0; t < 3; t++) {
            if (!U[u].in[t]) continue;
            int p = U[u].slot[t];
            if (lslot[t][2 * p] != U[u].let[0] || lslot[t][2 * p + 1] != U[u].let[1]) return O_ELAYOUT;
        }
    }
    /* ---- scale V3 by f2 ---- */
    i64 len3 = o_desc_len(d3);
    if (f2 == 0.0) memset(v3, 0, (size_t)len3 * sizeof(double));
    else if (f2 != 1.0)
        for (i64 i = 0; i < len3; i++) v3[i] *= f2;
    /* ---- enumerate irrep assignments ---- */
    i64 nirr = o_nirrep();
    i64 ncomb = 1;
    for (int k = 0; k < nlet; k++) ncomb *= nirr;
    task_t *tasks = (task_t *)malloc(sizeof(task_t) * (size_t)(ncomb > 0 ? ncomb : 1));
    if (!tasks) return O_EMEM;
    i64 ntask = 0;
    for (i64 c = 0; c < ncomb; c++) {
        i64 lir[6];
        i64 cc = c;
        for (int k = 0; k < nlet; k++) { lir[k] = cc % nirr + 1; cc /= nirr; }
        int ok = 1;
        i64 sirr[3][4];
        for (int t = 0; t < 3 && ok; t++) {
            i64 prod = 1;
            for (int s = 0; s < 4; s++) {
                sirr[t][s] = lslot[t][s] < 0 ? 1 : lir[lslot[t][s]];
                prod = o_dirprd(prod, sirr[t][s]);
                if (D[t]->pop[s][sirr[t][s] - 1] == 0) ok = 0;
            }
            if (prod != D[t]->sym) ok = 0;
        }
        if (!ok) continue;
        task_t tk;
        for (int u = 0; u < nu && ok; u++) {
            if (U[u].nlet == 2) {
                i64 ia = lir[U[u].let[0]], ib = lir[U[u].let[1]];
                if (ia > ib) { ok = 0; break; }
                int t0 = U[u].in[0] ? 0 : 1;
                const o_desc *d = D[t0];
                int p = U[u].slot[t0];
                i64 na = d->pop[2 * p][ia - 1], nb = d->pop[2 * p + 1][ib - 1];
                if (ia < ib) tk.ext[u] = na * nb;
                else tk.ext[u] = (U[u].iop == 0) ? na * (na - 1) / 2 : na * (na + 1) / 2;
                if (tk.ext[u] == 0) ok = 0;
            } else {
                int k = U[u].let[0];
                int t0 = where[k][0] >= 0 ? 0 : 1;
                tk.ext[u] = D[t0]->pop[where[k][t0]][lir[k] - 1];
            }
        }
        if (!ok) continue;
        for (int t = 0; t < 3; t++) {
            i64 st4[4], nleft;
            block_geom(D[t], sirr[t], &tk.base[t], st4, &nleft);
            for (int u = 0; u < nu; u++) {
                if (!U[u].in[t]) { tk.st[t][u] = 0; continue; }
                if (U[u].nlet == 2) tk.st[t][u] = (U[u].slot[t] == 0) ? 1 : nleft;
                else tk.st[t][u] = st4[U[u].slot[t]];
            }
        }
        i64 key = 0;
        for (int k = 0; k < nlet; k++) {
            int u = lunit[k];
            if (U[u].cls != 2) key = key * 9 + lir[k];
        }
        tk.key = key;
        tasks[ntask++] = tk;
    }
    qsort(tasks, (size_t)ntask, sizeof(task_t), cmp_task);
    /* group boundaries (tasks writing the same V3 region) */
    i64 *gstart = (i64 *)malloc(sizeof(i64) * (size_t)(ntask + 1));
    i64 ng = 0;
    for (i64 i = 0; i < ntask; i++)
        if (i == 0 || tasks[i].key != tasks[i - 1].key) gstart[ng++] = i;
    gstart[ng] = ntask;

    int mu[MAXU], nuu[MAXU], ku[MAXU];
    int nm = 0, nn = 0, nk = 0;
    for (int u = 0; u < nu; u++) {
        if (U[u].cls == 0) mu[nm++] = u;
        else if (U[u].cls == 1) nuu[nn++] = u;
        else ku[nk++] = u;
    }
    int par = (ng > 1 && g_threads > 1);
    if (par) scipy_openblas_set_num_threads64_(1);
    int err = 0;
#pragma omp parallel for schedule(dynamic, 1) if (par)
    for (i64 g = 0; g < ng; g++) {
        for (i64 ti = gstart[g]; ti < gstart[g + 1]; ti++) {
            const task_t *tk = &tasks[ti];
            i64 M = 1, N = 1, K = 1;
            for (int i = 0; i < nm; i++) M *= tk->ext[mu[i]];
            for (int i = 0; i < nn; i++) N *= tk->ext[nuu[i]];
            for (int i = 0; i < nk; i++) K *= tk->ext[ku[i]];
            if (M == 0 || N == 0 || K == 0) continue;
            double *A = (double *)malloc(sizeof(double) * (size_t)(M * K));
            double *B = (double *)malloc(sizeof(double) * (size_t)(K * N));
            double *C = (double *)malloc(sizeof(double) * (size_t)(M * N));
            if (!A || !B || !C) { err = 1; free(A); free(B); free(C); continue; }
            /* offsets of M/N/K composite indices in each tensor */
            i64 *offmA = (i64 *)malloc(sizeof(i64) * (size_t)M), *offmC = (i64 *)malloc(sizeof(i64) * (size_t)M);
            i64 *offnB = (i64 *)malloc(sizeof(i64) * (size_t)N), *offnC = (i64 *)malloc(sizeof(i64) * (size_t)N);
            i64 *offkA = (i64 *)malloc(sizeof(i64) * (size_t)K), *offkB = (i64 *)malloc(sizeof(i64) * (size_t)K);
            for (i64 m = 0; m < M; m++) {
                i64 r = m, oa = 0, oc = 0;
                for (int i = 0; i < nm; i++) {
                    i64 e = tk->ext[mu[i]], x = r % e;
                    r /= e;
                    oa += x * tk->st[0][mu[i]];
                    oc += x * tk->st[2][mu[i]];
                }
                offmA[m] = oa; offmC[m] = oc;
            }
            for (i64 n = 0; n < N; n++) {
                i64 r = n, ob = 0, oc = 0;
                for (int i = 0; i < nn; i++) {
                    i64 e = tk->ext[nuu[i]], x = r % e;
                    r /= e;
                    ob += x * tk->st[1][nuu[i]];
                    oc += x * tk->st[2][nuu[i]];
                }
                offnB[n] = ob; offnC[n] = oc;
            }
            for (i64 k = 0; k < K; k++) {
                i64 r = k, oa = 0, ob = 0;
                for (int i = 0; i < nk; i++) {
                    i64 e = tk->ext[ku[i]], x = r % e;
                    r /= e;
                    oa += x * tk->st[0][ku[i]];
                    ob += x * tk->st[1][ku[i]];
                }
                offkA[k] = oa; offkB[k] = ob;
            }
            for (i64 k = 0; k < K; k++)
                for (i64 m = 0; m < M; m++) A[m + k * M] = v1[tk->base[0] + offmA[m] + offkA[k]];
            for (i64 n = 0; n < N; n++)
                for (i64 k = 0; k < K; k++) B[k + n * K] = v2[tk->base[1] + offkB[k] + offnB[n]];
            const double one = 1.0, zero = 0.0;
            scipy_dgemm_64_("N", "N", &M, &N, &K, &one, A, &M, B, &K, &zero, C, &M, 1, 1);
            for (i64 n = 0; n < N; n++)
                for (i64 m = 0; m < M; m++) v3[tk->base[2] + offmC[m] + offnC[n]] += f1 * C[m + n * M];
            free(A); free(B); free(C);
            free(offmA); free(offmC); free(offnB); free(offnC); free(offkA); free(offkB);
        }
    }
    if (par) scipy_openblas_set_num_threads64_((int)g_threads);
    free(gstart);
    free(tasks);
    return err ? O_EMEM : O_OK;
}
