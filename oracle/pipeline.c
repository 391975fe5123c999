/*
 * CPU ORACLE (test infrastructure only): the SF-CIS, ground CPS(D) and
 * EE-CPS(D-3) drivers, restating
 *   src/EE-CIS.SF/run.f90, src/EE-CIS.SF/calAR.f90,
 *   src/CPSd.SF/run1.f90, src/CPSd.SF/run2.f90, src/CPSd.SF/calC1.f90, calC2.f90,
 *   src/EE-CPSd.SF/run.f90, run_order.f90, calV_C.f90, calE_C.f90, calJ.f90,
 *   calC1_VR2.f90, calC2_VR1.f90, calC2_VR2.f90, calC_JR.f90, calC_VTR.f90,
 *   solver.f90, orthogonalR2L.f90.
 * The reference's disk records (IO_stream files CIS_sym<n>, CPSd_T__,
 * CPSd_sym<n>, CPSdC_sym<n>) are held in memory.
 */
#include "cpsd_oracle.h"
#include "oracle_internal.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

int o_system_init(o_system *s)
{
    int rc = o_set_symmetry(s->nirrep, s->dirprd);
    if (rc != O_OK) return rc;
    for (i64 r = 1; r <= 8; r++) {
        if (r > s->nirrep) { s->popo[r - 1] = s->popv[r - 1] = 0; continue; }
        i64 rb = o_dirprd(r, s->symry);
        s->popo[r - 1] = s->popa[r - 1] + s->popb[rb - 1];
        s->popv[r - 1] = s->vrta[r - 1] + s->vrtb[rb - 1];
    }
    return O_OK;
}

/* defaults of src/lib_cc/mod_common.f90:11-44 */
void o_params_default(o_params *p)
{
    memset(p, 0, sizeof(*p));
    p->davidson_dim = 20;
    p->davidson_cyc = 50;
    p->davidson_conv = 8;
    p->lowest = 0;
    p->diis_dim = 10;
    p->diis_cyc = 50;
    p->diis_max_err = 10.0e-8;
    p->spin_flip = 1;
    p->open_shell = 1;
    p->ex_mult = 1;
    p->nthreads = 1;
}

static const i64 Z[8] = {1, 0, 0, 0, 0, 0, 0, 0};

/* integral tensor views (src/EE-CPSd.SF/allocate_mem.f90) */
typedef struct {
    o_opt ijkl, ijka, abij, iabj, abci, abcd;
} ints_t;

static void ints_view(const o_system *s, const o_integrals *I, ints_t *v)
{
    const i64 *o = s->popo, *V = s->popv;
    o_opt_view(&v->ijkl, o, o, o, o, 0, 0, 1, (double *)I->ijkl);
    o_opt_view(&v->ijka, o, o, o, V, 0, 1, 1, (double *)I->ijka);
    o_opt_view(&v->abij, V, V, o, o, 0, 0, 1, (double *)I->abij);
    o_opt_view(&v->iabj, V, o, V, o, 1, 1, 1, (double *)I->iabj);
    o_opt_view(&v->abci, V, V, V, o, 0, 1, 1, (double *)I->abci);
    o_opt_view(&v->abcd, V, V, V, V, 0, 0, 1, (double *)I->abcd);
}

static double *zalloc(i64 n) { return (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }

/* ---------------- SF-CIS ---------------- */
typedef struct {
    const o_system *s;
    const ints_t *I;
    const double *oed1;
    i64 sym;
} cis_ctx;

/* calAR (src/EE-CIS.SF/calAR.f90:6-34): AR = e(a,i)*r(a,i) + V(fn,ai) r(fn) */
static void cis_sigma(void *vctx, const double *R, double *AR)
{
    cis_ctx *c = (cis_ctx *)vctx;
    o_opt r1, ar1;
    o_opt_view(&r1, c->s->popv, c->s->popo, Z, Z, 1, 1, c->sym, (double *)R);
    o_opt_view(&ar1, c->s->popv, c->s->popo, Z, Z, 1, 1, c->sym, AR);
    for (i64 i = 0; i < r1.len; i++) AR[i] = c->oed1[i] * R[i];
    o_c1_r1iabj(&ar1, &r1, &c->I->iabj, 1.0);
}

int o_cis_run(const o_system *s, const o_integrals *I, const o_params *p,
              double *omega, double *R, i64 *iters)
{
    ints_t v;
    ints_view(s, I, &v);
    i64 kroot = 0, roff = 0, itsum = 0;
    for (i64 sym = 1; sym <= s->nirrep; sym++) {
        i64 nroot = p->estate_sym[sym - 1];
        if (nroot == 0) continue;
        i64 len = o_irpdso(sym, s->popv, s->popo, 1);
        double *oed1 = zalloc(len);
        o_eorb_diff1(oed1, I->eorb, s->popv, s->popo, sym);
        double *file = zalloc((1 + len) * nroot);
        int rc = o_guess(s, I->eorb, p, sym, nroot, file);
        if (rc != O_OK) { free(oed1); free(file); return rc; }
        cis_ctx ctx = {s, &v, oed1, sym};
        i64 it = 0;
        rc = o_davidson(file, oed1, len, nroot, 1, p, cis_sigma, &ctx, &it);
        itsum += it;
        for (i64 k = 0; k < nroot; k++) {
            omega[kroot + k] = file[(1 + len) * k];
            memcpy(R + roff + len * k, file + (1 + len) * k + 1, sizeof(double) * (size_t)len);
        }
        kroot += nroot;
        roff += len * nroot;
        free(oed1);
        free(file);
        if (rc != O_OK) return rc;
    }
    if (iters) *iters = itsum;
    return O_OK;
}

/* ---------------- CIS(D-infinity) (src/CISdoo.SD.SF/run.f90, calAR.f90) ----
 * Davidson over (R1, R2) of one irrep with the sigma of calAR.f90:19-49:
 *   C1 = Fac R1 - R1 Fki + Wkaci R1 + c1_r2abci(R2) + c1_r2ijka(R2)
 *   C2 = e(ab,ij) R2 + c2_r1abci(R1) + c2_r1ijka(R1)
 * with MP2t = denomT2(abij), Fac = diag(e_v) + Fae_r2abij(MP2t),
 * Fki = diag(e_o) + Fmi_r2abij(MP2t), Wkaci = iabj + 2 Wmbej_r2abij(MP2t)
 * (run.f90:25-39, putDiagFock.f90); the diagonal preconditioner is
 * (Eorb_diff1, Eorb_diff2) and the guesses the singles' (run.f90:42-60). */
typedef struct {
    const o_system *s;
    const ints_t *I;
    const o_opt *fac, *fki, *wk;
    const double *oed2;
    i64 sym, l1, l2;
} doo_ctx;

static void doo_sigma(void *vctx, const double *R, double *AR)
{
    doo_ctx *c = (doo_ctx *)vctx;
    const i64 *o = c->s->popo, *V = c->s->popv;
    o_opt r1, r2, c1, c2;
    o_opt_view(&r1, V, o, Z, Z, 1, 1, c->sym, (double *)R);
    o_opt_view(&r2, V, V, o, o, 0, 0, c->sym, (double *)R + c->l1);
    o_opt_view(&c1, V, o, Z, Z, 1, 1, c->sym, AR);
    o_opt_view(&c2, V, V, o, o, 0, 0, c->sym, AR + c->l1);
    memset(AR, 0, sizeof(double) * (size_t)c->l1);
    o_c1_r1Fae(&c1, &r1, c->fac, 1.0);
    o_c1_r1Fmi(&c1, &r1, c->fki, 1.0);
    o_c1_r1iabj(&c1, &r1, c->wk, 1.0);
    o_c1_r2abci(&c1, &r2, &c->I->abci, 1.0);
    o_c1_r2ijka(&c1, &r2, &c->I->ijka, 1.0);
    for (i64 k = 0; k < c->l2; k++) AR[c->l1 + k] = c->oed2[k] * R[c->l1 + k];
    o_c2_r1abci(&c2, &r1, &c->I->abci, 1.0);
    o_c2_r1ijka(&c2, &r1, &c->I->ijka, 1.0);
}

/* putDiagFock (src/lib_cc/putDiagFock.f90:6-56): f(p,p) = e_p on the
 * diagonal of the (pop, pop) block of every irrep; eorb holds the occupied
 * orbitals of all irreps, then the virtual ones */
static void put_diag(double *F, const double *eorb, const o_system *s, int vir)
{
    const i64 *pp = vir ? s->popv : s->popo;
    i64 e0 = 0;
    if (vir)
        for (i64 h = 0; h < s->nirrep; h++) e0 += s->popo[h];
    i64 off = 0;
    for (i64 h = 0; h < s->nirrep; h++) {
        for (i64 p = 0; p < pp[h]; p++) F[off + p * pp[h] + p] = eorb[e0 + p];
        off += pp[h] * pp[h];
        e0 += pp[h];
    }
}

int o_cisdoo_run(const o_system *s, const o_integrals *I, const o_params *p, double *omega, double *R,
                 i64 *iters)
{
    ints_t v;
    ints_view(s, I, &v);
    const i64 *o = s->popo, *V = s->popv;
    i64 l2g = o_idsymsoc(1, V, V, 0, o, o, 0);
    double *mp2 = zalloc(l2g), *fa = zalloc(o_irpdso(1, V, V, 1)), *fk = zalloc(o_irpdso(1, o, o, 1));
    double *wka = zalloc(v.iabj.len);
    o_opt mp2t, fac, fki, wk;
    o_opt_view(&mp2t, V, V, o, o, 0, 0, 1, mp2);
    o_opt_view(&fac, V, V, Z, Z, 1, 1, 1, fa);
    o_opt_view(&fki, o, o, Z, Z, 1, 1, 1, fk);
    o_opt_view(&wk, V, o, V, o, 1, 1, 1, wka);
    o_denomT2(mp2, I->abij, I->eorb, V, o, 1, 0);
    put_diag(fa, I->eorb, s, 1);
    put_diag(fk, I->eorb, s, 0);
    memcpy(wka, I->iabj, sizeof(double) * (size_t)v.iabj.len);
    int rc = o_Fae_r2abij(&fac, &mp2t, &v.abij, 1.0);
    if (rc == O_OK) rc = o_Fmi_r2abij(&fki, &mp2t, &v.abij, 1.0);
    if (rc == O_OK) rc = o_Wmbej_r2abij(&wk, &mp2t, &v.abij, 2.0);
    i64 kroot = 0, roff = 0, itsum = 0;
    for (i64 sym = 1; sym <= s->nirrep && rc == O_OK; sym++) {
        i64 nroot = p->estate_sym[sym - 1];
        if (nroot == 0) continue;
        i64 l1 = o_irpdso(sym, V, o, 1), l2 = o_idsymsoc(sym, V, V, 0, o, o, 0), len = l1 + l2;
        double *diag = zalloc(len), *g1 = zalloc((1 + l1) * nroot), *file = zalloc((1 + len) * nroot);
        o_eorb_diff1(diag, I->eorb, V, o, sym);
        o_eorb_diff2(diag + l1, I->eorb, V, o, sym, 0);
        rc = o_guess(s, I->eorb, p, sym, nroot, g1);
        for (i64 k = 0; k < nroot && rc == O_OK; k++)
            memcpy(file + (1 + len) * k, g1 + (1 + l1) * k, sizeof(double) * (size_t)(1 + l1));
        doo_ctx ctx = {s, &v, &fac, &fki, &wk, diag + l1, sym, l1, l2};
        i64 it = 0;
        if (rc == O_OK) rc = o_davidson(file, diag, len, nroot, 1, p, doo_sigma, &ctx, &it);
        itsum += it;
        for (i64 k = 0; k < nroot; k++) {
            omega[kroot + k] = file[(1 + len) * k];
            memcpy(R + roff + len * k, file + (1 + len) * k + 1, sizeof(double) * (size_t)len);
        }
        kroot += nroot;
        roff += len * nroot;
        free(diag);
        free(g1);
        free(file);
    }
    if (iters) *iters = itsum;
    free(mp2); free(fa); free(fk); free(wka);
    return rc;
}

/* ---------------- ground CPS(D) ---------------- */
int o_cpsd_ground(const o_system *s, const o_integrals *I, const o_params *p,
                  double *T2_1, double *T1_2, double *T2_2, double *E2, double *E3,
                  i64 *diis_iters)
{
    ints_t v;
    ints_view(s, I, &v);
    const i64 *o = s->popo, *V = s->popv;
    o_opt t1, t2, t2b, c1, c2, r1;
    i64 l1 = o_irpdso(1, V, o, 1);
    i64 l2 = o_idsymsoc(1, V, V, 0, o, o, 0);
    double *c1a = zalloc(l1), *c2a = zalloc(l2), *r1a = zalloc(l1);
    o_opt_view(&t1, V, o, Z, Z, 1, 1, 1, T1_2);
    o_opt_view(&t2, V, V, o, o, 0, 0, 1, T2_1);
    o_opt_view(&t2b, V, V, o, o, 0, 0, 1, T2_2);
    o_opt_view(&c1, V, o, Z, Z, 1, 1, 1, c1a);
    o_opt_view(&c2, V, V, o, o, 0, 0, 1, c2a);
    o_opt_view(&r1, V, o, Z, Z, 1, 1, 1, r1a);
    /* run1 (src/CPSd.SF/run1.f90:9-38): T1^(1)=0, T2^(1) = <ab||ij>/D */
    o_denomT2(T2_1, I->abij, I->eorb, V, o, 1, 0);
    *E2 = o_ddot(l2, T2_1, I->abij);
    /* run2 (src/CPSd.SF/run2.f90:8-95) */
    int rc = o_c1_r2abci(&c1, &t2, &v.abci, 1.0);           /* calC1 -> calC1_VR2 */
    if (rc == O_OK) rc = o_c1_r2ijka(&c1, &t2, &v.ijka, 1.0);
    if (rc == O_OK) rc = o_c2_r2Wmbej(&c2, &t2, &v.iabj, 1.0); /* calC2 -> calC2_VR2 */
    if (rc == O_OK) rc = o_c2_r2Wmnij(&c2, &t2, &v.ijkl, 1.0);
    if (rc == O_OK) rc = o_c2_r2abcd(&c2, &t2, &v.abcd, 1.0);
    if (rc != O_OK) goto out;
    o_denomT2(T2_2, c2a, I->eorb, V, o, 1, 0);
    memcpy(r1a, c1a, sizeof(double) * (size_t)l1);
    o_diis dst;
    o_diis_init(&dst, l1, p->diis_dim);
    i64 iter = 0;
    for (;;) {
        iter++;
        o_denomT1(T1_2, r1a, I->eorb, V, o, 1);
        double err = o_diis_step(&dst, iter, T1_2);
        if (iter > 1 && fabs(err) < p->diis_max_err) break;
        if (iter > p->diis_cyc) break;
        memcpy(r1a, c1a, sizeof(double) * (size_t)l1);
        rc = o_c1_r1iabj(&r1, &t1, &v.iabj, 1.0);
        if (rc != O_OK) break;
    }
    o_diis_free(&dst);
    if (diis_iters) *diis_iters = iter;
    *E3 = o_ddot(l2, T2_2, I->abij);
out:
    free(c1a); free(c2a); free(r1a);
    return rc;
}

/* ---------------- ground state, third order (src/CPSd.SF/run3.f90:8-97) ----
 * C1^(3) = calC1_VR2(T2^(2))                               (calC1.f90)
 * C2^(3) = calC2_VR1(T1^(2)) + calC2_VR2(T2^(2))            (calC2.f90, calC2_VR.f90)
 *        + calC2_VTT(T2^(1)) with T1^(1) = 0: Fli, Fad, Wkaci, Wklij terms
 *          (calC2_VTT.f90:82-207)
 * T2^(3) = denomT2(C2^(3)); T1^(3) by the DIIS loop of run2 on C1^(3);
 * E^(4) = T2^(3) . abij (calEcorr.f90) */
int o_cpsd_ground3(const o_system *s, const o_integrals *I, const o_params *p,
                   const double *T2_1, const double *T1_2, const double *T2_2,
                   double *T1_3, double *T2_3, double *E4, i64 *diis_iters)
{
    ints_t v;
    ints_view(s, I, &v);
    const i64 *o = s->popo, *V = s->popv;
    o_opt t1b, t2a, t2b, t1c, c1, c2, r1, fli, fad, wkaci, wklij;
    i64 l1 = o_irpdso(1, V, o, 1);
    i64 l2 = o_idsymsoc(1, V, V, 0, o, o, 0);
    double *c1a = zalloc(l1), *c2a = zalloc(l2), *r1a = zalloc(l1);
    double *fo = zalloc(o_irpdso(1, o, o, 1)), *fv = zalloc(o_irpdso(1, V, V, 1));
    double *wk = zalloc(o_idsymsoc(1, V, o, 1, V, o, 1)), *wl = zalloc(o_idsymsoc(1, o, o, 0, o, o, 0));
    o_opt_view(&t1b, V, o, Z, Z, 1, 1, 1, (double *)T1_2);
    o_opt_view(&t2a, V, V, o, o, 0, 0, 1, (double *)T2_1);
    o_opt_view(&t2b, V, V, o, o, 0, 0, 1, (double *)T2_2);
    o_opt_view(&t1c, V, o, Z, Z, 1, 1, 1, T1_3);
    o_opt_view(&c1, V, o, Z, Z, 1, 1, 1, c1a);
    o_opt_view(&c2, V, V, o, o, 0, 0, 1, c2a);
    o_opt_view(&r1, V, o, Z, Z, 1, 1, 1, r1a);
    o_opt_view(&fli, o, o, Z, Z, 1, 1, 1, fo);
    o_opt_view(&fad, V, V, Z, Z, 1, 1, 1, fv);
    o_opt_view(&wkaci, V, o, V, o, 1, 1, 1, wk);
    o_opt_view(&wklij, o, o, o, o, 0, 0, 1, wl);
    int rc = o_c1_r2abci(&c1, &t2b, &v.abci, 1.0);
    if (rc == O_OK) rc = o_c1_r2ijka(&c1, &t2b, &v.ijka, 1.0);
    if (rc == O_OK) rc = o_c2_r1ijka(&c2, &t1b, &v.ijka, 1.0);
    if (rc == O_OK) rc = o_c2_r1abci(&c2, &t1b, &v.abci, 1.0);
    if (rc == O_OK) rc = o_c2_r2Wmbej(&c2, &t2b, &v.iabj, 1.0);
    if (rc == O_OK) rc = o_c2_r2Wmnij(&c2, &t2b, &v.ijkl, 1.0);
    if (rc == O_OK) rc = o_c2_r2abcd(&c2, &t2b, &v.abcd, 1.0);
    if (rc == O_OK) rc = o_Fmi_r2abij(&fli, &t2a, &v.abij, 1.0);
    if (rc == O_OK) rc = o_c2_r2Fmi(&c2, &t2a, &fli, 1.0);
    if (rc == O_OK) rc = o_Fae_r2abij(&fad, &t2a, &v.abij, 1.0);
    if (rc == O_OK) rc = o_c2_r2Fae(&c2, &t2a, &fad, 1.0);
    if (rc == O_OK) rc = o_Wmbej_r2abij(&wkaci, &t2a, &v.abij, 1.0);
    if (rc == O_OK) rc = o_c2_r2Wmbej(&c2, &t2a, &wkaci, 1.0);
    if (rc == O_OK) rc = o_Wmnij_r2abij(&wklij, &t2a, &v.abij, 0.5);
    if (rc == O_OK) rc = o_c2_r2Wmnij(&c2, &t2a, &wklij, 2.0);
    if (rc != O_OK) goto out;
    o_denomT2(T2_3, c2a, I->eorb, V, o, 1, 0);
    memcpy(r1a, c1a, sizeof(double) * (size_t)l1);
    o_diis dst;
    o_diis_init(&dst, l1, p->diis_dim);
    i64 iter = 0;
    for (;;) {
        iter++;
        o_denomT1(T1_3, r1a, I->eorb, V, o, 1);
        double err = o_diis_step(&dst, iter, T1_3);
        if (iter > 1 && fabs(err) < p->diis_max_err) break;
        if (iter > p->diis_cyc) break;
        memcpy(r1a, c1a, sizeof(double) * (size_t)l1);
        rc = o_c1_r1iabj(&r1, &t1c, &v.iabj, 1.0);
        if (rc != O_OK) break;
    }
    o_diis_free(&dst);
    if (diis_iters) *diis_iters = iter;
    *E4 = o_ddot(l2, T2_3, I->abij);
out:
    free(c1a); free(c2a); free(r1a); free(fo); free(fv); free(wk); free(wl);
    return rc;
}

/* ---------------- grCPS(D) ground state (src/grCPSd.SF) ----------------
 * Intermediates (run.f90:27-47): MP2t = denomT2(abij), Fli = -Fmi_r2abij(MP2t),
 * Fad = -Fae_r2abij(MP2t), Wkaci = iabj + 2 Wmbej_r2abij(MP2t).
 * Order k solves (solver.f90:1-77), from R = C^(k):
 *   T1 = denomT1(R1), T2 = denomT2(R2), DIIS on (T1, T2),
 *   E = calEcorr(k), R1 = C1 + calA0R1(T), R2 = C2 + calA0R2(T1)
 * with calA0R1 = Wkaci T1 - Fli T1 + Fad T1 + c1_r2ijka(T2) + c1_r2abci(T2)
 * (calA0R1.f90:19-30) and calA0R2 = c2_r1ijka(T1) + c2_r1abci(T1)
 * (calA0R2.f90:13-19).  Constants: C^(1) = (0, abij) (run1.f90:17-19);
 * C^(2) = (0, calA1R2(T2^(1))) (run2.f90, calA1R2.f90:30-37); C^(3) =
 * (calA2R1(T1^(1)) + calL1_VTT(T^(1)), calA1R2(T2^(2)) + calL2_VTT(T^(1)))
 * (run3.f90, calC1.f90, calC2.f90). */
typedef struct {
    const o_system *s;
    const ints_t *v;
    o_opt fli, fad, wk;
    i64 l1, l2;
} gr_ctx;

/* <ab,ij|[V,T2]|0> = c2_r2Wmbej + c2_r2Wmnij + c2_r2abcd (calA1R2.f90:30-37) */
static int gr_A1R2(const gr_ctx *g, o_opt *C2, const double *T2)
{
    const i64 *o = g->s->popo, *V = g->s->popv;
    o_opt t2;
    o_opt_view(&t2, V, V, o, o, 0, 0, 1, (double *)T2);
    int rc = o_c2_r2Wmbej(C2, &t2, &g->v->iabj, 1.0);
    if (rc == O_OK) rc = o_c2_r2Wmnij(C2, &t2, &g->v->ijkl, 1.0);
    if (rc == O_OK) rc = o_c2_r2abcd(C2, &t2, &g->v->abcd, 1.0);
    return rc;
}

/* calA2R1.f90:27-47: C1 -= (Wkaci - iabj) T1 + Fli T1 - Fad T1, i.e.
 * c1_r1iabj(Wkaci - iabj, -1), c1_r1Fmi(Fli, +1), c1_r1Fae(Fad, +1).  The
 * reference forms Wkaci - iabj in place and adds iabj back afterwards, so
 * Wkaci leaves rounded as (Wkaci - iabj) + iabj; so does this. */
static int gr_A2R1(gr_ctx *g, o_opt *C1, const double *T1)
{
    const i64 *o = g->s->popo, *V = g->s->popv;
    o_opt t1;
    o_opt_view(&t1, V, o, Z, Z, 1, 1, 1, (double *)T1);
    for (i64 k = 0; k < g->wk.len; k++) g->wk.arr[k] -= g->v->iabj.arr[k];
    int rc = o_c1_r1iabj(C1, &t1, &g->wk, -1.0);
    for (i64 k = 0; k < g->wk.len; k++) g->wk.arr[k] += g->v->iabj.arr[k];
    if (rc == O_OK) rc = o_c1_r1Fmi(C1, &t1, &g->fli, 1.0);
    if (rc == O_OK) rc = o_c1_r1Fae(C1, &t1, &g->fad, 1.0);
    return rc;
}

/* calL1_VTT.f90:30-75: L1 += Gli t(a,l) - Gad t(d,i) + Gld t(da,li) with
 * Gli = -Fmi_r1ijka(T1) - Fmi_r2abij(T2), Gad = -Fae_r1abci(T1) -
 * Fae_r2abij(T2), Gld = Fme_r1abij(T1) */
static int gr_L1_VTT(const gr_ctx *g, o_opt *L1, const double *T1, const double *T2)
{
    const i64 *o = g->s->popo, *V = g->s->popv;
    o_opt t1, t2, gli, gad, gld;
    o_opt_view(&t1, V, o, Z, Z, 1, 1, 1, (double *)T1);
    o_opt_view(&t2, V, V, o, o, 0, 0, 1, (double *)T2);
    double *a = zalloc(o_irpdso(1, o, o, 1)), *b = zalloc(o_irpdso(1, V, V, 1)), *c = zalloc(g->l1);
    o_opt_view(&gli, o, o, Z, Z, 1, 1, 1, a);
    o_opt_view(&gad, V, V, Z, Z, 1, 1, 1, b);
    o_opt_view(&gld, V, o, Z, Z, 1, 1, 1, c);
    int rc = o_Fmi_r1ijka(&gli, &t1, &g->v->ijka, -1.0);
    if (rc == O_OK) rc = o_Fmi_r2abij(&gli, &t2, &g->v->abij, -1.0);
    if (rc == O_OK) rc = o_Fae_r1abci(&gad, &t1, &g->v->abci, -1.0);
    if (rc == O_OK) rc = o_Fae_r2abij(&gad, &t2, &g->v->abij, -1.0);
    if (rc == O_OK) rc = o_Fme_r1abij(&gld, &t1, &g->v->abij, 1.0);
    if (rc == O_OK) rc = o_c1_r1Fmi(L1, &t1, &gli, -1.0);
    if (rc == O_OK) rc = o_c1_r1Fae(L1, &t1, &gad, -1.0);
    if (rc == O_OK) rc = o_c1_r2Fme(L1, &t2, &gld, 1.0);
    free(a); free(b); free(c);
    return rc;
}

/* calL2_VTT.f90:50-163, the eight terms of 0.5 <ab,ij|[[V,T],T]|0> */
static int gr_L2_VTT(const gr_ctx *g, o_opt *L2, const double *T1, const double *T2)
{
    const o_system *s = g->s;
    const i64 *o = s->popo, *V = s->popv;
    const ints_t *v = g->v;
    o_opt t1, t2, w;
    o_opt_view(&t1, V, o, Z, Z, 1, 1, 1, (double *)T1);
    o_opt_view(&t2, V, V, o, o, 0, 0, 1, (double *)T2);
    i64 n = v->abci.len;
    if (v->ijka.len > n) n = v->ijka.len;
    if (v->iabj.len > n) n = v->iabj.len;
    if (v->ijkl.len > n) n = v->ijkl.len;
    double *buf = zalloc(n);
#define GR_TMP(P0, P1, P2, P3, I0, I1)                                   \
    do {                                                                \
        o_opt_view(&w, P0, P1, P2, P3, I0, I1, 1, buf);                 \
        memset(buf, 0, sizeof(double) * (size_t)w.len);                 \
    } while (0)
    int rc = O_OK;
    /* -PijPab{V(kb,cj) t(c,i) t(a,k)}: W(ij,kb) = Wkbij_r1iabj(T1); c2_r1ijka(W, -1) */
    GR_TMP(o, o, o, V, 0, 1);
    rc = o_Wkbij_r1iabj(&w, &t1, &v->iabj, 1.0);
    if (rc == O_OK) rc = o_c2_r1ijka(L2, &t1, &w, -1.0);
    /* 0.5 Pij{V(ab,cd) t(c,i) t(d,j)}: W(ab,dj) = Wabdj_r1abcd(T1); c2_r1abci(W, 0.5) */
    if (rc == O_OK) {
        GR_TMP(V, V, V, o, 0, 1);
        rc = o_Wabdj_r1abcd(&w, &t1, &v->abcd, 1.0);
    }
    if (rc == O_OK) rc = o_c2_r1abci(L2, &t1, &w, 0.5);
    /* 0.5 Pab{V(kl,ij) t(a,k) t(b,l)}: W(ij,kb) = Wkbij_r1Uklij(T1); c2_r1ijka(W, 0.5) */
    if (rc == O_OK) {
        GR_TMP(o, o, o, V, 0, 1);
        rc = o_Wkbij_r1Uklij(&w, &t1, &v->ijkl, 1.0);
    }
    if (rc == O_OK) rc = o_c2_r1ijka(L2, &t1, &w, 0.5);
    /* -Pij{Gli t(ab,lj)}, Gli = Fmi_r1ijka(T1) + Fmi_r2abij(T2) */
    if (rc == O_OK) {
        GR_TMP(o, o, Z, Z, 1, 1);
        rc = o_Fmi_r1ijka(&w, &t1, &v->ijka, 1.0);
    }
    if (rc == O_OK) rc = o_Fmi_r2abij(&w, &t2, &v->abij, 1.0);
    if (rc == O_OK) rc = o_c2_r2Fmi(L2, &t2, &w, 1.0);
    /* Pab{Gad t(db,ij)}, Gad = Fae_r1abci(T1) + Fae_r2abij(T2) */
    if (rc == O_OK) {
        GR_TMP(V, V, Z, Z, 1, 1);
        rc = o_Fae_r1abci(&w, &t1, &v->abci, 1.0);
    }
    if (rc == O_OK) rc = o_Fae_r2abij(&w, &t2, &v->abij, 1.0);
    if (rc == O_OK) rc = o_c2_r2Fae(L2, &t2, &w, 1.0);
    /* PijPab{Wkbcj t(ac,ik)}, W = Wmbej_r1ijka(T1) + Wmbej_r1abci(T1) + Wmbej_r2abij(T2) */
    if (rc == O_OK) {
        GR_TMP(V, o, V, o, 1, 1);
        rc = o_Wmbej_r1ijka(&w, &t1, &v->ijka, 1.0);
    }
    if (rc == O_OK) rc = o_Wmbej_r1abci(&w, &t1, &v->abci, 1.0);
    if (rc == O_OK) rc = o_Wmbej_r2abij(&w, &t2, &v->abij, 1.0);
    if (rc == O_OK) rc = o_c2_r2Wmbej(L2, &t2, &w, 1.0);
    /* -0.5 Pab{V(kb,cd) t(cd,ij) t(a,k)}: W(ij,kb) = Wkbij_r2abci(T2); c2_r1ijka(W, 1) */
    if (rc == O_OK) {
        GR_TMP(o, o, o, V, 0, 1);
        rc = o_Wkbij_r2abci(&w, &t2, &v->abci, 1.0);
    }
    if (rc == O_OK) rc = o_c2_r1ijka(L2, &t1, &w, 1.0);
    /* Wklij t(ab,kl), Wklij = Wmnij_r1ijka(T1, 0.5) + Wmnij_r2abij(T2, 0.5); c2_r2Wmnij(W, 2) */
    if (rc == O_OK) {
        GR_TMP(o, o, o, o, 0, 0);
        rc = o_Wmnij_r1ijka(&w, &t1, &v->ijka, 0.5);
    }
    if (rc == O_OK) rc = o_Wmnij_r2abij(&w, &t2, &v->abij, 0.5);
    if (rc == O_OK) rc = o_c2_r2Wmnij(L2, &t2, &w, 2.0);
#undef GR_TMP
    free(buf);
    return rc;
}

int o_grcpsd_ground(const o_system *s, const o_integrals *I, const o_params *p, double *T, double *E,
                    i64 *iters)
{
    ints_t v;
    ints_view(s, I, &v);
    const i64 *o = s->popo, *V = s->popv;
    const i64 l1 = o_irpdso(1, V, o, 1), l2 = o_idsymsoc(1, V, V, 0, o, o, 0), lt = l1 + l2;
    gr_ctx g;
    g.s = s;
    g.v = &v;
    g.l1 = l1;
    g.l2 = l2;
    double *mp2 = zalloc(l2), *fo = zalloc(o_irpdso(1, o, o, 1)), *fv = zalloc(o_irpdso(1, V, V, 1));
    double *wk = zalloc(v.iabj.len), *C = zalloc(lt), *R = zalloc(lt), *tau = zalloc(l2);
    o_opt mp2t, c1, c2, r1, r2, t1, t2, ta, x1, y1;
    o_opt_view(&mp2t, V, V, o, o, 0, 0, 1, mp2);
    o_opt_view(&g.fli, o, o, Z, Z, 1, 1, 1, fo);
    o_opt_view(&g.fad, V, V, Z, Z, 1, 1, 1, fv);
    o_opt_view(&g.wk, V, o, V, o, 1, 1, 1, wk);
    o_opt_view(&c1, V, o, Z, Z, 1, 1, 1, C);
    o_opt_view(&c2, V, V, o, o, 0, 0, 1, C + l1);
    o_opt_view(&r1, V, o, Z, Z, 1, 1, 1, R);
    o_opt_view(&r2, V, V, o, o, 0, 0, 1, R + l1);
    o_opt_view(&ta, V, V, o, o, 0, 0, 1, tau);
    o_denomT2(mp2, I->abij, I->eorb, V, o, 1, 0);
    memcpy(wk, I->iabj, sizeof(double) * (size_t)v.iabj.len);
    int rc = o_Fmi_r2abij(&g.fli, &mp2t, &v.abij, -1.0);
    if (rc == O_OK) rc = o_Fae_r2abij(&g.fad, &mp2t, &v.abij, -1.0);
    if (rc == O_OK) rc = o_Wmbej_r2abij(&g.wk, &mp2t, &v.abij, 2.0);
    for (int k = 1; k <= 3 && rc == O_OK; k++) {
        double *Tk = T + (k - 1) * lt;
        o_opt_view(&t1, V, o, Z, Z, 1, 1, 1, Tk);
        o_opt_view(&t2, V, V, o, o, 0, 0, 1, Tk + l1);
        /* the constant C^(k) */
        memset(C, 0, sizeof(double) * (size_t)lt);
        if (k == 1) memcpy(C + l1, I->abij, sizeof(double) * (size_t)l2);
        if (k >= 2) rc = gr_A1R2(&g, &c2, T + (k - 2) * lt + l1);
        if (k == 3 && rc == O_OK) rc = gr_A2R1(&g, &c1, T);
        if (k == 3 && rc == O_OK) rc = gr_L1_VTT(&g, &c1, T, T + l1);
        if (k == 3 && rc == O_OK) rc = gr_L2_VTT(&g, &c2, T, T + l1);
        if (rc != O_OK) break;
        /* solver.f90:24-73 */
        memcpy(R, C, sizeof(double) * (size_t)lt);
        o_diis dst;
        o_diis_init(&dst, lt, p->diis_dim);
        i64 iter = 0;
        double Ek = 0.0;
        for (;;) {
            iter++;
            o_denomT1(Tk, R, I->eorb, V, o, 1);
            o_denomT2(Tk + l1, R + l1, I->eorb, V, o, 1, 0);
            double err = o_diis_step(&dst, iter, Tk);
            /* calEcorr.f90:21-52 */
            memcpy(tau, Tk + l1, sizeof(double) * (size_t)l2);
            if (k == 2) {
                o_opt_view(&x1, V, o, Z, Z, 1, 1, 1, T);
                rc = o_effectT2(&ta, &x1, &x1, 1.0, 1);
            } else if (k == 3) {
                o_opt_view(&x1, V, o, Z, Z, 1, 1, 1, T + lt);
                o_opt_view(&y1, V, o, Z, Z, 1, 1, 1, T);
                rc = o_effectT2(&ta, &x1, &y1, 1.0, 2);
            }
            if (rc != O_OK) break;
            Ek = o_ddot(l2, tau, I->abij);
            if (iter > 1 && fabs(err) < p->diis_max_err) break;
            if (iter > p->diis_cyc) break;
            memcpy(R, C, sizeof(double) * (size_t)lt);
            rc = o_c1_r1iabj(&r1, &t1, &g.wk, 1.0); /* calA0R1 */
            if (rc == O_OK) rc = o_c1_r1Fmi(&r1, &t1, &g.fli, -1.0);
            if (rc == O_OK) rc = o_c1_r1Fae(&r1, &t1, &g.fad, -1.0);
            if (rc == O_OK) rc = o_c1_r2ijka(&r1, &t2, &v.ijka, 1.0);
            if (rc == O_OK) rc = o_c1_r2abci(&r1, &t2, &v.abci, 1.0);
            if (rc == O_OK) rc = o_c2_r1ijka(&r2, &t1, &v.ijka, 1.0); /* calA0R2 */
            if (rc == O_OK) rc = o_c2_r1abci(&r2, &t1, &v.abci, 1.0);
            if (rc != O_OK) break;
        }
        o_diis_free(&dst);
        E[k - 1] = Ek;
        if (iters) iters[k - 1] = iter;
    }
    free(mp2); free(fo); free(fv); free(wk); free(C); free(R); free(tau);
    return rc;
}

/* ---------------- EE-grCPS(D) (src/EE-grCPSd.SF) ----------------
 * Per root of the CIS(D-infinity) problem (R^(0), w0): the left vector L
 * (calEigenCISDoo.f90: L1 by DIIS on L1 [Ass - Asd (Add - w)^-1 Ads - w] = 0,
 * L2 = L1 Asd (w - Add)^-1, <L|R> = 1), w^(1) = L J^(1) R^(0); then orders
 * 1, 2 (run1.f90, run2.f90): (A0 - w0) R^(n) = sum_k w^(k) R^(n-k) - C^(n)
 * by the DIIS solver with R orthogonal to L (solver.f90), w^(n+1) =
 * L C^(n+1) with C^(n) of calE_C.f90. */
static double *opt_new(o_opt *t, const i64 *p0, const i64 *p1, const i64 *p2, const i64 *p3, i64 i0, i64 i1,
                       i64 sym)
{
    o_opt_view(t, p0, p1, p2, p3, i0, i1, sym, NULL);
    t->arr = zalloc(t->len);
    return t->arr;
}

/* one J^(k) set: Foo, Fvv, Fov, Woooo, Wooov, Wovoo, Wovvo (allocate_mem.f90:54-81) */
typedef struct {
    o_opt Foo, Fvv, Fov, Woooo, Wooov, Wovoo, Wovvo;
} ee_J;

static void ee_J_alloc(const o_system *s, ee_J *J)
{
    const i64 *o = s->popo, *V = s->popv;
    opt_new(&J->Foo, o, o, Z, Z, 1, 1, 1);
    opt_new(&J->Fvv, V, V, Z, Z, 1, 1, 1);
    opt_new(&J->Fov, V, o, Z, Z, 1, 1, 1);
    opt_new(&J->Woooo, o, o, o, o, 0, 0, 1);
    opt_new(&J->Wooov, o, o, o, V, 0, 1, 1);
    opt_new(&J->Wovoo, o, o, o, V, 0, 1, 1);
    opt_new(&J->Wovvo, V, o, V, o, 1, 1, 1);
}
static void ee_J_free(ee_J *J)
{
    free(J->Foo.arr); free(J->Fvv.arr); free(J->Fov.arr); free(J->Woooo.arr);
    free(J->Wooov.arr); free(J->Wovoo.arr); free(J->Wovvo.arr);
}

/* the [V,T] part of calJ2 / calJ3 (calJ.f90:14-95, 104-170) */
static int ee_J_VT(const ints_t *v, ee_J *J, const o_opt *t1, const o_opt *t2)
{
    int rc = o_Fmi_r1ijka(&J->Foo, t1, &v->ijka, 1.0);
    if (rc == O_OK) rc = o_Fmi_r2abij(&J->Foo, t2, &v->abij, 1.0);
    if (rc == O_OK) rc = o_Fae_r1abci(&J->Fvv, t1, &v->abci, 1.0);
    if (rc == O_OK) rc = o_Fae_r2abij(&J->Fvv, t2, &v->abij, 1.0);
    if (rc == O_OK) rc = o_Fme_r1abij(&J->Fov, t1, &v->abij, 1.0);
    if (rc == O_OK) rc = o_Wkbij_r1iabj(&J->Wovoo, t1, &v->iabj, -1.0);
    if (rc == O_OK) rc = o_Wkbij_r1Uklij(&J->Wovoo, t1, &v->ijkl, 1.0);
    if (rc == O_OK) rc = o_Wkbij_r2ijka(&J->Wovoo, t2, &v->ijka, 1.0);
    if (rc == O_OK) rc = o_Wkbij_r2abci(&J->Wovoo, t2, &v->abci, 1.0);
    if (rc == O_OK) rc = o_Wmbej_r1ijka(&J->Wovvo, t1, &v->ijka, 1.0);
    if (rc == O_OK) rc = o_Wmbej_r1abci(&J->Wovvo, t1, &v->abci, 1.0);
    if (rc == O_OK) rc = o_Wmbej_r2abij(&J->Wovvo, t2, &v->abij, 2.0);
    if (rc == O_OK) rc = o_Wmnij_r1ijka(&J->Woooo, t1, &v->ijka, 1.0);
    if (rc == O_OK) rc = o_Wmnij_r2abij(&J->Woooo, t2, &v->abij, 1.0);
    if (rc == O_OK) rc = o_Wlkjd_r1abij(&J->Wooov, t1, &v->abij, 1.0);
    return rc;
}

/* the [[V,T^(1)],T^(1)] part of calJ3 (calJ.f90:172-218) */
static int ee_J_VTT(const o_system *s, const ints_t *v, ee_J *J, const o_opt *t1, const o_opt *t2)
{
    const i64 *o = s->popo, *V = s->popv;
    o_opt w;
    opt_new(&w, V, o, Z, Z, 1, 1, 1);
    int rc = o_Fme_r1abij(&w, t1, &v->abij, 1.0);
    if (rc == O_OK) rc = o_Fmi_r1fia(&J->Foo, t1, &w, 1.0);
    if (rc == O_OK) rc = o_Fae_r1fia(&J->Fvv, t1, &w, 1.0);
    if (rc == O_OK) rc = o_Wkbij_r2Fkc(&J->Wovoo, t2, &w, -1.0);
    free(w.arr);
    if (rc != O_OK) return rc;
    opt_new(&w, o, o, o, V, 0, 1, 1);
    rc = o_Wlkjd_r1abij(&w, t1, &v->abij, 1.0);
    if (rc == O_OK) rc = o_Wmbej_r1ijka(&J->Wovvo, t1, &w, 1.0);
    if (rc == O_OK) rc = o_Wmnij_r1ijka(&J->Woooo, t1, &w, 0.5);
    if (rc == O_OK) rc = o_Wkbij_r2ijka(&J->Wovoo, t2, &w, 1.0);
    free(w.arr);
    if (rc != O_OK) return rc;
    opt_new(&w, o, o, o, o, 0, 0, 1);
    rc = o_Wmnij_r1ijka(&w, t1, &v->ijka, 1.0);
    if (rc == O_OK) rc = o_Wmnij_r2abij(&w, t2, &v->abij, 1.0);
    if (rc == O_OK) rc = o_Wkbij_r1Uklij(&J->Wovoo, t1, &w, 1.0);
    free(w.arr);
    if (rc != O_OK) return rc;
    opt_new(&w, V, o, V, o, 1, 1, 1);
    rc = o_Wmbej_r1abci(&w, t1, &v->abci, 1.0);
    if (rc == O_OK) rc = o_Wkbij_r1iabj(&J->Wovoo, t1, &w, -0.5);
    free(w.arr);
    return rc;
}

/* calC_J2R / calC_J3R (calC_JR.f90:3-29, 32-58) */
static int ee_CJR(const ee_J *J, o_opt *C1, o_opt *C2, const o_opt *r1, const o_opt *r2, double f)
{
    int rc = o_c2_r1ijka(C2, r1, &J->Wovoo, f);
    if (rc == O_OK) rc = o_c1_r1iabj(C1, r1, &J->Wovvo, f);
    if (rc == O_OK) rc = o_c2_r2Wmbej(C2, r2, &J->Wovvo, f);
    if (rc == O_OK) rc = o_c2_r2Wmnij(C2, r2, &J->Woooo, f);
    if (rc == O_OK) rc = o_c1_r1Fmi(C1, r1, &J->Foo, f);
    if (rc == O_OK) rc = o_c2_r2Fmi(C2, r2, &J->Foo, f);
    if (rc == O_OK) rc = o_c1_r1Fae(C1, r1, &J->Fvv, f);
    if (rc == O_OK) rc = o_c2_r2Fae(C2, r2, &J->Fvv, f);
    if (rc == O_OK) rc = o_c1_r2ijka(C1, r2, &J->Wooov, f);
    if (rc == O_OK) rc = o_c1_r2Fme(C1, r2, &J->Fov, f);
    return rc;
}

/* calC_VTR.f90:3-78: C += f <u|[[V,T],R]|0> without intermediates */
static int ee_VTR(const o_system *s, const ints_t *v, o_opt *C1, o_opt *C2, const o_opt *t1, const o_opt *t2,
                  const o_opt *r1, const o_opt *r2, i64 symR, double f)
{
    const i64 *o = s->popo, *V = s->popv;
    o_opt w;
    int rc;
    opt_new(&w, o, o, Z, Z, 1, 1, symR);
    rc = o_Fmi_r2abij(&w, r2, &v->abij, 1.0);
    if (rc == O_OK) rc = o_c1_r1Fmi(C1, t1, &w, f);
    free(w.arr);
    if (rc != O_OK) return rc;
    opt_new(&w, o, o, o, V, 0, 1, symR);
    rc = o_Wkbij_r1iabj(&w, r1, &v->iabj, -1.0);
    if (rc == O_OK) rc = o_Wkbij_r2abci(&w, r2, &v->abci, 1.0);
    if (rc == O_OK) rc = o_c2_r1ijka(C2, t1, &w, f);
    free(w.arr);
    if (rc != O_OK) return rc;
    opt_new(&w, V, V, V, o, 0, 1, 1);
    rc = o_Wabdj_r1abcd(&w, t1, &v->abcd, 1.0);
    if (rc == O_OK) rc = o_c2_r1abci(C2, r1, &w, f);
    free(w.arr);
    if (rc != O_OK) return rc;
    opt_new(&w, o, o, o, o, 0, 0, symR);
    rc = o_Wmnij_r2abij(&w, r2, &v->abij, 1.0);
    if (rc == O_OK) rc = o_Wmnij_r1ijka(&w, r1, &v->ijka, 1.0);
    if (rc == O_OK) rc = o_c2_r2Wmnij(C2, t2, &w, f);
    free(w.arr);
    if (rc != O_OK) return rc;
    opt_new(&w, V, o, V, o, 1, 1, symR);
    rc = o_Wmbej_r1abci(&w, r1, &v->abci, 1.0);
    if (rc == O_OK) rc = o_c2_r2Wmbej(C2, t2, &w, f);
    free(w.arr);
    if (rc != O_OK) return rc;
    opt_new(&w, o, o, Z, Z, 1, 1, symR);
    rc = o_Fmi_r1ijka(&w, r1, &v->ijka, 1.0);
    if (rc == O_OK) rc = o_Fmi_r2abij(&w, r2, &v->abij, 1.0);
    if (rc == O_OK) rc = o_c2_r2Fmi(C2, t2, &w, f);
    free(w.arr);
    if (rc != O_OK) return rc;
    opt_new(&w, V, V, Z, Z, 1, 1, symR);
    rc = o_Fae_r1abci(&w, r1, &v->abci, 1.0);
    if (rc == O_OK) rc = o_Fae_r2abij(&w, r2, &v->abij, 1.0);
    if (rc == O_OK) rc = o_c2_r2Fae(C2, t2, &w, f);
    free(w.arr);
    return rc;
}

/* calC_VTTR.f90:3-86: C2 += f <u|[[[V,T],T],R]|0> */
static int ee_VTTR(const o_system *s, const ints_t *v, o_opt *C2, const o_opt *t1, const o_opt *t2,
                   const o_opt *r1, const o_opt *r2, i64 symR, double f)
{
    const i64 *o = s->popo, *V = s->popv;
    o_opt a, b, c;
    int rc;
    opt_new(&a, V, o, Z, Z, 1, 1, symR);  /* Gld = V(kl,cd) r(c,k) */
    rc = o_Fme_r1abij(&a, r1, &v->abij, 1.0);
    opt_new(&b, V, V, Z, Z, 1, 1, symR);  /* F(a,d) -= Gld t(a,l) */
    if (rc == O_OK) rc = o_Fae_r1fia(&b, t1, &a, 1.0);
    if (rc == O_OK) rc = o_c2_r2Fae(C2, t2, &b, f);
    free(b.arr);
    opt_new(&b, o, o, Z, Z, 1, 1, symR);  /* F(l,i) = Gld t(d,i) + Fld r(d,i) */
    if (rc == O_OK) rc = o_Fmi_r1fia(&b, t1, &a, 1.0);
    opt_new(&c, V, o, Z, Z, 1, 1, 1);     /* F(l,d) = V(kl,cd) t(c,k) */
    if (rc == O_OK) rc = o_Fme_r1abij(&c, t1, &v->abij, 1.0);
    if (rc == O_OK) rc = o_Fmi_r1fia(&b, r1, &c, 1.0);
    if (rc == O_OK) rc = o_c2_r2Fmi(C2, t2, &b, f);
    free(a.arr); free(b.arr); free(c.arr);
    if (rc != O_OK) return rc;
    /* 0.5 V(kl,cd) r(c,i) t(d,j) t(ab,kl) */
    opt_new(&a, o, o, o, V, 0, 1, symR);
    rc = o_Wlkjd_r1abij(&a, r1, &v->abij, 1.0);
    opt_new(&b, o, o, o, o, 0, 0, symR);
    if (rc == O_OK) rc = o_Wmnij_r1ijka(&b, t1, &a, 1.0);
    if (rc == O_OK) rc = o_c2_r2Wmnij(C2, t2, &b, f);
    free(a.arr); free(b.arr);
    if (rc != O_OK) return rc;
    /* W(kb,ij) = -0.5 W(kl,ij) t(b,l) + W(kb,cj) r(c,i) + W(kl,id) t(db,lj) */
    opt_new(&a, o, o, o, V, 0, 1, symR);
    opt_new(&b, o, o, o, o, 0, 0, symR);
    rc = o_Wmnij_r2abij(&b, r2, &v->abij, 1.0);
    if (rc == O_OK) rc = o_Wmnij_r1ijka(&b, r1, &v->ijka, 1.0);
    if (rc == O_OK) rc = o_Wkbij_r1Uklij(&a, t1, &b, 0.5);
    free(b.arr);
    opt_new(&b, V, o, V, o, 1, 1, 1);
    if (rc == O_OK) rc = o_Wmbej_r1abci(&b, t1, &v->abci, 1.0);
    if (rc == O_OK) rc = o_Wkbij_r1iabj(&a, r1, &b, -1.0);
    free(b.arr);
    opt_new(&b, o, o, o, V, 0, 1, symR);
    if (rc == O_OK) rc = o_Wlkjd_r1abij(&b, r1, &v->abij, 1.0);
    if (rc == O_OK) rc = o_Wkbij_r2ijka(&a, t2, &b, 1.0);
    free(b.arr);
    if (rc == O_OK) rc = o_c2_r1ijka(C2, t1, &a, f);
    free(a.arr);
    return rc;
}

/* calC2_VR2.f90:3-24: C2 += f <ab,ij|[V,R2]|0> */
static int ee_C2VR2(const ints_t *v, o_opt *C2, const o_opt *r2, double f)
{
    int rc = o_c2_r2Wmbej(C2, r2, &v->iabj, f);
    if (rc == O_OK) rc = o_c2_r2Wmnij(C2, r2, &v->ijkl, f);
    if (rc == O_OK) rc = o_c2_r2abcd(C2, r2, &v->abcd, f);
    return rc;
}

/* calC1_VMP2R1.f90:9-30: C1 -= f <a,i|[[V,MP2t],R1]|0>, Wkaci - iabj formed
 * in place and restored */
static int ee_VMP2R1(gr_ctx *g, o_opt *C1, const o_opt *r1, double f)
{
    for (i64 k = 0; k < g->wk.len; k++) g->wk.arr[k] -= g->v->iabj.arr[k];
    int rc = o_c1_r1iabj(C1, r1, &g->wk, -f);
    for (i64 k = 0; k < g->wk.len; k++) g->wk.arr[k] += g->v->iabj.arr[k];
    if (rc == O_OK) rc = o_c1_r1Fmi(C1, r1, &g->fli, f);
    if (rc == O_OK) rc = o_c1_r1Fae(C1, r1, &g->fad, f);
    return rc;
}

/* calE_C.f90:4-66: C^(n) of one root (C, R^(k) as (R1, R2) vectors of irrep
 * symR; T^(1), T^(2) of irrep 1) */
static int ee_calE_C(gr_ctx *g, const ee_J *J2, const ee_J *J3, const double *T, i64 lt, double *C,
                     double *const *R, i64 symR, i64 l1, int order)
{
    const o_system *s = g->s;
    const i64 *o = s->popo, *V = s->popv;
    const ints_t *v = g->v;
    const i64 g1 = o_irpdso(1, V, o, 1);
    o_opt c1, c2, r1, r2, t1, t2;
    o_opt_view(&c1, V, o, Z, Z, 1, 1, symR, C);
    o_opt_view(&c2, V, V, o, o, 0, 0, symR, C + l1);
    memset(C, 0, sizeof(double) * (size_t)(c1.len + c2.len));
    o_opt_view(&r2, V, V, o, o, 0, 0, symR, R[order - 1] + l1);
    int rc = ee_C2VR2(v, &c2, &r2, 1.0);
    if (order == 1 || rc != O_OK) return rc;
    o_opt_view(&r1, V, o, Z, Z, 1, 1, symR, R[order - 2]);
    o_opt_view(&r2, V, V, o, o, 0, 0, symR, R[order - 2] + l1);
    o_opt_view(&t1, V, o, Z, Z, 1, 1, 1, (double *)T);
    o_opt_view(&t2, V, V, o, o, 0, 0, 1, (double *)T + g1);
    rc = ee_VMP2R1(g, &c1, &r1, 1.0);
    if (rc == O_OK) rc = ee_CJR(J2, &c1, &c2, &r1, &r2, 1.0);
    if (rc == O_OK) rc = ee_VTR(s, v, &c1, &c2, &t1, &t2, &r1, &r2, symR, 1.0);
    if (order == 2 || rc != O_OK) return rc;
    o_opt_view(&r1, V, o, Z, Z, 1, 1, symR, R[0]);
    o_opt_view(&r2, V, V, o, o, 0, 0, symR, R[0] + l1);
    rc = ee_CJR(J3, &c1, &c2, &r1, &r2, 1.0);
    o_opt_view(&t1, V, o, Z, Z, 1, 1, 1, (double *)T + lt);
    o_opt_view(&t2, V, V, o, o, 0, 0, 1, (double *)T + lt + g1);
    if (rc == O_OK) rc = ee_VTR(s, v, &c1, &c2, &t1, &t2, &r1, &r2, symR, 1.0);
    o_opt_view(&t1, V, o, Z, Z, 1, 1, 1, (double *)T);
    o_opt_view(&t2, V, V, o, o, 0, 0, 1, (double *)T + g1);
    if (rc == O_OK) rc = ee_VTTR(s, v, &c2, &t1, &t2, &r1, &r2, symR, 1.0);
    return rc;
}

/* orthogonalR2L.f90:5-21: R -= (<L|R> / |L|) L (the reference divides by the
 * norm, not its square) */
static void ee_orth(double *R, const double *L, i64 n)
{
    double nrm = o_dnrm2(n, L), dot = o_ddot(n, L, R);
    o_daxpy(n, -dot / nrm, L, R);
}

int o_eegrcpsd_roots(const o_system *s, const o_integrals *I, const o_params *p, const double *T,
                     const double *omega, const double *R0, double *w, double *Lout, double *Rout,
                     i64 *iters)
{
    ints_t v;
    ints_view(s, I, &v);
    const i64 *o = s->popo, *V = s->popv;
    const i64 g1 = o_irpdso(1, V, o, 1), lt = g1 + o_idsymsoc(1, V, V, 0, o, o, 0);
    gr_ctx g;
    g.s = s;
    g.v = &v;
    g.l1 = g1;
    g.l2 = lt - g1;
    double *mp2 = zalloc(g.l2), *fo = zalloc(o_irpdso(1, o, o, 1)), *fv = zalloc(o_irpdso(1, V, V, 1));
    double *wk = zalloc(v.iabj.len);
    o_opt mp2t;
    o_opt_view(&mp2t, V, V, o, o, 0, 0, 1, mp2);
    o_opt_view(&g.fli, o, o, Z, Z, 1, 1, 1, fo);
    o_opt_view(&g.fad, V, V, Z, Z, 1, 1, 1, fv);
    o_opt_view(&g.wk, V, o, V, o, 1, 1, 1, wk);
    /* run.f90:41-60 */
    o_denomT2(mp2, I->abij, I->eorb, V, o, 1, 0);
    memcpy(wk, I->iabj, sizeof(double) * (size_t)v.iabj.len);
    int rc = o_Fmi_r2abij(&g.fli, &mp2t, &v.abij, -1.0);
    if (rc == O_OK) rc = o_Fae_r2abij(&g.fad, &mp2t, &v.abij, -1.0);
    if (rc == O_OK) rc = o_Wmbej_r2abij(&g.wk, &mp2t, &v.abij, 2.0);
    i64 nroot = 0, rlen = 0, itsum = 0;
    for (i64 h = 0; h < s->nirrep; h++) {
        nroot += p->estate_sym[h];
        rlen += p->estate_sym[h] * (o_irpdso(h + 1, V, o, 1) + o_idsymsoc(h + 1, V, V, 0, o, o, 0));
    }
    /* per root: R^(0..2), L, C^(n) */
    double *Rall = zalloc(3 * rlen), *Lall = zalloc(rlen), *Call = zalloc(rlen);
    memcpy(Rall, R0, sizeof(double) * (size_t)rlen);
    /* calEigenCISDoo for every root (run.f90:64-69) */
    i64 off = 0, k = 0;
    for (i64 sym = 1; sym <= s->nirrep && rc == O_OK; sym++) {
        const i64 l1 = o_irpdso(sym, V, o, 1), l2 = o_idsymsoc(sym, V, V, 0, o, o, 0), n = l1 + l2;
        double *oed1 = zalloc(l1), *demw = zalloc(l2), *c = zalloc(n);
        o_eorb_diff1(oed1, I->eorb, V, o, sym);
        for (i64 r = 0; r < p->estate_sym[sym - 1] && rc == O_OK; r++, k++, off += n) {
            const double wv = omega[k];
            double *R = Rall + off, *L = Lall + off;
            double nrm = o_dnrm2(n, R);
            if (fabs(nrm - 1.0) > p->diis_max_err) /* dscal by 1/norm */
                for (i64 q = 0; q < n; q++) R[q] *= 1.0 / nrm;
            o_eorb_diff2(demw, I->eorb, V, o, sym, 0);
            for (i64 q = 0; q < l2; q++) demw[q] = 1.0 / (wv - demw[q]);
            o_opt L1, L2, C1, R1, R2;
            o_opt_view(&L1, V, o, Z, Z, 1, 1, sym, L);
            o_opt_view(&L2, V, V, o, o, 0, 0, sym, L + l1);
            o_opt_view(&C1, V, o, Z, Z, 1, 1, sym, c);
            o_opt_view(&R1, V, o, Z, Z, 1, 1, sym, R);
            o_opt_view(&R2, V, V, o, o, 0, 0, sym, R + l1);
            memcpy(L, R, sizeof(double) * (size_t)l1);
            o_diis dst;
            o_diis_init(&dst, l1, p->diis_dim);
            i64 iter = 0;
            for (;;) { /* calEigenCISDoo.f90:94-140 */
                iter++;
                double d = 1.0 / o_ddot(l1, L, R);
                for (i64 q = 0; q < l1; q++) L[q] *= d;
                double err = o_diis_step(&dst, iter, L);
                d = 1.0 / o_ddot(l1, L, R);
                for (i64 q = 0; q < l1; q++) L[q] *= d;
                if (fabs(err) < p->diis_max_err && iter > 1) break;
                if (iter > p->diis_cyc) break;
                for (i64 q = 0; q < l1; q++) c[q] = -wv * L[q];
                rc = o_c1d_l1Wibaj(&C1, &L1, &g.wk, 1.0);
                if (rc == O_OK) rc = o_c1d_l1fab(&C1, &L1, &g.fad, 1.0);
                if (rc == O_OK) rc = o_c1d_l1fij(&C1, &L1, &g.fli, 1.0);
                memset(L + l1, 0, sizeof(double) * (size_t)l2);
                if (rc == O_OK) rc = o_c2_r1ijka(&L2, &L1, &v.ijka, 1.0); /* calL2d_VL1 */
                if (rc == O_OK) rc = o_c2_r1abci(&L2, &L1, &v.abci, 1.0);
                for (i64 q = 0; q < l2; q++) L[l1 + q] *= demw[q];
                if (rc == O_OK) rc = o_c1_r2ijka(&C1, &L2, &v.ijka, 1.0); /* calL1d_VL2 */
                if (rc == O_OK) rc = o_c1_r2abci(&C1, &L2, &v.abci, 1.0);
                if (rc != O_OK) break;
                o_denomT1(L, c, I->eorb, V, o, sym);
            }
            o_diis_free(&dst);
            itsum += iter;
            if (rc != O_OK) break;
            /* L2 = L1 Asd (w - Add)^-1, L /= 1 + <L2|R2> (calEigenCISDoo.f90:142-157) */
            memset(L + l1, 0, sizeof(double) * (size_t)l2);
            rc = o_c2_r1ijka(&L2, &L1, &v.ijka, 1.0);
            if (rc == O_OK) rc = o_c2_r1abci(&L2, &L1, &v.abci, 1.0);
            for (i64 q = 0; q < l2; q++) L[l1 + q] *= demw[q];
            double nl = 1.0 / (1.0 + o_ddot(l2, L + l1, R + l1));
            for (i64 q = 0; q < n; q++) L[q] *= nl;
            /* w^(1) = L J^(1) R^(0) (calEigenCISDoo.f90:170-186) */
            double *Rk[3] = {R, NULL, NULL};
            if (rc == O_OK) rc = ee_calE_C(&g, NULL, NULL, T, lt, Call + off, Rk, sym, l1, 1);
            w[3 * k] = o_ddot(n, L, Call + off);
        }
        free(oed1); free(demw); free(c);
    }
    ee_J J2, J3;
    ee_J_alloc(s, &J2);
    ee_J_alloc(s, &J3);
    if (rc == O_OK) { /* calJ2 / calJ3 (run.f90:72-73) */
        o_opt t1, t2;
        o_opt_view(&t1, V, o, Z, Z, 1, 1, 1, (double *)T + lt);
        o_opt_view(&t2, V, V, o, o, 0, 0, 1, (double *)T + lt + g1);
        rc = ee_J_VT(&v, &J3, &t1, &t2);
        o_opt_view(&t1, V, o, Z, Z, 1, 1, 1, (double *)T);
        o_opt_view(&t2, V, V, o, o, 0, 0, 1, (double *)T + g1);
        if (rc == O_OK) rc = ee_J_VT(&v, &J2, &t1, &t2);
        if (rc == O_OK) rc = ee_J_VTT(s, &v, &J3, &t1, &t2);
    }
    /* run1 / run2 per root (run.f90:75-82) */
    off = 0;
    k = 0;
    for (i64 sym = 1; sym <= s->nirrep && rc == O_OK; sym++) {
        const i64 l1 = o_irpdso(sym, V, o, 1), l2 = o_idsymsoc(sym, V, V, 0, o, o, 0), n = l1 + l2;
        double *C = zalloc(n), *pr = zalloc(n);
        o_opt r1, r2, p1, p2;
        for (i64 r = 0; r < p->estate_sym[sym - 1] && rc == O_OK; r++, k++, off += n) {
            const double w0 = omega[k];
            double *L = Lall + off;
            double *Rk[3] = {Rall + off, Rall + rlen + off, Rall + 2 * rlen + off};
            for (int order = 1; order <= 2 && rc == O_OK; order++) {
                /* calV_C: Ctilde = -C^(n) + sum_k w^(k) R^(n-k); solver.f90 negates it */
                for (i64 q = 0; q < n; q++) C[q] = -Call[off + q];
                for (int kk = 1; kk <= order; kk++) o_daxpy(n, w[3 * k + kk - 1], Rk[order - kk], C);
                for (i64 q = 0; q < n; q++) C[q] = -C[q];
                double *Rn = Rk[order];
                o_opt_view(&r1, V, o, Z, Z, 1, 1, sym, Rn);
                o_opt_view(&r2, V, V, o, o, 0, 0, sym, Rn + l1);
                o_opt_view(&p1, V, o, Z, Z, 1, 1, sym, pr);
                o_opt_view(&p2, V, V, o, o, 0, 0, sym, pr + l1);
                memcpy(pr, C, sizeof(double) * (size_t)n);
                o_diis dst;
                o_diis_init(&dst, n, p->diis_dim);
                i64 iter = 0;
                for (;;) { /* solver.f90:31-77 */
                    iter++;
                    o_denomT1(Rn, pr, I->eorb, V, o, sym);
                    o_denomT2(Rn + l1, pr + l1, I->eorb, V, o, sym, 0);
                    ee_orth(Rn, L, n);
                    double err = o_diis_step(&dst, iter, Rn);
                    ee_orth(Rn, L, n);
                    if (iter > 1 && fabs(err) < p->diis_max_err) break;
                    if (iter > p->diis_cyc) break;
                    memcpy(pr, C, sizeof(double) * (size_t)n);
                    o_daxpy(n, -w0, Rn, pr);
                    rc = o_c1_r1iabj(&p1, &r1, &g.wk, 1.0); /* calA0R1 */
                    if (rc == O_OK) rc = o_c1_r1Fmi(&p1, &r1, &g.fli, -1.0);
                    if (rc == O_OK) rc = o_c1_r1Fae(&p1, &r1, &g.fad, -1.0);
                    if (rc == O_OK) rc = o_c1_r2ijka(&p1, &r2, &v.ijka, 1.0);
                    if (rc == O_OK) rc = o_c1_r2abci(&p1, &r2, &v.abci, 1.0);
                    if (rc == O_OK) rc = o_c2_r1ijka(&p2, &r1, &v.ijka, 1.0); /* calA0R2 */
                    if (rc == O_OK) rc = o_c2_r1abci(&p2, &r1, &v.abci, 1.0);
                    if (rc != O_OK) break;
                }
                o_diis_free(&dst);
                itsum += iter;
                if (rc != O_OK) break;
                rc = ee_calE_C(&g, &J2, &J3, T, lt, Call + off, Rk, sym, l1, order + 1);
                w[3 * k + order] = o_ddot(n, L, Call + off);
            }
        }
        free(C); free(pr);
    }
    if (rc == O_OK && Lout) memcpy(Lout, Lall, sizeof(double) * (size_t)rlen);
    if (rc == O_OK && Rout) memcpy(Rout, Rall + rlen, sizeof(double) * (size_t)(2 * rlen));
    if (iters) *iters = itsum;
    ee_J_free(&J2);
    ee_J_free(&J3);
    free(Rall); free(Lall); free(Call);
    free(mp2); free(fo); free(fv); free(wk);
    return rc;
}

/* ---------------- J^(2), J^(3) (src/EE-CPSd.SF/calJ.f90) ---------------- */
int o_calJ(const o_system *s, const o_integrals *I, const double *T2_1,
           const double *T1_2, const double *T2_2, o_jints *J)
{
    ints_t v;
    ints_view(s, I, &v);
    const i64 *o = s->popo, *V = s->popv;
    o_opt t2a, t1b, t2b, foo, fvv, wvo, woo, foo3, fvv3, wvo3;
    o_opt_view(&t2a, V, V, o, o, 0, 0, 1, (double *)T2_1);
    o_opt_view(&t1b, V, o, Z, Z, 1, 1, 1, (double *)T1_2);
    o_opt_view(&t2b, V, V, o, o, 0, 0, 1, (double *)T2_2);
    o_opt_view(&foo, o, o, Z, Z, 1, 1, 1, J->J2_Foo);
    o_opt_view(&fvv, V, V, Z, Z, 1, 1, 1, J->J2_Fvv);
    o_opt_view(&wvo, V, o, V, o, 1, 1, 1, J->J2_Wovvo);
    o_opt_view(&woo, o, o, o, V, 0, 1, 1, J->J2_Wovoo);
    o_opt_view(&foo3, o, o, Z, Z, 1, 1, 1, J->J3_Foo);
    o_opt_view(&fvv3, V, V, Z, Z, 1, 1, 1, J->J3_Fvv);
    o_opt_view(&wvo3, V, o, V, o, 1, 1, 1, J->J3_Wovvo);
    memset(foo.arr, 0, sizeof(double) * (size_t)foo.len);
    memset(fvv.arr, 0, sizeof(double) * (size_t)fvv.len);
    memset(wvo.arr, 0, sizeof(double) * (size_t)wvo.len);
    memset(woo.arr, 0, sizeof(double) * (size_t)woo.len);
    memset(foo3.arr, 0, sizeof(double) * (size_t)foo3.len);
    memset(fvv3.arr, 0, sizeof(double) * (size_t)fvv3.len);
    memset(wvo3.arr, 0, sizeof(double) * (size_t)wvo3.len);
    int rc = O_OK;
    /* calJ2 (calJ.f90:6-99) */
    if (rc == O_OK) rc = o_Fmi_r2abij(&foo, &t2a, &v.abij, 1.0);
    if (rc == O_OK) rc = o_Fae_r2abij(&fvv, &t2a, &v.abij, 1.0);
    if (rc == O_OK) rc = o_Wkbij_r2ijka(&woo, &t2a, &v.ijka, 1.0);
    if (rc == O_OK) rc = o_Wkbij_r2abci(&woo, &t2a, &v.abci, 1.0);
    if (rc == O_OK) rc = o_Wmbej_r2abij(&wvo, &t2a, &v.abij, 2.0);
    /* calJ3 (calJ.f90:104-228) */
    if (rc == O_OK) rc = o_Fmi_r1ijka(&foo3, &t1b, &v.ijka, 1.0);
    if (rc == O_OK) rc = o_Fmi_r2abij(&foo3, &t2b, &v.abij, 1.0);
    if (rc == O_OK) rc = o_Fae_r1abci(&fvv3, &t1b, &v.abci, 1.0);
    if (rc == O_OK) rc = o_Fae_r2abij(&fvv3, &t2b, &v.abij, 1.0);
    if (rc == O_OK) rc = o_Wmbej_r1ijka(&wvo3, &t1b, &v.ijka, 1.0);
    if (rc == O_OK) rc = o_Wmbej_r1abci(&wvo3, &t1b, &v.abci, 1.0);
    if (rc == O_OK) rc = o_Wmbej_r2abij(&wvo3, &t2b, &v.abij, 2.0);
    return rc;
}

/* orthogonalR2L (src/EE-CPSd.SF/orthogonalR2L.f90:5-34): note the division
 * by ||L|| (not ||L||^2), as in the reference */
static void orth_r2l(double *R, const double *L, i64 n)
{
    double nrm = o_dnrm2(n, L);
    double dot = o_ddot(n, L, R);
    o_daxpy(n, -dot / nrm, L, R);
}

/* ---------------- one EE-CPS(D-3) root ---------------- */
int o_eecpsd_root(const o_system *s, const o_integrals *I, const o_params *p,
                  const double *T2_1, const o_jints *J, i64 symR, double w0,
                  const double *L, double *w, double *R2_1_out, double *R1_2_out,
                  double *R2_2_out, i64 *solver_iters)
{
    ints_t v;
    ints_view(s, I, &v);
    const i64 *o = s->popo, *V = s->popv;
    i64 l1 = o_irpdso(symR, V, o, 1);
    i64 l2 = o_idsymsoc(symR, V, V, 0, o, o, 0);
    double *R0_1 = zalloc(l1);
    double *Rn_1[3], *Rn_2[3], *Cn_1 = zalloc(l1), *Cn_2 = zalloc(l2);
    double *C1a = zalloc(l1), *C2a = zalloc(l2), *tmpa;
    for (int k = 0; k < 3; k++) { Rn_1[k] = zalloc(l1); Rn_2[k] = zalloc(l2); }
    double *oed2 = zalloc(l2);
    o_eorb_diff2(oed2, I->eorb, V, o, symR, 0);
    memcpy(Rn_1[0], L, sizeof(double) * (size_t)l1);
    double wk[4] = {0, 0, 0, 0}; /* w^(1..3) at [1..3] */
    o_opt C1, C2, pR1, pR2, T2, jfoo, jfvv, jwvo, jwoo, j3foo, j3fvv, j3wvo;
    o_opt_view(&C1, V, o, Z, Z, 1, 1, symR, C1a);
    o_opt_view(&C2, V, V, o, o, 0, 0, symR, C2a);
    o_opt_view(&T2, V, V, o, o, 0, 0, 1, (double *)T2_1);
    o_opt_view(&jfoo, o, o, Z, Z, 1, 1, 1, J->J2_Foo);
    o_opt_view(&jfvv, V, V, Z, Z, 1, 1, 1, J->J2_Fvv);
    o_opt_view(&jwvo, V, o, V, o, 1, 1, 1, J->J2_Wovvo);
    o_opt_view(&jwoo, o, o, o, V, 0, 1, 1, J->J2_Wovoo);
    o_opt_view(&j3foo, o, o, Z, Z, 1, 1, 1, J->J3_Foo);
    o_opt_view(&j3fvv, V, V, Z, Z, 1, 1, 1, J->J3_Fvv);
    o_opt_view(&j3wvo, V, o, V, o, 1, 1, 1, J->J3_Wovvo);
    int rc = O_OK;
    i64 sit = 0;
    for (i64 order = 1; order <= 3 && rc == O_OK; order++) {
        if (order != 1) {
            /* calV_C (calV_C.f90): Ctilde^(n-1) = sum_k w^(k) R^(n-1-k) - C^(n-1) */
            i64 m = order - 1;
            for (i64 i = 0; i < l1; i++) C1a[i] = -Cn_1[i];
            for (i64 i = 0; i < l2; i++) C2a[i] = -Cn_2[i];
            for (i64 k = 2; k <= m; k++) {
                o_daxpy(l1, wk[k], Rn_1[m - k], C1a);
                o_daxpy(l2, wk[k], Rn_2[m - k], C2a);
            }
            /* R2 = C2/(e2 - w0) (run_order.f90:54-58) */
            double *R1 = Rn_1[m], *R2 = Rn_2[m];
            for (i64 i = 0; i < l2; i++) R2[i] = C2a[i] / (oed2[i] - w0);
            if (order != 2) {
                /* solver (solver.f90:4-66) */
                double *pR = zalloc(l1);
                o_opt oR1, opR;
                o_opt_view(&oR1, V, o, Z, Z, 1, 1, symR, R1);
                o_opt_view(&opR, V, o, Z, Z, 1, 1, symR, pR);
                for (i64 i = 0; i < l1; i++) C1a[i] = -C1a[i];
                memcpy(pR, C1a, sizeof(double) * (size_t)l1);
                o_diis dst;
                o_diis_init(&dst, l1, p->diis_dim);
                i64 iter = 0;
                for (;;) {
                    iter++;
                    o_denomT1(R1, pR, I->eorb, V, o, symR);
                    orth_r2l(R1, L, l1);
                    double err = o_diis_step(&dst, iter, R1);
                    orth_r2l(R1, L, l1);
                    if (iter > 1 && fabs(err) < p->diis_max_err) break;
                    if (iter > p->diis_cyc) break;
                    memcpy(pR, C1a, sizeof(double) * (size_t)l1);
                    o_daxpy(l1, -w0, R1, pR);
                    rc = o_c1_r1iabj(&opR, &oR1, &v.iabj, 1.0);
                    if (rc != O_OK) break;
                }
                sit += iter;
                o_diis_free(&dst);
                free(pR);
            } else {
                memset(R1, 0, sizeof(double) * (size_t)l1);
            }
        }
        if (rc != O_OK) break;
        /* calE_C (calE_C.f90:3-83): C^(n) = sum_k J^(k) R^(n-k) */
        memset(C1a, 0, sizeof(double) * (size_t)l1);
        memset(C2a, 0, sizeof(double) * (size_t)l2);
        o_opt_view(&pR1, V, o, Z, Z, 1, 1, symR, Rn_1[order - 1]);
        o_opt_view(&pR2, V, V, o, o, 0, 0, symR, Rn_2[order - 1]);
        if (order != 1) rc = o_c1_r2abci(&C1, &pR2, &v.abci, 1.0);   /* calC1_VR2 */
        if (rc == O_OK && order != 1) rc = o_c1_r2ijka(&C1, &pR2, &v.ijka, 1.0);
        if (rc == O_OK && order != 3) {
            if (order != 2) { /* calC2_VR1 */
                rc = o_c2_r1ijka(&C2, &pR1, &v.ijka, 1.0);
                if (rc == O_OK) rc = o_c2_r1abci(&C2, &pR1, &v.abci, 1.0);
            }
            if (rc == O_OK && order != 1) { /* calC2_VR2 */
                rc = o_c2_r2Wmbej(&C2, &pR2, &v.iabj, 1.0);
                if (rc == O_OK) rc = o_c2_r2Wmnij(&C2, &pR2, &v.ijkl, 1.0);
                if (rc == O_OK) rc = o_c2_r2abcd(&C2, &pR2, &v.abcd, 1.0);
            }
        }
        if (rc == O_OK && order == 2) {
            /* calC_J2R (calC_JR.f90:4-52) with R^(0) */
            o_opt_view(&pR1, V, o, Z, Z, 1, 1, symR, Rn_1[0]);
            rc = o_c2_r1ijka(&C2, &pR1, &jwoo, 1.0);
            if (rc == O_OK) rc = o_c1_r1iabj(&C1, &pR1, &jwvo, 1.0);
            if (rc == O_OK) rc = o_c1_r1Fmi(&C1, &pR1, &jfoo, 1.0);
            if (rc == O_OK) rc = o_c1_r1Fae(&C1, &pR1, &jfvv, 1.0);
            /* calC_VTR (calC_VTR.f90:6-111) with T^(1) = (0, T2^(1)) */
            o_opt tmp;
            if (rc == O_OK) {
                tmpa = zalloc(o_idsymsoc(symR, o, o, 0, o, o, 0));
                o_opt_view(&tmp, o, o, o, o, 0, 0, symR, tmpa);
                rc = o_Wmnij_r1ijka(&tmp, &pR1, &v.ijka, 1.0);
                if (rc == O_OK) rc = o_c2_r2Wmnij(&C2, &T2, &tmp, 1.0);
                free(tmpa);
            }
            if (rc == O_OK) {
                tmpa = zalloc(o_idsymsoc(symR, V, o, 1, V, o, 1));
                o_opt_view(&tmp, V, o, V, o, 1, 1, symR, tmpa);
                rc = o_Wmbej_r1abci(&tmp, &pR1, &v.abci, 1.0);
                if (rc == O_OK) rc = o_c2_r2Wmbej(&C2, &T2, &tmp, 1.0);
                free(tmpa);
            }
            if (rc == O_OK) {
                tmpa = zalloc(o_irpdso(symR, o, o, 1));
                o_opt_view(&tmp, o, o, Z, Z, 1, 1, symR, tmpa);
                rc = o_Fmi_r1ijka(&tmp, &pR1, &v.ijka, 1.0);
                if (rc == O_OK) rc = o_c2_r2Fmi(&C2, &T2, &tmp, 1.0);
                free(tmpa);
            }
            if (rc == O_OK) {
                tmpa = zalloc(o_irpdso(symR, V, V, 1));
                o_opt_view(&tmp, V, V, Z, Z, 1, 1, symR, tmpa);
                rc = o_Fae_r1abci(&tmp, &pR1, &v.abci, 1.0);
                if (rc == O_OK) rc = o_c2_r2Fae(&C2, &T2, &tmp, 1.0);
                free(tmpa);
            }
        }
        if (rc == O_OK && order == 3) {
            /* calC_J3R (calC_JR.f90:56-106) with R^(0) */
            o_opt_view(&pR1, V, o, Z, Z, 1, 1, symR, Rn_1[0]);
            rc = o_c1_r1iabj(&C1, &pR1, &j3wvo, 1.0);
            if (rc == O_OK) rc = o_c1_r1Fmi(&C1, &pR1, &j3foo, 1.0);
            if (rc == O_OK) rc = o_c1_r1Fae(&C1, &pR1, &j3fvv, 1.0);
        }
        if (rc != O_OK) break;
        wk[order] = o_ddot(l1, L, C1a);
        memcpy(Cn_1, C1a, sizeof(double) * (size_t)l1);
        memcpy(Cn_2, C2a, sizeof(double) * (size_t)l2);
    }
    w[0] = wk[1]; w[1] = wk[2]; w[2] = wk[3];
    if (R2_1_out) memcpy(R2_1_out, Rn_2[1], sizeof(double) * (size_t)l2);
    if (R1_2_out) memcpy(R1_2_out, Rn_1[2], sizeof(double) * (size_t)l1);
    if (R2_2_out) memcpy(R2_2_out, Rn_2[2], sizeof(double) * (size_t)l2);
    if (solver_iters) *solver_iters = sit;
    for (int k = 0; k < 3; k++) { free(Rn_1[k]); free(Rn_2[k]); }
    free(R0_1); free(Cn_1); free(Cn_2); free(C1a); free(C2a); free(oed2);
    return rc;
}

/* ---------------- the whole pipeline (one "step" of the metric) --------- */
int o_sfcpsd_pipeline(const o_system *s, const o_integrals *I, const o_params *p,
                      double *omega_cis, double *w2, double *w3, i64 *nroots_out)
{
    const i64 *o = s->popo, *V = s->popv;
    i64 nroot = 0, rlen = 0;
    for (i64 sym = 1; sym <= s->nirrep; sym++) {
        nroot += p->estate_sym[sym - 1];
        rlen += p->estate_sym[sym - 1] * o_irpdso(sym, V, o, 1);
    }
    double *R = zalloc(rlen);
    int rc = o_cis_run(s, I, p, omega_cis, R, NULL);
    i64 l1 = o_irpdso(1, V, o, 1), l2 = o_idsymsoc(1, V, V, 0, o, o, 0);
    double *T2_1 = zalloc(l2), *T1_2 = zalloc(l1), *T2_2 = zalloc(l2);
    double E2, E3;
    if (rc == O_OK) rc = o_cpsd_ground(s, I, p, T2_1, T1_2, T2_2, &E2, &E3, NULL);
    o_jints J;
    J.J2_Foo = zalloc(o_irpdso(1, o, o, 1));
    J.J2_Fvv = zalloc(o_irpdso(1, V, V, 1));
    J.J2_Wovvo = zalloc(o_idsymsoc(1, V, o, 1, V, o, 1));
    J.J2_Wovoo = zalloc(o_idsymsoc(1, o, o, 0, o, V, 1));
    J.J3_Foo = zalloc(o_irpdso(1, o, o, 1));
    J.J3_Fvv = zalloc(o_irpdso(1, V, V, 1));
    J.J3_Wovvo = zalloc(o_idsymsoc(1, V, o, 1, V, o, 1));
    if (rc == O_OK) rc = o_calJ(s, I, T2_1, T1_2, T2_2, &J);
    i64 k = 0, roff = 0;
    for (i64 sym = 1; sym <= s->nirrep && rc == O_OK; sym++) {
        i64 len = o_irpdso(sym, V, o, 1);
        for (i64 r = 0; r < p->estate_sym[sym - 1] && rc == O_OK; r++) {
            double w[3];
            rc = o_eecpsd_root(s, I, p, T2_1, &J, sym, omega_cis[k], R + roff + r * len, w,
                               NULL, NULL, NULL, NULL);
            w2[k] = w[1];
            w3[k] = w[2];
            k++;
        }
        roff += len * p->estate_sym[sym - 1];
    }
    if (nroots_out) *nroots_out = nroot;
    free(R); free(T2_1); free(T1_2); free(T2_2);
    free(J.J2_Foo); free(J.J2_Fvv); free(J.J2_Wovvo); free(J.J2_Wovoo);
    free(J.J3_Foo); free(J.J3_Fvv); free(J.J3_Wovvo);
    return rc;
}
