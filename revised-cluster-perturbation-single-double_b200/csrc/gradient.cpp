// SF-CIS(D) excitation energies of one irrep and their gradient with respect
// to the spin-free DPD integrals and the orbital energies.
//
// Per root: the SF-CIS energy w0 with unit vector L (src/EE-CIS.SF/run.f90,
// Davidson of src/lib_cc/mod_davidson.f90) and the second-order correction
// w^(2) of the EE-CPS(D-3) chain (src/EE-CPSd.SF/run_order.f90, order 2):
//   T2   = <ab||ij> / (ei+ej-ea-eb)                        run1.f90:20-36
//   Foo  = Fmi_r2abij(T2), Fvv = Fae_r2abij(T2),
//   Wvo  = 2 Wmbej_r2abij(T2)                               calJ.f90:6-99
//   C2   = c2_r1ijka(L) + c2_r1abci(L)                     calE_C.f90 order 1
//   R2   = -C2 / (e(ab,ij) - w0)                           run_order.f90:54-58
//   C1   = c1_r2abci(R2) + c1_r2ijka(R2)                   calC1_VR2
//        + c1_r1iabj(L, Wvo) + c1_r1Fmi(L, Foo) + c1_r1Fae(L, Fvv)   calC_J2R
//   w2   = L . C1                                          run_order.f90:89
// The reference has no derivative code.  The gradient of sum_k (g0_k w0_k +
// g2_k w2_k) is reverse mode through these steps: every contraction by the
// adjoint contractions vjp_* (ops.cpp), the denominators by their
// derivatives, and the response of the CIS vector by the Z-vector equation
// (A - w0) z = P Lbar, L.z = 0 (P = 1 - L L^T), solved by the device solver
// of solver.f90.  For a unit right eigenvector L of A = e(a,i) + V(fn,ai)
// that is symmetric at the expansion point, dw0 = L^T dA L and
// Lbar.dL = -z^T dA L, so A's integrals and energies receive the outer
// product (w0bar L - z) L^T.  The doubles amplitudes T2 and R2 are
// recomputed from the singles, not stored by the forward call.
//
// The third-order correction w^(3) of the same chain (run_order.f90 order 3,
// calE_C.f90, calC_JR.f90, calC_VTR.f90) adds, per root,
//   C2^(2) = calC2_VR2(R2) + c2_r1ijka(L, J2_Wovoo)
//          + c2_r2Wmnij(T2, Wmnij_r1ijka(L)) + c2_r2Wmbej(T2, Wmbej_r1abci(L))
//          + c2_r2Fmi(T2, Fmi_r1ijka(L)) + c2_r2Fae(T2, Fae_r1abci(L))
//   R2^(2) = -C2^(2) / (e(ab,ij) - w0)
//   C1^(3) = c1_r2abci(R2^(2)) + c1_r2ijka(R2^(2)) + c1_r1iabj(L, J3_Wovvo)
//          + c1_r1Fmi(L, J3_Foo) + c1_r1Fae(L, J3_Fvv);   w3 = L . C1^(3)
// with the ground state's second order (run2.f90): T2^(2) = calC2_VR2(T2) /
// D and T1^(2) from (ei - ea) T1 = calC1_VR2(T2) + V(fn,ai) T1 (its DIIS
// solve; reversed by one solve of the same operator, symmetric at the
// expansion point), and J^(3) of T1^(2), T2^(2) (calJ.f90:104-228).  R1^(2)
// of the order-3 solver does not enter w^(3) (C1^(3) has no J^(1) R1^(2)
// term), so its solve is not reversed.
#include <algorithm>
#include <vector>

#include "drivers.hpp"

namespace cpsd {

namespace {

// contractions of the gradient always run in FP64
struct Fp64Only {
    int saved;
    Fp64Only() : saved(ctx().oz_digits) { ctx().oz_digits = 0; }
    ~Fp64Only() { ctx().oz_digits = saved; }
};

i64 occupied(const Sys &S) {
    i64 n = 0;
    for (int r = 0; r < 8; r++) n += S.popo[r];
    return n;
}

// T2^(1) (run1.f90) and the J^(2) intermediates on the w^(2) path (calJ.f90)
struct Ground {
    double *t2, *foo, *fvv, *wvo;
    Ten T2, Foo, Fvv, Wvo;
};

int ground_j2(const Sys &S, const Ints &X, Ground *g) {
    const i64 *o = S.popo, *v = S.popv;
    g->T2 = ten(v, v, o, o, 0, 0, 1, nullptr);
    g->Foo = ten(o, o, ZORB, ZORB, 1, 1, 1, nullptr);
    g->Fvv = ten(v, v, ZORB, ZORB, 1, 1, 1, nullptr);
    g->Wvo = ten(v, o, v, o, 1, 1, 1, nullptr);
    for (Ten *t : {&g->T2, &g->Foo, &g->Fvv, &g->Wvo}) {
        CPSD_TRY(scratch(t->len(), &t->arr));
        CPSD_TRY(launch_scale(t->arr, t->len(), 0.0));
    }
    g->t2 = g->T2.arr;
    g->foo = g->Foo.arr;
    g->fvv = g->Fvv.arr;
    g->wvo = g->Wvo.arr;
    const EnergyPlan *e2;
    CPSD_TRY(plan_energy(make_desc(v, v, o, o, 0, 0, 1), "vvoo", &e2));
    CPSD_TRY(launch_energy(e2, 2, X.eorb, X.abij.arr, g->t2));
    CPSD_TRY(k_Fmi_r2abij(g->Foo, g->T2, X.abij, 1.0));
    CPSD_TRY(k_Fae_r2abij(g->Fvv, g->T2, X.abij, 1.0));
    CPSD_TRY(k_Wmbej_r2abij(g->Wvo, g->T2, X.abij, 2.0));
    return CPSD_OK;
}

// w^(2) of nb roots (L: nb x l1, w0d their CIS energies on the device):
// C2, R2 (nb x l2), C1 (nb x l1) and w2d (nb) on the device
int w2_forward(const Sys &S, const Ints &X, const Ground &g, i64 symR, i64 nb, const double *L, const double *w0d,
               double *c2, double *r2, double *c1, double *w2d) {
    const i64 *o = S.popo, *v = S.popv;
    const i64 l1 = irpdso(symR, v, o, 1), l2 = idsymsoc(symR, v, v, 0, o, o, 0);
    Ten Lt = ten(v, o, ZORB, ZORB, 1, 1, symR, (double *)L, l1);
    Ten C1 = ten(v, o, ZORB, ZORB, 1, 1, symR, c1, l1), C2 = ten(v, v, o, o, 0, 0, symR, c2, l2);
    Ten R2 = ten(v, v, o, o, 0, 0, symR, r2, l2);
    const EnergyPlan *e2;
    CPSD_TRY(plan_energy(make_desc(v, v, o, o, 0, 0, symR), "vvoo", &e2));
    CPSD_TRY(launch_scale(c2, nb * l2, 0.0));
    CPSD_TRY(k_c2_r1ijka(C2, Lt, X.ijka, 1.0, nb));
    CPSD_TRY(k_c2_r1abci(C2, Lt, X.abci, 1.0, nb));
    CPSD_TRY(launch_copy(r2, c2, nb * l2));
    CPSD_TRY(launch_scale(r2, nb * l2, -1.0));
    CPSD_TRY(launch_energy(e2, 1, X.eorb, r2, r2, w0d, nb, l2, l2));
    CPSD_TRY(launch_scale(c1, nb * l1, 0.0));
    CPSD_TRY(k_c1_r2abci(C1, R2, X.abci, 1.0, nb));
    CPSD_TRY(k_c1_r2ijka(C1, R2, X.ijka, 1.0, nb));
    CPSD_TRY(k_c1_r1iabj(C1, Lt, g.Wvo, 1.0, nb));
    CPSD_TRY(k_c1_r1Fmi(C1, Lt, g.Foo, 1.0, nb));
    CPSD_TRY(k_c1_r1Fae(C1, Lt, g.Fvv, 1.0, nb));
    for (i64 r = 0; r < nb; r++) CPSD_TRY(launch_dot(L + r * l1, c1 + r * l1, l1, w2d + r, true));
    return CPSD_OK;
}

int upload(double *dev, const double *host, i64 n) {
    return cuda_check(cudaMemcpyAsync(dev, host, sizeof(double) * n, cudaMemcpyHostToDevice, stream()), "upload");
}

// t's layout in zeroed scratch, nb copies stacked
int fresh(Ten *t, i64 nb = 1) {
    CPSD_TRY(scratch(nb * t->len(), &t->arr));
    t->bs = nb > 1 ? t->len() : 0;
    return launch_scale(t->arr, nb * t->len(), 0.0);
}

// the ground state beyond T2^(1) on the w^(3) path: J2_Wovoo (calJ.f90:6-99),
// T2^(2) and T1^(2) (run2.f90:8-95), J^(3) (calJ.f90:104-228)
struct Ground3 {
    Ten Woo, T1b, T2b, Foo3, Fvv3, Wvo3;
};

int ground3(const Sys &S, const Ints &X, const cpsd_params *p, const Ground &g, Ground3 *h) {
    const i64 *o = S.popo, *v = S.popv;
    h->Woo = ten(o, o, o, v, 0, 1, 1, nullptr);
    h->T1b = ten(v, o, ZORB, ZORB, 1, 1, 1, nullptr);
    h->T2b = ten(v, v, o, o, 0, 0, 1, nullptr);
    h->Foo3 = ten(o, o, ZORB, ZORB, 1, 1, 1, nullptr);
    h->Fvv3 = ten(v, v, ZORB, ZORB, 1, 1, 1, nullptr);
    h->Wvo3 = ten(v, o, v, o, 1, 1, 1, nullptr);
    for (Ten *t : {&h->Woo, &h->T1b, &h->T2b, &h->Foo3, &h->Fvv3, &h->Wvo3}) CPSD_TRY(fresh(t));
    CPSD_TRY(k_Wkbij_r2ijka(h->Woo, g.T2, X.ijka, 1.0));
    CPSD_TRY(k_Wkbij_r2abci(h->Woo, g.T2, X.abci, 1.0));
    Ten C1 = h->T1b, C2 = h->T2b;
    CPSD_TRY(fresh(&C1));
    CPSD_TRY(fresh(&C2));
    CPSD_TRY(k_c1_r2abci(C1, g.T2, X.abci, 1.0));
    CPSD_TRY(k_c1_r2ijka(C1, g.T2, X.ijka, 1.0));
    CPSD_TRY(k_c2_r2Wmbej(C2, g.T2, X.iabj, 1.0));
    CPSD_TRY(k_c2_r2Wmnij(C2, g.T2, X.ijkl, 1.0));
    CPSD_TRY(k_c2_r2abcd(C2, g.T2, X.abcd, 1.0));
    const EnergyPlan *e2g, *e1g;
    CPSD_TRY(plan_energy(make_desc(v, v, o, o, 0, 0, 1), "vvoo", &e2g));
    CPSD_TRY(plan_energy(make_desc(v, o, ZORB, ZORB, 1, 1, 1), "vozz", &e1g));
    CPSD_TRY(launch_energy(e2g, 2, X.eorb, C2.arr, h->T2b.arr));
    i64 it = 0;
    CPSD_TRY(solve_r1(S, X, p, 1, 1, C1.len(), e1g, C1.arr, nullptr, nullptr, h->T1b.arr, &it));
    CPSD_TRY(k_Fmi_r1ijka(h->Foo3, h->T1b, X.ijka, 1.0));
    CPSD_TRY(k_Fmi_r2abij(h->Foo3, h->T2b, X.abij, 1.0));
    CPSD_TRY(k_Fae_r1abci(h->Fvv3, h->T1b, X.abci, 1.0));
    CPSD_TRY(k_Fae_r2abij(h->Fvv3, h->T2b, X.abij, 1.0));
    CPSD_TRY(k_Wmbej_r1ijka(h->Wvo3, h->T1b, X.ijka, 1.0));
    CPSD_TRY(k_Wmbej_r1abci(h->Wvo3, h->T1b, X.abci, 1.0));
    return k_Wmbej_r2abij(h->Wvo3, h->T2b, X.abij, 2.0);
}

// the one-index intermediates of calC_VTR (calC_VTR.f90:6-111) for nb roots
struct VtrTemps {
    Ten mn, mb, fo, fv;
};

int vtr_layouts(const Sys &S, i64 symR, i64 nb, VtrTemps *t) {
    const i64 *o = S.popo, *v = S.popv;
    t->mn = ten(o, o, o, o, 0, 0, symR, nullptr);
    t->mb = ten(v, o, v, o, 1, 1, symR, nullptr);
    t->fo = ten(o, o, ZORB, ZORB, 1, 1, symR, nullptr);
    t->fv = ten(v, v, ZORB, ZORB, 1, 1, symR, nullptr);
    for (Ten *x : {&t->mn, &t->mb, &t->fo, &t->fv}) CPSD_TRY(fresh(x, nb));
    return CPSD_OK;
}

int vtr_temps(const Sys &S, const Ints &X, i64 symR, const Ten &Lt, i64 nb, VtrTemps *t) {
    CPSD_TRY(vtr_layouts(S, symR, nb, t));
    CPSD_TRY(k_Wmnij_r1ijka(t->mn, Lt, X.ijka, 1.0, nb));
    CPSD_TRY(k_Wmbej_r1abci(t->mb, Lt, X.abci, 1.0, nb));
    CPSD_TRY(k_Fmi_r1ijka(t->fo, Lt, X.ijka, 1.0, nb));
    return k_Fae_r1abci(t->fv, Lt, X.abci, 1.0, nb);
}

// w^(3) of nb roots from R2^(1) (r21) of w2_forward: R2^(2) (r22), C1^(3)
// (c1c) and w3d on the device
int w3_forward(const Sys &S, const Ints &X, const Ground &g, const Ground3 &h, i64 symR, i64 nb, const double *L,
               const double *w0d, const double *r21, double *r22, double *c1c, double *w3d) {
    const i64 *o = S.popo, *v = S.popv;
    const i64 l1 = irpdso(symR, v, o, 1), l2 = idsymsoc(symR, v, v, 0, o, o, 0);
    Ten Lt = ten(v, o, ZORB, ZORB, 1, 1, symR, (double *)L, l1);
    Ten R21 = ten(v, v, o, o, 0, 0, symR, (double *)r21, l2);
    Ten C2 = ten(v, v, o, o, 0, 0, symR, r22, l2);
    Ten C1 = ten(v, o, ZORB, ZORB, 1, 1, symR, c1c, l1);
    CPSD_TRY(launch_scale(r22, nb * l2, 0.0));
    CPSD_TRY(k_c2_r2Wmbej(C2, R21, X.iabj, 1.0, nb));  // calC2_VR2
    CPSD_TRY(k_c2_r2Wmnij(C2, R21, X.ijkl, 1.0, nb));
    CPSD_TRY(k_c2_r2abcd(C2, R21, X.abcd, 1.0, nb));
    CPSD_TRY(k_c2_r1ijka(C2, Lt, h.Woo, 1.0, nb));  // calC_J2R
    {
        ScratchScope sc;
        VtrTemps t;
        CPSD_TRY(vtr_temps(S, X, symR, Lt, nb, &t));
        CPSD_TRY(k_c2_r2Wmnij(C2, g.T2, t.mn, 1.0, nb));
        CPSD_TRY(k_c2_r2Wmbej(C2, g.T2, t.mb, 1.0, nb));
        CPSD_TRY(k_c2_r2Fmi(C2, g.T2, t.fo, 1.0, nb));
        CPSD_TRY(k_c2_r2Fae(C2, g.T2, t.fv, 1.0, nb));
    }
    const EnergyPlan *e2;
    CPSD_TRY(plan_energy(make_desc(v, v, o, o, 0, 0, symR), "vvoo", &e2));
    CPSD_TRY(launch_scale(r22, nb * l2, -1.0));
    CPSD_TRY(launch_energy(e2, 1, X.eorb, r22, r22, w0d, nb, l2, l2));
    Ten R22 = C2;
    CPSD_TRY(launch_scale(c1c, nb * l1, 0.0));
    CPSD_TRY(k_c1_r2abci(C1, R22, X.abci, 1.0, nb));
    CPSD_TRY(k_c1_r2ijka(C1, R22, X.ijka, 1.0, nb));
    CPSD_TRY(k_c1_r1iabj(C1, Lt, h.Wvo3, 1.0, nb));  // calC_J3R
    CPSD_TRY(k_c1_r1Fmi(C1, Lt, h.Foo3, 1.0, nb));
    CPSD_TRY(k_c1_r1Fae(C1, Lt, h.Fvv3, 1.0, nb));
    for (i64 r = 0; r < nb; r++) CPSD_TRY(launch_dot(L + r * l1, c1c + r * l1, l1, w3d + r, true));
    return CPSD_OK;
}

}  // namespace
}  // namespace cpsd

using namespace cpsd;

extern "C" {

int cpsd_cisd_energies(const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p, int64_t symR,
                       int64_t nroot, double *w0_host, double *w2_host, double *L_dev) {
    Sys S;
    CPSD_TRY(make_sys(s, &S));
    if (!p || !I || !w0_host || !w2_host || !L_dev) return set_error(CPSD_EARG, "cisd_energies: null argument");
    if (symR < 1 || symR > S.nirrep || nroot <= 0) return set_error(CPSD_EARG, "cisd_energies: bad irrep or roots");
    Ints X = make_ints(S, I);
    IntegralScope keep(I);
    cpsd_params q = *p;
    for (int h = 0; h < 8; h++) q.estate_sym[h] = h == symR - 1 ? nroot : 0;
    CPSD_TRY(cpsd_cis_run(s, I, &q, w0_host, L_dev, nullptr));
    const i64 *o = S.popo, *v = S.popv;
    const i64 l1 = irpdso(symR, v, o, 1), l2 = idsymsoc(symR, v, v, 0, o, o, 0);
    ScratchScope sc;
    Ground g;
    CPSD_TRY(ground_j2(S, X, &g));
    double *c2, *r2, *c1, *w0d, *w2d;
    CPSD_TRY(scratch(nroot * l2, &c2));
    CPSD_TRY(scratch(nroot * l2, &r2));
    CPSD_TRY(scratch(nroot * l1, &c1));
    CPSD_TRY(scratch(nroot, &w0d));
    CPSD_TRY(scratch(nroot, &w2d));
    CPSD_TRY(upload(w0d, w0_host, nroot));
    CPSD_TRY(w2_forward(S, X, g, symR, nroot, L_dev, w0d, c2, r2, c1, w2d));
    return read_back(w2_host, w2d, sizeof(double) * nroot);
}

int cpsd_cpsd3_energies(const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p, int64_t symR,
                        int64_t nroot, double *w0_host, double *w2_host, double *w3_host, double *L_dev) {
    Sys S;
    CPSD_TRY(make_sys(s, &S));
    if (!p || !I || !w0_host || !w2_host || !w3_host || !L_dev)
        return set_error(CPSD_EARG, "cpsd3_energies: null argument");
    if (!I->ijkl || !I->abcd) return set_error(CPSD_EARG, "cpsd3_energies: ijkl and abcd are required");
    if (symR < 1 || symR > S.nirrep || nroot <= 0) return set_error(CPSD_EARG, "cpsd3_energies: bad irrep or roots");
    Ints X = make_ints(S, I);
    IntegralScope keep(I);
    cpsd_params q = *p;
    for (int h = 0; h < 8; h++) q.estate_sym[h] = h == symR - 1 ? nroot : 0;
    CPSD_TRY(cpsd_cis_run(s, I, &q, w0_host, L_dev, nullptr));
    const i64 *o = S.popo, *v = S.popv;
    const i64 l1 = irpdso(symR, v, o, 1), l2 = idsymsoc(symR, v, v, 0, o, o, 0);
    ScratchScope sc;
    Ground g;
    Ground3 h;
    CPSD_TRY(ground_j2(S, X, &g));
    CPSD_TRY(ground3(S, X, p, g, &h));
    double *c2, *r2, *c1, *r22, *c1c, *w0d, *wd;
    CPSD_TRY(scratch(nroot * l2, &c2));
    CPSD_TRY(scratch(nroot * l2, &r2));
    CPSD_TRY(scratch(nroot * l1, &c1));
    CPSD_TRY(scratch(nroot * l2, &r22));
    CPSD_TRY(scratch(nroot * l1, &c1c));
    CPSD_TRY(scratch(nroot, &w0d));
    CPSD_TRY(scratch(2 * nroot, &wd));
    CPSD_TRY(upload(w0d, w0_host, nroot));
    CPSD_TRY(w2_forward(S, X, g, symR, nroot, L_dev, w0d, c2, r2, c1, wd));
    CPSD_TRY(w3_forward(S, X, g, h, symR, nroot, L_dev, w0d, r2, r22, c1c, wd + nroot));
    std::vector<double> w((size_t)(2 * nroot));
    CPSD_TRY(read_back(w.data(), wd, sizeof(double) * w.size()));
    for (i64 r = 0; r < nroot; r++) {
        w2_host[r] = w[(size_t)r];
        w3_host[r] = w[(size_t)(nroot + r)];
    }
    return CPSD_OK;
}

}  // extern "C"

namespace cpsd {
namespace {

// the gradient of sum_k g0_k w0_k + g2_k w2_k (+ g3_k w3_k when g3 is given)
int gradient_impl(const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p, int64_t symR, int64_t nroot,
                  const double *w0_host, const double *L_dev, const double *g0_host, const double *g2_host,
                  const double *g3_host, cpsd_integral_grads *G) {
    Sys S;
    CPSD_TRY(make_sys(s, &S));
    const bool third = g3_host != nullptr;
    Ints X = make_ints(S, I);
    IntegralScope keep(I);
    Fp64Only fp64;
    const i64 *o = S.popo, *v = S.popv;
    const i64 l1 = irpdso(symR, v, o, 1), l2 = idsymsoc(symR, v, v, 0, o, o, 0), nocc = occupied(S);
    const i64 nb = nroot;
    ScratchScope sc;
    Ground g;
    Ground3 h;
    CPSD_TRY(ground_j2(S, X, &g));
    if (third) CPSD_TRY(ground3(S, X, p, g, &h));
    // forward recomputation of the doubles (R2^(1), R2^(2)) and C1 of every root
    double *c2, *r2, *c1, *r22 = nullptr, *c1c = nullptr, *w0d, *w2d, *wbar, *wbar3, *lbar, *z, *dots, *g0d;
    CPSD_TRY(scratch(nb * l2, &c2));
    CPSD_TRY(scratch(nb * l2, &r2));
    CPSD_TRY(scratch(nb * l1, &c1));
    CPSD_TRY(scratch(nb, &w0d));
    CPSD_TRY(scratch(2 * nb, &w2d));
    CPSD_TRY(scratch(nb, &wbar));
    CPSD_TRY(scratch(nb, &wbar3));
    CPSD_TRY(scratch(nb, &dots));
    CPSD_TRY(scratch(nb, &g0d));
    CPSD_TRY(scratch(nb * l1, &lbar));
    CPSD_TRY(scratch(nb * l1, &z));
    CPSD_TRY(launch_scale(lbar, nb * l1, 0.0));
    CPSD_TRY(launch_scale(wbar3, nb, 0.0));
    CPSD_TRY(upload(w0d, w0_host, nb));
    CPSD_TRY(upload(g0d, g0_host, nb));
    CPSD_TRY(w2_forward(S, X, g, symR, nb, L_dev, w0d, c2, r2, c1, w2d));
    if (third) {
        CPSD_TRY(scratch(nb * l2, &r22));
        CPSD_TRY(scratch(nb * l1, &c1c));
        CPSD_TRY(w3_forward(S, X, g, h, symR, nb, L_dev, w0d, r2, r22, c1c, w2d + nb));
    }
    // cotangents of the ground-state intermediates, summed over the roots
    Ten Foob = g.Foo, Fvvb = g.Fvv, Wvob = g.Wvo, T2b = g.T2;
    for (Ten *t : {&Foob, &Fvvb, &Wvob, &T2b}) CPSD_TRY(fresh(t));
    Ground3 hb = h;
    if (third)
        for (Ten *t : {&hb.Woo, &hb.Foo3, &hb.Fvv3, &hb.Wvo3}) CPSD_TRY(fresh(t));
    Ten Gijkl = X.ijkl, Gijka = X.ijka, Gabij = X.abij, Giabj = X.iabj, Gabci = X.abci, Gabcd = X.abcd;
    Gijkl.arr = G->ijkl;
    Gijka.arr = G->ijka;
    Gabij.arr = G->abij;
    Giabj.arr = G->iabj;
    Gabci.arr = G->abci;
    Gabcd.arr = G->abcd;
    const EnergyPlan *e2, *e1, *e2g, *e1g;
    CPSD_TRY(plan_energy(make_desc(v, v, o, o, 0, 0, symR), "vvoo", &e2));
    CPSD_TRY(plan_energy(make_desc(v, o, ZORB, ZORB, 1, 1, symR), "vozz", &e1));
    CPSD_TRY(plan_energy(make_desc(v, v, o, o, 0, 0, 1), "vvoo", &e2g));
    CPSD_TRY(plan_energy(make_desc(v, o, ZORB, ZORB, 1, 1, 1), "vozz", &e1g));
    double *cb1, *r2b, *q, *r22b = nullptr;
    CPSD_TRY(scratch(l1, &cb1));
    CPSD_TRY(scratch(l2, &r2b));
    CPSD_TRY(scratch(l2, &q));
    if (third) CPSD_TRY(scratch(l2, &r22b));
    for (i64 r = 0; r < nb; r++) {
        const double *Lr = L_dev + r * l1;
        Ten Lt = ten(v, o, ZORB, ZORB, 1, 1, symR, (double *)Lr);
        Ten R2 = ten(v, v, o, o, 0, 0, symR, r2 + r * l2);
        Ten Cb1 = ten(v, o, ZORB, ZORB, 1, 1, symR, cb1);
        Ten Lb = ten(v, o, ZORB, ZORB, 1, 1, symR, lbar + r * l1);
        Ten R2b = ten(v, v, o, o, 0, 0, symR, r2b);
        Ten C2b = ten(v, v, o, o, 0, 0, symR, q);
        CPSD_TRY(launch_scale(r2b, l2, 0.0));
        if (third) {
            Ten R22 = ten(v, v, o, o, 0, 0, symR, r22 + r * l2);
            Ten R22b = ten(v, v, o, o, 0, 0, symR, r22b);
            // w3 = L . C1^(3): C1^(3)bar = g3 L, Lbar += g3 C1^(3)
            CPSD_TRY(launch_copy(cb1, Lr, l1));
            CPSD_TRY(launch_scale(cb1, l1, g3_host[r]));
            CPSD_TRY(launch_axpy(l1, g3_host[r], c1c + r * l1, Lb.arr));
            CPSD_TRY(launch_scale(r22b, l2, 0.0));
            CPSD_TRY(vjp_c1_r2abci(R22, X.abci, Cb1, R22b, 0, 1.0));
            CPSD_TRY(vjp_c1_r2abci(R22, X.abci, Cb1, Gabci, 1, 1.0));
            CPSD_TRY(vjp_c1_r2ijka(R22, X.ijka, Cb1, R22b, 0, 1.0));
            CPSD_TRY(vjp_c1_r2ijka(R22, X.ijka, Cb1, Gijka, 1, 1.0));
            CPSD_TRY(vjp_c1_r1iabj(Lt, h.Wvo3, Cb1, Lb, 0, 1.0));
            CPSD_TRY(vjp_c1_r1iabj(Lt, h.Wvo3, Cb1, hb.Wvo3, 1, 1.0));
            CPSD_TRY(vjp_c1_r1Fmi(Lt, h.Foo3, Cb1, Lb, 0, 1.0));
            CPSD_TRY(vjp_c1_r1Fmi(Lt, h.Foo3, Cb1, hb.Foo3, 1, 1.0));
            CPSD_TRY(vjp_c1_r1Fae(Lt, h.Fvv3, Cb1, Lb, 0, 1.0));
            CPSD_TRY(vjp_c1_r1Fae(Lt, h.Fvv3, Cb1, hb.Fvv3, 1, 1.0));
            // R2^(2) = -C2^(2)/(e2 - w0): q = R2^(2)bar/(e2 - w0), C2^(2)bar = -q
            CPSD_TRY(launch_energy(e2, 1, X.eorb, r22b, q, w0d + r));
            CPSD_TRY(launch_energy_adjoint(e2, q, R22.arr, -1.0, nocc, G->eorb));
            CPSD_TRY(launch_dot(q, R22.arr, l2, wbar3 + r, true));
            CPSD_TRY(launch_scale(q, l2, -1.0));
            // C2^(2) = calC2_VR2(R2^(1)) + c2_r1ijka(L, J2_Wovoo) + calC_VTR(T2, L)
            CPSD_TRY(vjp_c2_r2Wmbej(R2, X.iabj, C2b, R2b, 0, 1.0));
            CPSD_TRY(vjp_c2_r2Wmbej(R2, X.iabj, C2b, Giabj, 1, 1.0));
            CPSD_TRY(vjp_c2_r2Wmnij(R2, X.ijkl, C2b, R2b, 0, 1.0));
            CPSD_TRY(vjp_c2_r2Wmnij(R2, X.ijkl, C2b, Gijkl, 1, 1.0));
            CPSD_TRY(vjp_c2_r2abcd(R2, X.abcd, C2b, R2b, 0, 1.0));
            CPSD_TRY(vjp_c2_r2abcd(R2, X.abcd, C2b, Gabcd, 1, 1.0));
            CPSD_TRY(vjp_c2_r1ijka(Lt, h.Woo, C2b, Lb, 0, 1.0));
            CPSD_TRY(vjp_c2_r1ijka(Lt, h.Woo, C2b, hb.Woo, 1, 1.0));
            ScratchScope s2;
            VtrTemps t, tb;
            CPSD_TRY(vtr_temps(S, X, symR, Lt, 1, &t));
            CPSD_TRY(vtr_layouts(S, symR, 1, &tb));
            CPSD_TRY(vjp_c2_r2Wmnij(g.T2, t.mn, C2b, T2b, 0, 1.0));
            CPSD_TRY(vjp_c2_r2Wmnij(g.T2, t.mn, C2b, tb.mn, 1, 1.0));
            CPSD_TRY(vjp_c2_r2Wmbej(g.T2, t.mb, C2b, T2b, 0, 1.0));
            CPSD_TRY(vjp_c2_r2Wmbej(g.T2, t.mb, C2b, tb.mb, 1, 1.0));
            CPSD_TRY(vjp_c2_r2Fmi(g.T2, t.fo, C2b, T2b, 0, 1.0));
            CPSD_TRY(vjp_c2_r2Fmi(g.T2, t.fo, C2b, tb.fo, 1, 1.0));
            CPSD_TRY(vjp_c2_r2Fae(g.T2, t.fv, C2b, T2b, 0, 1.0));
            CPSD_TRY(vjp_c2_r2Fae(g.T2, t.fv, C2b, tb.fv, 1, 1.0));
            CPSD_TRY(vjp_Wmnij_r1ijka(Lt, X.ijka, tb.mn, Lb, 0, 1.0));
            CPSD_TRY(vjp_Wmnij_r1ijka(Lt, X.ijka, tb.mn, Gijka, 1, 1.0));
            CPSD_TRY(vjp_Wmbej_r1abci(Lt, X.abci, tb.mb, Lb, 0, 1.0));
            CPSD_TRY(vjp_Wmbej_r1abci(Lt, X.abci, tb.mb, Gabci, 1, 1.0));
            CPSD_TRY(vjp_Fmi_r1ijka(Lt, X.ijka, tb.fo, Lb, 0, 1.0));
            CPSD_TRY(vjp_Fmi_r1ijka(Lt, X.ijka, tb.fo, Gijka, 1, 1.0));
            CPSD_TRY(vjp_Fae_r1abci(Lt, X.abci, tb.fv, Lb, 0, 1.0));
            CPSD_TRY(vjp_Fae_r1abci(Lt, X.abci, tb.fv, Gabci, 1, 1.0));
        }
        // w2 = L . C1: C1bar = g2 L, Lbar += g2 C1
        CPSD_TRY(launch_copy(cb1, Lr, l1));
        CPSD_TRY(launch_scale(cb1, l1, g2_host[r]));
        CPSD_TRY(launch_axpy(l1, g2_host[r], c1 + r * l1, Lb.arr));
        // C1 = c1_r2abci(R2) + c1_r2ijka(R2) + c1_r1iabj(L,Wvo) + c1_r1Fmi(L,Foo) + c1_r1Fae(L,Fvv)
        CPSD_TRY(vjp_c1_r2abci(R2, X.abci, Cb1, R2b, 0, 1.0));
        CPSD_TRY(vjp_c1_r2abci(R2, X.abci, Cb1, Gabci, 1, 1.0));
        CPSD_TRY(vjp_c1_r2ijka(R2, X.ijka, Cb1, R2b, 0, 1.0));
        CPSD_TRY(vjp_c1_r2ijka(R2, X.ijka, Cb1, Gijka, 1, 1.0));
        CPSD_TRY(vjp_c1_r1iabj(Lt, g.Wvo, Cb1, Lb, 0, 1.0));
        CPSD_TRY(vjp_c1_r1iabj(Lt, g.Wvo, Cb1, Wvob, 1, 1.0));
        CPSD_TRY(vjp_c1_r1Fmi(Lt, g.Foo, Cb1, Lb, 0, 1.0));
        CPSD_TRY(vjp_c1_r1Fmi(Lt, g.Foo, Cb1, Foob, 1, 1.0));
        CPSD_TRY(vjp_c1_r1Fae(Lt, g.Fvv, Cb1, Lb, 0, 1.0));
        CPSD_TRY(vjp_c1_r1Fae(Lt, g.Fvv, Cb1, Fvvb, 1, 1.0));
        // R2 = -C2/(e2 - w0): q = R2bar/(e2 - w0); C2bar = -q,
        // e2bar = -q R2, w0bar = q . R2
        CPSD_TRY(launch_energy(e2, 1, X.eorb, r2b, q, w0d + r));
        CPSD_TRY(launch_energy_adjoint(e2, q, R2.arr, -1.0, nocc, G->eorb));
        CPSD_TRY(launch_dot(q, R2.arr, l2, wbar + r, true));
        CPSD_TRY(launch_scale(q, l2, -1.0));
        // C2 = c2_r1ijka(L) + c2_r1abci(L)
        CPSD_TRY(vjp_c2_r1ijka(Lt, X.ijka, C2b, Lb, 0, 1.0));
        CPSD_TRY(vjp_c2_r1ijka(Lt, X.ijka, C2b, Gijka, 1, 1.0));
        CPSD_TRY(vjp_c2_r1abci(Lt, X.abci, C2b, Lb, 0, 1.0));
        CPSD_TRY(vjp_c2_r1abci(Lt, X.abci, C2b, Gabci, 1, 1.0));
    }
    // Z-vector: (A - w0) z = P Lbar with L.z = 0; solve_r1 solves
    // (A - w0) z = -cc for cc orthogonal to L
    for (i64 r = 0; r < nb; r++) CPSD_TRY(launch_dot(L_dev + r * l1, lbar + r * l1, l1, dots + r, false));
    CPSD_TRY(launch_axpy_dev(l1, dots, -1.0, L_dev, lbar, nb, l1, l1));
    CPSD_TRY(launch_scale(lbar, nb * l1, -1.0));
    i64 sit = 0;
    CPSD_TRY(solve_r1(S, X, p, symR, nb, l1, e1, lbar, L_dev, w0d, z, &sit));
    // A-bar = (w0bar L - z) L^T with w0bar = g0 + q.R2 (+ q.R2^(2)): into V(fn,ai) and e(a,i)
    CPSD_TRY(launch_axpy(nb, 1.0, g0d, wbar));
    CPSD_TRY(launch_axpy(nb, 1.0, wbar3, wbar));
    CPSD_TRY(launch_scale(z, nb * l1, -1.0));
    CPSD_TRY(launch_axpy_dev(l1, wbar, 1.0, L_dev, z, nb, l1, l1));
    for (i64 r = 0; r < nb; r++) {
        Ten Lt = ten(v, o, ZORB, ZORB, 1, 1, symR, (double *)(L_dev + r * l1));
        Ten U = ten(v, o, ZORB, ZORB, 1, 1, symR, z + r * l1);
        CPSD_TRY(vjp_c1_r1iabj(Lt, X.iabj, U, Giabj, 1, 1.0));
        CPSD_TRY(launch_energy_adjoint(e1, U.arr, Lt.arr, 1.0, nocc, G->eorb));
    }
    if (third) {
        // J^(3) back to T1^(2), T2^(2) and the integrals
        Ten T1bb = h.T1b, T2bb = h.T2b;
        CPSD_TRY(fresh(&T1bb));
        CPSD_TRY(fresh(&T2bb));
        CPSD_TRY(vjp_Fmi_r1ijka(h.T1b, X.ijka, hb.Foo3, T1bb, 0, 1.0));
        CPSD_TRY(vjp_Fmi_r1ijka(h.T1b, X.ijka, hb.Foo3, Gijka, 1, 1.0));
        CPSD_TRY(vjp_Fmi_r2abij(h.T2b, X.abij, hb.Foo3, T2bb, 0, 1.0));
        CPSD_TRY(vjp_Fmi_r2abij(h.T2b, X.abij, hb.Foo3, Gabij, 1, 1.0));
        CPSD_TRY(vjp_Fae_r1abci(h.T1b, X.abci, hb.Fvv3, T1bb, 0, 1.0));
        CPSD_TRY(vjp_Fae_r1abci(h.T1b, X.abci, hb.Fvv3, Gabci, 1, 1.0));
        CPSD_TRY(vjp_Fae_r2abij(h.T2b, X.abij, hb.Fvv3, T2bb, 0, 1.0));
        CPSD_TRY(vjp_Fae_r2abij(h.T2b, X.abij, hb.Fvv3, Gabij, 1, 1.0));
        CPSD_TRY(vjp_Wmbej_r1ijka(h.T1b, X.ijka, hb.Wvo3, T1bb, 0, 1.0));
        CPSD_TRY(vjp_Wmbej_r1ijka(h.T1b, X.ijka, hb.Wvo3, Gijka, 1, 1.0));
        CPSD_TRY(vjp_Wmbej_r1abci(h.T1b, X.abci, hb.Wvo3, T1bb, 0, 1.0));
        CPSD_TRY(vjp_Wmbej_r1abci(h.T1b, X.abci, hb.Wvo3, Gabci, 1, 1.0));
        CPSD_TRY(vjp_Wmbej_r2abij(h.T2b, X.abij, hb.Wvo3, T2bb, 0, 2.0));
        CPSD_TRY(vjp_Wmbej_r2abij(h.T2b, X.abij, hb.Wvo3, Gabij, 1, 2.0));
        // T2^(2) = C2g / D: t = T2^(2)bar / D is C2g's cotangent, e2bar = T2^(2) t
        const i64 lg = g.T2.len();
        Ten tt = g.T2;
        CPSD_TRY(scratch(lg, &tt.arr));
        CPSD_TRY(launch_energy(e2g, 2, X.eorb, T2bb.arr, tt.arr));
        CPSD_TRY(launch_energy_adjoint(e2g, h.T2b.arr, tt.arr, 1.0, nocc, G->eorb));
        CPSD_TRY(vjp_c2_r2Wmbej(g.T2, X.iabj, tt, T2b, 0, 1.0));
        CPSD_TRY(vjp_c2_r2Wmbej(g.T2, X.iabj, tt, Giabj, 1, 1.0));
        CPSD_TRY(vjp_c2_r2Wmnij(g.T2, X.ijkl, tt, T2b, 0, 1.0));
        CPSD_TRY(vjp_c2_r2Wmnij(g.T2, X.ijkl, tt, Gijkl, 1, 1.0));
        CPSD_TRY(vjp_c2_r2abcd(g.T2, X.abcd, tt, T2b, 0, 1.0));
        CPSD_TRY(vjp_c2_r2abcd(g.T2, X.abcd, tt, Gabcd, 1, 1.0));
        // T1^(2): (ei - ea) T1 - V T1 = C1g.  lam solves the same (symmetric)
        // system with T1^(2)bar: C1g-bar = lam, V-bar += lam T1^T, and the
        // orbital energies get -lam T1 d(ei - ea)
        Ten lam = h.T1b;
        CPSD_TRY(scratch(lam.len(), &lam.arr));
        i64 it = 0;
        CPSD_TRY(solve_r1(S, X, p, 1, 1, lam.len(), e1g, T1bb.arr, nullptr, nullptr, lam.arr, &it));
        CPSD_TRY(launch_energy_adjoint(e1g, lam.arr, h.T1b.arr, 1.0, nocc, G->eorb));
        CPSD_TRY(vjp_c1_r1iabj(h.T1b, X.iabj, lam, Giabj, 1, 1.0));
        CPSD_TRY(vjp_c1_r2abci(g.T2, X.abci, lam, T2b, 0, 1.0));
        CPSD_TRY(vjp_c1_r2abci(g.T2, X.abci, lam, Gabci, 1, 1.0));
        CPSD_TRY(vjp_c1_r2ijka(g.T2, X.ijka, lam, T2b, 0, 1.0));
        CPSD_TRY(vjp_c1_r2ijka(g.T2, X.ijka, lam, Gijka, 1, 1.0));
        // J2_Wovoo = Wkbij_r2ijka(T2) + Wkbij_r2abci(T2)
        CPSD_TRY(vjp_Wkbij_r2ijka(g.T2, X.ijka, hb.Woo, T2b, 0, 1.0));
        CPSD_TRY(vjp_Wkbij_r2ijka(g.T2, X.ijka, hb.Woo, Gijka, 1, 1.0));
        CPSD_TRY(vjp_Wkbij_r2abci(g.T2, X.abci, hb.Woo, T2b, 0, 1.0));
        CPSD_TRY(vjp_Wkbij_r2abci(g.T2, X.abci, hb.Woo, Gabci, 1, 1.0));
    }
    // J^(2) intermediates back to T2 and <ab||ij>; T2 = <ab||ij>/D, D = -e2
    CPSD_TRY(vjp_Fmi_r2abij(g.T2, X.abij, Foob, T2b, 0, 1.0));
    CPSD_TRY(vjp_Fmi_r2abij(g.T2, X.abij, Foob, Gabij, 1, 1.0));
    CPSD_TRY(vjp_Fae_r2abij(g.T2, X.abij, Fvvb, T2b, 0, 1.0));
    CPSD_TRY(vjp_Fae_r2abij(g.T2, X.abij, Fvvb, Gabij, 1, 1.0));
    CPSD_TRY(vjp_Wmbej_r2abij(g.T2, X.abij, Wvob, T2b, 0, 2.0));
    CPSD_TRY(vjp_Wmbej_r2abij(g.T2, X.abij, Wvob, Gabij, 1, 2.0));
    const i64 lg = g.T2.len();
    double *t;
    CPSD_TRY(scratch(lg, &t));
    CPSD_TRY(launch_energy(e2g, 2, X.eorb, T2b.arr, t));  // t = T2bar / D
    CPSD_TRY(launch_axpy(lg, 1.0, t, G->abij));
    CPSD_TRY(launch_energy_adjoint(e2g, g.t2, t, 1.0, nocc, G->eorb));  // e2bar = T2 t
    return cuda_check(cudaStreamSynchronize(stream()), "cisd gradient");
}

}  // namespace
}  // namespace cpsd

extern "C" {

int cpsd_cisd_gradient(const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p, int64_t symR,
                       int64_t nroot, const double *w0_host, const double *L_dev, const double *g0_host,
                       const double *g2_host, cpsd_integral_grads *G) {
    Sys S;
    CPSD_TRY(make_sys(s, &S));
    if (!p || !I || !w0_host || !L_dev || !g0_host || !g2_host || !G)
        return set_error(CPSD_EARG, "cisd_gradient: null argument");
    if (!G->ijka || !G->abij || !G->iabj || !G->abci || !G->eorb)
        return set_error(CPSD_EARG, "cisd_gradient: ijka, abij, iabj, abci and eorb gradients are required");
    if (symR < 1 || symR > S.nirrep || nroot <= 0) return set_error(CPSD_EARG, "cisd_gradient: bad irrep or roots");
    return gradient_impl(s, I, p, symR, nroot, w0_host, L_dev, g0_host, g2_host, nullptr, G);
}

int cpsd_cpsd3_gradient(const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p, int64_t symR,
                        int64_t nroot, const double *w0_host, const double *L_dev, const double *g0_host,
                        const double *g2_host, const double *g3_host, cpsd_integral_grads *G) {
    Sys S;
    CPSD_TRY(make_sys(s, &S));
    if (!p || !I || !w0_host || !L_dev || !g0_host || !g2_host || !g3_host || !G)
        return set_error(CPSD_EARG, "cpsd3_gradient: null argument");
    if (!I->ijkl || !I->abcd) return set_error(CPSD_EARG, "cpsd3_gradient: ijkl and abcd are required");
    if (!G->ijkl || !G->ijka || !G->abij || !G->iabj || !G->abci || !G->abcd || !G->eorb)
        return set_error(CPSD_EARG, "cpsd3_gradient: all six list gradients and eorb are required");
    if (symR < 1 || symR > S.nirrep || nroot <= 0) return set_error(CPSD_EARG, "cpsd3_gradient: bad irrep or roots");
    return gradient_impl(s, I, p, symR, nroot, w0_host, L_dev, g0_host, g2_host, g3_host, G);
}

}  // extern "C"
