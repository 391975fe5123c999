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
    Ints X = make_ints(S, I);
    IntegralScope keep(I);
    Fp64Only fp64;
    const i64 *o = S.popo, *v = S.popv;
    const i64 l1 = irpdso(symR, v, o, 1), l2 = idsymsoc(symR, v, v, 0, o, o, 0), nocc = occupied(S);
    const i64 nb = nroot;
    ScratchScope sc;
    Ground g;
    CPSD_TRY(ground_j2(S, X, &g));
    // forward recomputation of the doubles (R2) and C1 of every root
    double *c2, *r2, *c1, *w0d, *w2d, *wbar, *lbar, *z, *dots, *g0d;
    CPSD_TRY(scratch(nb * l2, &c2));
    CPSD_TRY(scratch(nb * l2, &r2));
    CPSD_TRY(scratch(nb * l1, &c1));
    CPSD_TRY(scratch(nb, &w0d));
    CPSD_TRY(scratch(nb, &w2d));
    CPSD_TRY(scratch(nb, &wbar));
    CPSD_TRY(scratch(nb, &dots));
    CPSD_TRY(scratch(nb, &g0d));
    CPSD_TRY(scratch(nb * l1, &lbar));
    CPSD_TRY(scratch(nb * l1, &z));
    CPSD_TRY(upload(w0d, w0_host, nb));
    CPSD_TRY(upload(g0d, g0_host, nb));
    CPSD_TRY(w2_forward(S, X, g, symR, nb, L_dev, w0d, c2, r2, c1, w2d));
    // cotangents of the J^(2) intermediates, summed over the roots
    Ten Foob = g.Foo, Fvvb = g.Fvv, Wvob = g.Wvo;
    for (Ten *t : {&Foob, &Fvvb, &Wvob}) {
        CPSD_TRY(scratch(t->len(), &t->arr));
        CPSD_TRY(launch_scale(t->arr, t->len(), 0.0));
    }
    Ten Gijka = X.ijka, Gabij = X.abij, Giabj = X.iabj, Gabci = X.abci;
    Gijka.arr = G->ijka;
    Gabij.arr = G->abij;
    Giabj.arr = G->iabj;
    Gabci.arr = G->abci;
    const EnergyPlan *e2, *e1, *e2g;
    CPSD_TRY(plan_energy(make_desc(v, v, o, o, 0, 0, symR), "vvoo", &e2));
    CPSD_TRY(plan_energy(make_desc(v, o, ZORB, ZORB, 1, 1, symR), "vozz", &e1));
    CPSD_TRY(plan_energy(make_desc(v, v, o, o, 0, 0, 1), "vvoo", &e2g));
    double *cb1, *r2b, *q;
    CPSD_TRY(scratch(l1, &cb1));
    CPSD_TRY(scratch(l2, &r2b));
    CPSD_TRY(scratch(l2, &q));
    for (i64 r = 0; r < nb; r++) {
        const double *Lr = L_dev + r * l1;
        Ten Lt = ten(v, o, ZORB, ZORB, 1, 1, symR, (double *)Lr);
        Ten R2 = ten(v, v, o, o, 0, 0, symR, r2 + r * l2);
        Ten Cb1 = ten(v, o, ZORB, ZORB, 1, 1, symR, cb1);
        Ten Lb = ten(v, o, ZORB, ZORB, 1, 1, symR, lbar + r * l1);
        Ten R2b = ten(v, v, o, o, 0, 0, symR, r2b);
        Ten C2b = ten(v, v, o, o, 0, 0, symR, q);
        // w2 = L . C1: C1bar = g2 L, Lbar = g2 C1
        CPSD_TRY(launch_copy(cb1, Lr, l1));
        CPSD_TRY(launch_scale(cb1, l1, g2_host[r]));
        CPSD_TRY(launch_copy(Lb.arr, c1 + r * l1, l1));
        CPSD_TRY(launch_scale(Lb.arr, l1, g2_host[r]));
        // C1 = c1_r2abci(R2) + c1_r2ijka(R2) + c1_r1iabj(L,Wvo) + c1_r1Fmi(L,Foo) + c1_r1Fae(L,Fvv)
        CPSD_TRY(launch_scale(r2b, l2, 0.0));
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
    // A-bar = (w0bar L - z) L^T with w0bar = g0 + q.R2: into V(fn,ai) and e(a,i)
    CPSD_TRY(launch_axpy(nb, 1.0, g0d, wbar));
    CPSD_TRY(launch_scale(z, nb * l1, -1.0));
    CPSD_TRY(launch_axpy_dev(l1, wbar, 1.0, L_dev, z, nb, l1, l1));
    for (i64 r = 0; r < nb; r++) {
        Ten Lt = ten(v, o, ZORB, ZORB, 1, 1, symR, (double *)(L_dev + r * l1));
        Ten U = ten(v, o, ZORB, ZORB, 1, 1, symR, z + r * l1);
        CPSD_TRY(vjp_c1_r1iabj(Lt, X.iabj, U, Giabj, 1, 1.0));
        CPSD_TRY(launch_energy_adjoint(e1, U.arr, Lt.arr, 1.0, nocc, G->eorb));
    }
    // J^(2) intermediates back to T2 and <ab||ij>; T2 = <ab||ij>/D, D = -e2
    Ten T2b = g.T2;
    CPSD_TRY(scratch(T2b.len(), &T2b.arr));
    CPSD_TRY(launch_scale(T2b.arr, T2b.len(), 0.0));
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

}  // extern "C"
