// Internal tensor operations of libcpsd_b200 (mod_contract wrappers and the
// spin-free lib_cc kernels) with optional batching over independent
// copies (the roots of one irrep): a Ten with bs != 0 is a stack of nb
// tensors bs elements apart; the output of a batched call is always
// stacked.
#pragma once
#include "runtime.hpp"

namespace cpsd {

struct Ten {
    Desc d;
    double *arr = nullptr;
    i64 bs = 0;  // batch stride in elements (0 = one tensor shared by the batch)
    i64 len() const { return d.len(); }
};
Ten ten_of(const cpsd_opt *t);
Ten ten(const i64 *p0, const i64 *p1, const i64 *p2, const i64 *p3, i64 iop0, i64 iop1, i64 sym, double *arr,
        i64 bs = 0);

// Scope during which the given device arrays (a program's integrals) are
// not written: expanded copies made of them are kept and reused until the
// outermost scope ends.
struct ConstOperands {
    ConstOperands(const double *const *arrs, int n);
    ~ConstOperands();
    ConstOperands(const ConstOperands &) = delete;
    ConstOperands &operator=(const ConstOperands &) = delete;
};

// V3 = f1 * V1 (x) V2 + f2 * V3 (the vv2v_dpd engines)
int engine(const Ten &v1, const char *t1, const Ten &v2, const char *t2, Ten &v3, const char *t3, double f1,
           double f2, i64 nb = 1);

int w444(const Ten &v1, const Ten &v2, Ten &v3, double fact, const char *t1, const char *t2, const char *t3,
         i64 anti, i64 nb = 1);
int w424(const Ten &v1, const Ten &v2, Ten &v3, double fact, const char *t1, const char *t2, const char *t3,
         i64 anti, i64 nb = 1);
int w442(const Ten &v1, const Ten &v2, Ten &v3, double fact, const char *t1, const char *t2, const char *t3,
         i64 nb = 1);
int w422(const Ten &v1, const Ten &v2, Ten &v3, double fact, const char *t1, const char *t2, const char *t3,
         i64 nb = 1);
int w222(const Ten &v1, const Ten &v2, Ten &v3, double fact, const char *t1, const char *t2, const char *t3,
         i64 nb = 1);
int w224(const Ten &v1, const Ten &v2, Ten &v3, double fact, const char *t1, const char *t2, const char *t3,
         i64 anti, i64 nb = 1);

// lib_cc kernels: out += f * kernel(a, b)
#define CPSD_IK(name) int k_##name(Ten &out, const Ten &a, const Ten &b, double f, i64 nb = 1)
CPSD_IK(c1_r1iabj);
CPSD_IK(c1_r1Fae);
CPSD_IK(c1_r1Fmi);
CPSD_IK(c1_r2abci);
CPSD_IK(c1_r2ijka);
CPSD_IK(c2_r1abci);
CPSD_IK(c2_r1ijka);
CPSD_IK(c2_r2Wmbej);
CPSD_IK(c2_r2Wmnij);
CPSD_IK(c2_r2abcd);
CPSD_IK(c2_r2Fae);
CPSD_IK(c2_r2Fmi);
CPSD_IK(Fmi_r2abij);
CPSD_IK(Fae_r2abij);
CPSD_IK(Fmi_r1ijka);
CPSD_IK(Fae_r1abci);
CPSD_IK(Wkbij_r2ijka);
CPSD_IK(Wkbij_r2abci);
CPSD_IK(Wmbej_r2abij);
CPSD_IK(Wmbej_r1abci);
CPSD_IK(Wmbej_r1ijka);
CPSD_IK(Wmnij_r1ijka);
CPSD_IK(Wmnij_r2abij);
CPSD_IK(Wkbij_r1iabj);
CPSD_IK(Wabdj_r1abcd);
CPSD_IK(Wkbij_r1Uklij);
CPSD_IK(Fme_r1abij);
CPSD_IK(c1_r2Fme);
CPSD_IK(c1d_l1Wibaj);
CPSD_IK(c1d_l1fab);
CPSD_IK(c1d_l1fij);
CPSD_IK(Fae_r1fia);
CPSD_IK(Fmi_r1fia);
CPSD_IK(Wkbij_r2Fkc);
CPSD_IK(Wlkjd_r1abij);
#undef CPSD_IK

// Vector-Jacobian product of the vv2v_444 form v3 += fact * P{v1 v2}:
// G += d<Y, v3>/d(v1) (which 0) or d(v2) (which 1); Y has v3's layout, G
// the operand's.  One copy (no batch).
int vjp444(const Ten &v1, const Ten &v2, const Ten &Y, Ten &G, int which, double fact, const char *t1,
           const char *t2, const char *t3, i64 anti);
// adjoints of the kernels on the SF-CIS(D) energy path: G += d<Y, out>/da
// (which 0) or d<Y, out>/db (which 1) of out += f * kernel(a, b)
#define CPSD_VJP(name) int vjp_##name(const Ten &a, const Ten &b, const Ten &Y, Ten &G, int which, double f)
CPSD_VJP(c1_r1iabj);
CPSD_VJP(c1_r1Fae);
CPSD_VJP(c1_r1Fmi);
CPSD_VJP(c1_r2abci);
CPSD_VJP(c1_r2ijka);
CPSD_VJP(c2_r1abci);
CPSD_VJP(c2_r1ijka);
CPSD_VJP(Fmi_r2abij);
CPSD_VJP(Fae_r2abij);
CPSD_VJP(Wmbej_r2abij);
// and the further ones of the third-order correction w^(3)
CPSD_VJP(c2_r2Wmbej);
CPSD_VJP(c2_r2Wmnij);
CPSD_VJP(c2_r2abcd);
CPSD_VJP(c2_r2Fae);
CPSD_VJP(c2_r2Fmi);
CPSD_VJP(Fmi_r1ijka);
CPSD_VJP(Fae_r1abci);
CPSD_VJP(Wkbij_r2ijka);
CPSD_VJP(Wkbij_r2abci);
CPSD_VJP(Wmbej_r1abci);
CPSD_VJP(Wmbej_r1ijka);
CPSD_VJP(Wmnij_r1ijka);
#undef CPSD_VJP

}  // namespace cpsd
