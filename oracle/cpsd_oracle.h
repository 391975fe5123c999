/*
 * CPU ORACLE — test infrastructure only.
 *
 * A plain FP64 CPU restatement of the reference's spin-free SF-CIS /
 * SF-CPS(D-3) hot path (lishun-1208/revised-cluster-perturbation-single-double),
 * used ONLY by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * `--impl reference` arm, as the checker and as the timed CPU baseline.
 * Nothing in the product library links or calls this code.
 *
 * Parity status: the reference is Fortran (nvfortran/OpenACC/CUDA Fortran)
 * and cannot be compiled here (no Fortran compiler), and its example goldens
 * need PySCF integrals that are not available.  This restatement is
 * therefore "parity unpinned" against reference-produced numbers; it is
 * cross-checked against independent dense numpy formulas (nirrep = 1 and
 * symmetry-blocked cases), a dense diagonalisation of the CIS matrix and the
 * reference's own built-in runtime assertions (Davidson residual test,
 * <L|R^(n)> = 0).
 *
 * Conventions follow the reference exactly: irreps are 1-based, integers are
 * int64 (the reference is built with -i8), tensors are DPD-packed with irrep
 * blocks ordered by the irrep of the right pair, column-major inside a block,
 * left index fastest; iop 0 = p<q packed antisymmetric pair, 1 = full pair,
 * 2 = p<=q.
 */
#ifndef CPSD_ORACLE_H
#define CPSD_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int64_t i64;

/* error codes (the reference STOPs; the oracle returns) */
#define O_OK 0
#define O_EARG (-1)
#define O_ELAYOUT (-2)
#define O_EMEM (-3)
#define O_ELAPACK (-4)

/* ---------------- symmetry / size math ----------------
 * mod_symm (src/lib_mod/mod_symm.f:1-9); dirprd is column-major 8x8,
 * dirprd[(j-1)*8 + (i-1)] = DIRPRD(i,j). */
int o_set_symmetry(i64 nirrep, const i64 *dirprd);
i64 o_nirrep(void);
i64 o_dirprd(i64 i, i64 j);
/* src/libsrint/irpdso.f:1-52 */
i64 o_irpdso(i64 sym, const i64 *popp, const i64 *popq, i64 ioppq);
/* src/libsrint/idsymsoc.f:1-30 */
i64 o_idsymsoc(i64 irrepx, const i64 *popp, const i64 *popq, i64 ioppq,
               const i64 *popr, const i64 *pops, i64 ioprs);
/* src/libsrint/isymoffso.f:1-54 (1-based start) */
i64 o_isymoffso(i64 irrepq1, i64 irrep, const i64 *popp, const i64 *popq, i64 iop);

/* DPD tensor descriptor: the data part of type(opt)
 * (src/lib_cc/mod_operator.f90:8-25) */
typedef struct {
    i64 pop[4][8]; /* popp, popq, popr, pops */
    i64 iop[2];    /* ioppq, ioprs */
    i64 sym;
} o_desc;

void o_desc_init(o_desc *d, const i64 *popp, const i64 *popq, const i64 *popr,
                 const i64 *pops, i64 ioppq, i64 ioprs, i64 sym);
i64 o_desc_len(const o_desc *d);
/* Linear 0-based offset of element (irr[k], idx[k]) (irreps 1-based, indices
 * 0-based within the irrep) — the element addressing of putidx
 * (src/lib_cc/putidx.f90).  Returns -1 if the element is structurally zero
 * (p==q in a p<q pair, or a symmetry-forbidden combination).  For packed
 * pairs presented in the non-stored order, *sign is set to -1 (iop 0) or
 * +1 (iop 2) and the stored partner's offset is returned. */
i64 o_elem_offset(const o_desc *d, const i64 irr[4], const i64 idx[4], int *sign);

/* ---------------- DPD contraction engine ----------------
 * V3 = f1 * sum_contracted V1*V2 + f2 * V3 over the symmetry-allowed
 * elements; the semantics of vv2v_dpd_444 (src/libsrint/vv2v_dpd_444.f90:55,
 * src/libsrint/vv2v_dpd_444_d.f90:4-529) generalised to every rank used by
 * the 424/442/422/222/224 siblings.  Types are 4 characters per tensor; a
 * '.' slot is a dummy index of extent 1 (zorb population). Packed (iop != 1)
 * pairs must be intact: the same two letters, same order, same iop, as a
 * pair of the partner tensor. */
int o_vv2v_dpd(const double *v1, const o_desc *d1, const char *t1,
               const double *v2, const o_desc *d2, const char *t2,
               double *v3, const o_desc *d3, const char *t3,
               double f1, double f2);

/* ---------------- layout transforms ----------------
 * iexpso (src/libsrint/iexpso.f90:24-120): expand pq and/or rs to iop 1 */
int o_iexpso(const double *in, double *out, const o_desc *din, i64 exppq, i64 exprs);
/* icompso (src/libsrint/icompso.f:1): compress an iop 1 pair to iop cpq/crs */
int o_icompso(const double *in, double *out, const o_desc *din, i64 cpq, i64 crs);
/* isymtrso (src/libsrint/isymtrso.f:1-351): out(qp / sr) = in(pq / rs) */
int o_isymtrso(const double *in, double *out, const o_desc *din, i64 swpq, i64 swrs);

/* ---------------- tensor objects and mod_contract wrappers ----------------
 * (src/lib_cc/mod_contract.f90:10-455) */
typedef struct {
    o_desc d;
    double *arr;
    i64 len;
} o_opt;

void o_opt_view(o_opt *t, const i64 *popp, const i64 *popq, const i64 *popr,
                const i64 *pops, i64 ioppq, i64 ioprs, i64 sym, double *arr);
int o_vv2v_444(const o_opt *v1, const o_opt *v2, o_opt *v3, double fact,
               const char *t1, const char *t2, const char *t3, i64 anti);
int o_vv2v_424(const o_opt *v1, const o_opt *v2, o_opt *v3, double fact,
               const char *t1, const char *t2, const char *t3, i64 anti);
int o_vv2v_442(const o_opt *v1, const o_opt *v2, o_opt *v3, double fact,
               const char *t1, const char *t2, const char *t3);
int o_vv2v_422(const o_opt *v1, const o_opt *v2, o_opt *v3, double fact,
               const char *t1, const char *t2, const char *t3);
int o_vv2v_222(const o_opt *v1, const o_opt *v2, o_opt *v3, double fact,
               const char *t1, const char *t2, const char *t3);
int o_vv2v_224(const o_opt *v1, const o_opt *v2, o_opt *v3, double fact,
               const char *t1, const char *t2, const char *t3, i64 anti);

/* ---------------- spin-free contraction kernels (src/lib_cc/<name>.f90) -------- */
int o_c1_r1iabj(o_opt *c1, const o_opt *r1, const o_opt *iabj, double f);
int o_c1_r1Fae(o_opt *c1, const o_opt *r1, const o_opt *Fae, double f);
int o_c1_r1Fmi(o_opt *c1, const o_opt *r1, const o_opt *Fmi, double f);
int o_c1_r2abci(o_opt *c1, const o_opt *r2, const o_opt *abci, double f);
int o_c1_r2ijka(o_opt *c1, const o_opt *r2, const o_opt *ijka, double f);
int o_c2_r1abci(o_opt *c2, const o_opt *r1, const o_opt *abci, double f);
int o_c2_r1ijka(o_opt *c2, const o_opt *r1, const o_opt *ijka, double f);
int o_c2_r2Wmbej(o_opt *c2, const o_opt *r2, const o_opt *W, double f);
int o_c2_r2Wmnij(o_opt *c2, const o_opt *r2, const o_opt *W, double f);
int o_c2_r2abcd(o_opt *c2, const o_opt *r2, const o_opt *abcd, double f);
int o_c2_r2Fae(o_opt *c2, const o_opt *r2, const o_opt *F, double f);
int o_c2_r2Fmi(o_opt *c2, const o_opt *r2, const o_opt *F, double f);
int o_Fmi_r2abij(o_opt *F, const o_opt *r2, const o_opt *abij, double f);
int o_Fae_r2abij(o_opt *F, const o_opt *r2, const o_opt *abij, double f);
int o_Fmi_r1ijka(o_opt *F, const o_opt *r1, const o_opt *ijka, double f);
int o_Fae_r1abci(o_opt *F, const o_opt *r1, const o_opt *abci, double f);
int o_Wkbij_r2ijka(o_opt *W, const o_opt *r2, const o_opt *ijka, double f);
int o_Wkbij_r2abci(o_opt *W, const o_opt *r2, const o_opt *abci, double f);
int o_Wmbej_r2abij(o_opt *W, const o_opt *r2, const o_opt *abij, double f);
int o_Wmbej_r1abci(o_opt *W, const o_opt *r1, const o_opt *abci, double f);
/* second-order ground state kernels (src/lib_cc/Wkbij_r1iabj.f90,
 * Wabdj_r1abcd.f90, Wkbij_r1Uklij.f90, Fme_r1abij.f90, c1_r2Fme.f90) */
int o_Wkbij_r1iabj(o_opt *W, const o_opt *r1, const o_opt *iabj, double f);
int o_Wabdj_r1abcd(o_opt *W, const o_opt *r1, const o_opt *abcd, double f);
int o_Wkbij_r1Uklij(o_opt *W, const o_opt *r1, const o_opt *U, double f);
int o_Fme_r1abij(o_opt *F, const o_opt *r1, const o_opt *abij, double f);
int o_c1_r2Fme(o_opt *c1, const o_opt *r2, const o_opt *F, double f);
/* excited-state grCPS(D) kernels (src/lib_cc/c1d_l1Wibaj.f90, c1d_l1fab.f90,
 * c1d_l1fij.f90, Fae_r1fia.f90, Fmi_r1fia.f90, Wkbij_r2Fkc.f90, Wlkjd_r1abij.f90) */
int o_c1d_l1Wibaj(o_opt *c1, const o_opt *l1, const o_opt *W, double f);
int o_c1d_l1fab(o_opt *c1, const o_opt *l1, const o_opt *F, double f);
int o_c1d_l1fij(o_opt *c1, const o_opt *l1, const o_opt *F, double f);
int o_Fae_r1fia(o_opt *c1, const o_opt *r1, const o_opt *F, double f);
int o_Fmi_r1fia(o_opt *c1, const o_opt *r1, const o_opt *F, double f);
int o_Wkbij_r2Fkc(o_opt *c1, const o_opt *r2, const o_opt *F, double f);
int o_Wlkjd_r1abij(o_opt *c1, const o_opt *r1, const o_opt *V, double f);
/* effectT2 (src/lib_cc/effectT2.f90:47-140), types 1 and 2 */
int o_effectT2(o_opt *t2, const o_opt *x, const o_opt *y, double f, int type);
int o_Wmbej_r1ijka(o_opt *W, const o_opt *r1, const o_opt *ijka, double f);
int o_Wmnij_r1ijka(o_opt *W, const o_opt *r1, const o_opt *ijka, double f);
int o_Wmnij_r2abij(o_opt *W, const o_opt *r2, const o_opt *abij, double f);

/* ---------------- molecular system and the pipeline ---------------- */
typedef struct {
    i64 nirrep;
    i64 dirprd[64];
    i64 symry;
    i64 popa[8], popb[8], vrta[8], vrtb[8];
    i64 popo[8], popv[8]; /* spin-free: popa(irr)+popb(irr x symry) (readmodule.f90:36-41) */
} o_system;

/* fills popo/popv from popa/popb/vrta/vrtb and installs the symmetry table */
int o_system_init(o_system *s);

/* spin-free integrals, DPD layout with iop = 0 (loadSCF, allocate_mem.f90) */
typedef struct {
    const double *ijkl, *ijka, *abij, *iabj, *abci, *abcd;
    const double *eorb; /* spin-free orbital energies (resortEorb layout) */
} o_integrals;

typedef struct {
    i64 davidson_dim, davidson_cyc, davidson_conv, lowest;
    i64 diis_dim, diis_cyc;
    double diis_max_err;
    i64 spin_flip;   /* 0 none, 1 alpha->beta ("ab"), 2 beta->alpha ("ba") */
    i64 open_shell;  /* shell=open (1) / close (0) */
    i64 ex_mult;     /* 1 or 3 (closed shell guesses) */
    i64 estate_sym[8];
    i64 nthreads;    /* OpenMP/OpenBLAS threads for the oracle */
} o_params;

void o_params_default(o_params *p);

/* Eorb_diff1 / Eorb_diff2 (src/lib_cc/Eorb_diff.f90:6,68) */
void o_eorb_diff1(double *oed1, const double *eorb, const i64 *pop_a, const i64 *pop_i, i64 sym);
void o_eorb_diff2(double *oed2, const double *eorb, const i64 *pop_a, const i64 *pop_i, i64 sym, i64 iop);
/* denomT1 / denomT2 (src/lib_cc/denomT.f90:1-249): t = r / D */
void o_denomT1(double *t1, const double *r1, const double *eorb, const i64 *pop_a, const i64 *pop_i, i64 sym);
void o_denomT2(double *t2, const double *r2, const double *eorb, const i64 *pop_a, const i64 *pop_i, i64 sym, i64 iop);

/* SF-CIS (src/EE-CIS.SF/run.f90:2-100).  For each irrep with roots, omega
 * and R1 are written to omega[k] and R[k*lenR(sym)], roots of irrep 1 first.
 * Returns the number of Davidson iterations summed over irreps in *iters. */
int o_cis_run(const o_system *s, const o_integrals *I, const o_params *p,
              double *omega, double *R, i64 *iters);
/* CIS(D-infinity) (src/CISdoo.SD.SF/run.f90): roots of the (R1, R2) problem;
 * R receives per root the R1 (l1) and R2 (l2, packed) of its irrep */
int o_cisdoo_run(const o_system *s, const o_integrals *I, const o_params *p, double *omega, double *R,
                 i64 *iters);

/* ground CPS(D) first and second order (src/CPSd.SF/run1.f90, run2.f90):
 * T2^(1), T1^(2), T2^(2), E^(2), E^(3) */
int o_cpsd_ground(const o_system *s, const o_integrals *I, const o_params *p,
                  double *T2_1, double *T1_2, double *T2_2, double *E2, double *E3,
                  i64 *diis_iters);
/* third order: T1^(3), T2^(3), E^(4) (src/CPSd.SF/run3.f90) */
/* second-order-dressed ground state grCPS(D) (src/grCPSd.SF/run.f90): for
 * order k = 1, 2, 3 the coupled (T1, T2)^(k) of solver.f90 with their DIIS
 * loop; T receives per order T1 (l1) then T2 (l2) of irrep 1, E[k-1] the
 * energy E^(k+1) of calEcorr.f90 at convergence, iters[k-1] the DIIS
 * iterations */
int o_grcpsd_ground(const o_system *s, const o_integrals *I, const o_params *p, double *T, double *E,
                    i64 *iters);
/* excited-state grCPS(D) (src/EE-grCPSd.SF/run.f90) from the grCPS(D)
 * amplitudes T (orders 1, 2 used; layout of o_grcpsd_ground) and the
 * CIS(D-infinity) roots omega / R0 (layout of o_cisdoo_run): w[3k..3k+2] =
 * w^(1), w^(2), w^(3) of root k; Lout (nullable) the normalised left vectors
 * (R0's layout), Rout (nullable) R^(1) of every root then R^(2) of every
 * root; *iters the DIIS iterations summed */
int o_eegrcpsd_roots(const o_system *s, const o_integrals *I, const o_params *p, const double *T,
                     const double *omega, const double *R0, double *w, double *Lout, double *Rout,
                     i64 *iters);
int o_cpsd_ground3(const o_system *s, const o_integrals *I, const o_params *p,
                   const double *T2_1, const double *T1_2, const double *T2_2,
                   double *T1_3, double *T2_3, double *E4, i64 *diis_iters);

/* J^(2) / J^(3) intermediates (src/EE-CPSd.SF/calJ.f90:6-228) */
typedef struct {
    double *J2_Foo, *J2_Fvv, *J2_Wovvo, *J2_Wovoo;
    double *J3_Foo, *J3_Fvv, *J3_Wovvo;
} o_jints;
int o_calJ(const o_system *s, const o_integrals *I, const double *T2_1,
           const double *T1_2, const double *T2_2, o_jints *J);

/* One root of EE-CPS(D-3) (src/EE-CPSd.SF/run.f90:86-107, run_order.f90):
 * orders 1..3 for CIS (w0, L = R1^CIS) of irrep symR.  Outputs
 * w[0..2] = w^(1), w^(2), w^(3); optionally R1_2 (R1^(2)), R2_1, R2_2. */
int o_eecpsd_root(const o_system *s, const o_integrals *I, const o_params *p,
                  const double *T2_1, const o_jints *J, i64 symR, double w0,
                  const double *L, double *w, double *R2_1, double *R1_2,
                  double *R2_2, i64 *solver_iters);

/* Full pipeline: CIS + ground + J + every root, the metric's unit of work */
int o_sfcpsd_pipeline(const o_system *s, const o_integrals *I, const o_params *p,
                      double *omega_cis, double *w2, double *w3, i64 *nroots_out);

/* set OpenBLAS / OpenMP threads used by the oracle */
void o_set_threads(i64 n);

#ifdef __cplusplus
}
#endif
#endif
