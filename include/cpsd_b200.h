/*
 * cpsd_b200 — C-ABI of the B200-native SF-CIS / SF-CPS(D-3) hot path.
 *
 * Drop-in for the reference's GPU path of libsrint / lib_cc
 * (lishun-1208/revised-cluster-perturbation-single-double): every entry
 * point takes DEVICE pointers (the reference's igpu=1 contract,
 * src/libsrint/vv2v_dpd_444.f90:45-46), int64 integers (the reference is
 * built with -i8, src/make.config:110), 1-based irreps and the DPD layout
 * of src/libsrint/irpdso.f / isymoffso.f / idsymsoc.f.  Errors are returned
 * as negative codes instead of the reference's STOP; cpsd_last_error()
 * gives the message.  All work is queued on the stream set with
 * cpsd_set_stream (default: the legacy default stream); entry points that
 * return host scalars synchronise that stream.
 */
#ifndef CPSD_B200_H
#define CPSD_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CPSD_OK 0
#define CPSD_EARG (-1)    /* invalid argument / index specification */
#define CPSD_ELAYOUT (-2) /* packed pair not intact, population mismatch */
#define CPSD_EMEM (-3)    /* device allocation failed */
#define CPSD_ECUDA (-4)   /* CUDA runtime error */
#define CPSD_ESTATE (-5)  /* library not initialised */
#define CPSD_ENUM (-6)    /* numerical failure: an eigen-solve did not converge */
#define CPSD_ETIMEOUT (-7) /* a bounded device wait (int8-digit path) timed out; results invalid */

/* ------------------------------------------------------------------ setup */
/* Symmetry tables; replaces module mod_symm (src/lib_mod/mod_symm.f:1-9) as
 * filled by readmodule (src/lib_cc/readmodule.f90:23-27).  dirprd is the
 * column-major 8x8 DIRPRD table, dirprd[(j-1)*8+(i-1)] = DIRPRD(i,j). */
int cpsd_init(int64_t nirrep, const int64_t *dirprd);
/* cudaStream_t to queue work on (NULL = legacy default stream) */
int cpsd_set_stream(void *stream);
/* Caller-owned device scratch for expansions / split-K partials.  Without
 * it the library allocates (cudaMalloc) its own and grows it on demand. */
int cpsd_set_workspace(void *dev_ptr, size_t bytes);
/* bytes of scratch the last operations needed (high-water mark) */
size_t cpsd_workspace_high_water(void);
const char *cpsd_last_error(void);
/* number of kernels this library launched since cpsd_init / last reset */
int64_t cpsd_launch_count(int reset);
/* useful contraction flops (2*M*N*K over the irrep blocks) issued since
 * the last reset */
double cpsd_flop_count(int reset);
/* CUDA-event timing of every contraction-kernel launch on its stream
 * (off by default); cpsd_contract_time synchronises the recorded events
 * and returns total milliseconds, launches and useful flops. */
int cpsd_contract_timing(int enable);
int cpsd_contract_time(double *ms, int64_t *launches, double *flops, int reset);
/* Sliced-integer tensor-core contractions (no counterpart in the
 * reference): contractions of at least min_gflop useful GFLOP whose irrep
 * blocks regroup into dense GEMMs run on the int8 tensor cores with every
 * FP64 operand split into `digits` signed 7-bit digits under a power-of-two
 * scale per row / column, exact int32 sums and an FP64 epilogue; the error
 * per element is below (digits+1) K 128^-digits max|a_row| max|b_col|.
 * digits = 0 (default) keeps the FP64 tensor-pipe path everywhere.
 * cpsd_mixed_error returns 1 if a wait in that path timed out since the
 * last reset; cpsd_cis_run, cpsd_cisdoo_run, cpsd_ground, cpsd_ground3,
 * cpsd_eecpsd_roots and so
 * cpsd_pipeline / cpsd_pipeline_batch check it themselves and return
 * CPSD_ETIMEOUT instead of results. */
int cpsd_set_mixed(int digits, double min_gflop);
int cpsd_mixed_error(int reset);
/* Davidson subspace problem (src/lib_cc/mod_davidson.f90:185-219, dgeev on
 * the Ritz matrix Abar): a step whose Abar is symmetric to 1e-12 of its
 * largest element takes the parallel Jacobi on the symmetric part (same
 * eigenpairs to rounding); any other takes the general Hessenberg + Francis
 * QR solve.  Counts, for the calling thread since the last reset, of steps
 * that took the general solve and of Ritz values with an imaginary part
 * above 1e-10 (the reference prints a warning for each; their real parts
 * are used, as there). */
int cpsd_davidson_stats(int64_t *nonsym_steps, int64_t *imag_warnings, int reset);
/* bytes of each of the two device staging buffers through which a
 * host-resident abcd is streamed (default 1 GiB; no counterpart in the
 * reference, which sizes its row blocks by the free iCore) */
int cpsd_set_host_panel_bytes(size_t bytes);

/* -------------------------------------------------------------- size math */
/* irpdso (src/libsrint/irpdso.f:1-52) */
int64_t cpsd_irpdso(int64_t sym, const int64_t *popp, const int64_t *popq, int64_t ioppq);
/* idsymsoc (src/libsrint/idsymsoc.f:1-30) */
int64_t cpsd_idsymsoc(int64_t irrepx, const int64_t *popp, const int64_t *popq, int64_t ioppq,
                      const int64_t *popr, const int64_t *pops, int64_t ioprs);
/* isymoffso (src/libsrint/isymoffso.f:1-54), 1-based */
int64_t cpsd_isymoffso(int64_t irrepq1, int64_t irrep, const int64_t *popp, const int64_t *popq,
                       int64_t iop);

/* --------------------------------------------------------- DPD engines
 * V3 = fact1 * (V1 (x) V2) + fact2 * V3 over symmetry-allowed elements,
 * arbitrary 4-letter aliases.  fact2 = 0 overwrites V3 without reading it.
 * Packed (iop 0/2) pairs must stay intact (same letters, order and iop in
 * the partner operand), as the reference's dispatcher requires
 * (src/libsrint/vv2v_dpd_444.f90:171-186). */

/* vv2v_dpd_444 (src/libsrint/vv2v_dpd_444.f90:55-72) */
int cpsd_vv2v_dpd_444(const double *v1, const int64_t *p1_1, const int64_t *p1_2, int64_t iop1_12,
                      const int64_t *p1_3, const int64_t *p1_4, int64_t iop1_34, int64_t sym1,
                      const char *type1,
                      const double *v2, const int64_t *p2_1, const int64_t *p2_2, int64_t iop2_12,
                      const int64_t *p2_3, const int64_t *p2_4, int64_t iop2_34, int64_t sym2,
                      const char *type2,
                      double *v3, const int64_t *p3_1, const int64_t *p3_2, int64_t iop3_12,
                      const int64_t *p3_3, const int64_t *p3_4, int64_t iop3_34, int64_t sym3,
                      const char *type3, double fact1, double fact2);
/* vv2v_dpd_424 (src/libsrint/vv2v_dpd_424.f90:21-24): V2 is 2-index */
int cpsd_vv2v_dpd_424(const double *v1, const int64_t *p1_1, const int64_t *p1_2, int64_t iop1_12,
                      const int64_t *p1_3, const int64_t *p1_4, int64_t iop1_34, int64_t sym1,
                      const char *type1,
                      const double *v2, const int64_t *p2_1, const int64_t *p2_2, int64_t iop2_12,
                      int64_t sym2, const char *type2,
                      double *v3, const int64_t *p3_1, const int64_t *p3_2, int64_t iop3_12,
                      const int64_t *p3_3, const int64_t *p3_4, int64_t iop3_34, int64_t sym3,
                      const char *type3, double fact1, double fact2);
/* vv2v_dpd_442 (src/libsrint/vv2v_dpd_442.f90:22-25): V3 is 2-index */
int cpsd_vv2v_dpd_442(const double *v1, const int64_t *p1_1, const int64_t *p1_2, int64_t iop1_12,
                      const int64_t *p1_3, const int64_t *p1_4, int64_t iop1_34, int64_t sym1,
                      const char *type1,
                      const double *v2, const int64_t *p2_1, const int64_t *p2_2, int64_t iop2_12,
                      const int64_t *p2_3, const int64_t *p2_4, int64_t iop2_34, int64_t sym2,
                      const char *type2,
                      double *v3, const int64_t *p3_1, const int64_t *p3_2, int64_t iop3_12,
                      int64_t sym3, const char *type3, double fact1, double fact2);
/* vv2v_dpd_422 (src/libsrint/vv2v_dpd_422.f90:21): V2, V3 2-index */
int cpsd_vv2v_dpd_422(const double *v1, const int64_t *p1_1, const int64_t *p1_2, int64_t iop1_12,
                      const int64_t *p1_3, const int64_t *p1_4, int64_t iop1_34, int64_t sym1,
                      const char *type1,
                      const double *v2, const int64_t *p2_1, const int64_t *p2_2, int64_t iop2_12,
                      int64_t sym2, const char *type2,
                      double *v3, const int64_t *p3_1, const int64_t *p3_2, int64_t iop3_12,
                      int64_t sym3, const char *type3, double fact1, double fact2);
/* vv2v_dpd_222 (src/libsrint/vv2v_dpd_222.f90:19): all 2-index */
int cpsd_vv2v_dpd_222(const double *v1, const int64_t *p1_1, const int64_t *p1_2, int64_t iop1_12,
                      int64_t sym1, const char *type1,
                      const double *v2, const int64_t *p2_1, const int64_t *p2_2, int64_t iop2_12,
                      int64_t sym2, const char *type2,
                      double *v3, const int64_t *p3_1, const int64_t *p3_2, int64_t iop3_12,
                      int64_t sym3, const char *type3, double fact1, double fact2);

/* vv2v_dpd_224 (src/libsrint/vv2v_dpd_224.f90:16-19): V1, V2 2-index, V3
 * 4-index (the outer product V3(pqrs) += fact1 V1(pq) V2(rs)) */
int cpsd_vv2v_dpd_224(const double *v1, const int64_t *p1_1, const int64_t *p1_2, int64_t iop1_12,
                      int64_t sym1, const char *type1,
                      const double *v2, const int64_t *p2_1, const int64_t *p2_2, int64_t iop2_12,
                      int64_t sym2, const char *type2,
                      double *v3, const int64_t *p3_1, const int64_t *p3_2, int64_t iop3_12,
                      const int64_t *p3_3, const int64_t *p3_4, int64_t iop3_34, int64_t sym3,
                      const char *type3, double fact1, double fact2);

/* No counterpart in the reference.  cpsd_vv2v_dpd_444's contraction with
 * the same arguments, for callers that may not allocate device memory
 * during the call (all of HBM handed to their own pool, or no cudaMalloc /
 * cudaFree stalls allowed in a time-critical loop): the contraction's plan
 * tables and split-K partial tiles live in a fixed region compiled into
 * the library, CPSD_NOALLOC_SCRATCH_BYTES (32 MiB) per device, instead of
 * cudaMalloc'ed memory.  It always runs the FP64 tile kernel (k_contract),
 * whatever cpsd_set_mixed selected and whether or not cpsd_vv2v_dpd_444
 * would take its narrow-output kernels: results equal cpsd_vv2v_dpd_444's
 * in FP64 mode to rounding, and differ from its mixed-mode results by that
 * mode's digit error.  A contraction that needs more than the region is
 * rejected with CPSD_EARG before any work is queued.  Nothing in the
 * region has to start at zero.  The region is shared by all calls on a
 * device: calls queued on one stream are ordered, calls that overlap in
 * time (other streams, other host threads) race.  The plan tables are
 * copied from pageable host memory, which CUDA starts only after the work
 * queued earlier on the stream: a call can block the host until then.  The
 * first call on each device does the set-up (region address, kernel
 * attributes); make it before any stream capture begins. */
#define CPSD_NOALLOC_SCRATCH_BYTES (32u << 20)
int cpsd_vv2v_dpd_444_noalloc(const double *v1, const int64_t *p1_1, const int64_t *p1_2, int64_t iop1_12,
                              const int64_t *p1_3, const int64_t *p1_4, int64_t iop1_34, int64_t sym1,
                              const char *type1,
                              const double *v2, const int64_t *p2_1, const int64_t *p2_2, int64_t iop2_12,
                              const int64_t *p2_3, const int64_t *p2_4, int64_t iop2_34, int64_t sym2,
                              const char *type2,
                              double *v3, const int64_t *p3_1, const int64_t *p3_2, int64_t iop3_12,
                              const int64_t *p3_3, const int64_t *p3_4, int64_t iop3_34, int64_t sym3,
                              const char *type3, double fact1, double fact2);

/* Fortran-callable binding of the same engine (gfortran/nvfortran ABI:
 * lower case + trailing underscore, every argument by reference, hidden
 * character lengths last), so the reference's call sites
 * (src/lib_cc/mod_contract.f90:104-107) link against it unchanged when
 * igpu=1 and prec=8.  Like the reference's dispatcher, which STOPs on a
 * failed check (src/libsrint/vv2v_dpd_444.f90:150-200), it prints the
 * error and ends the program (exit status 1) when the call fails.
 * vv2v_dpd_444_ierr_ (no counterpart in the reference) takes one more
 * integer, ierr, after fact2 and returns the code there instead. */
void vv2v_dpd_444_(const double *v1, const int64_t *p1_1, const int64_t *p1_2, const int64_t *iop1_12,
                   const int64_t *p1_3, const int64_t *p1_4, const int64_t *iop1_34, const int64_t *sym1,
                   const char *type1,
                   const double *v2, const int64_t *p2_1, const int64_t *p2_2, const int64_t *iop2_12,
                   const int64_t *p2_3, const int64_t *p2_4, const int64_t *iop2_34, const int64_t *sym2,
                   const char *type2,
                   double *v3, const int64_t *p3_1, const int64_t *p3_2, const int64_t *iop3_12,
                   const int64_t *p3_3, const int64_t *p3_4, const int64_t *iop3_34, const int64_t *sym3,
                   const char *type3, const double *fact1, const double *fact2,
                   size_t len_type1, size_t len_type2, size_t len_type3);
void vv2v_dpd_444_ierr_(const double *v1, const int64_t *p1_1, const int64_t *p1_2, const int64_t *iop1_12,
                        const int64_t *p1_3, const int64_t *p1_4, const int64_t *iop1_34, const int64_t *sym1,
                        const char *type1,
                        const double *v2, const int64_t *p2_1, const int64_t *p2_2, const int64_t *iop2_12,
                        const int64_t *p2_3, const int64_t *p2_4, const int64_t *iop2_34, const int64_t *sym2,
                        const char *type2,
                        double *v3, const int64_t *p3_1, const int64_t *p3_2, const int64_t *iop3_12,
                        const int64_t *p3_3, const int64_t *p3_4, const int64_t *iop3_34, const int64_t *sym3,
                        const char *type3, const double *fact1, const double *fact2, int64_t *ierr,
                        size_t len_type1, size_t len_type2, size_t len_type3);

/* ------------------------------------------------- tensor descriptor
 * POD mirror of type(opt) (src/lib_cc/mod_operator.f90:8-25): populations,
 * iops, irrep, length (filled by cpsd_opt_init) and a device array. */
typedef struct {
    int64_t popp[8], popq[8], popr[8], pops[8];
    int64_t ioppq, ioprs;
    int64_t sym;
    int64_t len;
    double *arr;
} cpsd_opt;

/* init_opt (src/lib_cc/mod_operator.f90:70-115): fills len */
int cpsd_opt_init(cpsd_opt *t, const int64_t *popp, const int64_t *popq, const int64_t *popr,
                  const int64_t *pops, int64_t ioppq, int64_t ioprs, int64_t sym, double *dev_arr);

/* layout transforms on cpsd_opt (device arrays), out described by its own
 * cpsd_opt: iexpso (src/libsrint/iexpso.f90:24-120), icompso
 * (src/libsrint/icompso.f:1-80; c = 1 keeps a pair), isymtrso
 * (src/libsrint/isymtrso.f:1-351). */
int cpsd_iexpso(const cpsd_opt *in, cpsd_opt *out, int64_t exppq, int64_t exprs);
int cpsd_icompso(const cpsd_opt *in, cpsd_opt *out, int64_t cpq, int64_t crs);
int cpsd_isymtrso(const cpsd_opt *in, cpsd_opt *out, int64_t swpq, int64_t swrs);

/* mod_contract wrappers (src/lib_cc/mod_contract.f90:10-455):
 * v3 += fact * P{v1 * v2}; anti 0/1/2/3 antisymmetrises none / 1st / 2nd /
 * both pairs of v3.  2-index operands carry popr = pops = (1,0,...). */
int cpsd_vv2v_444(const cpsd_opt *v1, const cpsd_opt *v2, cpsd_opt *v3, double fact,
                  const char *t1, const char *t2, const char *t3, int64_t anti);
int cpsd_vv2v_424(const cpsd_opt *v1, const cpsd_opt *v2, cpsd_opt *v3, double fact,
                  const char *t1, const char *t2, const char *t3, int64_t anti);
int cpsd_vv2v_442(const cpsd_opt *v1, const cpsd_opt *v2, cpsd_opt *v3, double fact,
                  const char *t1, const char *t2, const char *t3);
int cpsd_vv2v_422(const cpsd_opt *v1, const cpsd_opt *v2, cpsd_opt *v3, double fact,
                  const char *t1, const char *t2, const char *t3);
int cpsd_vv2v_222(const cpsd_opt *v1, const cpsd_opt *v2, cpsd_opt *v3, double fact,
                  const char *t1, const char *t2, const char *t3);
int cpsd_vv2v_224(const cpsd_opt *v1, const cpsd_opt *v2, cpsd_opt *v3, double fact,
                  const char *t1, const char *t2, const char *t3, int64_t anti);

/* ---------------------------------------- spin-free lib_cc kernels
 * out += fact * kernel(a, b); each replaces the subroutine of the same name
 * in src/lib_cc/<name>.f90 (plain spin-free variant). */
#define CPSD_KERNEL(name) int cpsd_##name(cpsd_opt *out, const cpsd_opt *a, const cpsd_opt *b, double fact)
CPSD_KERNEL(c1_r1iabj);  /* c1_r1iabj.f90:3   c(a,i) += r(f,n) V(fn,ai)        */
CPSD_KERNEL(c1_r1Fae);   /* c1_r1Fae.f90:3    c(a,i) += r(e,i) F(a,e)          */
CPSD_KERNEL(c1_r1Fmi);   /* c1_r1Fmi.f90:3    c(a,i) -= r(a,m) F(m,i)          */
CPSD_KERNEL(c1_r2abci);  /* c1_r2abci.f90:3   c(a,i) += .5 r(fe,im) V(fe,am)   */
CPSD_KERNEL(c1_r2ijka);  /* c1_r2ijka.f90:3   c(a,i) -= .5 r(ae,mn) V(mn,ie)   */
CPSD_KERNEL(c2_r1abci);  /* c2_r1abci.f90:3   c(ab,ij) += P(ij) r(e,i) V(ab,ej) */
CPSD_KERNEL(c2_r1ijka);  /* c2_r1ijka.f90:3   c(ab,ij) -= P(ab) r(a,m) V(ij,mb) */
CPSD_KERNEL(c2_r2Wmbej); /* c2_r2Wmbej.f90:3  c(ab,ij) += P(ab|ij) r(ae,im) W(em,bj) */
CPSD_KERNEL(c2_r2Wmnij); /* c2_r2Wmnij.f90:3  c(ab,ij) += .5 r(ab,mn) W(mn,ij) */
CPSD_KERNEL(c2_r2abcd);  /* c2_r2abcd.f90:3   c(ab,ij) += .5 r(ef,ij) V(ab,ef) */
CPSD_KERNEL(c2_r2Fae);   /* c2_r2Fae.f90:3    c(ab,ij) += P(ab) r(ae,ij) F(b,e) */
CPSD_KERNEL(c2_r2Fmi);   /* c2_r2Fmi.f90:3    c(ab,ij) -= P(ij) r(ab,im) F(m,j) */
CPSD_KERNEL(Fmi_r2abij); /* Fmi_r2abij.f90:3  F(m,i) += .5 r(ef,in) V(ef,mn)   */
CPSD_KERNEL(Fae_r2abij); /* Fae_r2abij.f90:3  F(a,e) -= .5 r(af,mn) V(ef,mn)   */
CPSD_KERNEL(Fmi_r1ijka); /* Fmi_r1ijka.f90:3  F(m,i) += r(e,n) V(mn,ie)        */
CPSD_KERNEL(Fae_r1abci); /* Fae_r1abci.f90:3  F(a,e) += r(f,m) V(ef,am)        */
CPSD_KERNEL(Wkbij_r2ijka); /* Wkbij_r2ijka.f90:3 W(ij,kb) += P(ij) V(kl,ic) r(bc,jl) */
CPSD_KERNEL(Wkbij_r2abci); /* Wkbij_r2abci.f90:3 W(ij,kb) += .5 V(dc,bk) r(cd,ij)   */
CPSD_KERNEL(Wmbej_r2abij); /* Wmbej_r2abij.f90:3 W(em,bj) += .5 r(bf,jn) V(fe,nm)   */
CPSD_KERNEL(Wmbej_r1abci); /* Wmbej_r1abci.f90:3 W(em,bj) += r(f,j) V(fe,bm)        */
CPSD_KERNEL(Wmbej_r1ijka); /* Wmbej_r1ijka.f90:3 W(em,bj) -= r(b,n) V(nm,je)        */
CPSD_KERNEL(Wmnij_r1ijka); /* Wmnij_r1ijka.f90:3 W(mn,ij) += P(ij) r(e,j) V(mn,ie)  */
CPSD_KERNEL(Wmnij_r2abij); /* Wmnij_r2abij.f90:1 W(mn,ij) += .5 V(ef,mn) r(ef,ij)   */
/* the second-order ground state's (src/grCPSd.SF/calL1_VTT.f90, calL2_VTT.f90) */
CPSD_KERNEL(Wkbij_r1iabj);  /* Wkbij_r1iabj.f90:1  W(ij,kb) -= P(ij) V(ck,bj) r(c,i) */
CPSD_KERNEL(Wabdj_r1abcd);  /* Wabdj_r1abcd.f90:1  W(ab,dj) += V(ab,dc) r(c,j)       */
CPSD_KERNEL(Wkbij_r1Uklij); /* Wkbij_r1Uklij.f90:1 W(ij,kb) -= U(kl,ij) r(b,l)       */
CPSD_KERNEL(Fme_r1abij);    /* Fme_r1abij.f90:1    F(e,m) += r(f,n) V(ef,mn)         */
CPSD_KERNEL(c1_r2Fme);      /* c1_r2Fme.f90:1      c(a,i) += r(ae,im) F(e,m)         */
/* the excited-state grCPS(D)'s (src/EE-grCPSd.SF/calEigenCISDoo.f90, calJ.f90, calC_VTTR.f90) */
CPSD_KERNEL(c1d_l1Wibaj);   /* c1d_l1Wibaj.f90:1 c(a,i) += W(ai,bj) l(b,j) */
CPSD_KERNEL(c1d_l1fab);     /* c1d_l1fab.f90:1 c(a,i) -= f(b,a) l(b,i) */
CPSD_KERNEL(c1d_l1fij);     /* c1d_l1fij.f90:1 c(a,i) += f(i,j) l(a,j) */
CPSD_KERNEL(Fae_r1fia);     /* Fae_r1fia.f90:1 F(a,e) -= f(e,l) r(a,l) */
CPSD_KERNEL(Fmi_r1fia);     /* Fmi_r1fia.f90:1 F(m,i) += r(d,i) f(d,m) */
CPSD_KERNEL(Wkbij_r2Fkc);   /* Wkbij_r2Fkc.f90:1 W(ij,kb) -= F(c,k) r(cb,ij) */
CPSD_KERNEL(Wlkjd_r1abij);  /* Wlkjd_r1abij.f90:1 W(lk,jd) += r(c,j) V(cd,lk) */
#undef CPSD_KERNEL

/* --------------------------------------------- planner introspection
 * Host-only (no GPU needed; no counterpart in the reference): the tables
 * the planner builds for a contraction / pair transform, for verification
 * tools.  Layouts are TaskDev / SegDev / TileDev / PMBlockDev of
 * csrc/runtime.hpp; pointers stay valid for the life of the process.
 * op codes: 0 copy, 1 expand, 2 compress, 3 antisymmetrise,
 * 4 antisymmetrise+compress, 5 swap. */
int cpsd_debug_contract_plan(const cpsd_opt *v1, const char *t1, const cpsd_opt *v2, const char *t2,
                             const cpsd_opt *v3, const char *t3, int64_t nb, int64_t sA, int64_t sB, int64_t sC,
                             const void **tasks, int64_t *ntasks, const void **segs, int64_t *nsegs,
                             const void **tiles, int64_t *ntiles, int64_t *tile_bm, int64_t *tile_bn);
/* per-launch records of the contraction timing buffer: milliseconds,
 * useful flops and (tasks, segments, tiles, tile shape) */
int cpsd_contract_records(double *ms, double *flops, int64_t *shape, int64_t maxrec, int64_t *nrec);
/* work items of the narrow-output kernels for a contraction (layouts
 * NarrowItem / NarrowRed of csrc/narrow.cuh); flags[5] = {narrow, rows over
 * the second operand, lanes over K, partial slots, columns per long-K item
 * (its rows: 32 / columns)}; items = NULL when the contraction runs on the
 * tensor-core tiles instead */
int cpsd_debug_narrow_plan(const cpsd_opt *v1, const char *t1, const cpsd_opt *v2, const char *t2,
                           const cpsd_opt *v3, const char *t3, int64_t nb, int64_t sA, int64_t sB, int64_t sC,
                           const void **items, int64_t *nitems, const void **reds, int64_t *nreds, int64_t *flags);
/* work items of the row-dot kernel for a contraction (layout RowDotItem of
 * csrc/rowdot.cuh) and the task / segment tables it reads (the plan's,
 * row units reordered by stride); flags = {row-dot, rows over N, K / 32
 * rounded up, columns per item rounded up}; items = NULL when it does not
 * qualify */
int cpsd_debug_rowdot_plan(const cpsd_opt *v1, const char *t1, const cpsd_opt *v2, const char *t2,
                           const cpsd_opt *v3, const char *t3, int64_t nb, int64_t sA, int64_t sB, int64_t sC,
                           const void **items, int64_t *nitems, const void **tasks, const void **segs,
                           int64_t *flags);
/* work items of the short-K kernel for a contraction (layout ShortKItem of
 * csrc/shortk.cuh); flags = {short-K, f runs along M, tile extent BS along
 * the other side, largest contracted range}; items = NULL when it does not
 * qualify */
int cpsd_debug_shortk_plan(const cpsd_opt *v1, const char *t1, const cpsd_opt *v2, const char *t2,
                           const cpsd_opt *v3, const char *t3, int64_t nb, int64_t sA, int64_t sB, int64_t sC,
                           const void **items, int64_t *nitems, int64_t *flags);
/* tables of the sliced-integer plan of a contraction (layouts OzGroup,
 * OzTile, OzSliceJob of csrc/ozaki.cuh): tables[0..12] = groups, tiles,
 * A jobs, B jobs, A row / K offsets, B row / K offsets, C row / column
 * offsets, M / N / K combination ids, sizes[0..12] their counts;
 * sizes[13..19] = A digit bytes, B digit bytes, A / B exponents, K stages
 * per launch, most K stages, B tile width; tables[20..21] = the A / B
 * OzStage tables (affine K stages), sizes[20..21] their counts.  Both
 * arrays hold 22 entries.  tables[0] = NULL when the contraction does not
 * regroup into dense GEMMs. */
int cpsd_debug_ozaki_plan(const cpsd_opt *v1, const char *t1, const cpsd_opt *v2, const char *t2,
                          const cpsd_opt *v3, const char *t3, int64_t nb, int64_t sA, int64_t sB, int64_t sC,
                          int digits, const void **tables, int64_t *sizes);
/* the Davidson step's general eigen-solve (one warp, n <= 32) on the
 * row-major n x n host matrix A: eigenvalues wr / wi and row-major V whose
 * columns are dgeev's right eigenvectors (a complex pair k, k+1 with
 * wi[k] > 0: real and imaginary parts; unit norm, largest component real);
 * *sweeps = QR sweeps or -1 when the iteration did not converge */
int cpsd_debug_geev(const double *A_host, int64_t n, double *wr, double *wi, double *V_host, int64_t *sweeps);
int cpsd_debug_pairmap_plan(const cpsd_opt *in, int64_t op0, int64_t op1, int64_t tgt0, int64_t tgt1,
                            const void **blocks, int64_t *nblocks, const void **idx, const void **sgn,
                            int64_t *nidx, int64_t *lterms, int64_t *rterms);

/* -------------------------------------------------- molecular programs */
typedef struct {
    int64_t nirrep;
    int64_t dirprd[64];
    int64_t symry;
    int64_t popa[8], popb[8], vrta[8], vrtb[8];
} cpsd_system;

/* spin-free integrals in DPD layout, iop 0 on antisymmetric pairs, device
 * pointers (allocate_mem, src/EE-CPSd.SF/allocate_mem.f90:14-44).  abcd
 * may instead be host memory, for systems whose abcd does not fit in HBM
 * (the reference keeps it on disk then, vvvv_incore = .false.,
 * allocate_mem.f90:38-43): the particle ladder then streams it through two
 * device staging buffers (cpsd_set_host_panel_bytes), FP64 also in the
 * mixed mode; pinned host memory (cudaHostAlloc / cudaHostRegister) keeps
 * the copies at full link speed. */
typedef struct {
    const double *ijkl, *ijka, *abij, *iabj, *abci, *abcd;
    const double *eorb; /* spin-free orbital energies (src/getHF/resortEorb.f90) */
} cpsd_integrals;

typedef struct {
    int64_t davidson_dim, davidson_cyc, davidson_conv, lowest; /* mod_common.f90:37-40 */
    int64_t diis_dim, diis_cyc;                                 /* mod_common.f90:17-18 */
    double diis_max_err;                                        /* mod_common.f90:20 */
    int64_t spin_flip;  /* 0 none, 1 "ab", 2 "ba" (preDavidson.f90:64-95) */
    int64_t open_shell; /* shell=open */
    int64_t ex_mult;
    int64_t estate_sym[8];
    int64_t batch_roots; /* 1: the roots of one irrep share each contraction launch */
} cpsd_params;

void cpsd_params_default(cpsd_params *p);

/* SF-CIS (src/EE-CIS.SF/run.f90:2-100): omega_host[k] and the unit-norm
 * R1 of every requested root (irrep 1 first) into R_dev (device). */
int cpsd_cis_run(const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p,
                 double *omega_host, double *R_dev, int64_t *iterations);

/* CIS(D-infinity) (src/CISdoo.SD.SF/run.f90:25-110, calAR.f90:19-49): the
 * (R1, R2) eigenproblem with the MP2-dressed Fac, Fki and Wkaci; per
 * requested root omega_host[k] and its unit-norm R1 then R2 (lengths
 * irpdso(sym,v,o) and idsymsoc(sym,v,v,0,o,o,0) of its irrep) into R_dev
 * (device), irrep 1 first.  The matrix is not symmetric: the Ritz steps
 * take the general eigen-solve (cpsd_davidson_stats counts them). */
int cpsd_cisdoo_run(const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p,
                    double *omega_host, double *R_dev, int64_t *iterations);

/* grCPS(D) ground state (src/grCPSd.SF/run.f90): orders k = 1..3 of the
 * coupled (T1, T2) equations with the MP2-dressed Fli, Fad, Wkaci and their
 * DIIS loops (solver.f90).  T_dev (device) receives per order T1 (l1 =
 * irpdso(1,v,o)) then T2 (l2 = idsymsoc(1,v,v,0,o,o,0)); E_host[k-1] =
 * E^(k+1) of calEcorr.f90; iters[k-1] the DIIS iterations of order k. */
int cpsd_grcpsd_ground(const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p, double *T_dev,
                       double *E_host, int64_t *iters);

/* excited-state grCPS(D) (src/EE-grCPSd.SF/run.f90) from the grCPS(D)
 * amplitudes T_dev (cpsd_grcpsd_ground's layout; orders 1, 2 used) and the
 * CIS(D-infinity) roots (omega_host, R0_dev in cpsd_cisdoo_run's layout):
 * per root k the left vector (calEigenCISDoo.f90) and w_host[3k..3k+2] =
 * w^(1), w^(2), w^(3); L_dev (nullable) receives the left vectors (R0's
 * layout, <L|R0> = 1), R_dev (nullable) R^(1) of every root then R^(2);
 * iterations = DIIS iterations summed. */
int cpsd_eegrcpsd_roots(const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p, const double *T_dev,
                        const double *omega_host, const double *R0_dev, double *w_host, double *L_dev, double *R_dev,
                        int64_t *iterations);

/* The spin-free DPD lists as a linear function of the spatial integrals
 * (pq|rs), and its adjoint (no counterpart in the reference, whose lists
 * come from src/pyscf2cc/py2cc.py).  orb_mo / orb_spin (host, one entry per
 * spin-free orbital in the lists' order: occupied orbitals of irreps 1..n,
 * then virtual ones) give each orbital's spatial index (< nmo) and spin
 * (0 alpha, 1 beta); a list element is <PQ||RS> = [sP=sR, sQ=sS] (PR|QS) -
 * [sP=sS, sQ=sR] (PS|QR), iabj(b,i,a,j) = <ia||bj>.  The dense (pq|rs) array
 * is nmo^4 doubles on the device, (pr|qs) at ((p*nmo + r)*nmo + q)*nmo + s.
 * cpsd_eri_lists fills every non-NULL list of `lists` (device, irrep 1);
 * cpsd_eri_adjoint adds d/d(pq|rs) of sum_e g(e) list(e) over the non-NULL
 * lists g of `grads` into geri_dev (atomic adds: the last bits vary). */
int cpsd_eri_lists(const cpsd_system *s, const int64_t *orb_mo, const int64_t *orb_spin, int64_t nmo,
                   const double *eri_dev, const cpsd_integrals *lists);
int cpsd_eri_adjoint(const cpsd_system *s, const int64_t *orb_mo, const int64_t *orb_spin, int64_t nmo,
                     const cpsd_integrals *grads, double *geri_dev);

/* ground CPS(D) T^(1), T^(2) (src/CPSd.SF/run1.f90, run2.f90); device outputs */
int cpsd_ground(const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p,
                double *T2_1, double *T1_2, double *T2_2, double *E2_host, double *E3_host,
                int64_t *diis_iters);

/* ground CPS(D) third order T^(3) and E^(4) (src/CPSd.SF/run3.f90:8-97)
 * from T2^(1), T1^(2), T2^(2) of cpsd_ground; device in- and outputs,
 * E^(4) on the host */
int cpsd_ground3(const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p, const double *T2_1,
                 const double *T1_2, const double *T2_2, double *T1_3, double *T2_3, double *E4_host,
                 int64_t *diis_iters);

/* J^(2) / J^(3) intermediates (src/EE-CPSd.SF/calJ.f90:6-228); device */
typedef struct {
    double *J2_Foo, *J2_Fvv, *J2_Wovvo, *J2_Wovoo;
    double *J3_Foo, *J3_Fvv, *J3_Wovvo;
} cpsd_jints;
int cpsd_calJ(const cpsd_system *s, const cpsd_integrals *I, const double *T2_1,
              const double *T1_2, const double *T2_2, cpsd_jints *J);

/* EE-CPS(D-3) orders 1..3 (src/EE-CPSd.SF/run.f90:86-107, run_order.f90)
 * for nroot roots of irrep symR with CIS energies w0_host[k] and CIS
 * vectors L_dev (nroot x lenR1, device).  w_host[3k..3k+2] = w^(1..3).
 * Optional device outputs (NULL to skip): R2_1, R1_2, R2_2 per root. */
int cpsd_eecpsd_roots(const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p,
                      const double *T2_1, const cpsd_jints *J, int64_t symR, int64_t nroot,
                      const double *w0_host, const double *L_dev, double *w_host,
                      double *R2_1, double *R1_2, double *R2_2, int64_t *solver_iters);

/* The whole SF-CIS + SF-CPS(D-3) pipeline: one step of the roots/s metric.
 * Integrals are device pointers; outputs on the host.  By default the
 * SF-CIS Davidson and the ground state + J^(2)/J^(3) run at once on two
 * library worker threads (own streams), then the excited orders; results
 * equal the sequential order's.  The sequential order is used inside
 * cpsd_pipeline_batch workers, while per-launch timing is on and when the
 * integrals take a fifth of the device memory or more. */
int cpsd_pipeline(const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p,
                  double *omega_cis, double *w2, double *w3, int64_t *nroots);
/* on = 0: run the pipeline's phases one after the other on the caller's
 * stream (default 1: SF-CIS beside the ground state) */
int cpsd_set_phase_overlap(int on);
/* Empirical tile-shape choice for the FP64 tile kernel (off by default):
 * with it on, the first launch of each contraction plan runs its four tile
 * shapes (128x64, 128x32, 64x128, 64x64) on a scratch copy of the output,
 * times them with CUDA events and keeps the fastest (the cost model's shape
 * unless another is 3 % faster) for every later launch of that plan.  The
 * sums of different shapes differ in rounding, and the choice can differ
 * from run to run.  cpsd_tile_autotune_stats: plans tuned, plans whose
 * shape the tuning changed, since the process started. */
int cpsd_set_tile_autotune(int on);
int cpsd_tile_autotune_stats(int64_t *tuned, int64_t *changed);

/* Independent molecules in one call (no counterpart in the reference, which
 * runs one molecule per program invocation): cpsd_pipeline of molecule m
 * with s[m], I[m], p[m] (each with its own nirrep / populations), run by
 * nworkers (1..64) persistent host threads, each with its own CUDA stream
 * and library state, largest molecules first; the batch starts after the
 * work queued so far on the calling thread's stream and the call returns
 * when every molecule is done.  Roots go to omega_cis / w2 / w3 in molecule
 * order (molecule m's roots start after those of molecules 0..m-1);
 * *nroots = their total.  The mixed-precision setting of the calling thread
 * applies to every molecule.  The first failing molecule's error is
 * returned (the remaining ones are not started). */
int cpsd_pipeline_batch(int64_t nmol, const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p,
                        int64_t nworkers, double *omega_cis, double *w2, double *w3, int64_t *nroots);

/* Gives back device memory the library keeps between calls: the idle
 * buffers of its constant-operand copies and the calling thread's scratch
 * arena (batch workers free theirs at the end of every batch).  Later
 * calls allocate again as needed. */
int cpsd_release_device_cache(void);

/* ------------------------------------------ the reference's input files
 * Host-side readers (and writers) of the files the reference's programs
 * read their input from; no GPU is needed.  The files are those of its
 * gfortran / nvfortran builds with 8-byte default integers: sequential
 * records framed by 4-byte length markers, 32768-byte direct-access records.
 *
 * DPD list `<dir>/<name>` + `<dir>/<name>.c` (clmoioso0.f:30-67 writes the
 * sidecar; getallso_d.f:31-79 / getlstso.f:50-125 read the data): the
 * sidecar's records, Fortran (10, 20) arrays as [list - 1][irrep - 1]. */
typedef struct {
    int64_t irrepx;
    int64_t popp[8], popq[8], popr[8], pops[8];
    int64_t ioppq[8], ioprs[8], irrepr[8], irrepi[8];
    int64_t moionuml[20][10], moionumr[20][10], rectmp[20][10];
} cpsd_dpd_list_meta;
int cpsd_dpd_list_meta_read(const char *dir, const char *name, cpsd_dpd_list_meta *m);
/* getallso(z, 1, name): list 1, all irrep blocks, into host[0..len) (len
 * must equal the list's DPD length); needs cpsd_init for the symmetry */
int cpsd_dpd_list_read(const char *dir, const char *name, double *host, int64_t len);
/* clmoioso0 + putlstso of list 1: writes a whole DPD tensor (host) */
int cpsd_dpd_list_write(const char *dir, const char *name, int64_t irrepx, const int64_t *popp, const int64_t *popq,
                        int64_t ioppq, const int64_t *popr, const int64_t *pops, int64_t ioprs, const double *host);
/* the "interface" node file (src/pyscf2cc/mod_interface.f90): stream file,
 * header (table position, node count), data, table of 36-byte nodes (name
 * blank-padded to 20 lower-case characters, 1-based byte position, byte
 * size).  read_node: the node's size must equal `bytes`; add_node: a new
 * node's data goes where the table was, the table behind it. */
int cpsd_interface_size(const char *path, const char *node, int64_t *bytes);
int cpsd_interface_read(const char *path, const char *node, void *out, int64_t bytes);
int cpsd_interface_write(const char *path, const char *node, const void *data, int64_t bytes);
/* readmodule (src/lib_cc/readmodule.f90:17-40): symry, dirprd, nirrep and
 * the (8, 2) pop / vrt nodes into a cpsd_system */
int cpsd_load_system(const char *interface_path, cpsd_system *s);
/* loadSCF (src/EE-CPSd.SF/loadSCF.f90:13-48): the spin-free orbital
 * energies ('orb_energy_no_spin') and the six integral lists 'ijkl_ns_' ...
 * 'abcd_ns_' (src/EE-CPSd.SF/mod_variable.f90:37-47, layouts of
 * allocate_mem.f90:22-43) into host arrays of the cpsd_integrals layouts
 * (NULL skips one); dir NULL reads the interface's 'tmpdir' node (else the
 * current directory).  Populations and iops are checked against s. */
int cpsd_load_inputs(const char *dir, const char *interface_path, const cpsd_system *s, double *ijkl, double *ijka,
                     double *abij, double *iabj, double *abci, double *abcd, double *eorb);

/* -------------------------------------------- SF-CIS(D) energy gradient
 * No counterpart in the reference (it has no derivative code).
 *
 * cpsd_cisd_energies: the SF-CIS roots of irrep symR (Davidson as in
 * cpsd_cis_run, roots requested only in symR) and their second-order
 * corrections w^(2) (src/EE-CPSd.SF/run_order.f90 order 2, the same terms
 * as cpsd_eecpsd_roots).  w0_host[k], w2_host[k] per root; the unit CIS
 * vectors go to L_dev (nroot x lenR1, device).  ijkl and abcd are not read.
 *
 * cpsd_cisd_gradient: ADDS to G the gradient of
 *     sum_k g0_host[k] w0_k + g2_host[k] w2_k
 * with respect to the DPD integral tensors (same layouts as cpsd_integrals)
 * and Eorb, at the roots w0_host / L_dev of cpsd_cisd_energies.  The doubles
 * amplitudes are recomputed; the CIS vector response is one Z-vector solve
 * by the solver of solver.f90 (p->diis_dim / diis_cyc / diis_max_err; its
 * tolerance bounds the gradient's accuracy).  ijkl and abcd do not enter
 * w0 / w^(2): G->ijkl and G->abcd are not written and may be NULL.
 * Contractions run in FP64 whatever cpsd_set_mixed selected. */
typedef struct {
    double *ijkl, *ijka, *abij, *iabj, *abci, *abcd;
    double *eorb;
} cpsd_integral_grads;
int cpsd_cisd_energies(const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p,
                       int64_t symR, int64_t nroot, double *w0_host, double *w2_host, double *L_dev);
int cpsd_cisd_gradient(const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p,
                       int64_t symR, int64_t nroot, const double *w0_host, const double *L_dev,
                       const double *g0_host, const double *g2_host, cpsd_integral_grads *G);

/* The same with the third-order correction (run_order.f90 order 3):
 *
 * cpsd_cpsd3_energies: w0, w^(2) and w^(3) per root of irrep symR, the terms
 * of cpsd_eecpsd_roots with the ground state (T2^(1), T1^(2), T2^(2), J^(2),
 * J^(3)) computed inside; all six integral lists are read (abcd in device
 * or host memory).
 *
 * cpsd_cpsd3_gradient: ADDS to G the gradient of
 *     sum_k g0_host[k] w0_k + g2_host[k] w2_k + g3_host[k] w3_k
 * with respect to all six DPD integral lists and Eorb (every member of G
 * required; abcd must be in device memory).  Besides the Z-vector solve of
 * the CIS vector, the ground state's T1^(2) (a DIIS solve in the forward
 * direction) is reversed by one more solve of the same operator; both
 * tolerances bound the gradient's accuracy.  FP64 contractions. */
int cpsd_cpsd3_energies(const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p,
                        int64_t symR, int64_t nroot, double *w0_host, double *w2_host, double *w3_host,
                        double *L_dev);
int cpsd_cpsd3_gradient(const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p,
                        int64_t symR, int64_t nroot, const double *w0_host, const double *L_dev,
                        const double *g0_host, const double *g2_host, const double *g3_host,
                        cpsd_integral_grads *G);

#ifdef __cplusplus
}
#endif
#endif
