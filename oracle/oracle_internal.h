/* CPU ORACLE (test infrastructure only): internal helpers shared by the
 * oracle's translation units. */
#ifndef CPSD_ORACLE_INTERNAL_H
#define CPSD_ORACLE_INTERNAL_H
#include "cpsd_oracle.h"

typedef struct {
    i64 n;
    i64 *ip, *p, *iq, *q;
} o_pairs;
void o_pairs_build(o_pairs *pl, const i64 *popp, const i64 *popq, i64 iop, i64 irr);
void o_pairs_free(o_pairs *pl);

double o_ddot(i64 n, const double *x, const double *y);
double o_dnrm2(i64 n, const double *x);
void o_daxpy(i64 n, double a, const double *x, double *y);
i64 o_idamax(i64 n, const double *x);

typedef void (*o_sigma_fn)(void *ctx, const double *R, double *AR);
int o_davidson(double *fileEV, const double *diagA, i64 dimA, i64 nroot, i64 istate,
               const o_params *p, o_sigma_fn calAR, void *ctx, i64 *iters_out);
int o_guess(const o_system *s, const double *eorb, const o_params *p, i64 irrepex,
            i64 nroot, double *guess);

typedef struct {
    i64 len, maxdim, ndimr, idimr;
    double *prev, *err, *amp;
} o_diis;
void o_diis_init(o_diis *st, i64 len, i64 maxdim);
void o_diis_free(o_diis *st);
double o_diis_step(o_diis *st, i64 iter, double *vec);
void o_dgefa(double *a, i64 lda, i64 n, i64 *ipvt);
void o_dgesl(const double *a, i64 lda, i64 n, const i64 *ipvt, double *b);

const i64 *o_zorb(void);
#endif
