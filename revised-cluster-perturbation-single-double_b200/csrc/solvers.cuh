// Device state of the Davidson eigensolver and the DIIS extrapolator.
#pragma once
#include "runtime.hpp"

namespace cpsd {

constexpr int DAV_MAXD = 32;  // davidson_dim limit (reference default 20)

// Everything the reference keeps in local variables / scratch files
// (src/lib_cc/mod_davidson.f90:40-560), resident on the device.
struct DavState {
    int D, dimA, nroot, lowest, maxcyc;
    int dimIter, dimFree, dim_exceed, ndimIter, ndimFree, dimDel;
    int iterations, cur, nNew, newpos, done, converged;
    // steps that took the general (non-symmetric) eigen-solve, Ritz values
    // with an imaginary part above 1e-10 (the reference's warning,
    // mod_davidson.f90:193-196), QR iteration failure
    int nonsym_steps, warn_imag, eig_fail, pad;
    double maxError, max_resid;
    int conv[DAV_MAXD];
    int lowestE[DAV_MAXD];
    double eigenVal[DAV_MAXD];
    double valR[DAV_MAXD];
    double Abar[DAV_MAXD * DAV_MAXD];
    double vecR[DAV_MAXD * DAV_MAXD];
    double vecNeed[DAV_MAXD * DAV_MAXD];
    double oldE[DAV_MAXD * DAV_MAXD];
    double newE[DAV_MAXD * DAV_MAXD];
};

struct DavBuffers {
    double *B[2], *AB[2];  // basis and sigma "files", D x dimA each
    const double *diag;    // OED1 of the irrep
    double *fileEV;        // nroot records (w, R)
    double *w0, *w1;       // work vectors, nroot x dimA (one slice per root)
    // device-driven loop: the step stages its new vectors in W (nroot x dimA,
    // zero beyond nNew), the sigma of W goes to AW and the Ritz update moves
    // it in place; mailbox[0] (mapped host memory) = 1 while iterating
    double *W = nullptr, *AW = nullptr;
    int *mailbox = nullptr;
};

int dav_init_launch(DavState *st, const DavBuffers &b);      // Abar of the guesses
int dav_step_launch(DavState *st, const DavBuffers &b);
int dav_abar_launch(DavState *st, const DavBuffers &b);
int dav_final_launch(DavState *st, const DavBuffers &b);     // eigen test residual
// the Davidson step's general eigen-solve on one row-major n x n device
// matrix: eigenvalues wr / wi, eigenvectors V (row-major, dgeev's columns),
// QR sweeps (-1: no convergence); all device pointers
int geev_probe(const double *A_dev, int n, double *wr, double *wi, double *V, int *sweeps);

constexpr int DIIS_MAXDIM = 16;
struct DiisState {
    int len, maxdim, ndimr, idimr;
    double res;
    double Bm[DIIS_MAXDIM * DIIS_MAXDIM];  // error-vector overlaps of the stored steps
};
struct DiisBuffers {
    double *prev, *err, *amp;  // len, maxdim*len, maxdim*len
};
// Device-driven solver steps for nb independent roots: the EE solver
// (solver.f90:4-66), without L and w0 the ground T1^(2) DIIS loop
// (run2.f90) and the grCPS(D) (T1, T2) loop, with nrmv the CIS(D-infinity)
// left-vector loop (src/EE-grCPSd.SF/calEigenCISDoo.f90:94-140).  One CTA
// per root and step does
//   pr = cc - w0 R1 + S      (S = the sigma of the previous step's R1; from step 2)
//   R1 = pr / den (den = ei - ea, or ei + ej - ea - eb on the doubles; kept
//   as given at step 1 with keep_first);  orthogonalR2L or the <R1|nrmv> = 1
//   scaling; dosodiis2_d (LINPACK solve of the bordered -1e-4 system,
//   dodiis.f / minv.f); orthogonalR2L or the scaling again
// (orthogonalR2L: R -= (<L|R>/||L||) L, orthogonalR2L.f90:5-34)
// and stops the root (active = 0) once |DIIS residual| < tol after step 1 or
// after step cyc + 1, exactly where the reference's loop exits.  The host
// keeps launching steps without reading anything back; mailbox (mapped host
// memory) tells it when every root has stopped.
struct SolverState {
    int iter, active, pad0, pad1;
    double res;
};
struct SolverArgs {
    int len = 0, nb = 0, cyc = 0;
    double tol = 0;
    SolverState *ss = nullptr;      // nb
    DiisState *ds = nullptr;        // nb
    DiisBuffers db{};               // root r at db.prev + r * sprev, db.err / db.amp + r * serr
    i64 sprev = 0, serr = 0;
    double *pr = nullptr, *R1 = nullptr;  // nb x len
    const double *cc = nullptr, *S = nullptr, *den = nullptr, *L = nullptr, *w0 = nullptr;
    int *mailbox = nullptr;         // nb (device view of mapped host memory)
    const double *nrmv = nullptr;   // nb x len: scale R1 to <R1|nrmv> = 1 around the DIIS step
    int keep_first = 0;             // iteration 1 keeps R1 as given instead of pr / den
};
int solver_step_launch(const SolverArgs &a);

}  // namespace cpsd
