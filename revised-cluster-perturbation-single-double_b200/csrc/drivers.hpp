// Program-level pieces shared by the molecular drivers (drivers.cpp) and the
// gradient program (gradient.cpp): the orbital spaces of a system, the DPD
// views of its integrals and the device solver of solver.f90.
#pragma once
#include <functional>

#include "ops.hpp"

namespace cpsd {

// orbital populations per irrep; popo / popv are the spin-free occupied /
// virtual spaces (alpha + beta of the spin-flipped irrep, readmodule.f90:36-41)
struct Sys {
    i64 nirrep, symry;
    i64 popa[8], popb[8], vrta[8], vrtb[8], popo[8], popv[8];
};
int make_sys(const cpsd_system *s, Sys *S);

// the six spin-free integral tensors (allocate_mem.f90:14-44) and Eorb
struct Ints {
    Ten ijkl, ijka, abij, iabj, abci, abcd;
    const double *eorb;
};
Ints make_ints(const Sys &S, const cpsd_integrals *I);

// a program does not write its integrals: expanded copies of them are kept
// for the whole run (ConstOperands)
struct IntegralScope {
    const double *a[6];
    ConstOperands scope;
    explicit IntegralScope(const cpsd_integrals *I)
        : a{I->ijkl, I->ijka, I->abij, I->iabj, I->abci, I->abcd}, scope(a, 6) {}
};

// pinned host mailbox for the few scalars the host control flow needs
double *mailbox();
// synchronous device -> host copy on the library stream
int read_back(void *host, const void *dev, size_t bytes);

// The solver of solver.f90:4-66 for nb vectors of irrep symR at once: the
// fixed point of R1 = P[(cc - w0 R1 + V(fn,ai) R1) / (ei - ea)] with
// P = orthogonalR2L against L (no P and no w0 term when L / w0d are null).
// For cc orthogonal to a unit eigenvector L of A = e(a,i) + V this is
// (A - w0) R1 = -cc with L.R1 = 0.  *sit receives the summed step counts.
int solve_r1(const Sys &S, const Ints &X, const cpsd_params *p, i64 symR, i64 nb, i64 l1, const EnergyPlan *e1,
             const double *cc, const double *L, const double *w0d, double *R1, i64 *sit);

// CPSD_ETIMEOUT (word cleared) if a bounded wait of the int8-digit path
// timed out on this thread since the last check; synchronises the stream
int digit_error_check();

// Host worker threads (batch.cpp), each with its own non-blocking stream
// and library context, started on demand up to nthreads; in_pool_worker()
// is true on them.
void pool_submit(int nthreads, std::function<void()> job);
bool &in_pool_worker();

}  // namespace cpsd
