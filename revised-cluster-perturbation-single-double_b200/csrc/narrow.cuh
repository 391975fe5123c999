// Contractions with a narrow output side (at most 16 columns after
// batching, or 16 rows with the operands' roles swapped): sigma vectors of
// CIS and of the R1 solver, one-index intermediates.  Tensor-core tiles would
// be mostly padding there; these kernels stream the wide operand once.
#pragma once
#include <atomic>
#include "runtime.hpp"

namespace cpsd {

constexpr int NARROW_COLS = 8;  // output columns per work item (short K; at most, long K)
constexpr int NARROW_ROWS = 4;  // rows per warp in the long-K kernel at 8 columns

// one warp's work: rows [r0, r0 + rows) of a task, columns [c0, c0 + 8),
// contracted range [k0, k1) of the task's concatenated K; partial slot when
// the K range is split (deterministic reduce afterwards)
struct NarrowItem {
    int task, c0;
    i64 r0, k0, k1;
    i64 part;
};
struct NarrowRed {  // split items of one (task, r0, c0), in K order
    int task, c0, nparts, pad;
    i64 r0, part0;
};

struct NarrowPlan {
    bool swap = false;   // rows run over the N side (the second operand)
    bool longk = false;  // lanes over K (warp reductions) instead of over rows
    int kc = NARROW_COLS;  // long K: columns per item (4, 5, 6 or 8), rows 32 / kc
    std::vector<NarrowItem> items;
    std::vector<NarrowRed> reds;
    i64 nparts = 0;
    std::atomic<bool> uploaded{false};
    NarrowItem *d_items = nullptr;
    NarrowRed *d_reds = nullptr;
    int upload();
};

// nullptr in *out when the contraction is not narrow
int plan_narrow(const ContractPlan *cp, const NarrowPlan **out);
int launch_narrow(const ContractPlan *cp, const NarrowPlan *np, const double *A, const double *B, double *C,
                  double alpha);

}  // namespace cpsd
