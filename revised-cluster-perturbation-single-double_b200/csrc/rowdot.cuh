// Contractions whose narrow output side (at most 8 columns) meets rows
// that are strided in the row operand but contiguous along a short
// contracted range (at most 128), one K segment per output block: the
// singles update of the ring intermediate W(em,bj) += r(f,j) V(fe,bm).
#pragma once
#include <atomic>
#include "runtime.hpp"

namespace cpsd {

// one warp's run: rows [r0, r1) of a task, columns [c0, c0 + ncol)
struct RowDotItem {
    int task, seg, c0, ncol;
    i64 r0, r1;
};

struct RowDotPlan {
    bool swap = false;  // rows over the N side (the second operand)
    int kq = 1;         // contracted range / 32, rounded up (1..4)
    int nc = 8;         // columns per item rounded up: 2, 4 or 8
    std::vector<RowDotItem> items;
    // the contraction's task / segment tables with the row units of each
    // task ordered by their stride in the row operand
    std::vector<TaskDev> tasks;
    std::vector<SegDev> segs;
    std::atomic<bool> uploaded{false};
    RowDotItem *d_items = nullptr;
    TaskDev *d_tasks = nullptr;
    SegDev *d_segs = nullptr;
    int upload();
};

// nullptr in *out when the contraction does not qualify
int plan_rowdot(const ContractPlan *cp, const RowDotPlan **out);
int launch_rowdot(const ContractPlan *cp, const RowDotPlan *rp, const double *A, const double *B, double *C,
                  double alpha);

}  // namespace cpsd
