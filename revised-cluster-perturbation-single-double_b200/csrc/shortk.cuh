// Contractions with a short contracted range (at most SHORTK_KMAX over the
// K segments of every output block) and a wide output: the updates of
// doubles-sized tensors by singles or by small intermediates
// (c2_r1ijka, c2_r2Fmi/Fae, the Wmbej_r1 terms, the hole ladder).  Their
// cost is the read-modify-write of the output, not the arithmetic.
#pragma once
#include <atomic>
#include "runtime.hpp"

namespace cpsd {

constexpr int SHORTK_KMAX = 64;

// one CTA's work: the BF x BS output tile of a task starting at (f0, s0)
// along the output's contiguous side (f) and the other side (s); seg0 = the
// task's first segment (fetched beside the task)
struct ShortKItem {
    int task, seg0;
    i64 f0, s0;
};

struct ShortKPlan {
    bool fm = true;   // the contiguous side of the output is M (else N)
    int bs = 32;      // tile extent along s: 8, 16 or 32 (BF = 2048 / bs)
    int kmax = 0;     // largest contracted range of a task
    std::vector<ShortKItem> items;
    std::atomic<bool> uploaded{false};
    ShortKItem *d_items = nullptr;
    int upload();
};

// nullptr in *out when the contraction does not qualify
int plan_shortk(const ContractPlan *cp, const ShortKPlan **out);
int launch_shortk(const ContractPlan *cp, const ShortKPlan *sp, const double *A, const double *B, double *C,
                  double alpha);

}  // namespace cpsd
