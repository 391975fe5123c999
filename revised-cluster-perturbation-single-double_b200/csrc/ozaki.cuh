// Sliced-integer (int8 digit) contraction on tcgen05: device tables and
// launchers.  See ozaki.cu for the method.
#pragma once
#include <atomic>
#include "runtime.hpp"

namespace cpsd {

// One dense GEMM C_g(M x N) += A_g(M x K) B_g(K x N) of a contraction: the
// rows concatenate the M-index irrep combinations, the columns the N ones,
// K the contracted ones.
struct OzGroup {
    i64 M, N, K;
    int KT;      // K stages of 64
    int nI, nL;  // M- and N-combinations of the group
    i64 aoff, boff;        // byte offsets of the group's digit tiles
    i64 eaoff, eboff;      // offsets of its row / column exponents
    i64 moff, noff;        // offsets into mcombo / ncombo
    i64 crowoff, ccoloff;  // offsets into crow (M x nL) / ccol (N x nI)
};
struct OzTile {
    int g, mt, nt, pad;
};
// slicing work item: one row tile of one group of one operand side.  When
// every row of the tile has the same row combination rc and the row offsets
// step by sr for every contracted combination (affine = 1), and a K stage
// lies in one contracted combination j with column offsets stepping by sk
// (the OzStage of (stage, rc)), element (r0 + dr, k0 + dk) of the tile is at
// roff[r0][j] + ko0 + dr sr + dk sk: the gather needs no per-element table.
struct OzSliceJob {
    i64 R, K;
    int KT, rt, nJ, nI;
    i64 roff, koff, rcoff, kcoff, eoff, doff;
    int affine, rc;
    i64 sr, soff;  // row stride; offset of the group's OzStage table (KT x nI)
};
struct OzStage {
    i64 ko0, sk;  // column offset of the stage's first index, column stride
    int j, ok;    // contracted combination; 1 when the stage is affine
};

struct OzSideDev {
    const OzSliceJob *jobs = nullptr;
    int njobs = 0;
    int kt_max = 0;  // most K stages of a job
    i64 nexpo = 0;   // exponents of this side
    const i64 *roff = nullptr, *koff = nullptr;
    const int *rcombo = nullptr, *kcombo = nullptr;
    const OzStage *stage = nullptr;
};
struct OzDevPlan {
    const OzTile *tiles = nullptr;
    int ntiles = 0;
    const OzGroup *groups = nullptr;
    const i64 *crow = nullptr, *ccol = nullptr;
    const int *mcombo = nullptr, *ncombo = nullptr;
};

// Host plan of a contraction as dense digit GEMMs: the tasks of a
// ContractPlan that share the same contracted irrep combinations form one
// group; its rows / columns run over all M / N combinations of the group.
struct OzPlan {
    int S = 0, BN = 0;
    std::vector<OzGroup> groups;
    std::vector<OzTile> tiles;
    std::vector<OzSliceJob> ajobs, bjobs;
    std::vector<OzStage> astage, bstage;
    std::vector<i64> aroff, akoff, broff, bkoff, crow, ccol;
    std::vector<int> mcombo, ncombo, kcombo;
    i64 adig = 0, bdig = 0;      // bytes of the A / B digit tiles
    i64 nea = 0, neb = 0;        // row / column exponents
    int kt_chunk = 0;            // K stages per launch (keeps the int32 sums exact)
    int kt_max = 0;              // largest K stage count of the groups
    double flops = 0;            // useful FP64-equivalent flops (2 M N K)
    double pad_eff = 0;          // useful / padded tile work
    i64 kmin = 0;                // shortest contracted length of a group
    uint64_t ahash = 0, bhash = 0;  // layout signatures of the A / B digits
    // device copies (uploaded at the first launch)
    std::atomic<bool> uploaded{false};
    OzDevPlan dev;
    OzSideDev adev, bdev;
    int upload();
};
// nullptr in *out when the contraction does not regroup into dense GEMMs
int plan_ozaki(const ContractPlan *cp, int S, const OzPlan **out);

// digits of one operand side (rows_per_tile 128 for A, oz_tile_n(S) for B)
int oz_slice(int S, int rows_per_tile, const OzSideDev &sd, const double *src, int8_t *dig, int *expo);
// C += alpha * sum over the groups, K stages [kt0, kt1) of every group
int oz_gemm(int S, const OzDevPlan &p, const int8_t *Adig, const int8_t *Bdig, const int *ea, const int *eb,
            double *C, double alpha, int kt0, int kt1, int *err);
int oz_tile_n(int S);

}  // namespace cpsd
