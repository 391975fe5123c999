// Internal runtime of libcpsd_b200: symmetry context, device scratch arena,
// DPD descriptors and the execution plans built by the host planner.
#pragma once
#include <mutex>
#include <atomic>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "cpsd_b200.h"

namespace cpsd {

using i64 = int64_t;

// ----------------------------------------------------------------- errors
int set_error(int code, const std::string &msg);
const std::string &last_error();
int cuda_check(cudaError_t e, const char *what);
#define CPSD_TRY(x)                  \
    do {                             \
        int _rc = (x);               \
        if (_rc != CPSD_OK) return _rc; \
    } while (0)

// ---------------------------------------------------------------- context
struct Context {
    bool init = false;
    i64 nirrep = 1;
    i64 dirprd[8][8] = {};  // [i-1][j-1]
    cudaStream_t stream = nullptr;
    int64_t launches = 0;
    double flops = 0;  // useful contraction flops issued (2 M N K per block)
    // sliced-integer (int8 digit) tensor-core path: digits per operand
    // element (0 = FP64 DMMA everywhere) and the smallest contraction, in
    // flops, that takes it; error word of its bounded waits
    int oz_digits = 0;
    double oz_min_flops = 1e9;
    int *oz_err = nullptr;
    // Davidson steps that solved the general (non-symmetric) Ritz problem and
    // complex Ritz values met (the reference's imaginary-eigenvalue warning)
    int64_t dav_nonsym_steps = 0, dav_imag_warnings = 0;
    // fraction of the free device memory this thread may plan its scratch
    // for (molecules running side by side share it)
    double mem_share = 1.0;
};
Context &ctx();
inline i64 dp(i64 a, i64 b) { return ctx().dirprd[a - 1][b - 1]; }
inline cudaStream_t stream() { return ctx().stream; }
inline void count_launch(int n = 1) { ctx().launches += n; }

// ------------------------------------------------------------ size math
i64 irpdso(i64 sym, const i64 *popp, const i64 *popq, i64 iop);
i64 idsymsoc(i64 irrepx, const i64 *popp, const i64 *popq, i64 ioppq, const i64 *popr,
             const i64 *pops, i64 ioprs);
i64 isymoffso(i64 irrepq1, i64 irrep, const i64 *popp, const i64 *popq, i64 iop);

struct Desc {
    i64 pop[4][8] = {};
    i64 iop[2] = {1, 1};
    i64 sym = 1;
    i64 len() const { return idsymsoc(sym, pop[0], pop[1], iop[0], pop[2], pop[3], iop[1]); }
    // offset of the right-pair block of irrep R
    i64 block_base(i64 R) const;
    i64 nleft(i64 L) const { return irpdso(L, pop[0], pop[1], iop[0]); }
    i64 nright(i64 R) const { return irpdso(R, pop[2], pop[3], iop[1]); }
    std::string key() const;
};
Desc make_desc(const i64 *p0, const i64 *p1, const i64 *p2, const i64 *p3, i64 iop0, i64 iop1, i64 sym);
Desc desc_of(const cpsd_opt *t);
extern const i64 ZORB[8];

// -------------------------------------------------------- scratch arena
// Bump allocator over device memory.  A caller-provided workspace is used
// as is; otherwise chunks are cudaMalloc'ed on demand and kept.
// CPSD_TRACE_MEM set in the environment: one line on stderr per device
// allocation or release of the scratch arena and the buffer pool, with the
// host time since the first line and the call's own duration (a profiling
// record of where a run meets the memory limit)
bool mem_trace_on();
void mem_trace(const char *what, size_t bytes, double ms, bool ok = true);
double host_ms();

struct Arena {
    struct Chunk {
        char *base;
        size_t size;
        bool owned;
    };
    std::vector<Chunk> chunks;
    size_t cur_chunk = 0, cur_off = 0;
    size_t in_use = 0, high_water = 0;
    bool external = false;
    int alloc(size_t bytes, void **out);
    struct Mark {
        size_t chunk, off, in_use;
    };
    Mark mark() const { return {cur_chunk, cur_off, in_use}; }
    void release(const Mark &m) {
        cur_chunk = m.chunk;
        cur_off = m.off;
        in_use = m.in_use;
    }
    void set_external(void *p, size_t bytes);
    void free_all();
    // frees the owned chunks past the allocation frontier (nothing there is
    // allocated; cudaFree waits for kernels still reading released scratch)
    void trim();
    // bytes of the owned chunks not in use (reusable without cudaMalloc)
    size_t spare() const {
        size_t t = 0;
        for (const Chunk &c : chunks) t += c.size;
        return t > in_use ? t - in_use : 0;
    }
};
Arena &arena();
// serialises the first upload of each cached plan's device tables (plans
// are shared by all host threads)
std::mutex &upload_mutex();
// frees the idle buffers of the device-buffer pool (constant-operand copies
// kept between program runs)
void pool_release_idle();
// frees the constant-operand copies a program keeps that the operation in
// progress was not handed (false: nothing to free)
bool evict_cached_copies(size_t need = 0);  // least recently used first until `need` bytes are free (0: all)
size_t pool_idle_bytes();
// takes the smallest idle pool buffer of min_bytes .. max_bytes out of the
// pool (its size in *bytes; nullptr if none): device memory that changes
// hands without a cudaFree / cudaMalloc
void *pool_take_idle(size_t min_bytes, size_t max_bytes, size_t *bytes);
struct ScratchScope {
    Arena::Mark m;
    ScratchScope() : m(arena().mark()) {}
    ~ScratchScope() { arena().release(m); }
};
template <class T>
int scratch(i64 n, T **out) {
    return arena().alloc(sizeof(T) * (size_t)(n > 0 ? n : 1), (void **)out);
}

// ----------------------------------------------------- contraction plans
constexpr int MAXU = 4;  // units per class (M, N or K)

struct SegDev {          // one K segment (irrep assignment of K letters) of a task
    i64 baseA, baseB, K, kstart;
    i64 mSA[MAXU], nSB[MAXU];
    i64 kExt[MAXU], kSA[MAXU], kSB[MAXU];
    int nk, aMfast, bKfast, pad;
};
struct TaskDev {         // one output region (irreps of M and N letters)
    i64 M, N, baseC, Ktot;
    i64 mExt[MAXU], mSC[MAXU];
    i64 nExt[MAXU], nSC[MAXU];
    int nm, nn, seg0, nseg;
};
struct TileDev {
    int task, mt, nt, nsplit;
    i64 k_lo, k_hi;
    i64 part;            // partial slot (split-K) or -1
};

// tile shapes of the contraction kernel: BM x BN = 128x64, 128x32, 64x128, 64x64
extern const int TILE_BM[4];
extern const int TILE_BN[4];

struct ContractPlan {
    bool empty = true;
    int cfg = 0;  // tile shape (index into TILE_BM / TILE_BN)
    int ntasks = 0, nsegs = 0, ntiles = 0;
    i64 nparts = 0;      // split-K partial tiles
    // host tables (kept for introspection) and their device copies,
    // uploaded at the first launch
    std::vector<TaskDev> h_tasks;
    std::vector<SegDev> h_segs;
    std::vector<TileDev> h_tiles;
    std::vector<int> h_reduce;
    std::atomic<bool> uploaded{false};
    TaskDev *d_tasks = nullptr;
    SegDev *d_segs = nullptr;
    TileDev *d_tiles = nullptr;
    int *d_reduce = nullptr;  // (task, mt, nt, part0, nsplit) groups for split-K
    int nreduce = 0;
    double flops = 0;    // 2*sum M*N*K
    // irreps of the M / N units of each task and of the K units of each
    // segment (one character per unit), for regrouping into dense GEMMs
    std::vector<std::string> task_mkey, task_nkey, seg_kkey;
    int upload();
};
// A batched operand / result: `nb` copies with the given element stride
struct Batch {
    i64 nb = 1;
    i64 strideA = 0, strideB = 0, strideC = 0;
};
int plan_contract(const Desc &d1, const char *t1, const Desc &d2, const char *t2, const Desc &d3,
                  const char *t3, const Batch &batch, const ContractPlan **out);
// tiles of a plan whose tasks and segments are built (force_cfg >= 0: that
// tile shape instead of the cost model's)
void finish_plan(ContractPlan *plan, std::vector<TaskDev> tasks, std::vector<SegDev> dsegs, int force_cfg = -1);
// empirical tile-shape choice (off by default): with it on, the first
// launch of each FP64 tile plan times the four tile shapes on a scratch
// copy of the output and later launches use the fastest
int set_tile_autotune(int on);
int tile_autotune_stats(int64_t *tuned, int64_t *changed);

// C[m + n ldc + r sC] += A[m + k lda] B[k + n ldb + r sB] (m < M, n < N,
// k < K, r < nb) as a one-task plan of the tile kernel
int plan_gemm(i64 M, i64 N, i64 K, i64 lda, i64 ldb, i64 ldc, i64 nb, i64 sB, i64 sC, const ContractPlan **out);

// ------------------------------------------------------- pair-map plans
// out[ob + r*nlo + l] = beta*out + alpha * sum_terms s_l s_r in[ib + ri*nli + li]
struct PMBlockDev {
    i64 outBase, nlo, nro, inBase, nli, lmap, rmap, start;
};
struct PairMapPlan {
    int nblocks = 0;
    i64 total = 0;
    int lterms = 1, rterms = 1;
    std::vector<PMBlockDev> h_blocks;
    std::vector<long long> h_idx;
    std::vector<double> h_sgn;
    std::atomic<bool> uploaded{false};
    PMBlockDev *d_blocks = nullptr;
    long long *d_idx = nullptr;  // index maps (terms interleaved)
    double *d_sgn = nullptr;
    // column tiling (256 rows x 8 columns per tile) when the blocks are
    // tall: first tile of each block and the tile count
    bool tiled = false;
    std::vector<i64> h_tstart;
    i64 ntiles = 0;
    i64 *d_tstart = nullptr;
    int upload();
};
enum PairOp { PAIR_ID = 0, PAIR_EXPAND, PAIR_COMPRESS, PAIR_ANTI, PAIR_ANTI_COMPRESS, PAIR_SWAP };
// the stored (irrep, index) pairs of the pair space of irrep irr, in DPD
// storage order (blocks by the second index's irrep, first index fastest,
// p<q packing for iop 0, p<=q for iop 2)
struct PairEl {
    i64 ip, p, iq, q;
};
std::vector<PairEl> pair_list(const i64 *pp, const i64 *pq, i64 iop, i64 irr);
int plan_pairmap(const Desc &din, int op0, int op1, i64 target_iop0, i64 target_iop1, Desc *dout,
                 const PairMapPlan **out);

// ------------------------------------------------------------- launches
int launch_contract(const ContractPlan *p, const double *A, const double *B, double *C, double alpha);
// same contraction with its tables and partial tiles in the library's fixed
// device region (no allocation); bytes of that region a plan needs
int launch_contract_noalloc(const ContractPlan *p, const double *A, const double *B, double *C, double alpha);
size_t contract_noalloc_bytes(const ContractPlan *p);
// CUDA-event record of one more launch in the timing buffer (when timing is
// on): kind 0-3 DMMA tile shapes, 10 / 11 digit slicing of A / B, 12 digit
// GEMM, 20 / 21 narrow-output kernels (rows / K), 22 short-K kernel (tasks,
// tiles, output elements), 23 row-dot kernel (tasks, warps, output
// elements), 30 / 31 Davidson step /
// Ritz update, 32 solver step, 40 pair transform; a, b, c describe its
// size.  Kinds below 30 are contraction work (cpsd_contract_time).
int timing_begin(double flops, int64_t a, int64_t b, int64_t c, int64_t kind, cudaEvent_t *end);
int timing_end(cudaEvent_t end);
int contract_timing(int enable);
bool contract_timing_on();  // per-launch timing of this thread is on
int contract_time(double *ms, int64_t *launches, double *flops, int reset);
int contract_records(double *ms, double *flops, int64_t *shape, int64_t maxrec, int64_t *nrec);
int launch_pairmap(const PairMapPlan *p, const double *in, double *out, double alpha, double beta, i64 nb = 1,
                   i64 in_stride = 0, i64 out_stride = 0);
int launch_scale(double *x, i64 n, double beta);                  // x *= beta (beta 0: zero fill)
int launch_axpy(i64 n, double a, const double *x, double *y);     // y += a x
int launch_copy(double *y, const double *x, i64 n);
int launch_dot(const double *x, const double *y, i64 n, double *dev_out, bool compensated);
// orbital-energy kernels on (v,o) and (v,v,o,o) DPD tensors
// Element -> orbital-energy indices of the (p,q) and (r,s) pairs; eorb is
// read on the device at launch time.
struct EnergyPlan {
    i64 n = 0;
    int nblocks = 0;
    std::vector<i64> h_blk, h_lidx, h_ridx;
    std::atomic<bool> uploaded{false};
    i64 *d_blk = nullptr;      // per block: base, nl, nr, lpair offset, rpair offset
    i64 *d_lidx = nullptr;     // per left pair: eorb index of p, q (-1 = none)
    i64 *d_ridx = nullptr;     // per right pair: eorb index of r, s (-1 = none)
    int upload();
};
// the tensor's slots are (vir, vir|occ, occ, occ) or (vir, occ) spaces;
// kinds[k] = 'o' / 'v' / 'z' gives the orbital space of slot k
int plan_energy(const Desc &d, const char *kinds, const EnergyPlan **out);
// mode 0: out = e(ab,ij) = ea+eb-ei-ej  (e(a,i) = ea-ei for 2-index)
// mode 1: out = in / (e(ab,ij) - w0)           (run_order.f90:54-58)
// mode 2: out = in / (ei+ej-ea-eb)             (denomT2, denomT.f90:175)
// mode 3: out = in / (ei-ea)                   (denomT1, denomT.f90:82)
// mode 4: out = e(a,i) * in, e(ab,ij) * in     (calAR vdmul: src/EE-CIS.SF/calAR.f90:29,
//                                               src/CISdoo.SD.SF/calAR.f90:69)
// mode 5: out = ei-ea, ei+ej-ea-eb              (the divisor of mode 3 / mode 2)
// mode 6: out = in * (1 / (w0 - e(ab,ij)))      (dEmw, calEigenCISDoo.f90:80-86)
int launch_energy(const EnergyPlan *p, int mode, const double *eorb, const double *in, double *out,
                  const double *w0_dev = nullptr, i64 nb = 1, i64 in_stride = 0, i64 out_stride = 0);
// gorb[k] += d/d eorb[k] of sum_e alpha x(e) y(e) e(pq,rs) (y null: y = 1),
// e(pq,rs) the plan's orbital-energy difference; nocc = occupied orbitals
int launch_energy_adjoint(const EnergyPlan *p, const double *x, const double *y, double alpha, i64 nocc,
                          double *gorb);
// y_c += sgn * a_dev[c] * x_c for nb copies
int launch_axpy_dev(i64 n, const double *a_dev, double sgn, const double *x, double *y, i64 nb = 1, i64 sx = 0,
                    i64 sy = 0);

}  // namespace cpsd
