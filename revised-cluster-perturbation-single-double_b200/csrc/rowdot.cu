// Row-dot contractions (FP64): an output with at most 8 columns whose
// rows are strided in the row operand while the contracted index is
// contiguous there and short (at most 128), one K segment per output block.
// The case is the singles update of the ring intermediate,
// W(em,bj) += r(f,j) V(fe,bm) (Wmbej_r1abci): the expanded (vv|vo)
// integral is read along f for each row (e,b,m), three to eight columns.
// The narrow kernels need contiguous rows (or a long K), the tile kernels'
// 32-wide column tiles would be mostly empty.
//
// A warp owns a run of rows of one task and one group of up to 8 columns:
// lane l keeps the column operand's values y[q][c] = Y(k = l + 32 q, c) in
// registers for the whole run (one segment per task, so they do not
// change), then takes the rows RB = 32 / ncol at a time.  Each lane copies
// its K elements of a batch's RB rows (coalesced along K) with 8-byte
// cp.async into its own slots of a per-warp ring of NS batches in shared
// memory, NS - 1 batches ahead of the one it works on, so the loads in
// flight do not hold registers; it forms the RB x ncol partial dot
// products from its slots, and one transpose reduction across the warp
// leaves output (row l / ncol, column l % ncol) in lane l, which adds it
// to C.  A lane only ever reads the slots it filled itself, so the
// cp.async group wait is the only synchronisation.  Sums run over k in
// lane order then the fixed butterfly, deterministic.
#include <algorithm>
#include <atomic>
#include <map>
#include <memory>
#include <mutex>

#include "rowdot.cuh"

namespace cpsd {

namespace {

constexpr int RW = 4;  // warps per CTA

__device__ __forceinline__ i64 rdecode(i64 x, int n, const i64 *ext, const i64 *st) {
    i64 off = 0;
    for (int u = 0; u < n - 1; u++) {
        const i64 e = ext[u];
        const i64 q = (x <= 0x7fffffffLL && e <= 0x7fffffffLL) ? (i64)((unsigned)x / (unsigned)e) : x / e;
        off += (x - q * e) * st[u];
        x = q;
    }
    return n > 0 ? off + x * st[n - 1] : off;
}

// 32 values per lane -> lane l holds the warp total of value l
__device__ __forceinline__ double reduce32(double (&v)[32]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        const bool up = (lane & s) != 0;
#pragma unroll
        for (int j = 0; j < s; j++) {
            const double send = up ? v[j] : v[j + s];
            const double recv = __shfl_xor_sync(0xffffffffu, send, s);
            v[j] = (up ? v[j + s] : v[j]) + recv;
        }
    }
    return v[0];
}

__device__ __forceinline__ void cp_async8(double *dst, const double *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int KQ, int NC>
struct RdCfg {
    static constexpr int RB = 32 / NC < 8 ? 32 / NC : 8;  // rows per batch
    static constexpr int SLOT = RB * KQ * 32;             // doubles of one batch of one warp
    // ring depth: about 12 KB per warp (48 KB a CTA, leaving L1 room), 2..6 batches
    static constexpr int NS = 12288 / (SLOT * 8) < 2 ? 2 : 12288 / (SLOT * 8) > 6 ? 6 : 12288 / (SLOT * 8);
    static constexpr int SMEM = RW * NS * SLOT * (int)sizeof(double);
};

// KQ = K / 32 rounded up (1..4); NC = columns per item rounded up to 2, 4,
// 5, 6 or 8 (RB x NC <= 32 outputs per batch: 5 and 6 columns take 6 and 5
// rows a batch instead of 4); SWAP: rows over the N side
template <int KQ, int NC, bool SWAP>
__global__ void __launch_bounds__(RW * 32) k_rowdot(const TaskDev *__restrict__ tasks, const SegDev *__restrict__ segs,
                                                    const RowDotItem *__restrict__ items, int nitems,
                                                    const double *__restrict__ A, const double *__restrict__ B,
                                                    double *__restrict__ C, double alpha) {
    using Cf = RdCfg<KQ, NC>;
    constexpr int RB = Cf::RB, RD_NS = Cf::NS;
    extern __shared__ double rd_ring[];
    __shared__ TaskDev tks[RW];
    __shared__ SegDev sgs[RW];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int iw = blockIdx.x * RW + warp;
    if (iw >= nitems) return;
    const RowDotItem item = items[iw];
    {  // the task and its segment, copied by the warp's lanes
        const long long *ts = reinterpret_cast<const long long *>(tasks + item.task);
        const long long *ss = reinterpret_cast<const long long *>(segs + item.seg);
        long long *td = reinterpret_cast<long long *>(&tks[warp]), *sd = reinterpret_cast<long long *>(&sgs[warp]);
        for (int w = lane; w < (int)(sizeof(TaskDev) / 8); w += 32) td[w] = ts[w];
        for (int w = lane; w < (int)(sizeof(SegDev) / 8); w += 32) sd[w] = ss[w];
        __syncwarp();
    }
    const TaskDev &tk = tks[warp];
    const SegDev &sg = sgs[warp];
    const double *X = SWAP ? B : A, *Y = SWAP ? A : B;
    const int rn = SWAP ? tk.nn : tk.nm, cn = SWAP ? tk.nm : tk.nn;
    const i64 *rext = SWAP ? tk.nExt : tk.mExt, *cext = SWAP ? tk.mExt : tk.nExt;
    const i64 *rsx = SWAP ? sg.nSB : sg.mSA, *csy = SWAP ? sg.mSA : sg.nSB;
    const i64 *rsc = SWAP ? tk.nSC : tk.mSC, *csc = SWAP ? tk.mSC : tk.nSC;
    const i64 kyst = SWAP ? sg.kSA[0] : sg.kSB[0];  // the contracted unit's stride in Y (1 in X)
    const i64 xb = SWAP ? sg.baseB : sg.baseA, yb = SWAP ? sg.baseA : sg.baseB;
    const int K = (int)sg.K, ncol = item.ncol;
    double *ring = rd_ring + (size_t)warp * RD_NS * Cf::SLOT;
    // batch b covers rows item.r0 + b RB ..; its copies go to slot b % RD_NS,
    // element (row i, k = lane + 32 q) at [(i KQ + q) 32 + lane]
    const i64 nrows = item.r1 - item.r0;
    const int nbatch = (int)((nrows + RB - 1) / RB);
    auto issue = [&](int b) {
        if (b < nbatch) {
            const i64 r0 = item.r0 + (i64)b * RB;
            const int nr = (int)min((i64)RB, item.r1 - r0);
            const i64 myrow = lane < nr ? xb + rdecode(r0 + lane, rn, rext, rsx) : 0;
            double *buf = ring + (size_t)(b % RD_NS) * Cf::SLOT + lane;
#pragma unroll
            for (int i = 0; i < RB; i++) {
                const i64 ox = __shfl_sync(0xffffffffu, myrow, i);
#pragma unroll
                for (int q = 0; q < KQ; q++) {
                    const int k = lane + 32 * q;
                    double *d = buf + (i * KQ + q) * 32;
                    if (i < nr && k < K) cp_async8(d, X + ox + k);
                    else *d = 0.0;
                }
            }
        }
        cp_async_commit();  // an empty group past the end keeps the count
    };
    // column operand values of this lane (k = lane + 32 q), held for the run
    double y[KQ][NC];
#pragma unroll
    for (int c = 0; c < NC; c++) {
        const i64 oy = c < ncol ? yb + rdecode(item.c0 + c, cn, cext, csy) : 0;
#pragma unroll
        for (int q = 0; q < KQ; q++) {
            const int k = lane + 32 * q;
            y[q][c] = (c < ncol && k < K) ? __ldg(Y + oy + (i64)k * kyst) : 0.0;
        }
    }
#pragma unroll
    for (int b = 0; b < RD_NS - 1; b++) issue(b);
    const int ri = lane / NC, ci = lane % NC;
    const i64 ccol = ci < ncol ? rdecode(item.c0 + ci, cn, cext, csc) : 0;
    for (int b = 0; b < nbatch; b++) {
        issue(b + RD_NS - 1);  // into the slot consumed by batch b - 1
        cp_async_wait<RD_NS - 1>();
        const i64 r0 = item.r0 + (i64)b * RB;
        const int nr = (int)min((i64)RB, item.r1 - r0);
        // the output this lane updates, its old value fetched before the sums
        const bool mine = ri < nr && ci < ncol;
        const i64 o = mine ? tk.baseC + rdecode(r0 + ri, rn, rext, rsc) + ccol : 0;
        const double cold = mine ? C[o] : 0.0;
        const double *buf = ring + (size_t)(b % RD_NS) * Cf::SLOT + lane;
        double acc[32];
#pragma unroll
        for (int j = RB * NC; j < 32; j++) acc[j] = 0.0;  // lanes past the batch's outputs
#pragma unroll
        for (int i = 0; i < RB; i++) {
            double x[KQ];
#pragma unroll
            for (int q = 0; q < KQ; q++) x[q] = buf[(i * KQ + q) * 32];
#pragma unroll
            for (int c = 0; c < NC; c++) {
                double t = 0.0;
#pragma unroll
                for (int q = 0; q < KQ; q++) t = fma(x[q], y[q][c], t);
                acc[i * NC + c] = t;
            }
        }
        const double s = reduce32(acc);
        if (mine) C[o] = cold + alpha * s;
    }
    cp_async_wait<0>();  // no copy outlives the warp
}

template <class T>
int upload_vec(const std::vector<T> &v, T **d) {
    *d = nullptr;
    if (v.empty()) return CPSD_OK;
    CPSD_TRY(cuda_check(cudaMalloc(d, sizeof(T) * v.size()), "cudaMalloc(row-dot plan)"));
    return cuda_check(cudaMemcpyAsync(*d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, stream()),
                      "upload row-dot plan");
}

}  // namespace

int RowDotPlan::upload() {
    if (uploaded.load(std::memory_order_acquire)) return CPSD_OK;
    std::lock_guard<std::mutex> lock(upload_mutex());
    if (uploaded.load(std::memory_order_relaxed)) return CPSD_OK;
    CPSD_TRY(upload_vec(items, &d_items));
    CPSD_TRY(upload_vec(tasks, &d_tasks));
    CPSD_TRY(upload_vec(segs, &d_segs));
    // the table may next be read by kernels on another thread's stream
    CPSD_TRY(cuda_check(cudaStreamSynchronize(stream()), "plan upload"));
    uploaded.store(true, std::memory_order_release);
    return CPSD_OK;
}

// Qualifies: one side of every task has at most 8 columns (the other the
// rows), every task one segment, the row operand contiguous along a single
// contracted unit of at most 128 and strided along the rows.
int plan_rowdot(const ContractPlan *cp, const RowDotPlan **out) {
    static std::mutex m;
    std::lock_guard<std::mutex> lock(m);
    static std::map<const ContractPlan *, std::unique_ptr<RowDotPlan>> cache;
    *out = nullptr;
    auto it = cache.find(cp);
    if (it != cache.end()) {
        *out = it->second.get();
        return CPSD_OK;
    }
    std::unique_ptr<RowDotPlan> P;
    bool ok = !cp->empty && !cp->h_tasks.empty();
    i64 maxM = 0, maxN = 0, maxK = 0;
    for (const TaskDev &t : cp->h_tasks) {
        maxM = std::max(maxM, t.M);
        maxN = std::max(maxN, t.N);
        maxK = std::max(maxK, t.Ktot);
        ok = ok && t.nseg == 1;
    }
    const bool swap = !(maxN <= 8);
    ok = ok && (maxN <= 8 || maxM <= 8) && maxK >= 1 && maxK <= 128;
    if (ok)
        for (const TaskDev &t : cp->h_tasks) {
            const SegDev &sg = cp->h_segs[t.seg0];
            const i64 kst = swap ? sg.kSB[0] : sg.kSA[0];
            const i64 rst = swap ? sg.nSB[0] : sg.mSA[0];
            const int nr = swap ? t.nn : t.nm;
            ok = ok && sg.nk == 1 && kst == 1 && nr > 0 && rst != 1;
        }
    if (ok) {
        P = std::make_unique<RowDotPlan>();
        RowDotPlan &p = *P;
        p.swap = swap;
        p.kq = (int)((maxK + 31) / 32);
        const i64 cmax = std::min<i64>(8, swap ? maxM : maxN);
        p.nc = cmax <= 2 ? 2 : cmax <= 4 ? 4 : cmax <= 5 ? 5 : cmax <= 6 ? 6 : 8;
        // own copies of the tables with each task's row units reordered by
        // ascending stride in the row operand: consecutive rows are then
        // neighbours in memory (the same (row, column) -> (X, C) pairs, in
        // another order), not 2 MB pages apart
        p.tasks = cp->h_tasks;
        p.segs = cp->h_segs;
        for (TaskDev &t : p.tasks) {
            SegDev &sg = p.segs[t.seg0];
            const int n = swap ? t.nn : t.nm;
            i64 *ext = swap ? t.nExt : t.mExt, *sc = swap ? t.nSC : t.mSC, *sx = swap ? sg.nSB : sg.mSA;
            int ord[MAXU];
            for (int u = 0; u < n; u++) ord[u] = u;
            std::stable_sort(ord, ord + n, [&](int a, int b) { return sx[a] < sx[b]; });
            i64 e2[MAXU], c2[MAXU], x2[MAXU];
            for (int u = 0; u < n; u++) {
                e2[u] = ext[ord[u]];
                c2[u] = sc[ord[u]];
                x2[u] = sx[ord[u]];
            }
            for (int u = 0; u < n; u++) {
                ext[u] = e2[u];
                sc[u] = c2[u];
                sx[u] = x2[u];
            }
        }
        constexpr i64 RUN = 256;  // rows per warp
        for (int ti = 0; ti < (int)p.tasks.size(); ti++) {
            const TaskDev &t = p.tasks[ti];
            const i64 R = swap ? t.N : t.M, CN = swap ? t.M : t.N;
            for (i64 c0 = 0; c0 < CN; c0 += 8)
                for (i64 r0 = 0; r0 < R; r0 += RUN)
                    p.items.push_back(RowDotItem{ti, t.seg0, (int)c0, (int)std::min<i64>(8, CN - c0), r0,
                                                 std::min(R, r0 + RUN)});
        }
        *out = P.get();
    }
    cache[cp] = std::move(P);
    return CPSD_OK;
}

namespace {
template <int KQ, int NC, bool SWAP>
int rowdot_go(int grid, const RowDotPlan *rp, int ni, const double *A, const double *B, double *C, double alpha) {
    using Cf = RdCfg<KQ, NC>;
    static std::atomic<bool> attr{false};
    if (!attr.load(std::memory_order_acquire)) {
        CPSD_TRY(cuda_check(cudaFuncSetAttribute(k_rowdot<KQ, NC, SWAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 Cf::SMEM),
                            "row-dot smem attr"));
        attr.store(true, std::memory_order_release);
    }
    k_rowdot<KQ, NC, SWAP><<<grid, RW * 32, Cf::SMEM, stream()>>>(rp->d_tasks, rp->d_segs, rp->d_items, ni, A, B, C,
                                                                  alpha);
    return CPSD_OK;
}
}  // namespace

int launch_rowdot(const ContractPlan *cp, const RowDotPlan *rp, const double *A, const double *B, double *C,
                  double alpha) {
    if (rp->items.empty()) return CPSD_OK;
    CPSD_TRY(const_cast<RowDotPlan *>(rp)->upload());
    cudaEvent_t end;
    i64 outs = 0;
    for (const TaskDev &t : cp->h_tasks) outs += t.M * t.N;
    CPSD_TRY(timing_begin(cp->flops, cp->ntasks, (i64)rp->items.size(), outs, 23, &end));
    const int ni = (int)rp->items.size(), grid = (ni + RW - 1) / RW;
#define CPSD_ROWDOT(KQ, NC)                                                                                          \
    if (rp->swap)                                                                                                    \
        CPSD_TRY((rowdot_go<KQ, NC, true>(grid, rp, ni, A, B, C, alpha)));                                           \
    else                                                                                                             \
        CPSD_TRY((rowdot_go<KQ, NC, false>(grid, rp, ni, A, B, C, alpha)));
#define CPSD_ROWDOT_K(KQ)                                                                                            \
    switch (rp->nc) {                                                                                                \
    case 2: CPSD_ROWDOT(KQ, 2) break;                                                                                \
    case 4: CPSD_ROWDOT(KQ, 4) break;                                                                                \
    case 5: CPSD_ROWDOT(KQ, 5) break;                                                                                \
    case 6: CPSD_ROWDOT(KQ, 6) break;                                                                                \
    default: CPSD_ROWDOT(KQ, 8) break;                                                                               \
    }
    switch (rp->kq) {
    case 1: CPSD_ROWDOT_K(1) break;
    case 2: CPSD_ROWDOT_K(2) break;
    case 3: CPSD_ROWDOT_K(3) break;
    default: CPSD_ROWDOT_K(4) break;
    }
#undef CPSD_ROWDOT_K
#undef CPSD_ROWDOT
    count_launch();
    CPSD_TRY(cuda_check(cudaGetLastError(), "k_rowdot"));
    return timing_end(end);
}

}  // namespace cpsd
