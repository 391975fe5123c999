// Narrow-output contractions (FP64): CIS / solver sigma vectors, one-index
// intermediates and the other contractions whose output block has at most
// 16 columns (or rows), where tensor-core tiles would be mostly padding.
//
// Short contracted range: one thread per output row, the few columns in
// registers, the column operand read as warp-uniform broadcasts.  Long
// contracted range: one warp per 4 rows x 8 columns, lanes striding over K
// (loads along the contiguous K of both operands), a 31-shuffle transpose
// reduction of the 32 sums, and a K split with a fixed-order reduce when
// there are too few rows to fill the GPU.  Both use the planner's task /
// segment tables of the grouped contraction, so every layout that the
// tensor-core path handles is handled here too.
#include <atomic>
#include <mutex>
#include <algorithm>
#include <map>
#include <memory>

#include "narrow.cuh"

namespace cpsd {

namespace {

constexpr int NW = 4;  // warps per CTA

__device__ __forceinline__ i64 ndecode(i64 x, int n, const i64 *ext, const i64 *st) {
    // the last unit takes the remaining quotient whole (x < its extent), so
    // it needs no division; the others divide in 32 bits when both fit
    i64 off = 0;
    for (int u = 0; u < n - 1; u++) {
        const i64 e = ext[u];
        const i64 q = (x <= 0x7fffffffLL && e <= 0x7fffffffLL) ? (i64)((unsigned)x / (unsigned)e) : x / e;
        off += (x - q * e) * st[u];
        x = q;
    }
    return n > 0 ? off + x * st[n - 1] : off;
}

__device__ __forceinline__ void kdecode(i64 k, const SegDev &sg, const i64 *kx, const i64 *ky, i64 *ox, i64 *oy) {
    if (sg.nk == 1) {
        *ox = k * kx[0];
        *oy = k * ky[0];
        return;
    }
    if (sg.nk == 0) {  // no contracted unit: K = 1
        *ox = 0;
        *oy = 0;
        return;
    }
    i64 a = 0, b = 0;
    for (int u = 0; u < sg.nk - 1; u++) {
        const i64 e = sg.kExt[u];
        const i64 q = (k <= 0x7fffffffLL && e <= 0x7fffffffLL) ? (i64)((unsigned)k / (unsigned)e) : k / e;
        const i64 r = k - q * e;
        a += r * kx[u];
        b += r * ky[u];
        k = q;
    }
    *ox = a + k * kx[sg.nk - 1];
    *oy = b + k * ky[sg.nk - 1];
}

// row / column views of a task and segment: rows run over the M side
// (first operand), or over the N side when SWAP
template <bool SWAP>
struct View {
    const TaskDev &tk;
    __device__ View(const TaskDev &t) : tk(t) {}
    __device__ i64 R() const { return SWAP ? tk.N : tk.M; }
    __device__ i64 CN() const { return SWAP ? tk.M : tk.N; }
    __device__ i64 xrow(const SegDev &sg, i64 r) const {
        return SWAP ? sg.baseB + ndecode(r, tk.nn, tk.nExt, sg.nSB) : sg.baseA + ndecode(r, tk.nm, tk.mExt, sg.mSA);
    }
    __device__ i64 ycol(const SegDev &sg, i64 c) const {
        return SWAP ? sg.baseA + ndecode(c, tk.nm, tk.mExt, sg.mSA) : sg.baseB + ndecode(c, tk.nn, tk.nExt, sg.nSB);
    }
    __device__ i64 crow(i64 r) const {
        return SWAP ? ndecode(r, tk.nn, tk.nExt, tk.nSC) : ndecode(r, tk.nm, tk.mExt, tk.mSC);
    }
    __device__ i64 ccol(i64 c) const {
        return SWAP ? ndecode(c, tk.nm, tk.mExt, tk.mSC) : ndecode(c, tk.nn, tk.nExt, tk.nSC);
    }
    __device__ const i64 *kx(const SegDev &sg) const { return SWAP ? sg.kSB : sg.kSA; }
    __device__ const i64 *ky(const SegDev &sg) const { return SWAP ? sg.kSA : sg.kSB; }
};

// short K: thread = row, 8 columns in registers.  The contracted indices
// go in chunks of 32: lane l decodes index k0 + l once and loads its 8
// second-operand values into the warp's shared buffer, then every lane runs
// the 32 indices with its own first-operand loads in flight (same sums, in
// the same order, as one index at a time).
template <bool SWAP>
__global__ void __launch_bounds__(NW * 32) k_narrow_rows(const TaskDev *__restrict__ tasks,
                                                         const SegDev *__restrict__ segs,
                                                         const NarrowItem *__restrict__ items, int nitems,
                                                         const double *__restrict__ A, const double *__restrict__ B,
                                                         double *__restrict__ C, double alpha) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * NW + warp;
    if (it >= nitems) return;
    const NarrowItem item = items[it];
    const TaskDev &tk = tasks[item.task];
    const View<SWAP> v(tk);
    const double *X = SWAP ? B : A, *Y = SWAP ? A : B;
    const i64 r = item.r0 + lane;
    const bool rok = r < v.R();
    const int ncol = (int)min((i64)NARROW_COLS, v.CN() - item.c0);
    double acc[NARROW_COLS];
#pragma unroll
    for (int c = 0; c < NARROW_COLS; c++) acc[c] = 0.0;
    __shared__ i64 fxs[NW][32];
    __shared__ double ys[NW][NARROW_COLS][32];
    for (int si = 0; si < tk.nseg; si++) {
        const SegDev &sg = segs[tk.seg0 + si];
        const i64 ox = rok ? v.xrow(sg, r) : 0;
        i64 oy[NARROW_COLS];
#pragma unroll
        for (int c = 0; c < NARROW_COLS; c++) oy[c] = c < ncol ? v.ycol(sg, item.c0 + c) : 0;
        const i64 *kx = v.kx(sg), *ky = v.ky(sg);
        for (i64 k0 = 0; k0 < sg.K; k0 += 32) {
            const int nk = (int)min((i64)32, sg.K - k0);
            __syncwarp();
            if (lane < nk) {
                i64 fx, fy;
                kdecode(k0 + lane, sg, kx, ky, &fx, &fy);
                fxs[warp][lane] = fx;
#pragma unroll
                for (int c = 0; c < NARROW_COLS; c++) ys[warp][c][lane] = c < ncol ? __ldg(Y + oy[c] + fy) : 0.0;
            }
            __syncwarp();
#pragma unroll 8
            for (int j = 0; j < nk; j++) {
                const double x = rok ? __ldg(X + ox + fxs[warp][j]) : 0.0;
#pragma unroll
                for (int c = 0; c < NARROW_COLS; c++)
                    if (c < ncol) acc[c] = fma(x, ys[warp][c][j], acc[c]);
            }
        }
    }
    if (!rok) return;
    const i64 oc = tk.baseC + v.crow(r);
#pragma unroll
    for (int c = 0; c < NARROW_COLS; c++)
        if (c < ncol) C[oc + v.ccol(item.c0 + c)] += alpha * acc[c];
}

// 32 values per lane -> lane l holds the warp total of value l
__device__ __forceinline__ double transpose_reduce(double (&v)[32]) {
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

__device__ __forceinline__ void nk_cp8(double *dst, const double *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void nk_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void nk_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// long K: warp = KR rows x KC columns (KR x KC <= 32: 8 x 4, 6 x 5, 5 x 6 or
// 4 x 8, the plan's choice by the column count) over the K range of the
// item.  Lane l takes the indices k = kb + l + 32 s of each segment; the
// KR + KC operand values of step s are copied by cp.async into the lane's
// own slots of a per-warp ring of NK_NS steps, NK_NS - 1 steps ahead of the
// FMAs, so the loads in flight hold no registers (the lane reads back only
// what it copied itself: the group wait is the only synchronisation).  Per
// lane the sums run over its indices in order, then the fixed transpose
// reduction leaves output (row l / KC, column l % KC) in lane l.
constexpr int NK_NS = 4;                                   // ring depth (steps)
constexpr int NK_VALS = 12;                                // slots per lane and step (KR + KC <= 12)
constexpr int NK_SMEM = NW * NK_NS * NK_VALS * 32 * 8;     // dynamic shared memory per CTA
template <bool SWAP, int KC>
__global__ void __launch_bounds__(NW * 32) k_narrow_k(const TaskDev *__restrict__ tasks,
                                                      const SegDev *__restrict__ segs,
                                                      const NarrowItem *__restrict__ items, int nitems,
                                                      const double *__restrict__ A, const double *__restrict__ B,
                                                      double *__restrict__ C, double alpha,
                                                      double *__restrict__ partial) {
    extern __shared__ double ring_all[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * NW + warp;
    if (it >= nitems) return;
    const NarrowItem item = items[it];
    const TaskDev &tk = tasks[item.task];
    const View<SWAP> v(tk);
    const double *X = SWAP ? B : A, *Y = SWAP ? A : B;
    constexpr int KR = 32 / KC;
    static_assert(KR + KC <= NK_VALS, "ring slots");
    const int nrow = (int)min((i64)KR, v.R() - item.r0);
    const int ncol = (int)min((i64)KC, v.CN() - item.c0);
    // slot (step, value) of this lane at ring[(step * NK_VALS + value) * 32 + lane]
    double *ring = ring_all + (size_t)warp * NK_NS * NK_VALS * 32 + lane;
    double acc[32];
#pragma unroll
    for (int j = 0; j < 32; j++) acc[j] = 0.0;
    for (int si = 0; si < tk.nseg; si++) {
        const SegDev &sg = segs[tk.seg0 + si];
        i64 kb = item.k0 - sg.kstart, ke = item.k1 - sg.kstart;
        if (kb < 0) kb = 0;
        if (ke > sg.K) ke = sg.K;
        if (kb >= ke) continue;
        i64 ox[KR], oy[KC];
#pragma unroll
        for (int i = 0; i < KR; i++) ox[i] = i < nrow ? v.xrow(sg, item.r0 + i) : 0;
#pragma unroll
        for (int c = 0; c < KC; c++) oy[c] = c < ncol ? v.ycol(sg, item.c0 + c) : 0;
        const i64 *kx = v.kx(sg), *ky = v.ky(sg);
        const i64 nsteps = (ke - kb + 31) / 32;
        auto issue = [&](i64 st) {
            if (st < nsteps) {
                const i64 k = kb + lane + 32 * st;
                double *d = ring + (size_t)(st % NK_NS) * NK_VALS * 32;
                if (k < ke) {
                    i64 fx, fy;
                    kdecode(k, sg, kx, ky, &fx, &fy);
#pragma unroll
                    for (int i = 0; i < KR; i++) {
                        if (i < nrow) nk_cp8(d + i * 32, X + ox[i] + fx);
                        else d[i * 32] = 0.0;
                    }
#pragma unroll
                    for (int c = 0; c < KC; c++) {
                        if (c < ncol) nk_cp8(d + (KR + c) * 32, Y + oy[c] + fy);
                        else d[(KR + c) * 32] = 0.0;
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < KR + KC; j++) d[j * 32] = 0.0;
                }
            }
            nk_commit();  // an empty group past the end keeps the count
        };
#pragma unroll
        for (int st = 0; st < NK_NS - 1; st++) issue(st);
        for (i64 st = 0; st < nsteps; st++) {
            issue(st + NK_NS - 1);  // into the slot step st - 1 used
            nk_wait<NK_NS - 1>();
            const double *d = ring + (size_t)(st % NK_NS) * NK_VALS * 32;
            double x[KR], y[KC];
#pragma unroll
            for (int i = 0; i < KR; i++) x[i] = d[i * 32];
#pragma unroll
            for (int c = 0; c < KC; c++) y[c] = d[(KR + c) * 32];
#pragma unroll
            for (int i = 0; i < KR; i++)
#pragma unroll
                for (int c = 0; c < KC; c++) acc[i * KC + c] = fma(x[i], y[c], acc[i * KC + c]);
        }
        nk_wait<0>();
    }
    const double s = transpose_reduce(acc);
    if (item.part >= 0) {
        partial[item.part * 32 + lane] = s;
        return;
    }
    const int i = lane / KC, c = lane % KC;
    if (i < nrow && c < ncol) C[tk.baseC + v.crow(item.r0 + i) + v.ccol(item.c0 + c)] += alpha * s;
}

// split items of one output block, summed in K order
template <bool SWAP, int KC>
__global__ void __launch_bounds__(NW * 32) k_narrow_reduce(const TaskDev *__restrict__ tasks,
                                                           const NarrowRed *__restrict__ reds, int nreds,
                                                           const double *__restrict__ partial,
                                                           double *__restrict__ C, double alpha) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * NW + warp;
    if (it >= nreds) return;
    const NarrowRed rd = reds[it];
    const TaskDev &tk = tasks[rd.task];
    const View<SWAP> v(tk);
    double s = 0.0;
    for (int q = 0; q < rd.nparts; q++) s += partial[(rd.part0 + q) * 32 + lane];
    // lanes past the KR x KC outputs (KC = 5, 6) hold nothing and write nothing
    const int i = lane / KC, c = lane % KC;
    if (i < 32 / KC && rd.r0 + i < v.R() && rd.c0 + c < v.CN())
        C[tk.baseC + v.crow(rd.r0 + i) + v.ccol(rd.c0 + c)] += alpha * s;
}

template <class T>
int upload_vec(const std::vector<T> &v, T **d) {
    *d = nullptr;
    if (v.empty()) return CPSD_OK;
    CPSD_TRY(cuda_check(cudaMalloc(d, sizeof(T) * v.size()), "cudaMalloc(narrow plan)"));
    return cuda_check(cudaMemcpyAsync(*d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, stream()),
                      "upload narrow plan");
}

}  // namespace

int NarrowPlan::upload() {
    if (uploaded.load(std::memory_order_acquire)) return CPSD_OK;
    std::lock_guard<std::mutex> lock(upload_mutex());
    if (uploaded.load(std::memory_order_relaxed)) return CPSD_OK;
    CPSD_TRY(upload_vec(items, &d_items));
    CPSD_TRY(upload_vec(reds, &d_reds));
    // the tables may next be read by kernels on another thread's stream
    CPSD_TRY(cuda_check(cudaStreamSynchronize(stream()), "plan upload"));
    uploaded.store(true, std::memory_order_release);
    return CPSD_OK;
}

int plan_narrow(const ContractPlan *cp, const NarrowPlan **out) {
    static std::mutex m;
    std::lock_guard<std::mutex> lock(m);
    static std::map<const ContractPlan *, std::unique_ptr<NarrowPlan>> cache;
    *out = nullptr;
    auto it = cache.find(cp);
    if (it != cache.end()) {
        *out = it->second.get();
        return CPSD_OK;
    }
    i64 maxM = 0, maxN = 0, maxK = 0;
    for (const TaskDev &tk : cp->h_tasks) {
        maxM = std::max(maxM, tk.M);
        maxN = std::max(maxN, tk.N);
        maxK = std::max(maxK, tk.Ktot);
    }
    std::unique_ptr<NarrowPlan> P;
    bool ok = !cp->empty && (maxN <= 16 || maxM <= 16);
    const bool swap = !(maxN <= 16), longk = maxK > 96;
    if (ok) {  // the loads must be coalesced: along K (lanes over K) or along the rows
        const TaskDev &t0 = cp->h_tasks[0];
        const SegDev &s0 = cp->h_segs[t0.seg0];
        const i64 kst = swap ? s0.kSB[0] : s0.kSA[0];
        const i64 rst = swap ? s0.nSB[0] : s0.mSA[0];
        const int nr = swap ? t0.nn : t0.nm;
        ok = longk ? (s0.nk > 0 && kst == 1) : (nr > 0 && rst == 1);
    }
    if (ok) {
        P = std::make_unique<NarrowPlan>();
        NarrowPlan &p = *P;
        p.swap = swap;
        p.longk = longk;
        auto R = [&](const TaskDev &t) { return p.swap ? t.N : t.M; };
        auto CN = [&](const TaskDev &t) { return p.swap ? t.M : t.N; };
        if (!p.longk) {
            for (int ti = 0; ti < (int)cp->h_tasks.size(); ti++) {
                const TaskDev &t = cp->h_tasks[ti];
                for (i64 c0 = 0; c0 < CN(t); c0 += NARROW_COLS)
                    for (i64 r0 = 0; r0 < R(t); r0 += 32) p.items.push_back(NarrowItem{ti, (int)c0, r0, 0, t.Ktot, -1});
            }
        } else {
            // item shape by the column count: 8 x 4, 6 x 5, 5 x 6 or 4 x 8
            // rows x columns, so that few of a warp's 32 sums go unused
            i64 cmax = 0;
            for (const TaskDev &t : cp->h_tasks) cmax = std::max(cmax, CN(t));
            p.kc = cmax <= 4 ? 4 : cmax == 5 ? 5 : cmax == 6 ? 6 : 8;
            const int KC = p.kc, KR = 32 / p.kc;
            i64 base = 0;
            for (const TaskDev &t : cp->h_tasks) base += ((R(t) + KR - 1) / KR) * ((CN(t) + KC - 1) / KC);
            // K parts: about 8192 warp items (measured: 3552 and 16384 are
            // slower or no faster on d2h_nmo400)
            const i64 want = std::max<i64>(1, (8192 + base - 1) / base);
            for (int ti = 0; ti < (int)cp->h_tasks.size(); ti++) {
                const TaskDev &t = cp->h_tasks[ti];
                const i64 ns = std::max<i64>(1, std::min<i64>(want, t.Ktot / 256));
                // the row groups of one K part are neighbours in the item
                // list, so the warps running together read the same stretch
                // of the column operand (it stays in L2 across the row groups)
                for (i64 c0 = 0; c0 < CN(t); c0 += KC) {
                    const i64 part0 = p.nparts;
                    if (ns > 1)
                        for (i64 r0 = 0; r0 < R(t); r0 += KR) {
                            p.reds.push_back(NarrowRed{ti, (int)c0, (int)ns, 0, r0, p.nparts});
                            p.nparts += ns;
                        }
                    for (i64 q = 0; q < ns; q++)
                        for (i64 r0 = 0, ri = 0; r0 < R(t); r0 += KR, ri++)
                            p.items.push_back(NarrowItem{ti, (int)c0, r0, t.Ktot * q / ns, t.Ktot * (q + 1) / ns,
                                                         ns > 1 ? part0 + ri * ns + q : -1});
                }
            }
        }
        *out = P.get();
    }
    cache[cp] = std::move(P);
    return CPSD_OK;
}

namespace {
template <bool SWAP, int KC>
int narrow_k_launch(int grid, int ni, int nr, const ContractPlan *cp, const NarrowPlan *np, const double *A,
                    const double *B, double *C, double alpha, double *part) {
    static std::atomic<bool> attr{false};
    if (!attr.load(std::memory_order_acquire)) {
        CPSD_TRY(cuda_check(cudaFuncSetAttribute(k_narrow_k<SWAP, KC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 NK_SMEM),
                            "narrow smem attr"));
        attr.store(true, std::memory_order_release);
    }
    k_narrow_k<SWAP, KC><<<grid, NW * 32, NK_SMEM, stream()>>>(cp->d_tasks, cp->d_segs, np->d_items, ni, A, B, C,
                                                               alpha, part);
    count_launch();
    if (nr > 0) {
        const int rg = (nr + NW - 1) / NW;
        k_narrow_reduce<SWAP, KC><<<rg, NW * 32, 0, stream()>>>(cp->d_tasks, np->d_reds, nr, part, C, alpha);
        count_launch();
    }
    return CPSD_OK;
}

template <bool SWAP>
int narrow_k_kc(const NarrowPlan *np, int grid, int ni, int nr, const ContractPlan *cp, const double *A,
                const double *B, double *C, double alpha, double *part) {
    switch (np->kc) {
    case 4: return narrow_k_launch<SWAP, 4>(grid, ni, nr, cp, np, A, B, C, alpha, part);
    case 5: return narrow_k_launch<SWAP, 5>(grid, ni, nr, cp, np, A, B, C, alpha, part);
    case 6: return narrow_k_launch<SWAP, 6>(grid, ni, nr, cp, np, A, B, C, alpha, part);
    default: return narrow_k_launch<SWAP, 8>(grid, ni, nr, cp, np, A, B, C, alpha, part);
    }
}

int narrow_k_go(const NarrowPlan *np, int grid, int ni, int nr, const ContractPlan *cp, const double *A,
                const double *B, double *C, double alpha, double *part) {
    return np->swap ? narrow_k_kc<true>(np, grid, ni, nr, cp, A, B, C, alpha, part)
                    : narrow_k_kc<false>(np, grid, ni, nr, cp, A, B, C, alpha, part);
}
}  // namespace

int launch_narrow(const ContractPlan *cp, const NarrowPlan *np, const double *A, const double *B, double *C,
                  double alpha) {
    CPSD_TRY(const_cast<ContractPlan *>(cp)->upload());
    CPSD_TRY(const_cast<NarrowPlan *>(np)->upload());
    const int ni = (int)np->items.size(), nr = (int)np->reds.size();
    if (ni == 0) return CPSD_OK;
    cudaEvent_t end;
    CPSD_TRY(timing_begin(cp->flops, cp->ntasks, ni, np->nparts, 20 + (np->longk ? 1 : 0), &end));
    const int grid = (ni + NW - 1) / NW;
    if (!np->longk) {
        if (np->swap)
            k_narrow_rows<true><<<grid, NW * 32, 0, stream()>>>(cp->d_tasks, cp->d_segs, np->d_items, ni, A, B, C, alpha);
        else
            k_narrow_rows<false><<<grid, NW * 32, 0, stream()>>>(cp->d_tasks, cp->d_segs, np->d_items, ni, A, B, C, alpha);
        count_launch();
    } else {
        ScratchScope sc;
        double *part = nullptr;
        if (np->nparts > 0) CPSD_TRY(scratch(np->nparts * 32, &part));
        CPSD_TRY(narrow_k_go(np, grid, ni, nr, cp, A, B, C, alpha, part));
    }
    CPSD_TRY(cuda_check(cudaGetLastError(), "k_narrow"));
    return timing_end(end);
}

}  // namespace cpsd
