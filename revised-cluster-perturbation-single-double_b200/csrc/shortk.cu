// Short-K contractions (FP64): every output block has a contracted range of
// at most SHORTK_KMAX, so one CTA holds the whole K extent of its operand
// tiles in shared memory and the kernel's cost is the read-modify-write of
// the output.  Each CTA owns a BF x BS tile of one task, BF along the side
// that is contiguous in the output (so a warp's 32 output loads and stores
// are one run) and BS = 8, 16 or 32 along the other; a thread owns 8
// outputs of one f: it issues their 8 loads of C before the operand tiles
// are gathered, sums the K products with FMAs (the f-side operand read per
// lane, the s-side one as warp-uniform 16-byte broadcasts) in K order, and
// stores. Same task / segment tables and so the same layouts as the
// tensor-pipe tile kernel, whose 16-deep K stages would be mostly padding
// here and whose occupancy keeps too few loads in flight.
#include <algorithm>
#include <map>
#include <memory>
#include <mutex>

#include "shortk.cuh"

namespace cpsd {

namespace {

constexpr int ST = 256;  // threads per CTA

__device__ __forceinline__ i64 sdecode(i64 x, int n, const i64 *ext, const i64 *st) {
    i64 off = 0;
    for (int u = 0; u < n - 1; u++) {
        const i64 e = ext[u];
        const i64 q = (x <= 0x7fffffffLL && e <= 0x7fffffffLL) ? (i64)((unsigned)x / (unsigned)e) : x / e;
        off += (x - q * e) * st[u];
        x = q;
    }
    return n > 0 ? off + x * st[n - 1] : off;
}

// operand tile dst[(kk + k) * R + r] = src[offR[r] + offK[k]] (0 outside
// the task), r < R, k < K; consecutive threads walk r when rfast (else k),
// the source's contiguous side; eight loads of a thread are in flight
// before their stores
template <int R>
__device__ __forceinline__ void stage(double *dst, const double *__restrict__ src, const i64 *offR, const i64 *offK,
                                      int K, int kk, bool rfast) {
    constexpr int U = 8;
    const int total = R * K;
    auto split = [&](int e, int &r, int &k) {
        if (rfast) {
            r = e % R;
            k = e / R;
        } else {
            k = e % K;
            r = e / K;
        }
    };
    for (int e0 = threadIdx.x; e0 < total; e0 += ST * U) {
        double v[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int e = e0 + u * ST;
            v[u] = 0.0;
            if (e < total) {
                int r, k;
                split(e, r, k);
                const i64 o = offR[r];
                if (o >= 0) v[u] = __ldg(src + o + offK[k]);
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int e = e0 + u * ST;
            if (e < total) {
                int r, k;
                split(e, r, k);
                dst[(size_t)(kk + k) * R + r] = v[u];
            }
        }
    }
}

template <int BS, bool FM>
__global__ void __launch_bounds__(ST, 3) k_shortk(const double *__restrict__ A, const double *__restrict__ B,
                                               double *__restrict__ C, const TaskDev *__restrict__ tasks,
                                               const SegDev *__restrict__ segs, const ShortKItem *__restrict__ items,
                                               int kmax, double alpha) {
    constexpr int BF = 2048 / BS;
    constexpr int BM = FM ? BF : BS, BN = FM ? BS : BF;
    extern __shared__ __align__(16) double sk_sm[];
    double *As = sk_sm;                      // [kmax][BM]
    double *Bs = sk_sm + (size_t)kmax * BM;  // [kmax][BN]
    __shared__ i64 offCM[BM], offCN[BN], offAM[BM], offBN[BN], offKA[SHORTK_KMAX], offKB[SHORTK_KMAX];
    __shared__ TaskDev tk;
    __shared__ SegDev sg;
    const int tid = threadIdx.x;
    const ShortKItem it = items[blockIdx.x];
    // the task and its first segment are fetched side by side
    if (tid == 0) tk = tasks[it.task];
    if (tid == 32) sg = segs[it.seg0];
    __syncthreads();
    const i64 m0 = FM ? it.f0 : it.s0, n0 = FM ? it.s0 : it.f0;
    for (int i = tid; i < BM; i += ST) {
        const i64 m = m0 + i;
        offCM[i] = m < tk.M ? tk.baseC + sdecode(m, tk.nm, tk.mExt, tk.mSC) : -1;
    }
    for (int j = tid; j < BN; j += ST) {
        const i64 n = n0 + j;
        offCN[j] = n < tk.N ? sdecode(n, tk.nn, tk.nExt, tk.nSC) : -1;
    }
    __syncthreads();
    // outputs of this thread: (f, s0 + q), q < 8; their loads go out first
    const int f = tid % BF, s0 = (tid / BF) * 8;
    auto caddr = [&](int q) -> i64 {  // output address, -1 outside the task
        const i64 om = FM ? offCM[f] : offCM[s0 + q], on = FM ? offCN[s0 + q] : offCN[f];
        return (om >= 0 && on >= 0) ? om + on : -1;
    };
    double cval[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const i64 a = caddr(q);
        cval[q] = a >= 0 ? C[a] : 0.0;
    }
    // the operand tiles, segment after segment along K
    int kk = 0;
    for (int si = 0; si < tk.nseg; si++) {
        if (si > 0) {
            __syncthreads();
            if (tid == 0) sg = segs[tk.seg0 + si];
            __syncthreads();
        }
        const int K = (int)sg.K;
        for (int i = tid; i < BM; i += ST) {
            const i64 m = m0 + i;
            offAM[i] = m < tk.M ? sg.baseA + sdecode(m, tk.nm, tk.mExt, sg.mSA) : -1;
        }
        for (int j = tid; j < BN; j += ST) {
            const i64 n = n0 + j;
            offBN[j] = n < tk.N ? sg.baseB + sdecode(n, tk.nn, tk.nExt, sg.nSB) : -1;
        }
        for (int k = tid; k < K; k += ST) {
            i64 a = 0, b = 0, x = k;
            for (int u = 0; u < sg.nk - 1; u++) {
                const i64 e = sg.kExt[u];
                const i64 q = x / e, r = x - q * e;
                a += r * sg.kSA[u];
                b += r * sg.kSB[u];
                x = q;
            }
            if (sg.nk > 0) {  // the last unit takes the remaining quotient
                a += x * sg.kSA[sg.nk - 1];
                b += x * sg.kSB[sg.nk - 1];
            }
            offKA[k] = a;
            offKB[k] = b;
        }
        __syncthreads();
        stage<BM>(As, A, offAM, offKA, K, kk, sg.aMfast != 0);
        stage<BN>(Bs, B, offBN, offKB, K, kk, sg.bKfast == 0);
        kk += K;
    }
    __syncthreads();
    double acc[8];
#pragma unroll
    for (int q = 0; q < 8; q++) acc[q] = 0.0;
#pragma unroll 4
    for (int k = 0; k < kk; k++) {
        // f-side value per lane, s-side values broadcast (8 consecutive,
        // 16-byte aligned: s0 and the row lengths are multiples of 8)
        const double x = FM ? As[(size_t)k * BM + f] : Bs[(size_t)k * BN + f];
        const double2 *y = reinterpret_cast<const double2 *>(FM ? Bs + (size_t)k * BN + s0 : As + (size_t)k * BM + s0);
#pragma unroll
        for (int h = 0; h < 4; h++) {
            const double2 v = y[h];
            acc[2 * h] = fma(x, v.x, acc[2 * h]);
            acc[2 * h + 1] = fma(x, v.y, acc[2 * h + 1]);
        }
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const i64 a = caddr(q);
        if (a >= 0) C[a] = cval[q] + alpha * acc[q];
    }
}

template <int BS, bool FM>
constexpr size_t shortk_smem(int kmax) {
    return sizeof(double) * (size_t)kmax * (size_t)((2048 / BS) + BS);
}

template <class T>
int upload_vec(const std::vector<T> &v, T **d) {
    *d = nullptr;
    if (v.empty()) return CPSD_OK;
    CPSD_TRY(cuda_check(cudaMalloc(d, sizeof(T) * v.size()), "cudaMalloc(short-K plan)"));
    return cuda_check(cudaMemcpyAsync(*d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, stream()),
                      "upload short-K plan");
}

template <int BS, bool FM>
int launch_one(const ContractPlan *cp, const ShortKPlan *sp, const double *A, const double *B, double *C,
               double alpha) {
    static std::atomic<bool> attr{false};
    const size_t smem = shortk_smem<BS, FM>(sp->kmax);
    if (!attr.load()) {
        CPSD_TRY(cuda_check(cudaFuncSetAttribute(k_shortk<BS, FM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)shortk_smem<BS, FM>(SHORTK_KMAX)),
                            "short-K smem attribute"));
        attr.store(true);
    }
    k_shortk<BS, FM><<<(unsigned)sp->items.size(), ST, smem, stream()>>>(A, B, C, cp->d_tasks, cp->d_segs,
                                                                        sp->d_items, sp->kmax, alpha);
    count_launch();
    return cuda_check(cudaGetLastError(), "k_shortk");
}

}  // namespace

int ShortKPlan::upload() {
    if (uploaded.load(std::memory_order_acquire)) return CPSD_OK;
    std::lock_guard<std::mutex> lock(upload_mutex());
    if (uploaded.load(std::memory_order_relaxed)) return CPSD_OK;
    CPSD_TRY(upload_vec(items, &d_items));
    // the table may next be read by kernels on another thread's stream
    CPSD_TRY(cuda_check(cudaStreamSynchronize(stream()), "plan upload"));
    uploaded.store(true, std::memory_order_release);
    return CPSD_OK;
}

// A contraction qualifies when every task's contracted range is 1..KMAX;
// the output side whose first unit has stride 1 in C (in most tasks) runs
// along the tile's contiguous side, and the other side's extent picks BS.
int plan_shortk(const ContractPlan *cp, const ShortKPlan **out) {
    static std::mutex m;
    std::lock_guard<std::mutex> lock(m);
    static std::map<const ContractPlan *, std::unique_ptr<ShortKPlan>> cache;
    *out = nullptr;
    auto it = cache.find(cp);
    if (it != cache.end()) {
        *out = it->second.get();
        return CPSD_OK;
    }
    std::unique_ptr<ShortKPlan> P;
    bool ok = !cp->empty && !cp->h_tasks.empty();
    i64 kmax = 0, mfast = 0, nfast = 0;
    for (const TaskDev &t : cp->h_tasks) {
        ok = ok && t.Ktot >= 1 && t.Ktot <= SHORTK_KMAX;
        kmax = std::max(kmax, t.Ktot);
        mfast += (t.nm > 0 && t.mSC[0] == 1);
        nfast += (t.nn > 0 && t.nSC[0] == 1);
    }
    if (ok) {
        P = std::make_unique<ShortKPlan>();
        ShortKPlan &p = *P;
        p.fm = mfast >= nfast;
        p.kmax = (int)kmax;
        i64 smax = 0;
        for (const TaskDev &t : cp->h_tasks) smax = std::max(smax, p.fm ? t.N : t.M);
        p.bs = smax <= 8 ? 8 : smax <= 16 ? 16 : 32;
        const i64 bf = 2048 / p.bs;
        for (int ti = 0; ti < (int)cp->h_tasks.size(); ti++) {
            const TaskDev &t = cp->h_tasks[ti];
            const i64 F = p.fm ? t.M : t.N, S = p.fm ? t.N : t.M;
            for (i64 s0 = 0; s0 < S; s0 += p.bs)
                for (i64 f0 = 0; f0 < F; f0 += bf) p.items.push_back(ShortKItem{ti, t.seg0, f0, s0});
        }
        *out = P.get();
    }
    cache[cp] = std::move(P);
    return CPSD_OK;
}

int launch_shortk(const ContractPlan *cp, const ShortKPlan *sp, const double *A, const double *B, double *C,
                  double alpha) {
    if (sp->items.empty()) return CPSD_OK;
    CPSD_TRY(const_cast<ContractPlan *>(cp)->upload());
    CPSD_TRY(const_cast<ShortKPlan *>(sp)->upload());
    cudaEvent_t end;
    // record: tasks, tiles, output elements (each read and written once)
    i64 outs = 0;
    for (const TaskDev &t : cp->h_tasks) outs += t.M * t.N;
    CPSD_TRY(timing_begin(cp->flops, cp->ntasks, (i64)sp->items.size(), outs, 22, &end));
    if (sp->fm) {
        if (sp->bs == 8) CPSD_TRY((launch_one<8, true>(cp, sp, A, B, C, alpha)));
        else if (sp->bs == 16) CPSD_TRY((launch_one<16, true>(cp, sp, A, B, C, alpha)));
        else CPSD_TRY((launch_one<32, true>(cp, sp, A, B, C, alpha)));
    } else {
        if (sp->bs == 8) CPSD_TRY((launch_one<8, false>(cp, sp, A, B, C, alpha)));
        else if (sp->bs == 16) CPSD_TRY((launch_one<16, false>(cp, sp, A, B, C, alpha)));
        else CPSD_TRY((launch_one<32, false>(cp, sp, A, B, C, alpha)));
    }
    return timing_end(end);
}

}  // namespace cpsd
