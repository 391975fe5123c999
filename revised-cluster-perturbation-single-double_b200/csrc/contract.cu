// The grouped DPD contraction kernel (sm_100a, FP64).
//
// One launch executes every irrep block of a contraction: each CTA owns a
// BM x BN tile of one output block (task) and walks the K segments of that
// task (the irrep assignments of the contracted indices), gathering A / B
// tiles through the planner's stride tables (packed pairs are composite
// indices) into padded shared memory and multiplying them on the FP64
// tensor pipe with mma.sync.m8n8k4.f64 (tcgen05 has no FP64 kind).  The
// next K stage is fetched into registers while the current one is
// multiplied.  Split-K tiles write partial sums that k_splitk_reduce adds
// in a fixed order, so results are deterministic.
#include <atomic>
#include <array>
#include <vector>

#include <map>
#include <memory>
#include <mutex>
#include "runtime.hpp"

namespace cpsd {

namespace {
constexpr int NT = 256, BK = 16, PAD = 4;

__device__ __forceinline__ i64 decode1(i64 x, int n, const i64 *ext, const i64 *st) {
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

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

template <int BM, int BN>
constexpr int smem_bytes() {
    return (int)sizeof(double) * 2 * BK * ((BM + PAD) + (BN + PAD));
}

template <int BM, int BN, int WM, int WN>
__global__ void __launch_bounds__(NT, 2) k_contract(const double *__restrict__ A, const double *__restrict__ B,
                                                    double *__restrict__ C, const TaskDev *__restrict__ tasks,
                                                    const SegDev *__restrict__ segs, const TileDev *__restrict__ tiles,
                                                    double alpha, double *__restrict__ partial) {
    static_assert(WM * WN == NT / 32, "8 warps");
    constexpr int WTM = BM / WM, WTN = BN / WN, MI = WTM / 8, NI = WTN / 8;
    constexpr int LA = BM * BK / NT, LB = BN * BK / NT;
    static_assert(LA >= 1 && LB >= 1 && BM + BN <= NT, "tile shape");
    extern __shared__ double dsm[];
    double(*As)[BK][BM + PAD] = reinterpret_cast<double(*)[BK][BM + PAD]>(dsm);
    double(*Bs)[BK][BN + PAD] = reinterpret_cast<double(*)[BK][BN + PAD]>(dsm + 2 * BK * (BM + PAD));
    __shared__ i64 offM[BM], offN[BN], offKA[2][BK], offKB[2][BK];
    __shared__ TaskDev tk;
    __shared__ SegDev sg;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp % WM, wn = warp / WM;
    const TileDev tl = tiles[blockIdx.x];
    if (tid == 0) tk = tasks[tl.task];
    __syncthreads();
    const i64 m0 = (i64)tl.mt * BM, n0 = (i64)tl.nt * BN;
    double acc[MI][NI][2];
#pragma unroll
    for (int i = 0; i < MI; i++)
#pragma unroll
        for (int j = 0; j < NI; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
    double ra[LA], rb[LB];

    for (int si = 0; si < tk.nseg; si++) {
        __syncthreads();
        if (tid == 0) sg = segs[tk.seg0 + si];
        __syncthreads();
        i64 kb = tl.k_lo - sg.kstart, ke = tl.k_hi - sg.kstart;
        if (kb < 0) kb = 0;
        if (ke > sg.K) ke = sg.K;
        if (kb >= ke) continue;
        if (tid < BM) {
            i64 m = m0 + tid;
            offM[tid] = (m < tk.M) ? sg.baseA + decode1(m, tk.nm, tk.mExt, sg.mSA) : -1;
        } else if (tid < BM + BN) {
            i64 n = n0 + tid - BM;
            offN[tid - BM] = (n < tk.N) ? sg.baseB + decode1(n, tk.nn, tk.nExt, sg.nSB) : -1;
        }
        const int nst = (int)((ke - kb + BK - 1) / BK);
        auto decodeK = [&](int s, int buf) {
            if (tid < BK) {
                i64 k = kb + (i64)s * BK + tid;
                if (k < ke) {
                    i64 a = 0, b = 0, x = k;
                    for (int u = 0; u < sg.nk - 1; u++) {
                        const i64 e = sg.kExt[u];
                        const i64 q = (x <= 0x7fffffffLL && e <= 0x7fffffffLL) ? (i64)((unsigned)x / (unsigned)e)
                                                                               : x / e;
                        const i64 r = x - q * e;
                        a += r * sg.kSA[u];
                        b += r * sg.kSB[u];
                        x = q;
                    }
                    if (sg.nk > 0) {  // the last unit takes the remaining quotient
                        a += x * sg.kSA[sg.nk - 1];
                        b += x * sg.kSB[sg.nk - 1];
                    }
                    offKA[buf][tid] = a;
                    offKB[buf][tid] = b;
                } else {
                    offKA[buf][tid] = -1;
                    offKB[buf][tid] = -1;
                }
            }
        };
        auto loadRegs = [&](int buf) {
#pragma unroll
            for (int i = 0; i < LA; i++) {
                int e = tid + i * NT, m, k;
                if (sg.aMfast) {
                    m = e % BM;
                    k = e / BM;
                } else {
                    k = e % BK;
                    m = e / BK;
                }
                i64 om = offM[m], ok = offKA[buf][k];
                ra[i] = (om >= 0 && ok >= 0) ? __ldg(A + om + ok) : 0.0;
            }
#pragma unroll
            for (int i = 0; i < LB; i++) {
                int e = tid + i * NT, n, k;
                if (sg.bKfast) {
                    k = e % BK;
                    n = e / BK;
                } else {
                    n = e % BN;
                    k = e / BN;
                }
                i64 on = offN[n], ok = offKB[buf][k];
                rb[i] = (on >= 0 && ok >= 0) ? __ldg(B + on + ok) : 0.0;
            }
        };
        auto storeRegs = [&](int buf) {
#pragma unroll
            for (int i = 0; i < LA; i++) {
                int e = tid + i * NT;
                if (sg.aMfast) As[buf][e / BM][e % BM] = ra[i];
                else As[buf][e % BK][e / BK] = ra[i];
            }
#pragma unroll
            for (int i = 0; i < LB; i++) {
                int e = tid + i * NT;
                if (sg.bKfast) Bs[buf][e % BK][e / BK] = rb[i];
                else Bs[buf][e / BN][e % BN] = rb[i];
            }
        };
        decodeK(0, 0);
        __syncthreads();
        loadRegs(0);
        for (int s = 0; s < nst; s++) {
            const int buf = s & 1;
            storeRegs(buf);
            if (s + 1 < nst) decodeK(s + 1, buf ^ 1);
            __syncthreads();
            if (s + 1 < nst) loadRegs(buf ^ 1);
#pragma unroll
            for (int kk = 0; kk < BK / 4; kk++) {
                const int kr = kk * 4 + (lane & 3);
                double a[MI], b[NI];
#pragma unroll
                for (int i = 0; i < MI; i++) a[i] = As[buf][kr][wm * WTM + i * 8 + (lane >> 2)];
#pragma unroll
                for (int j = 0; j < NI; j++) b[j] = Bs[buf][kr][wn * WTN + j * 8 + (lane >> 2)];
#pragma unroll
                for (int i = 0; i < MI; i++)
#pragma unroll
                    for (int j = 0; j < NI; j++) dmma(acc[i][j], a[i], b[j]);
            }
        }
    }
    __syncthreads();
    const int rl = lane >> 2, cl = 2 * (lane & 3);
    if (tl.part >= 0) {
        double *P = partial + (size_t)tl.part * (BM * BN);
#pragma unroll
        for (int i = 0; i < MI; i++)
#pragma unroll
            for (int j = 0; j < NI; j++) {
                int r = wm * WTM + i * 8 + rl, c = wn * WTN + j * 8 + cl;
                P[r * BN + c] = acc[i][j][0];
                P[r * BN + c + 1] = acc[i][j][1];
            }
        return;
    }
    if (tid < BM) {
        i64 m = m0 + tid;
        offM[tid] = (m < tk.M) ? tk.baseC + decode1(m, tk.nm, tk.mExt, tk.mSC) : -1;
    } else if (tid < BM + BN) {
        i64 n = n0 + tid - BM;
        offN[tid - BM] = (n < tk.N) ? decode1(n, tk.nn, tk.nExt, tk.nSC) : -1;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < MI; i++) {
        i64 om = offM[wm * WTM + i * 8 + rl];
        if (om < 0) continue;
#pragma unroll
        for (int j = 0; j < NI; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                i64 on = offN[wn * WTN + j * 8 + cl + h];
                if (on < 0) continue;
                C[om + on] += alpha * acc[i][j][h];
            }
    }
}

// Sum the split-K partial tiles of the output tiles in a fixed order.  One
// thread per tile element: block b covers elements [NT*(b % chunks), +NT)
// of reduce group b / chunks (chunks = bm*bn / NT), with four independent
// partial sums so that the loads of several partial tiles are in flight.
__global__ void __launch_bounds__(NT) k_splitk_reduce(const int *__restrict__ red, const TaskDev *__restrict__ tasks,
                                                      const double *__restrict__ partial, double *__restrict__ C,
                                                      double alpha, int bm, int bn) {
    const int chunks = bm * bn / NT;
    const int *r = red + 5 * (blockIdx.x / chunks);
    const int e = (blockIdx.x % chunks) * NT + threadIdx.x;
    const TaskDev &tk = tasks[r[0]];
    const i64 m = (i64)r[1] * bm + e / bn, n = (i64)r[2] * bn + e % bn;
    if (m >= tk.M || n >= tk.N) return;
    const i64 p0 = r[3];
    const int ns = r[4];
    const size_t ts = (size_t)bm * bn;
    const double *P = partial + (size_t)p0 * ts + e;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int q = 0;
    for (; q + 4 <= ns; q += 4) {
        s0 += P[(size_t)q * ts];
        s1 += P[(size_t)(q + 1) * ts];
        s2 += P[(size_t)(q + 2) * ts];
        s3 += P[(size_t)(q + 3) * ts];
    }
    for (; q < ns; q++) s0 += P[(size_t)q * ts];
    const double s = (s0 + s1) + (s2 + s3);
    C[tk.baseC + decode1(m, tk.nm, tk.mExt, tk.mSC) + decode1(n, tk.nn, tk.nExt, tk.nSC)] += alpha * s;
}

// optional CUDA-event timing of every contraction launch (on its stream)
struct Timing {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    size_t used = 0;
    std::vector<double> flops;
    std::vector<std::array<int64_t, 4>> shape;  // tasks, segments, tiles, tile config
};
Timing &timing() {
    thread_local Timing t;
    return t;
}
int timing_event(cudaEvent_t *e) {
    Timing &t = timing();
    if (t.used == t.pool.size()) {
        cudaEvent_t ev;
        CPSD_TRY(cuda_check(cudaEventCreate(&ev), "event create"));
        t.pool.push_back(ev);
    }
    *e = t.pool[t.used++];
    return CPSD_OK;
}
}  // namespace

const int TILE_BM[4] = {128, 128, 64, 64};
const int TILE_BN[4] = {64, 32, 128, 64};

int contract_timing(int enable) {
    timing().on = enable != 0;
    return CPSD_OK;
}
bool contract_timing_on() { return timing().on; }

int timing_begin(double flops, int64_t a, int64_t b, int64_t c, int64_t kind, cudaEvent_t *end) {
    *end = nullptr;
    if (!timing().on) return CPSD_OK;
    cudaEvent_t e0;
    CPSD_TRY(timing_event(&e0));
    CPSD_TRY(timing_event(end));
    timing().flops.push_back(flops);
    timing().shape.push_back({a, b, c, kind});
    return cuda_check(cudaEventRecord(e0, stream()), "event record");
}

int timing_end(cudaEvent_t end) {
    if (!end) return CPSD_OK;
    return cuda_check(cudaEventRecord(end, stream()), "event record");
}

int contract_records(double *ms, double *flops, int64_t *shape, int64_t maxrec, int64_t *nrec) {
    Timing &t = timing();
    int64_t n = 0;
    for (size_t i = 0; i + 1 < t.used && n < maxrec; i += 2, n++) {
        CPSD_TRY(cuda_check(cudaEventSynchronize(t.pool[i + 1]), "event sync"));
        float x = 0.f;
        CPSD_TRY(cuda_check(cudaEventElapsedTime(&x, t.pool[i], t.pool[i + 1]), "event time"));
        ms[n] = x;
        flops[n] = t.flops[i / 2];
        for (int k = 0; k < 4; k++) shape[4 * n + k] = t.shape[i / 2][k];
    }
    *nrec = n;
    return CPSD_OK;
}

int contract_time(double *ms, int64_t *launches, double *flops, int reset) {
    Timing &t = timing();
    double tot = 0.0, fl = 0.0;
    for (size_t i = 0; i + 1 < t.used; i += 2) {
        if (t.shape[i / 2][3] >= 30) continue;  // solver / layout records are not contraction work
        CPSD_TRY(cuda_check(cudaEventSynchronize(t.pool[i + 1]), "event sync"));
        float x = 0.f;
        CPSD_TRY(cuda_check(cudaEventElapsedTime(&x, t.pool[i], t.pool[i + 1]), "event time"));
        tot += x;
        fl += t.flops[i / 2];
    }
    if (ms) *ms = tot;
    if (launches) *launches = (int64_t)(t.used / 2);
    if (flops) *flops = fl;
    if (reset) {
        t.used = 0;
        t.flops.clear();
        t.shape.clear();
    }
    return CPSD_OK;
}

namespace {
// the empirical tile-shape choice: per plan, the variant that ran fastest
std::atomic<int> g_autotune{0};
std::atomic<int64_t> g_tuned{0}, g_changed{0};
std::mutex &tune_mutex() {
    static std::mutex m;
    return m;
}
std::map<const ContractPlan *, const ContractPlan *> &tuned_plans() {
    static std::map<const ContractPlan *, const ContractPlan *> m;
    return m;
}
std::vector<std::unique_ptr<ContractPlan>> &tuned_variants() {
    static std::vector<std::unique_ptr<ContractPlan>> v;
    return v;
}
// one past the largest output offset a plan writes
i64 plan_c_extent(const ContractPlan *p) {
    i64 hi = 0;
    for (const TaskDev &t : p->h_tasks) {
        i64 e = t.baseC;
        for (int u = 0; u < t.nm; u++) e += (t.mExt[u] - 1) * t.mSC[u];
        for (int u = 0; u < t.nn; u++) e += (t.nExt[u] - 1) * t.nSC[u];
        hi = std::max(hi, e + 1);
    }
    return hi;
}
int launch_tiles(const ContractPlan *p, const double *A, const double *B, double *C, double alpha);
// the fastest of the four tile shapes for plan p, timed on a scratch output
int tune_plan(const ContractPlan *p, const double *A, const double *B, const ContractPlan **best) {
    *best = p;
    const i64 n = plan_c_extent(p);
    ScratchScope sc;
    double *Ct;
    CPSD_TRY(scratch(n, &Ct));
    CPSD_TRY(cuda_check(cudaMemsetAsync(Ct, 0, sizeof(double) * (size_t)n, stream()), "tune scratch"));
    cudaEvent_t e0, e1;
    CPSD_TRY(cuda_check(cudaEventCreate(&e0), "event"));
    CPSD_TRY(cuda_check(cudaEventCreate(&e1), "event"));
    float best_ms = 1e30f;
    int rc = CPSD_OK;
    for (int c = 0; c < 4 && rc == CPSD_OK; c++) {
        const ContractPlan *q = p;
        if (c != p->cfg) {
            auto v = std::make_unique<ContractPlan>();
            v->flops = p->flops;
            v->task_mkey = p->task_mkey;
            v->task_nkey = p->task_nkey;
            v->seg_kkey = p->seg_kkey;
            finish_plan(v.get(), p->h_tasks, p->h_segs, c);
            q = v.get();
            tuned_variants().push_back(std::move(v));
        }
        float ms = 0.f;
        for (int rep = 0; rep < 2 && rc == CPSD_OK; rep++) {  // the second run is timed
            rc = cuda_check(cudaEventRecord(e0, stream()), "event record");
            if (rc == CPSD_OK) rc = launch_tiles(q, A, B, Ct, 1.0);
            if (rc == CPSD_OK) rc = cuda_check(cudaEventRecord(e1, stream()), "event record");
            if (rc == CPSD_OK) rc = cuda_check(cudaEventSynchronize(e1), "event sync");
            if (rc == CPSD_OK) rc = cuda_check(cudaEventElapsedTime(&ms, e0, e1), "event time");
        }
        if (rc == CPSD_OK && ms < best_ms * 0.97f) {  // the cost model's shape unless 3 % faster
            best_ms = ms;
            *best = q;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}
}  // namespace

int set_tile_autotune(int on) {
    g_autotune.store(on ? 1 : 0);
    return CPSD_OK;
}
int tile_autotune_stats(int64_t *tuned, int64_t *changed) {
    if (tuned) *tuned = g_tuned.load();
    if (changed) *changed = g_changed.load();
    return CPSD_OK;
}

int launch_contract(const ContractPlan *p, const double *A, const double *B, double *C, double alpha) {
    if (p->empty) return CPSD_OK;
    if (g_autotune.load()) {
        const ContractPlan *q = nullptr;
        {
            std::lock_guard<std::mutex> lock(tune_mutex());
            auto it = tuned_plans().find(p);
            if (it != tuned_plans().end()) q = it->second;
        }
        if (!q) {
            std::lock_guard<std::mutex> lock(tune_mutex());
            CPSD_TRY(tune_plan(p, A, B, &q));
            tuned_plans()[p] = q;
            g_tuned++;
            if (q != p) g_changed++;
        }
        p = q;
    }
    return launch_tiles(p, A, B, C, alpha);
}

namespace {
int launch_tiles(const ContractPlan *p, const double *A, const double *B, double *C, double alpha) {
    CPSD_TRY(const_cast<ContractPlan *>(p)->upload());
    const int bm = TILE_BM[p->cfg], bn = TILE_BN[p->cfg];
    double *part = nullptr;
    ScratchScope scope;
    if (p->nparts > 0) CPSD_TRY(scratch(p->nparts * bm * bn, &part));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (timing().on) {
        CPSD_TRY(timing_event(&e0));
        CPSD_TRY(timing_event(&e1));
        timing().flops.push_back(p->flops);
        timing().shape.push_back({p->ntasks, p->nsegs, p->ntiles, p->cfg});
        CPSD_TRY(cuda_check(cudaEventRecord(e0, stream()), "event record"));
    }
    static std::atomic<bool> attr_set{false};
    if (!attr_set) {
        CPSD_TRY(cuda_check(cudaFuncSetAttribute(k_contract<128, 64, 4, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 smem_bytes<128, 64>()), "smem attr"));
        CPSD_TRY(cuda_check(cudaFuncSetAttribute(k_contract<128, 32, 4, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 smem_bytes<128, 32>()), "smem attr"));
        CPSD_TRY(cuda_check(cudaFuncSetAttribute(k_contract<64, 128, 2, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 smem_bytes<64, 128>()), "smem attr"));
        CPSD_TRY(cuda_check(cudaFuncSetAttribute(k_contract<64, 64, 2, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 smem_bytes<64, 64>()), "smem attr"));
        attr_set = true;
    }
    switch (p->cfg) {
    case 0:
        k_contract<128, 64, 4, 2><<<p->ntiles, NT, smem_bytes<128, 64>(), stream()>>>(
            A, B, C, p->d_tasks, p->d_segs, p->d_tiles, alpha, part);
        break;
    case 1:
        k_contract<128, 32, 4, 2><<<p->ntiles, NT, smem_bytes<128, 32>(), stream()>>>(
            A, B, C, p->d_tasks, p->d_segs, p->d_tiles, alpha, part);
        break;
    case 2:
        k_contract<64, 128, 2, 4><<<p->ntiles, NT, smem_bytes<64, 128>(), stream()>>>(
            A, B, C, p->d_tasks, p->d_segs, p->d_tiles, alpha, part);
        break;
    default:
        k_contract<64, 64, 2, 4><<<p->ntiles, NT, smem_bytes<64, 64>(), stream()>>>(
            A, B, C, p->d_tasks, p->d_segs, p->d_tiles, alpha, part);
        break;
    }
    count_launch();
    ctx().flops += p->flops;
    if (e1) CPSD_TRY(cuda_check(cudaEventRecord(e1, stream()), "event record"));
    if (p->nreduce > 0) {
        k_splitk_reduce<<<p->nreduce * (bm * bn / NT), NT, 0, stream()>>>(p->d_reduce, p->d_tasks, part, C, alpha,
                                                                          bm, bn);
        count_launch();
    }
    return cuda_check(cudaGetLastError(), "k_contract");
}
}  // namespace

// ------------------------------------------- contraction without allocation
// Some callers may not allocate device memory while they run a contraction:
// a host program that hands (nearly) all of HBM to its own pool at start-up
// sees cudaMalloc fail, and cudaMalloc / cudaFree can stall the device in
// the middle of a time-critical loop.  For them, launch_contract_noalloc
// keeps the plan tables and the split-K partial tiles in one fixed region
// compiled into this library instead of the cudaMalloc'ed plan copies and
// the scratch arena launch_contract uses.  Limits and rules:
//  - the region holds CPSD_NOALLOC_SCRATCH_BYTES; a contraction whose
//    tables plus partial tiles need more is rejected (CPSD_EARG) before any
//    work is queued;
//  - nothing in the region has to start at zero: every word a call reads
//    was written earlier in the same call (tables copied in, partial tiles
//    stored in full before the reduce reads them);
//  - there is one region per device, so two calls whose work overlaps in
//    time (different streams, or host threads) race on it; calls queued on
//    one stream are ordered and safe;
//  - the first call on each device does the set-up (symbol address of the
//    region, kernel attributes); make that first call before any stream
//    capture begins;
//  - the plan tables are copied from the plan's pageable host vectors
//    (pinned staging would itself be an allocation); CUDA lets such a copy
//    start only after the work queued earlier on the stream, so a call can
//    block the host until then.
namespace {
__device__ __align__(256) unsigned char g_noalloc_scratch[CPSD_NOALLOC_SCRATCH_BYTES];

constexpr int NOALLOC_MAXDEV = 64;
// region address per device ordinal (null until set up); the set-up runs
// under a lock so that two host threads' first calls do not race on it
std::atomic<unsigned char *> g_noalloc_base[NOALLOC_MAXDEV];
std::mutex g_noalloc_setup_mutex;

int noalloc_setup(unsigned char **base) {
    int dev = 0;
    CPSD_TRY(cuda_check(cudaGetDevice(&dev), "cudaGetDevice"));
    if (dev < 0 || dev >= NOALLOC_MAXDEV) return set_error(CPSD_EARG, "device ordinal beyond 63");
    if (!g_noalloc_base[dev].load()) {
        std::lock_guard<std::mutex> lock(g_noalloc_setup_mutex);
        if (g_noalloc_base[dev].load()) {
            *base = g_noalloc_base[dev].load();
            return CPSD_OK;
        }
        void *p = nullptr;
        CPSD_TRY(cuda_check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(noalloc scratch)"));
        CPSD_TRY(cuda_check(cudaFuncSetAttribute(k_contract<128, 64, 4, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 smem_bytes<128, 64>()), "smem attr"));
        CPSD_TRY(cuda_check(cudaFuncSetAttribute(k_contract<128, 32, 4, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 smem_bytes<128, 32>()), "smem attr"));
        CPSD_TRY(cuda_check(cudaFuncSetAttribute(k_contract<64, 128, 2, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 smem_bytes<64, 128>()), "smem attr"));
        CPSD_TRY(cuda_check(cudaFuncSetAttribute(k_contract<64, 64, 2, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 smem_bytes<64, 64>()), "smem attr"));
        g_noalloc_base[dev].store((unsigned char *)p);
    }
    *base = g_noalloc_base[dev].load();
    return CPSD_OK;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }
}  // namespace

size_t contract_noalloc_bytes(const ContractPlan *p) {
    if (p->empty) return 0;
    const size_t tile = (size_t)TILE_BM[p->cfg] * TILE_BN[p->cfg] * sizeof(double);
    return align256(p->h_tasks.size() * sizeof(TaskDev)) + align256(p->h_segs.size() * sizeof(SegDev)) +
           align256(p->h_tiles.size() * sizeof(TileDev)) + align256(p->h_reduce.size() * sizeof(int)) +
           align256((size_t)p->nparts * tile);
}

int launch_contract_noalloc(const ContractPlan *p, const double *A, const double *B, double *C, double alpha) {
    if (p->empty) return CPSD_OK;
    const size_t need = contract_noalloc_bytes(p);
    if (need > (size_t)CPSD_NOALLOC_SCRATCH_BYTES)
        return set_error(CPSD_EARG, "contraction needs " + std::to_string(need) +
                                        " bytes of scratch; the no-allocation entry point holds at most " +
                                        std::to_string((size_t)CPSD_NOALLOC_SCRATCH_BYTES));
    unsigned char *base = nullptr;
    CPSD_TRY(noalloc_setup(&base));
    size_t off = 0;
    auto place = [&](const void *src, size_t bytes, void **dst) -> int {
        *dst = base + off;
        off += align256(bytes);
        if (bytes == 0) return CPSD_OK;
        return cuda_check(cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, stream()), "copy plan tables");
    };
    void *d_tasks, *d_segs, *d_tiles, *d_reduce;
    CPSD_TRY(place(p->h_tasks.data(), p->h_tasks.size() * sizeof(TaskDev), &d_tasks));
    CPSD_TRY(place(p->h_segs.data(), p->h_segs.size() * sizeof(SegDev), &d_segs));
    CPSD_TRY(place(p->h_tiles.data(), p->h_tiles.size() * sizeof(TileDev), &d_tiles));
    CPSD_TRY(place(p->h_reduce.data(), p->h_reduce.size() * sizeof(int), &d_reduce));
    double *part = p->nparts > 0 ? (double *)(base + off) : nullptr;
    const TaskDev *tk = (const TaskDev *)d_tasks;
    const SegDev *sg = (const SegDev *)d_segs;
    const TileDev *tl = (const TileDev *)d_tiles;
    const int bm = TILE_BM[p->cfg], bn = TILE_BN[p->cfg];
    cudaEvent_t e0 = nullptr, e1 = nullptr;  // timing records, as launch_contract keeps them
    if (timing().on) {
        CPSD_TRY(timing_event(&e0));
        CPSD_TRY(timing_event(&e1));
        timing().flops.push_back(p->flops);
        timing().shape.push_back({p->ntasks, p->nsegs, p->ntiles, p->cfg});
        CPSD_TRY(cuda_check(cudaEventRecord(e0, stream()), "event record"));
    }
    switch (p->cfg) {
    case 0:
        k_contract<128, 64, 4, 2><<<p->ntiles, NT, smem_bytes<128, 64>(), stream()>>>(A, B, C, tk, sg, tl, alpha, part);
        break;
    case 1:
        k_contract<128, 32, 4, 2><<<p->ntiles, NT, smem_bytes<128, 32>(), stream()>>>(A, B, C, tk, sg, tl, alpha, part);
        break;
    case 2:
        k_contract<64, 128, 2, 4><<<p->ntiles, NT, smem_bytes<64, 128>(), stream()>>>(A, B, C, tk, sg, tl, alpha, part);
        break;
    default:
        k_contract<64, 64, 2, 4><<<p->ntiles, NT, smem_bytes<64, 64>(), stream()>>>(A, B, C, tk, sg, tl, alpha, part);
        break;
    }
    count_launch();
    ctx().flops += p->flops;
    if (e1) CPSD_TRY(cuda_check(cudaEventRecord(e1, stream()), "event record"));
    if (p->nreduce > 0) {
        k_splitk_reduce<<<p->nreduce * (bm * bn / NT), NT, 0, stream()>>>((const int *)d_reduce, tk, part, C, alpha,
                                                                          bm, bn);
        count_launch();
    }
    return cuda_check(cudaGetLastError(), "k_contract (no allocation)");
}

}  // namespace cpsd
