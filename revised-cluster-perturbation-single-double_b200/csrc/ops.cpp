// DPD engine entry points, layout transforms, the mod_contract wrappers and
// the spin-free lib_cc kernels (device side: libcpsd_b200).
#include "ops.hpp"

#include <algorithm>
#include <tuple>

#include "drivers.hpp"
#include "narrow.cuh"
#include "ozaki.cuh"
#include "rowdot.cuh"
#include "shortk.cuh"
#include "solvers.cuh"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

namespace cpsd {

Ten ten_of(const cpsd_opt *t) {
    Ten x;
    x.d = desc_of(t);
    x.arr = t->arr;
    return x;
}

Ten ten(const i64 *p0, const i64 *p1, const i64 *p2, const i64 *p3, i64 iop0, i64 iop1, i64 sym, double *arr,
        i64 bs) {
    Ten x;
    x.d = make_desc(p0, p1, p2, p3, iop0, iop1, sym);
    x.arr = arr;
    x.bs = bs;
    return x;
}

static int need_init() {
    if (!ctx().init) return set_error(CPSD_ESTATE, "cpsd_init has not been called");
    return CPSD_OK;
}

namespace {
int launch_ozaki(const OzPlan *oz, const double *A, const double *B, double *C, double alpha);
void op_enter();
void op_leave();
// One outermost operation (an engine, wrapper or kernel call): the cached
// constant-operand copies handed to it stay in place until it returns,
// whatever it allocates meanwhile; copies of earlier operations may be
// evicted when memory runs out.
struct OpScope {
    OpScope() { op_enter(); }
    ~OpScope() { op_leave(); }
    OpScope(const OpScope &) = delete;
    OpScope &operator=(const OpScope &) = delete;
};
}

// CPSD_TRACE set in the environment: one line per contraction on stderr
// with its index specification, the kernel path taken and the shapes of
// its tasks (a host-side record for profiling; nothing is synchronised)
static void trace_contraction(const ContractPlan *p, const char *t1, const char *t2, const char *t3, i64 nb,
                              const char *path) {
    static const bool on = getenv("CPSD_TRACE") != nullptr;
    if (!on) return;
    i64 mM = 0, mN = 0, mK = 0;
    double out = 0;
    for (const TaskDev &t : p->h_tasks) {
        mM = std::max(mM, t.M);
        mN = std::max(mN, t.N);
        mK = std::max(mK, t.Ktot);
        out += (double)t.M * (double)t.N;
    }
    fprintf(stderr, "[cpsd] %.4s*%.4s->%.4s nb=%lld path=%s tasks=%d segs=%d tiles=%d cfg=%d flops=%.4g maxM=%lld "
            "maxN=%lld maxK=%lld outelems=%.4g\n", t1, t2, t3, (long long)nb, path, p->ntasks, p->nsegs, p->ntiles,
            p->cfg, p->flops * (double)(nb > 1 ? nb : 1), (long long)mM, (long long)mN, (long long)mK,
            out * (double)(nb > 1 ? nb : 1));
}

int engine(const Ten &v1, const char *t1, const Ten &v2, const char *t2, Ten &v3, const char *t3, double f1,
           double f2, i64 nb) {
    CPSD_TRY(need_init());
    OpScope op;
    Batch b;
    b.nb = nb;
    if (nb > 1) {
        b.strideA = v1.bs;
        b.strideB = v2.bs;
        b.strideC = v3.bs ? v3.bs : v3.len();
    }
    const ContractPlan *p;
    CPSD_TRY(plan_contract(v1.d, t1, v2.d, t2, v3.d, t3, b, &p));
    // digit tensor-core path for large contractions whose dense regrouping
    // uses at least a quarter of the padded tiles and has K of at least 256
    // (min_gflop = 0 routes every contraction that regroups)
    const OzPlan *oz = nullptr;
    if (ctx().oz_digits > 0 && !p->empty && p->flops >= ctx().oz_min_flops) {
        CPSD_TRY(plan_ozaki(p, ctx().oz_digits, &oz));
        if (oz && ctx().oz_min_flops > 0 && (oz->pad_eff < 0.25 || oz->kmin < 256)) oz = nullptr;
    }
    i64 l3 = v3.len();
    if (f2 != 1.0) {
        if (nb <= 1 || b.strideC == l3) CPSD_TRY(launch_scale(v3.arr, l3 * (nb > 1 ? nb : 1), f2));
        else
            for (i64 c = 0; c < nb; c++) CPSD_TRY(launch_scale(v3.arr + c * b.strideC, l3, f2));
    }
    if (oz) {
        trace_contraction(p, t1, t2, t3, nb, "digits");
        ctx().flops += p->flops;
        return launch_ozaki(oz, v1.arr, v2.arr, v3.arr, f1);
    }
    // at most 16 output columns (or rows): streaming kernels instead of tiles
    const NarrowPlan *np = nullptr;
    if (!p->empty) CPSD_TRY(plan_narrow(p, &np));
    if (np) {
        trace_contraction(p, t1, t2, t3, nb, np->longk ? "narrow_k" : "narrow_rows");
        ctx().flops += p->flops;
        return launch_narrow(p, np, v1.arr, v2.arr, v3.arr, f1);
    }
    // a narrow output whose rows are strided but contiguous along a short K
    const RowDotPlan *rp = nullptr;
    if (!p->empty) CPSD_TRY(plan_rowdot(p, &rp));
    if (rp) {
        trace_contraction(p, t1, t2, t3, nb, "rowdot");
        ctx().flops += p->flops;
        return launch_rowdot(p, rp, v1.arr, v2.arr, v3.arr, f1);
    }
    // a contracted range of at most 64 everywhere: the output's
    // read-modify-write bounds it, streaming kernel instead of tiles
    const ShortKPlan *sp = nullptr;
    if (!p->empty) CPSD_TRY(plan_shortk(p, &sp));
    if (sp) {
        trace_contraction(p, t1, t2, t3, nb, "shortk");
        ctx().flops += p->flops;
        return launch_shortk(p, sp, v1.arr, v2.arr, v3.arr, f1);
    }
    if (!p->empty) trace_contraction(p, t1, t2, t3, nb, "tiles");
    return launch_contract(p, v1.arr, v2.arr, v3.arr, f1);
}

namespace {

bool check_flat(const char *cur, const char pairs[][2], int n, int self) {
    for (int i = 0; i < n; i++) {
        if (i == self) continue;
        if (pairs[i][0] == cur[0] && pairs[i][1] == cur[1]) return false;
    }
    return true;
}

// Operands that stay constant while a program runs (its integrals) keep the
// expanded copies made of them until the outermost ConstOperands scope
// ends, instead of being expanded again at every contraction that needs
// them.  Only with a library-owned arena: a caller that supplied its own
// workspace gets no extra allocation.
struct ExpEntry {
    const double *src;
    std::string key;
    Desc d;
    double *buf;
    size_t bytes;
    int64_t used;  // operation (epoch) that was last handed this copy
    int uses;      // operations handed this copy in this run
};
// digit tiles (and their exponents) made of a constant operand
struct DigEntry {
    const double *src;
    uint64_t hash;
    int8_t *dig;
    int *expo;
    size_t dbytes, ebytes;
    int64_t used;
    int uses;
};
// Uses per run of each copy (source array and layout / digit plan): a copy
// that served one operation in the last run is not kept for the next run
// (expanded copies go to scratch, digit tiles to pool buffers returned
// right after their launch), where it would only hold memory that later
// work then has to take back.  Counted per host thread over one run, merged
// into the process-wide record when the run ends.
using UseKey = std::pair<const void *, std::string>;
std::map<UseKey, int> &uses_last_run() {
    static std::map<UseKey, int> m;
    return m;
}
std::mutex &uses_mutex() {
    static std::mutex m;
    return m;
}
bool single_use_last_run(const void *src, const std::string &key) {
    std::lock_guard<std::mutex> lock(uses_mutex());
    auto it = uses_last_run().find({src, key});
    return it != uses_last_run().end() && it->second == 1;
}
std::string dig_key(uint64_t h) { return "digits:" + std::to_string(h); }
struct ConstOps {
    int depth = 0;
    std::vector<const double *> arrs;
    std::vector<ExpEntry> exp;
    std::vector<DigEntry> dig;
    int64_t epoch = 0;  // outermost operations so far
    int op_depth = 0;
    std::map<UseKey, int> uses;  // this run's counts (copies given way included)
    void note(const void *src, const std::string &key, int n) {  // a copy's count
        int &u = uses[{src, key}];
        u = std::max(u, n);
    }
    void bump(const void *src, const std::string &key) { uses[{src, key}]++; }  // a use made in scratch
};
ConstOps &const_ops() {
    thread_local ConstOps c;
    return c;
}

void op_enter() {
    ConstOps &c = const_ops();
    if (c.op_depth++ == 0) c.epoch++;
}
void op_leave() { const_ops().op_depth--; }

// Device buffers of the constant-operand copies are kept after a program
// run and reused by the next one (the same workload asks for the same
// sizes), so that runs do not pay cudaMalloc / cudaFree of gigabytes.
struct PoolBuf {
    void *p;
    size_t bytes;
};
// The pool is shared by all host threads (concurrent molecules of a batch):
// an idle buffer may serve any of them.  When the driver has no room, a
// larger idle buffer serves a request whole, and only then are idle buffers
// given back (smallest first) until the allocation fits.
std::vector<PoolBuf> &pool_free() {
    static std::vector<PoolBuf> v;
    return v;
}
std::mutex &pool_mutex() {
    static std::mutex m;
    return m;
}
// actual size of every buffer handed out (a request may be served by a
// larger idle buffer; pool_put gives back the whole buffer)
std::map<void *, size_t> &pool_sizes() {
    static std::map<void *, size_t> m;
    return m;
}
void *pool_get(size_t bytes) {
    std::lock_guard<std::mutex> lock(pool_mutex());
    auto &f = pool_free();
    auto take = [&](int i) {
        void *p = f[i].p;
        pool_sizes()[p] = f[i].bytes;
        f.erase(f.begin() + i);
        return p;
    };
    int best = -1;
    for (int i = 0; i < (int)f.size(); i++)
        if (f[i].bytes >= bytes && f[i].bytes <= 2 * bytes + (1u << 20) &&
            (best < 0 || f[i].bytes < f[best].bytes))
            best = i;
    if (best >= 0) return take(best);
    void *p = nullptr;
    double t = mem_trace_on() ? host_ms() : 0.0;
    if (cudaMalloc(&p, bytes) == cudaSuccess) {
        mem_trace("pool cudaMalloc", bytes, mem_trace_on() ? host_ms() - t : 0.0);
        pool_sizes()[p] = bytes;
        return p;
    }
    cudaGetLastError();
    // out of memory: a larger idle buffer serves the request whole (memory
    // changing hands without a driver call; a cudaFree at the memory limit
    // waits for the whole device)
    for (int i = 0; i < (int)f.size(); i++)
        if (f[i].bytes >= bytes && (best < 0 || f[i].bytes < f[best].bytes)) best = i;
    if (best >= 0) {
        mem_trace("pool: larger idle buffer handed out", f[best].bytes, 0.0);
        return take(best);
    }
    // else give back idle buffers, smallest first, until the allocation fits
    std::sort(f.begin(), f.end(), [](const PoolBuf &a, const PoolBuf &b) { return a.bytes < b.bytes; });
    size_t idle = 0;
    bool ok = false;
    while (!f.empty() && !ok) {
        idle += f.front().bytes;
        cudaFree(f.front().p);
        f.erase(f.begin());
        ok = cudaMalloc(&p, bytes) == cudaSuccess;
        if (!ok) cudaGetLastError();
    }
    if (!ok) {
        arena().trim();  // and this thread's unused scratch chunks
        ok = cudaMalloc(&p, bytes) == cudaSuccess;
    }
    if (mem_trace_on()) {
        mem_trace("pool: idle buffers released", idle, 0.0);
        mem_trace("pool cudaMalloc after release", bytes, host_ms() - t, ok);
    }
    if (ok) {
        pool_sizes()[p] = bytes;
        return p;
    }
    cudaGetLastError();
    return nullptr;
}
void pool_put(void *p, size_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(pool_mutex());
    auto it = pool_sizes().find(p);
    if (it != pool_sizes().end()) {
        bytes = it->second;
        pool_sizes().erase(it);
    }
    pool_free().push_back({p, bytes});
}

}  // namespace

void *pool_take_idle(size_t min_bytes, size_t max_bytes, size_t *bytes) {
    std::lock_guard<std::mutex> lock(pool_mutex());
    auto &f = pool_free();
    int best = -1;
    for (int i = 0; i < (int)f.size(); i++)
        if (f[i].bytes >= min_bytes && f[i].bytes <= max_bytes && (best < 0 || f[i].bytes < f[best].bytes)) best = i;
    if (best < 0) return nullptr;
    void *p = f[best].p;
    *bytes = f[best].bytes;
    f.erase(f.begin() + best);
    return p;
}

size_t pool_idle_bytes() {
    std::lock_guard<std::mutex> lock(pool_mutex());
    size_t t = 0;
    for (const PoolBuf &b : pool_free()) t += b.bytes;
    return t;
}

void pool_release_idle() {
    std::lock_guard<std::mutex> lock(pool_mutex());
    const double t = mem_trace_on() ? host_ms() : 0.0;
    size_t idle = 0;
    for (PoolBuf &b : pool_free()) {
        idle += b.bytes;
        cudaFree(b.p);
    }
    pool_free().clear();
    if (mem_trace_on() && idle) mem_trace("pool release idle (cudaFree)", idle, host_ms() - t);
}

namespace {

bool is_const_operand(const double *a) {
    ConstOps &c = const_ops();
    if (c.depth == 0 || arena().external) return false;
    for (const double *x : c.arrs)
        if (x == a) return true;
    return false;
}

// Cached copies give way when device memory runs out: copies the running
// program keeps, except those handed to the operation in progress and those
// made of `keep` (the operand being requested), go back to the pool once the
// stream has finished the kernels that read it, and the idle pool is freed.
// With a request of `need` bytes only what covers it goes: the smallest copy
// that does alone, else the smallest ones together (a copy is rebuilt at a
// cost that grows with its size, so the large digit tiles of abcd stay while
// smaller copies can make room); with need 0, all of them.  Returns false
// when there was nothing to evict.
bool evict_const_except(const double *keep, size_t need) {
    ConstOps &c = const_ops();
    auto kept_e = [&](const ExpEntry &e) { return e.used == c.epoch || e.src == keep || e.buf == keep; };
    auto kept_d = [&](const DigEntry &e) { return e.used == c.epoch || e.src == keep; };
    // candidates: (bytes, expanded copy?, index)
    std::vector<std::tuple<size_t, int, size_t>> cand;
    for (size_t i = 0; i < c.exp.size(); i++)
        if (!kept_e(c.exp[i])) cand.emplace_back(c.exp[i].bytes, 1, i);
    for (size_t i = 0; i < c.dig.size(); i++)
        if (!kept_d(c.dig[i])) cand.emplace_back(c.dig[i].dbytes + c.dig[i].ebytes, 0, i);
    if (cand.empty()) return false;
    std::sort(cand.begin(), cand.end());
    size_t fr = 0, tot = 0;
    if (need) cudaMemGetInfo(&fr, &tot);
    const size_t target = need + ((size_t)256 << 20);  // 256 MB to spare
    const size_t deficit = need ? (target > fr ? target - fr : 1) : 0;
    std::vector<char> drop_e(c.exp.size(), 0), drop_d(c.dig.size(), 0);
    auto drop = [&](const std::tuple<size_t, int, size_t> &t) {
        (std::get<1>(t) ? drop_e : drop_d)[std::get<2>(t)] = 1;
    };
    if (!need) {
        for (const auto &t : cand) drop(t);
    } else {
        auto one = std::find_if(cand.begin(), cand.end(), [&](const auto &t) { return std::get<0>(t) >= deficit; });
        if (one != cand.end()) {
            drop(*one);
        } else {
            size_t freed = 0;
            for (const auto &t : cand) {
                if (freed >= deficit) break;
                drop(t);
                freed += std::get<0>(t);
            }
        }
    }
    if (getenv("CPSD_TRACE")) {  // what gives way, for the memory picture of a run
        size_t eb = 0, db = 0, ne = 0, nd = 0;
        for (size_t i = 0; i < c.exp.size(); i++)
            if (drop_e[i]) eb += c.exp[i].bytes, ne++;
        for (size_t i = 0; i < c.dig.size(); i++)
            if (drop_d[i]) db += c.dig[i].dbytes + c.dig[i].ebytes, nd++;
        fprintf(stderr,
                "[cpsd] evict: expanded copies %.2f GB (%zu), digit tiles %.2f GB (%zu) for %.2f GB; free %.2f GB\n",
                eb / 1e9, ne, db / 1e9, nd, need / 1e9, fr / 1e9);
    }
    cudaStreamSynchronize(stream());
    std::vector<ExpEntry> ke;
    std::vector<DigEntry> kd;
    std::vector<const double *> dropped;
    for (size_t i = 0; i < c.exp.size(); i++) {
        if (drop_e[i]) {
            c.note(c.exp[i].src, c.exp[i].key, c.exp[i].uses);
            pool_put(c.exp[i].buf, c.exp[i].bytes);
            dropped.push_back(c.exp[i].buf);
        } else {
            ke.push_back(c.exp[i]);
        }
    }
    for (size_t i = 0; i < c.dig.size(); i++) {
        if (drop_d[i]) {
            c.note(c.dig[i].src, dig_key(c.dig[i].hash), c.dig[i].uses);
            pool_put(c.dig[i].dig, c.dig[i].dbytes);
            pool_put(c.dig[i].expo, c.dig[i].ebytes);
        } else {
            kd.push_back(c.dig[i]);
        }
    }
    c.exp.swap(ke);
    c.dig.swap(kd);
    // an evicted expanded copy is no longer a constant operand
    c.arrs.erase(std::remove_if(c.arrs.begin(), c.arrs.end(),
                                [&](const double *x) {
                                    return std::find(dropped.begin(), dropped.end(), x) != dropped.end();
                                }),
                 c.arrs.end());
    pool_release_idle();
    return true;
}

}  // namespace

bool evict_cached_copies(size_t need) { return evict_const_except(nullptr, need); }

namespace {

}  // namespace

// CPSD_ETIMEOUT when a bounded wait of the digit path timed out on this
// thread since the last check (the word is cleared): the results of the
// operations since then are invalid.  Synchronises the stream.
int digit_error_check() {
    if (!ctx().oz_err) return CPSD_OK;
    int h = 0;
    CPSD_TRY(read_back(&h, ctx().oz_err, sizeof h));
    if (!h) return CPSD_OK;
    CPSD_TRY(cuda_check(cudaMemsetAsync(ctx().oz_err, 0, sizeof(int), stream()), "clear error word"));
    return set_error(CPSD_ETIMEOUT, "int8-digit tensor-core path: a bounded device wait timed out; the results "
                                    "of this call are invalid");
}

namespace {

int oz_error_word(int **err) {
    if (!ctx().oz_err) {
        CPSD_TRY(cuda_check(cudaMalloc(&ctx().oz_err, sizeof(int)), "cudaMalloc(error word)"));
        CPSD_TRY(cuda_check(cudaMemsetAsync(ctx().oz_err, 0, sizeof(int), stream()), "clear error word"));
    }
    *err = ctx().oz_err;
    return CPSD_OK;
}

int slice_timed(const OzPlan *oz, bool sideA, const double *src, int8_t *dig, int *expo) {
    cudaEvent_t end;
    const i64 rows = sideA ? oz->nea : oz->neb, bytes = sideA ? oz->adig : oz->bdig;
    CPSD_TRY(timing_begin(0.0, rows, bytes, (i64)oz->groups.size(), sideA ? 10 : 11, &end));
    CPSD_TRY(oz_slice(oz->S, sideA ? 128 : oz->BN, sideA ? oz->adev : oz->bdev, src, dig, expo));
    return timing_end(end);
}

// digit tiles of one operand: kept for the program run when the operand is
// constant, otherwise made in scratch (released with the caller's scope).
// A constant operand whose tiles served a single launch in the last run
// gets pool buffers that go back to the pool right after this launch (into
// *release): its memory then serves the next request without a driver call.
int digits_of(const OzPlan *oz, bool sideA, const double *src, int8_t **dig, int **expo,
              std::vector<void *> *release) {
    const uint64_t h = sideA ? oz->ahash : oz->bhash;
    const i64 bytes = sideA ? oz->adig : oz->bdig, ne = sideA ? oz->nea : oz->neb;
    if (is_const_operand(src)) {
        ConstOps &c = const_ops();
        for (DigEntry &e : c.dig)
            if (e.src == src && e.hash == h) {
                e.used = c.epoch;
                e.uses++;
                *dig = e.dig;
                *expo = e.expo;
                return CPSD_OK;
            }
        const size_t db = (size_t)std::max<i64>(bytes, 16), eb = sizeof(int) * (size_t)std::max<i64>(ne, 1);
        if (single_use_last_run(src, dig_key(h))) {
            c.bump(src, dig_key(h));
            int8_t *d = (int8_t *)pool_get(db);
            int *x = d ? (int *)pool_get(eb) : nullptr;
            if (d && x) {
                release->push_back(d);
                release->push_back(x);
                *dig = d;
                *expo = x;
                return slice_timed(oz, sideA, src, d, x);
            }
            pool_put(d, db);
            CPSD_TRY(scratch(bytes, dig));
            CPSD_TRY(scratch(ne, expo));
            return slice_timed(oz, sideA, src, *dig, *expo);
        }
        int8_t *d = (int8_t *)pool_get(db);
        int *x = d ? (int *)pool_get(eb) : nullptr;
        if (!(d && x)) {
            pool_put(d, db);
            d = nullptr;
            if (evict_const_except(src, db + eb)) {
                d = (int8_t *)pool_get(db);
                x = d ? (int *)pool_get(eb) : nullptr;
            }
        }
        if (d && x) {
            c.dig.push_back({src, h, d, x, db, eb, c.epoch, 1});
            *dig = d;
            *expo = x;
            return slice_timed(oz, sideA, src, d, x);
        }
        pool_put(d, db);  // no room to keep them: make them in scratch
    }
    CPSD_TRY(scratch(bytes, dig));
    CPSD_TRY(scratch(ne, expo));
    return slice_timed(oz, sideA, src, *dig, *expo);
}

int launch_ozaki(const OzPlan *oz, const double *A, const double *B, double *C, double alpha) {
    CPSD_TRY(const_cast<OzPlan *>(oz)->upload());
    ScratchScope sc;
    int8_t *ad, *bd;
    int *ea, *eb, *err;
    CPSD_TRY(oz_error_word(&err));
    std::vector<void *> release;
    struct Release {  // after the launch's kernels are done
        std::vector<void *> &r;
        ~Release() {
            if (r.empty()) return;
            cudaStreamSynchronize(stream());
            for (void *p : r) pool_put(p, 0);
        }
    } rel{release};
    CPSD_TRY(digits_of(oz, true, A, &ad, &ea, &release));
    CPSD_TRY(digits_of(oz, false, B, &bd, &eb, &release));
    cudaEvent_t end;
    // record: groups, bytes of the digit tiles the launch streams, bytes of
    // C read and written (once per K chunk)
    i64 cbytes = 0;
    for (const OzGroup &g : oz->groups) cbytes += 16 * g.M * g.N;
    const i64 nchunk = (oz->kt_max + oz->kt_chunk - 1) / oz->kt_chunk;
    CPSD_TRY(timing_begin(oz->flops, (i64)oz->groups.size(), oz->adig + oz->bdig, cbytes * nchunk, 12, &end));
    for (int kt0 = 0; kt0 < oz->kt_max; kt0 += oz->kt_chunk)
        CPSD_TRY(oz_gemm(oz->S, oz->dev, ad, bd, ea, eb, C, alpha, kt0, kt0 + oz->kt_chunk, err));
    return timing_end(end);
}

int expand_cached(const Ten &v, bool e0, bool e1, Ten *out, bool *done) {
    *done = false;
    ConstOps &c = const_ops();
    if (c.depth == 0 || v.bs != 0 || arena().external) return CPSD_OK;
    bool is_const = false;
    for (const double *a : c.arrs) is_const |= (a == v.arr);
    if (!is_const) return CPSD_OK;
    std::string key = v.d.key() + (e0 ? "E" : "-") + (e1 ? "E" : "-");
    for (ExpEntry &e : c.exp)
        if (e.src == v.arr && e.key == key) {
            e.used = c.epoch;
            e.uses++;
            *out = v;
            out->d = e.d;
            out->arr = e.buf;
            *done = true;
            return CPSD_OK;
        }
    if (single_use_last_run(v.arr, key)) {  // expand into scratch as usual
        c.bump(v.arr, key);
        return CPSD_OK;
    }
    const PairMapPlan *pm;
    Desc d;
    CPSD_TRY(plan_pairmap(v.d, e0 ? PAIR_EXPAND : PAIR_ID, e1 ? PAIR_EXPAND : PAIR_ID, 1, 1, &d, &pm));
    const size_t bytes = sizeof(double) * (size_t)std::max<i64>(d.len(), 1);
    double *buf = (double *)pool_get(bytes);
    if (!buf && evict_const_except(v.arr, bytes)) buf = (double *)pool_get(bytes);
    if (!buf) return CPSD_OK;  // no room to keep it: expand into scratch as usual
    c.exp.push_back({v.arr, key, d, buf, bytes, c.epoch, 1});
    c.arrs.push_back(buf);  // derived from a constant operand: constant too
    CPSD_TRY(launch_pairmap(pm, v.arr, buf, 1.0, 0.0, 1, 0, d.len()));
    *out = v;
    out->d = d;
    out->arr = buf;
    *done = true;
    return CPSD_OK;
}

// iexpso into scratch: expanded copy (batched when v is)
int expand(const Ten &v, bool e0, bool e1, i64 nb, Ten *out) {
    *out = v;
    if (!e0 && !e1) return CPSD_OK;
    bool done;
    CPSD_TRY(expand_cached(v, e0, e1, out, &done));
    if (done) return CPSD_OK;
    const PairMapPlan *pm;
    Desc d;
    CPSD_TRY(plan_pairmap(v.d, e0 ? PAIR_EXPAND : PAIR_ID, e1 ? PAIR_EXPAND : PAIR_ID, 1, 1, &d, &pm));
    i64 n = d.len(), copies = v.bs ? nb : 1;
    double *buf;
    CPSD_TRY(scratch(n * copies, &buf));
    CPSD_TRY(launch_pairmap(pm, v.arr, buf, 1.0, 0.0, copies, v.bs, n));
    out->d = d;
    out->arr = buf;
    out->bs = v.bs ? n : 0;
    return CPSD_OK;
}

// v3 += P(X): antisymmetrise / compress pairs of the full-ish result X
int finish(const Ten &X, Ten &v3, bool anti0, bool anti1, bool comp0, bool comp1, i64 nb) {
    int op0 = anti0 ? (comp0 ? PAIR_ANTI_COMPRESS : PAIR_ANTI) : (comp0 ? PAIR_COMPRESS : PAIR_ID);
    int op1 = anti1 ? (comp1 ? PAIR_ANTI_COMPRESS : PAIR_ANTI) : (comp1 ? PAIR_COMPRESS : PAIR_ID);
    const PairMapPlan *pm;
    Desc d;
    CPSD_TRY(plan_pairmap(X.d, op0, op1, v3.d.iop[0], v3.d.iop[1], &d, &pm));
    if (d.iop[0] != v3.d.iop[0] || d.iop[1] != v3.d.iop[1]) return set_error(CPSD_ELAYOUT, "result layout mismatch");
    i64 s3 = nb > 1 ? (v3.bs ? v3.bs : v3.len()) : 0;
    return launch_pairmap(pm, X.arr, v3.arr, 1.0, 1.0, nb, X.bs, s3);
}

void pad(const char *t, int n, const char *tail, char out[5]) {
    for (int i = 0; i < 4; i++) out[i] = i < n ? t[i] : tail[i - n];
    out[4] = 0;
}

}  // namespace

ConstOperands::ConstOperands(const double *const *arrs, int n) {
    ConstOps &c = const_ops();
    if (c.depth++ == 0) c.arrs.assign(arrs, arrs + n);
}

ConstOperands::~ConstOperands() {
    ConstOps &c = const_ops();
    if (--c.depth > 0) return;
    // the buffers go back to the pool once the kernels that read them are
    // done (the next user may run on another stream)
    if (!c.exp.empty() || !c.dig.empty()) cudaStreamSynchronize(stream());
    for (ExpEntry &e : c.exp) {
        c.note(e.src, e.key, e.uses);
        pool_put(e.buf, e.bytes);
    }
    for (DigEntry &e : c.dig) {
        c.note(e.src, dig_key(e.hash), e.uses);
        pool_put(e.dig, e.dbytes);
        pool_put(e.expo, e.ebytes);
    }
    {
        std::lock_guard<std::mutex> lock(uses_mutex());
        for (const auto &u : c.uses) uses_last_run()[u.first] = u.second;
    }
    c.uses.clear();
    c.exp.clear();
    c.dig.clear();
    c.arrs.clear();
}

// vv2v_444 (src/lib_cc/mod_contract.f90:10-162): v3 += fact * P1 P2 {v1 v2}
int w444(const Ten &v1, const Ten &v2, Ten &v3, double fact, const char *t1, const char *t2, const char *t3,
         i64 anti, i64 nb) {
    OpScope op;
    if (anti < 0 || anti > 3) return set_error(CPSD_EARG, "vv2v_444: anti must be 0..3");
    const char pair[6][2] = {{t1[0], t1[1]}, {t1[2], t1[3]}, {t2[0], t2[1]},
                             {t2[2], t2[3]}, {t3[0], t3[1]}, {t3[2], t3[3]}};
    i64 iop[6] = {v1.d.iop[0], v1.d.iop[1], v2.d.iop[0], v2.d.iop[1], v3.d.iop[0], v3.d.iop[1]};
    bool iexp[6] = {};
    for (int i = 0; i < 6; i++)
        if (check_flat(pair[i], pair, 6, i) && iop[i] != 1) {
            iexp[i] = true;
            iop[i] = 1;
        }
    if (anti == 0 && (iexp[4] || iexp[5]))
        return set_error(CPSD_ELAYOUT, "vv2v_444: packed result pair needs antisymmetrisation");
    ScratchScope sc;
    Ten e1, e2;
    CPSD_TRY(expand(v1, iexp[0], iexp[1], nb, &e1));
    CPSD_TRY(expand(v2, iexp[2], iexp[3], nb, &e2));
    if (anti == 0) return engine(e1, t1, e2, t2, v3, t3, fact, 1.0, nb);
    Ten X = v3;
    X.d.iop[0] = iop[4];
    X.d.iop[1] = iop[5];
    i64 n = X.d.len();
    CPSD_TRY(scratch(n * nb, &X.arr));
    X.bs = nb > 1 ? n : 0;
    CPSD_TRY(launch_scale(X.arr, n * nb, 0.0));
    CPSD_TRY(engine(e1, t1, e2, t2, X, t3, fact, 1.0, nb));
    return finish(X, v3, anti == 1 || anti == 3, anti == 2 || anti == 3, iexp[4], iexp[5], nb);
}

// vv2v_424 (src/lib_cc/mod_contract.f90:220-367)
int w424(const Ten &v1, const Ten &v2, Ten &v3, double fact, const char *t1, const char *t2, const char *t3,
         i64 anti, i64 nb) {
    OpScope op;
    if (anti < 0 || anti > 2) return set_error(CPSD_EARG, "vv2v_424: anti must be 0..2");
    const char pair[4][2] = {{t1[0], t1[1]}, {t1[2], t1[3]}, {t3[0], t3[1]}, {t3[2], t3[3]}};
    i64 iop[4] = {v1.d.iop[0], v1.d.iop[1], v3.d.iop[0], v3.d.iop[1]};
    bool iexp[4] = {};
    for (int i = 0; i < 4; i++)
        if (check_flat(pair[i], pair, 4, i) && iop[i] != 1) {
            iexp[i] = true;
            iop[i] = 1;
        }
    if ((anti != 1 && iexp[2]) || (anti != 2 && iexp[3]))
        return set_error(CPSD_ELAYOUT, "vv2v_424: an expanded result pair must be antisymmetrised");
    char n2[5];
    pad(t2, 2, "..", n2);
    ScratchScope sc;
    Ten e1;
    CPSD_TRY(expand(v1, iexp[0], iexp[1], nb, &e1));
    if (anti == 0) return engine(e1, t1, v2, n2, v3, t3, fact, 1.0, nb);
    Ten X = v3;
    X.d.iop[0] = iop[2];
    X.d.iop[1] = iop[3];
    i64 n = X.d.len();
    CPSD_TRY(scratch(n * nb, &X.arr));
    X.bs = nb > 1 ? n : 0;
    CPSD_TRY(launch_scale(X.arr, n * nb, 0.0));
    CPSD_TRY(engine(e1, t1, v2, n2, X, t3, fact, 1.0, nb));
    return finish(X, v3, anti == 1, anti == 2, iexp[2], iexp[3], nb);
}

// vv2v_442 (src/lib_cc/mod_contract.f90:369-455)
int w442(const Ten &v1, const Ten &v2, Ten &v3, double fact, const char *t1, const char *t2, const char *t3,
         i64 nb) {
    OpScope op;
    const char pair[4][2] = {{t1[0], t1[1]}, {t1[2], t1[3]}, {t2[0], t2[1]}, {t2[2], t2[3]}};
    i64 iop[4] = {v1.d.iop[0], v1.d.iop[1], v2.d.iop[0], v2.d.iop[1]};
    bool iexp[4] = {};
    for (int i = 0; i < 4; i++)
        if (check_flat(pair[i], pair, 4, i) && iop[i] != 1) iexp[i] = true;
    char n3[5];
    pad(t3, 2, "..", n3);
    ScratchScope sc;
    Ten e1, e2;
    CPSD_TRY(expand(v1, iexp[0], iexp[1], nb, &e1));
    CPSD_TRY(expand(v2, iexp[2], iexp[3], nb, &e2));
    return engine(e1, t1, e2, t2, v3, n3, fact, 1.0, nb);
}

// vv2v_422 (src/lib_cc/mod_contract.f90:184-200)
int w422(const Ten &v1, const Ten &v2, Ten &v3, double fact, const char *t1, const char *t2, const char *t3,
         i64 nb) {
    char b[5], c[5];
    pad(t2, 2, "+-", b);
    pad(t3, 2, "+-", c);
    return w444(v1, v2, v3, fact, t1, b, c, 0, nb);
}

// vv2v_222 (src/lib_cc/mod_contract.f90:166-182)
int w222(const Ten &v1, const Ten &v2, Ten &v3, double fact, const char *t1, const char *t2, const char *t3,
         i64 nb) {
    char a[5], b[5], c[5];
    pad(t1, 2, "=+", a);
    pad(t2, 2, "=-", b);
    pad(t3, 2, "+-", c);
    return w444(v1, v2, v3, fact, a, b, c, 0, nb);
}

// vv2v_224 (src/lib_cc/mod_contract.f90:202-218)
int w224(const Ten &v1, const Ten &v2, Ten &v3, double fact, const char *t1, const char *t2, const char *t3,
         i64 anti, i64 nb) {
    char a[5], b[5];
    pad(t1, 2, "+-", a);
    pad(t2, 2, "+-", b);
    return w444(v1, v2, v3, fact, a, b, t3, anti, nb);
}

// Vector-Jacobian product of the vv2v_444 form v3 += fact * P{v1 v2}: G +=
// d<Y, v3> / d(operand `which`) (0: v1, 1: v2), the other operand fixed.
// Every wrapper above is this form with padded specs (422 / 222 / 224 pad
// with "+-" / "=+" / "=-", 424 / 442 pad the 2-index operand / result with
// ".."), so one routine reverses them all.  The forward chain expand ->
// contract -> antisymmetrise / compress is run backwards with each step
// replaced by its adjoint: antisymmetrise-and-compress by expansion (the
// cotangent of a packed p<q element goes to (p,q) and, negated, to (q,p)),
// antisymmetrise by itself, the contraction by the contraction of Y with
// the other operand onto the operand's letters, and the operand's
// expansion by antisymmetrise-and-compress.  One copy (nb = 1).
int vjp444(const Ten &v1, const Ten &v2, const Ten &Y, Ten &G, int which, double fact, const char *t1,
           const char *t2, const char *t3, i64 anti) {
    OpScope op;
    if (anti < 0 || anti > 3) return set_error(CPSD_EARG, "vjp444: anti must be 0..3");
    if (which != 0 && which != 1) return set_error(CPSD_EARG, "vjp444: operand must be 0 or 1");
    const char pair[6][2] = {{t1[0], t1[1]}, {t1[2], t1[3]}, {t2[0], t2[1]},
                             {t2[2], t2[3]}, {t3[0], t3[1]}, {t3[2], t3[3]}};
    const i64 iop[6] = {v1.d.iop[0], v1.d.iop[1], v2.d.iop[0], v2.d.iop[1], Y.d.iop[0], Y.d.iop[1]};
    bool iexp[6] = {};
    for (int i = 0; i < 6; i++)
        if (check_flat(pair[i], pair, 6, i) && iop[i] != 1) {
            if (iop[i] != 0) return set_error(CPSD_ELAYOUT, "vjp444: only antisymmetric (iop 0) pairs expand");
            iexp[i] = true;
        }
    const bool a0 = anti == 1 || anti == 3, a1 = anti == 2 || anti == 3;
    if ((!a0 && iexp[4]) || (!a1 && iexp[5]))
        return set_error(CPSD_ELAYOUT, "vjp444: packed result pair needs antisymmetrisation");
    ScratchScope sc;
    // cotangent of the contraction result: adjoint of finish()
    Ten X = Y;
    X.bs = 0;
    if (anti != 0) {
        const int op0 = a0 ? (iexp[4] ? PAIR_EXPAND : PAIR_ANTI) : PAIR_ID;
        const int op1 = a1 ? (iexp[5] ? PAIR_EXPAND : PAIR_ANTI) : PAIR_ID;
        const PairMapPlan *pm;
        Desc d;
        CPSD_TRY(plan_pairmap(Y.d, op0, op1, 1, 1, &d, &pm));
        X.d = d;
        CPSD_TRY(scratch(d.len(), &X.arr));
        CPSD_TRY(launch_pairmap(pm, Y.arr, X.arr, 1.0, 0.0));
    }
    const Ten &other = which == 0 ? v2 : v1;
    const char *ts = which == 0 ? t1 : t2, *to = which == 0 ? t2 : t1;
    const bool *ex_s = iexp + 2 * which, *ex_o = iexp + 2 * (1 - which);
    Ten eo;
    CPSD_TRY(expand(other, ex_o[0], ex_o[1], 1, &eo));
    if (!ex_s[0] && !ex_s[1]) return engine(X, t3, eo, to, G, ts, fact, 1.0);
    // the operand's packed pairs were expanded: contract into the full
    // layout, then antisymmetrise-and-compress into G
    Ten E = G;
    E.bs = 0;
    if (ex_s[0]) E.d.iop[0] = 1;
    if (ex_s[1]) E.d.iop[1] = 1;
    const i64 n = E.d.len();
    CPSD_TRY(scratch(n, &E.arr));
    CPSD_TRY(launch_scale(E.arr, n, 0.0));
    CPSD_TRY(engine(X, t3, eo, to, E, ts, fact, 1.0));
    const PairMapPlan *pm;
    Desc d;
    CPSD_TRY(plan_pairmap(E.d, ex_s[0] ? PAIR_ANTI_COMPRESS : PAIR_ID, ex_s[1] ? PAIR_ANTI_COMPRESS : PAIR_ID,
                          G.d.iop[0], G.d.iop[1], &d, &pm));
    if (d.iop[0] != G.d.iop[0] || d.iop[1] != G.d.iop[1]) return set_error(CPSD_ELAYOUT, "vjp444: layout mismatch");
    return launch_pairmap(pm, E.arr, G.arr, 1.0, 1.0);
}

// ------------------------------------------------ lib_cc kernels (spin-free)
int k_c1_r1iabj(Ten &c1, const Ten &r1, const Ten &V, double f, i64 nb) {
    return w422(V, r1, c1, f, "fnai", "fn", "ai", nb);
}
int k_c1_r1Fae(Ten &c1, const Ten &r1, const Ten &F, double f, i64 nb) {
    return w222(F, r1, c1, f, "ae", "ei", "ai", nb);
}
int k_c1_r1Fmi(Ten &c1, const Ten &r1, const Ten &F, double f, i64 nb) {
    return w222(r1, F, c1, -f, "am", "mi", "ai", nb);
}
int k_c1_r2abci(Ten &c1, const Ten &r2, const Ten &V, double f, i64 nb) {
    return w442(V, r2, c1, r2.d.iop[0] == 0 ? f : 0.5 * f, "feam", "feim", "ai", nb);
}
int k_c1_r2ijka(Ten &c1, const Ten &r2, const Ten &V, double f, i64 nb) {
    return w442(r2, V, c1, r2.d.iop[1] == 0 ? -f : -0.5 * f, "aemn", "mnie", "ai", nb);
}
int k_c2_r1abci(Ten &c2, const Ten &r1, const Ten &V, double f, i64 nb) {
    return w424(V, r1, c2, f, "abej", "ei", "abij", 2, nb);
}
int k_c2_r1ijka(Ten &c2, const Ten &r1, const Ten &V, double f, i64 nb) {
    return w424(V, r1, c2, -f, "ijmb", "am", "abij", 1, nb);
}
int k_c2_r2Wmbej(Ten &c2, const Ten &r2, const Ten &W, double f, i64 nb) {
    return w444(r2, W, c2, f, "aeim", "embj", "abij", 3, nb);
}
int k_c2_r2Wmnij(Ten &c2, const Ten &r2, const Ten &W, double f, i64 nb) {
    return w444(r2, W, c2, r2.d.iop[0] == 0 ? f : 0.5 * f, "abmn", "mnij", "abij", 0, nb);
}
namespace {
// ------------------------------------------- out-of-core particle ladder
// abcd in host memory (too large for HBM): the reference streams it from
// disk in blocks of rows (p_c2_r2abcd_h, src/lib_cc/c2_r2abcd.f90:29-95);
// here each irrep block V_h (n_ab x n_ef, column-major) is streamed in
// panels of whole columns (contiguous in host memory) through two device
// staging buffers on a copy stream, each panel's GEMM
//   C_g(ab, ij) += f V_h(ab, ef0..ef1) R_g(ef0..ef1, ij)   (g = h x sym(R))
// queued on the library stream as soon as its copy has landed, so the copy
// of the next panel overlaps the GEMM of this one.  Host memory allocated
// pinned (cudaHostAlloc / cudaHostRegister) is read at full PCIe / C2C
// speed; pageable memory works too, with staged copies.
std::atomic<size_t> g_panel_bytes{(size_t)1 << 30};

bool host_resident(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeUnregistered;
}

struct CopyLane {  // per host thread: copy stream and events
    cudaStream_t cs = nullptr;
    cudaEvent_t start = nullptr, copied[2] = {}, used[2] = {};
    int init() {
        if (cs) return CPSD_OK;
        CPSD_TRY(cuda_check(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "copy stream"));
        CPSD_TRY(cuda_check(cudaEventCreateWithFlags(&start, cudaEventDisableTiming), "event"));
        for (int b = 0; b < 2; b++) {
            CPSD_TRY(cuda_check(cudaEventCreateWithFlags(&copied[b], cudaEventDisableTiming), "event"));
            CPSD_TRY(cuda_check(cudaEventCreateWithFlags(&used[b], cudaEventDisableTiming), "event"));
        }
        return CPSD_OK;
    }
};

int stream_abcd(Ten &c2, const Ten &r2, const Ten &V, double f, i64 nb) {
    OpScope op;
    const Desc &dv = V.d, &dr = r2.d, &dc = c2.d;
    bool ok = dv.sym == 1 && dv.iop[0] == dc.iop[0] && dv.iop[1] == dr.iop[0] && dc.iop[1] == dr.iop[1] &&
              dc.sym == dr.sym;
    for (int h = 0; h < 8 && ok; h++)
        ok = dv.pop[0][h] == dc.pop[0][h] && dv.pop[1][h] == dc.pop[1][h] && dv.pop[2][h] == dr.pop[0][h] &&
             dv.pop[3][h] == dr.pop[1][h] && dc.pop[2][h] == dr.pop[2][h] && dc.pop[3][h] == dr.pop[3][h];
    if (!ok)
        return set_error(CPSD_ELAYOUT, "host-resident abcd: the ab / ef pairs of V, R2 and C2 must match (packed alike)");
    thread_local CopyLane lane;
    CPSD_TRY(lane.init());
    ScratchScope sc;
    const i64 words = std::max<i64>(1, (i64)(g_panel_bytes.load() / sizeof(double)));
    double *stg[2];
    CPSD_TRY(scratch(words, &stg[0]));
    CPSD_TRY(scratch(words, &stg[1]));
    // the staging memory may still be read by earlier work on the library
    // stream: the copy stream starts after it
    CPSD_TRY(cuda_check(cudaEventRecord(lane.start, stream()), "event record"));
    CPSD_TRY(cuda_check(cudaStreamWaitEvent(lane.cs, lane.start, 0), "stream wait"));
    int buf = 0;
    bool used[2] = {false, false};
    const i64 sB = nb > 1 ? (r2.bs ? r2.bs : dr.len()) : 0, sC = nb > 1 ? (c2.bs ? c2.bs : dc.len()) : 0;
    for (i64 h = 1; h <= ctx().nirrep; h++) {
        const i64 nab = dv.nleft(h), nef = dv.nright(h), g = dp(h, dr.sym), nij = dr.nright(g);
        if (nab == 0 || nef == 0 || nij == 0) continue;
        const double *Vh = V.arr + dv.block_base(h);
        const double *Rg = r2.arr + dr.block_base(g);
        double *Cg = c2.arr + dc.block_base(g);
        const i64 kc = std::max<i64>(1, std::min<i64>(nef, words / nab));
        if (nab > words) return set_error(CPSD_EARG, "host-resident abcd: one column exceeds the staging buffer");
        for (i64 k0 = 0; k0 < nef; k0 += kc) {
            const i64 kn = std::min(kc, nef - k0);
            if (used[buf]) CPSD_TRY(cuda_check(cudaStreamWaitEvent(lane.cs, lane.used[buf], 0), "stream wait"));
            CPSD_TRY(cuda_check(cudaMemcpyAsync(stg[buf], Vh + k0 * nab, sizeof(double) * (size_t)(nab * kn),
                                                cudaMemcpyHostToDevice, lane.cs),
                                "abcd panel copy"));
            CPSD_TRY(cuda_check(cudaEventRecord(lane.copied[buf], lane.cs), "event record"));
            CPSD_TRY(cuda_check(cudaStreamWaitEvent(stream(), lane.copied[buf], 0), "stream wait"));
            const ContractPlan *p;
            CPSD_TRY(plan_gemm(nab, nij, kn, nab, nef, nab, nb, sB, sC, &p));
            CPSD_TRY(launch_contract(p, stg[buf], Rg + k0, Cg, f));
            CPSD_TRY(cuda_check(cudaEventRecord(lane.used[buf], stream()), "event record"));
            used[buf] = true;
            buf ^= 1;
        }
    }
    return CPSD_OK;
}
}  // namespace

int k_c2_r2abcd(Ten &c2, const Ten &r2, const Ten &V, double f, i64 nb) {
    const double fr = r2.d.iop[0] == 1 ? 0.5 * f : f;
    if (V.arr && host_resident(V.arr)) return stream_abcd(c2, r2, V, fr, nb);
    return w444(V, r2, c2, fr, "abef", "efij", "abij", 0, nb);
}
int k_c2_r2Fae(Ten &c2, const Ten &r2, const Ten &F, double f, i64 nb) {
    return w424(r2, F, c2, f, "aeij", "be", "abij", 1, nb);
}
int k_c2_r2Fmi(Ten &c2, const Ten &r2, const Ten &F, double f, i64 nb) {
    return w424(r2, F, c2, -f, "abim", "mj", "abij", 2, nb);
}
int k_Fmi_r2abij(Ten &F, const Ten &r2, const Ten &V, double f, i64 nb) {
    return w442(V, r2, F, r2.d.iop[0] == 1 ? 0.5 * f : f, "efmn", "efin", "mi", nb);
}
int k_Fae_r2abij(Ten &F, const Ten &r2, const Ten &V, double f, i64 nb) {
    return w442(r2, V, F, r2.d.iop[1] == 0 ? -f : -0.5 * f, "afmn", "efmn", "ae", nb);
}
int k_Fmi_r1ijka(Ten &F, const Ten &r1, const Ten &V, double f, i64 nb) {
    return w422(V, r1, F, f, "mnie", "en", "mi", nb);
}
int k_Fae_r1abci(Ten &F, const Ten &r1, const Ten &V, double f, i64 nb) {
    return w422(V, r1, F, f, "efam", "fm", "ae", nb);
}
int k_Wkbij_r2ijka(Ten &W, const Ten &r2, const Ten &V, double f, i64 nb) {
    return w444(V, r2, W, f, "klic", "bcjl", "ijkb", 1, nb);
}
// Wkbij_r2abci.f90:3-43: tmp(ij,bk) = -.5 V(cd,bk) r(cd,ij); W(ij,kb) += tmp(ij,bk)
int k_Wkbij_r2abci(Ten &W, const Ten &r2, const Ten &V, double f, i64 nb) {
    OpScope op;
    ScratchScope sc;
    Ten tmp = W;
    std::swap(tmp.d.pop[2], tmp.d.pop[3]);
    tmp.d.iop[1] = 1;
    i64 n = tmp.d.len();
    CPSD_TRY(scratch(n * nb, &tmp.arr));
    tmp.bs = nb > 1 ? n : 0;
    CPSD_TRY(launch_scale(tmp.arr, n * nb, 0.0));
    CPSD_TRY(w444(r2, V, tmp, r2.d.iop[0] == 0 ? -f : -0.5 * f, "cdij", "cdbk", "ijbk", 0, nb));
    const PairMapPlan *pm;
    Desc d;
    CPSD_TRY(plan_pairmap(tmp.d, PAIR_ID, PAIR_SWAP, 1, 1, &d, &pm));
    i64 sw = nb > 1 ? (W.bs ? W.bs : W.len()) : 0;
    return launch_pairmap(pm, tmp.arr, W.arr, 1.0, 1.0, nb, tmp.bs, sw);
}
int k_Wmbej_r2abij(Ten &W, const Ten &r2, const Ten &V, double f, i64 nb) {
    return w444(V, r2, W, 0.5 * f, "fenm", "bfjn", "embj", 0, nb);
}
int k_Wmbej_r1abci(Ten &W, const Ten &r1, const Ten &V, double f, i64 nb) {
    return w424(V, r1, W, f, "febm", "fj", "embj", 0, nb);
}
int k_Wmbej_r1ijka(Ten &W, const Ten &r1, const Ten &V, double f, i64 nb) {
    return w424(V, r1, W, -f, "nmje", "bn", "embj", 0, nb);
}
int k_Wmnij_r1ijka(Ten &W, const Ten &r1, const Ten &V, double f, i64 nb) {
    return w424(V, r1, W, f, "mnie", "ej", "mnij", 2, nb);
}
int k_Wmnij_r2abij(Ten &W, const Ten &r2, const Ten &V, double f, i64 nb) {
    return w444(V, r2, W, r2.d.iop[0] == 0 ? f : 0.5 * f, "efmn", "efij", "mnij", 0, nb);
}
// kernels of the second-order ground state (grCPSd.SF calL1_VTT / calL2_VTT)
int k_Wkbij_r1iabj(Ten &W, const Ten &r1, const Ten &V, double f, i64 nb) {
    return w424(V, r1, W, -f, "ckbj", "ci", "ijkb", 1, nb);
}
int k_Wabdj_r1abcd(Ten &W, const Ten &r1, const Ten &V, double f, i64 nb) {
    return w424(V, r1, W, f, "abdc", "cj", "abdj", 0, nb);
}
int k_Wkbij_r1Uklij(Ten &W, const Ten &r1, const Ten &U, double f, i64 nb) {
    return w424(U, r1, W, -f, "klij", "bl", "ijkb", 0, nb);
}
int k_Fme_r1abij(Ten &F, const Ten &r1, const Ten &V, double f, i64 nb) {
    return w422(V, r1, F, f, "efmn", "fn", "em", nb);
}
int k_c1_r2Fme(Ten &c1, const Ten &r2, const Ten &F, double f, i64 nb) {
    return w422(r2, F, c1, f, "aeim", "em", "ai", nb);
}
// kernels of the excited-state grCPS(D) (EE-grCPSd.SF calEigenCISDoo, calJ, calC_VTTR)
int k_c1d_l1Wibaj(Ten &c1, const Ten &l1, const Ten &W, double f, i64 nb) {
    return w422(W, l1, c1, f, "aibj", "bj", "ai", nb);
}
int k_c1d_l1fab(Ten &c1, const Ten &l1, const Ten &F, double f, i64 nb) {
    return w222(F, l1, c1, -f, "ba", "bi", "ai", nb);
}
int k_c1d_l1fij(Ten &c1, const Ten &l1, const Ten &F, double f, i64 nb) {
    return w222(l1, F, c1, f, "aj", "ij", "ai", nb);
}
int k_Fae_r1fia(Ten &c1, const Ten &r1, const Ten &F, double f, i64 nb) {
    return w222(r1, F, c1, -f, "al", "el", "ae", nb);
}
int k_Fmi_r1fia(Ten &c1, const Ten &r1, const Ten &F, double f, i64 nb) {
    return w222(F, r1, c1, f, "dm", "di", "mi", nb);
}
int k_Wkbij_r2Fkc(Ten &c1, const Ten &r2, const Ten &F, double f, i64 nb) {
    return w424(r2, F, c1, -f, "cbij", "ck", "ijkb", 0, nb);
}
int k_Wlkjd_r1abij(Ten &c1, const Ten &r1, const Ten &V, double f, i64 nb) {
    return w424(V, r1, c1, f, "cdlk", "cj", "lkjd", 0, nb);
}

// ------------------------------------------ adjoints of the lib_cc kernels
// vjp_<name>(a, b, Y, G, which, f): G += d<Y, out>/da (which 0) or /db
// (which 1) of out += f * <name>(a, b), with the operand order, specs and
// factors of the forward kernels above (a 2-index operand or result padded
// the way its wrapper pads it).
int vjp_c1_r1iabj(const Ten &r1, const Ten &V, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(V, r1, Y, G, 1 - which, f, "fnai", "fn+-", "ai+-", 0);
}
int vjp_c1_r1Fae(const Ten &r1, const Ten &F, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(F, r1, Y, G, 1 - which, f, "ae=+", "ei=-", "ai+-", 0);
}
int vjp_c1_r1Fmi(const Ten &r1, const Ten &F, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(r1, F, Y, G, which, -f, "am=+", "mi=-", "ai+-", 0);
}
int vjp_c1_r2abci(const Ten &r2, const Ten &V, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(V, r2, Y, G, 1 - which, r2.d.iop[0] == 0 ? f : 0.5 * f, "feam", "feim", "ai..", 0);
}
int vjp_c1_r2ijka(const Ten &r2, const Ten &V, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(r2, V, Y, G, which, r2.d.iop[1] == 0 ? -f : -0.5 * f, "aemn", "mnie", "ai..", 0);
}
int vjp_c2_r1abci(const Ten &r1, const Ten &V, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(V, r1, Y, G, 1 - which, f, "abej", "ei..", "abij", 2);
}
int vjp_c2_r1ijka(const Ten &r1, const Ten &V, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(V, r1, Y, G, 1 - which, -f, "ijmb", "am..", "abij", 1);
}
int vjp_Fmi_r2abij(const Ten &r2, const Ten &V, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(V, r2, Y, G, 1 - which, r2.d.iop[0] == 1 ? 0.5 * f : f, "efmn", "efin", "mi..", 0);
}
int vjp_Fae_r2abij(const Ten &r2, const Ten &V, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(r2, V, Y, G, which, r2.d.iop[1] == 0 ? -f : -0.5 * f, "afmn", "efmn", "ae..", 0);
}
int vjp_Wmbej_r2abij(const Ten &r2, const Ten &V, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(V, r2, Y, G, 1 - which, 0.5 * f, "fenm", "bfjn", "embj", 0);
}
int vjp_c2_r2Wmbej(const Ten &r2, const Ten &W, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(r2, W, Y, G, which, f, "aeim", "embj", "abij", 3);
}
int vjp_c2_r2Wmnij(const Ten &r2, const Ten &W, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(r2, W, Y, G, which, r2.d.iop[0] == 0 ? f : 0.5 * f, "abmn", "mnij", "abij", 0);
}
int vjp_c2_r2abcd(const Ten &r2, const Ten &V, const Ten &Y, Ten &G, int which, double f) {
    if (V.arr && host_resident(V.arr))
        return set_error(CPSD_EARG, "adjoint of c2_r2abcd: abcd must be in device memory");
    return vjp444(V, r2, Y, G, 1 - which, r2.d.iop[0] == 1 ? 0.5 * f : f, "abef", "efij", "abij", 0);
}
int vjp_c2_r2Fae(const Ten &r2, const Ten &F, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(r2, F, Y, G, which, f, "aeij", "be..", "abij", 1);
}
int vjp_c2_r2Fmi(const Ten &r2, const Ten &F, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(r2, F, Y, G, which, -f, "abim", "mj..", "abij", 2);
}
int vjp_Fmi_r1ijka(const Ten &r1, const Ten &V, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(V, r1, Y, G, 1 - which, f, "mnie", "en+-", "mi+-", 0);
}
int vjp_Fae_r1abci(const Ten &r1, const Ten &V, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(V, r1, Y, G, 1 - which, f, "efam", "fm+-", "ae+-", 0);
}
int vjp_Wkbij_r2ijka(const Ten &r2, const Ten &V, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(V, r2, Y, G, 1 - which, f, "klic", "bcjl", "ijkb", 1);
}
// the forward wrote tmp(ij,bk) and swapped its right pair into W(ij,kb): the
// cotangent is swapped back (a permutation's adjoint is its inverse), then
// the contraction tmp(ij,bk) = fr r(cd,ij) V(cd,bk) is reversed
int vjp_Wkbij_r2abci(const Ten &r2, const Ten &V, const Ten &Y, Ten &G, int which, double f) {
    OpScope op;
    ScratchScope sc;
    const PairMapPlan *pm;
    Desc d;
    CPSD_TRY(plan_pairmap(Y.d, PAIR_ID, PAIR_SWAP, 1, 1, &d, &pm));
    Ten Yt = Y;
    Yt.d = d;
    Yt.bs = 0;
    CPSD_TRY(scratch(d.len(), &Yt.arr));
    CPSD_TRY(launch_pairmap(pm, Y.arr, Yt.arr, 1.0, 0.0));
    return vjp444(r2, V, Yt, G, which, r2.d.iop[0] == 0 ? -f : -0.5 * f, "cdij", "cdbk", "ijbk", 0);
}
int vjp_Wmbej_r1abci(const Ten &r1, const Ten &V, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(V, r1, Y, G, 1 - which, f, "febm", "fj..", "embj", 0);
}
int vjp_Wmbej_r1ijka(const Ten &r1, const Ten &V, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(V, r1, Y, G, 1 - which, -f, "nmje", "bn..", "embj", 0);
}
int vjp_Wmnij_r1ijka(const Ten &r1, const Ten &V, const Ten &Y, Ten &G, int which, double f) {
    return vjp444(V, r1, Y, G, 1 - which, f, "mnie", "ej..", "mnij", 2);
}

}  // namespace cpsd

// =============================================================== C-ABI
using namespace cpsd;

extern "C" {

int cpsd_init(int64_t nirrep, const int64_t *dirprd) {
    if (nirrep < 1 || nirrep > 8 || !dirprd) return set_error(CPSD_EARG, "cpsd_init: nirrep must be 1..8");
    Context &c = ctx();
    c.nirrep = nirrep;
    for (int j = 0; j < 8; j++)
        for (int i = 0; i < 8; i++) c.dirprd[i][j] = dirprd[j * 8 + i];
    for (int i = 1; i <= nirrep; i++)
        for (int j = 1; j <= nirrep; j++)
            if (c.dirprd[i - 1][j - 1] < 1 || c.dirprd[i - 1][j - 1] > nirrep)
                return set_error(CPSD_EARG, "cpsd_init: invalid direct-product table");
    c.init = true;
    return CPSD_OK;
}

int cpsd_set_stream(void *s) {
    // plan tables are uploaded on the stream in use when a plan is first
    // launched; finish those copies before kernels on another stream read them
    if (ctx().stream != (cudaStream_t)s) CPSD_TRY(cuda_check(cudaStreamSynchronize(ctx().stream), "sync"));
    ctx().stream = (cudaStream_t)s;
    return CPSD_OK;
}

int cpsd_set_workspace(void *p, size_t bytes) {
    if (p) arena().set_external(p, bytes);
    else arena().free_all();
    return CPSD_OK;
}

size_t cpsd_workspace_high_water(void) { return arena().high_water; }

const char *cpsd_last_error(void) { return last_error().c_str(); }

int64_t cpsd_launch_count(int reset) {
    int64_t n = ctx().launches;
    if (reset) ctx().launches = 0;
    return n;
}

int cpsd_contract_timing(int enable) { return contract_timing(enable); }

int cpsd_contract_time(double *ms, int64_t *launches, double *flops, int reset) {
    return contract_time(ms, launches, flops, reset);
}

double cpsd_flop_count(int reset) {
    double f = ctx().flops;
    if (reset) ctx().flops = 0;
    return f;
}

int cpsd_set_mixed(int digits, double min_gflop) {
    if (digits != 0 && (digits < 3 || digits > 7)) return set_error(CPSD_EARG, "digits must be 0 or 3..7");
    if (!(min_gflop >= 0.0)) return set_error(CPSD_EARG, "min_gflop must be >= 0");
    ctx().oz_digits = digits;
    ctx().oz_min_flops = min_gflop * 1e9;
    return CPSD_OK;
}

int cpsd_mixed_error(int reset) {
    if (!ctx().oz_err) return 0;
    int h = 0;
    CPSD_TRY(cuda_check(cudaMemcpyAsync(&h, ctx().oz_err, sizeof h, cudaMemcpyDeviceToHost, stream()), "read error word"));
    CPSD_TRY(cuda_check(cudaStreamSynchronize(stream()), "sync"));
    if (reset && h)
        CPSD_TRY(cuda_check(cudaMemsetAsync(ctx().oz_err, 0, sizeof(int), stream()), "clear error word"));
    return h;
}

int cpsd_set_host_panel_bytes(size_t bytes) {
    if (bytes < 4096) return set_error(CPSD_EARG, "staging buffers of at least 4096 bytes");
    g_panel_bytes.store(bytes);
    return CPSD_OK;
}

int cpsd_davidson_stats(int64_t *nonsym_steps, int64_t *imag_warnings, int reset) {
    if (nonsym_steps) *nonsym_steps = ctx().dav_nonsym_steps;
    if (imag_warnings) *imag_warnings = ctx().dav_imag_warnings;
    if (reset) ctx().dav_nonsym_steps = ctx().dav_imag_warnings = 0;
    return CPSD_OK;
}

int cpsd_debug_geev(const double *A_host, int64_t n, double *wr, double *wi, double *V_host, int64_t *sweeps) {
    if (n < 1 || n > DAV_MAXD) return set_error(CPSD_EARG, "n must be 1..32");
    ScratchScope sc;
    double *dA, *dwr, *dwi, *dV;
    int *dsw;
    CPSD_TRY(scratch(n * n, &dA));
    CPSD_TRY(scratch(n, &dwr));
    CPSD_TRY(scratch(n, &dwi));
    CPSD_TRY(scratch(n * n, &dV));
    CPSD_TRY(scratch(1, &dsw));
    CPSD_TRY(cuda_check(cudaMemcpyAsync(dA, A_host, sizeof(double) * n * n, cudaMemcpyHostToDevice, stream()), "geev A"));
    CPSD_TRY(geev_probe(dA, (int)n, dwr, dwi, dV, dsw));
    CPSD_TRY(read_back(wr, dwr, sizeof(double) * n));
    CPSD_TRY(read_back(wi, dwi, sizeof(double) * n));
    CPSD_TRY(read_back(V_host, dV, sizeof(double) * n * n));
    int sw = 0;
    CPSD_TRY(read_back(&sw, dsw, sizeof sw));
    if (sweeps) *sweeps = sw;
    return CPSD_OK;
}

int64_t cpsd_irpdso(int64_t sym, const int64_t *popp, const int64_t *popq, int64_t ioppq) {
    return irpdso(sym, popp, popq, ioppq);
}
int64_t cpsd_idsymsoc(int64_t irrepx, const int64_t *popp, const int64_t *popq, int64_t ioppq, const int64_t *popr,
                      const int64_t *pops, int64_t ioprs) {
    return idsymsoc(irrepx, popp, popq, ioppq, popr, pops, ioprs);
}
int64_t cpsd_isymoffso(int64_t irrepq1, int64_t irrep, const int64_t *popp, const int64_t *popq, int64_t iop) {
    return isymoffso(irrepq1, irrep, popp, popq, iop);
}

static void type4(const char *t, int n, char out[5]) {
    for (int i = 0; i < 4; i++) out[i] = i < n ? t[i] : '.';
    out[4] = 0;
}

int cpsd_vv2v_dpd_444(const double *v1, const int64_t *p1_1, const int64_t *p1_2, int64_t iop1_12,
                      const int64_t *p1_3, const int64_t *p1_4, int64_t iop1_34, int64_t sym1, const char *type1,
                      const double *v2, const int64_t *p2_1, const int64_t *p2_2, int64_t iop2_12,
                      const int64_t *p2_3, const int64_t *p2_4, int64_t iop2_34, int64_t sym2, const char *type2,
                      double *v3, const int64_t *p3_1, const int64_t *p3_2, int64_t iop3_12, const int64_t *p3_3,
                      const int64_t *p3_4, int64_t iop3_34, int64_t sym3, const char *type3, double fact1,
                      double fact2) {
    Ten a = ten(p1_1, p1_2, p1_3, p1_4, iop1_12, iop1_34, sym1, (double *)v1);
    Ten b = ten(p2_1, p2_2, p2_3, p2_4, iop2_12, iop2_34, sym2, (double *)v2);
    Ten c = ten(p3_1, p3_2, p3_3, p3_4, iop3_12, iop3_34, sym3, v3);
    char t1[5], t2[5], t3[5];
    type4(type1, 4, t1);
    type4(type2, 4, t2);
    type4(type3, 4, t3);
    return engine(a, t1, b, t2, c, t3, fact1, fact2);
}

// engine() for callers that may not allocate device memory: same plan and
// kernels, tables and partial tiles in the library's fixed region; the
// size check comes before V3 is scaled so a rejected call changes nothing
int cpsd_vv2v_dpd_444_noalloc(const double *v1, const int64_t *p1_1, const int64_t *p1_2, int64_t iop1_12,
                              const int64_t *p1_3, const int64_t *p1_4, int64_t iop1_34, int64_t sym1,
                              const char *type1, const double *v2, const int64_t *p2_1, const int64_t *p2_2,
                              int64_t iop2_12, const int64_t *p2_3, const int64_t *p2_4, int64_t iop2_34,
                              int64_t sym2, const char *type2, double *v3, const int64_t *p3_1,
                              const int64_t *p3_2, int64_t iop3_12, const int64_t *p3_3, const int64_t *p3_4,
                              int64_t iop3_34, int64_t sym3, const char *type3, double fact1, double fact2) {
    CPSD_TRY(need_init());
    Ten a = ten(p1_1, p1_2, p1_3, p1_4, iop1_12, iop1_34, sym1, (double *)v1);
    Ten b = ten(p2_1, p2_2, p2_3, p2_4, iop2_12, iop2_34, sym2, (double *)v2);
    Ten c = ten(p3_1, p3_2, p3_3, p3_4, iop3_12, iop3_34, sym3, v3);
    char t1[5], t2[5], t3[5];
    type4(type1, 4, t1);
    type4(type2, 4, t2);
    type4(type3, 4, t3);
    const ContractPlan *p;
    CPSD_TRY(plan_contract(a.d, t1, b.d, t2, c.d, t3, Batch{}, &p));
    size_t need = contract_noalloc_bytes(p);
    if (need > (size_t)CPSD_NOALLOC_SCRATCH_BYTES)
        return set_error(CPSD_EARG, "contraction needs " + std::to_string(need) +
                                        " bytes of scratch; the no-allocation entry point holds at most " +
                                        std::to_string((size_t)CPSD_NOALLOC_SCRATCH_BYTES));
    if (fact2 != 1.0) CPSD_TRY(launch_scale(c.arr, c.len(), fact2));
    return launch_contract_noalloc(p, a.arr, b.arr, c.arr, fact1);
}

int cpsd_vv2v_dpd_424(const double *v1, const int64_t *p1_1, const int64_t *p1_2, int64_t iop1_12,
                      const int64_t *p1_3, const int64_t *p1_4, int64_t iop1_34, int64_t sym1, const char *type1,
                      const double *v2, const int64_t *p2_1, const int64_t *p2_2, int64_t iop2_12, int64_t sym2,
                      const char *type2, double *v3, const int64_t *p3_1, const int64_t *p3_2, int64_t iop3_12,
                      const int64_t *p3_3, const int64_t *p3_4, int64_t iop3_34, int64_t sym3, const char *type3,
                      double fact1, double fact2) {
    Ten a = ten(p1_1, p1_2, p1_3, p1_4, iop1_12, iop1_34, sym1, (double *)v1);
    Ten b = ten(p2_1, p2_2, ZORB, ZORB, iop2_12, 1, sym2, (double *)v2);
    Ten c = ten(p3_1, p3_2, p3_3, p3_4, iop3_12, iop3_34, sym3, v3);
    char t1[5], t2[5], t3[5];
    type4(type1, 4, t1);
    type4(type2, 2, t2);
    type4(type3, 4, t3);
    return engine(a, t1, b, t2, c, t3, fact1, fact2);
}

int cpsd_vv2v_dpd_442(const double *v1, const int64_t *p1_1, const int64_t *p1_2, int64_t iop1_12,
                      const int64_t *p1_3, const int64_t *p1_4, int64_t iop1_34, int64_t sym1, const char *type1,
                      const double *v2, const int64_t *p2_1, const int64_t *p2_2, int64_t iop2_12,
                      const int64_t *p2_3, const int64_t *p2_4, int64_t iop2_34, int64_t sym2, const char *type2,
                      double *v3, const int64_t *p3_1, const int64_t *p3_2, int64_t iop3_12, int64_t sym3,
                      const char *type3, double fact1, double fact2) {
    Ten a = ten(p1_1, p1_2, p1_3, p1_4, iop1_12, iop1_34, sym1, (double *)v1);
    Ten b = ten(p2_1, p2_2, p2_3, p2_4, iop2_12, iop2_34, sym2, (double *)v2);
    Ten c = ten(p3_1, p3_2, ZORB, ZORB, iop3_12, 1, sym3, v3);
    char t1[5], t2[5], t3[5];
    type4(type1, 4, t1);
    type4(type2, 4, t2);
    type4(type3, 2, t3);
    return engine(a, t1, b, t2, c, t3, fact1, fact2);
}

int cpsd_vv2v_dpd_422(const double *v1, const int64_t *p1_1, const int64_t *p1_2, int64_t iop1_12,
                      const int64_t *p1_3, const int64_t *p1_4, int64_t iop1_34, int64_t sym1, const char *type1,
                      const double *v2, const int64_t *p2_1, const int64_t *p2_2, int64_t iop2_12, int64_t sym2,
                      const char *type2, double *v3, const int64_t *p3_1, const int64_t *p3_2, int64_t iop3_12,
                      int64_t sym3, const char *type3, double fact1, double fact2) {
    Ten a = ten(p1_1, p1_2, p1_3, p1_4, iop1_12, iop1_34, sym1, (double *)v1);
    Ten b = ten(p2_1, p2_2, ZORB, ZORB, iop2_12, 1, sym2, (double *)v2);
    Ten c = ten(p3_1, p3_2, ZORB, ZORB, iop3_12, 1, sym3, v3);
    char t1[5], t2[5], t3[5];
    type4(type1, 4, t1);
    type4(type2, 2, t2);
    type4(type3, 2, t3);
    return engine(a, t1, b, t2, c, t3, fact1, fact2);
}

int cpsd_vv2v_dpd_222(const double *v1, const int64_t *p1_1, const int64_t *p1_2, int64_t iop1_12, int64_t sym1,
                      const char *type1, const double *v2, const int64_t *p2_1, const int64_t *p2_2,
                      int64_t iop2_12, int64_t sym2, const char *type2, double *v3, const int64_t *p3_1,
                      const int64_t *p3_2, int64_t iop3_12, int64_t sym3, const char *type3, double fact1,
                      double fact2) {
    Ten a = ten(p1_1, p1_2, ZORB, ZORB, iop1_12, 1, sym1, (double *)v1);
    Ten b = ten(p2_1, p2_2, ZORB, ZORB, iop2_12, 1, sym2, (double *)v2);
    Ten c = ten(p3_1, p3_2, ZORB, ZORB, iop3_12, 1, sym3, v3);
    char t1[5], t2[5], t3[5];
    type4(type1, 2, t1);
    type4(type2, 2, t2);
    type4(type3, 2, t3);
    return engine(a, t1, b, t2, c, t3, fact1, fact2);
}

// vv2v_dpd_224 (src/libsrint/vv2v_dpd_224.f90:16-19): V1(pq) and V2(rs)
// become V1(pq+-) and V2(rs+-) over one-orbital dummy slots, so the
// contraction over + and - is the outer product V3(pqrs)
int cpsd_vv2v_dpd_224(const double *v1, const int64_t *p1_1, const int64_t *p1_2, int64_t iop1_12, int64_t sym1,
                      const char *type1, const double *v2, const int64_t *p2_1, const int64_t *p2_2,
                      int64_t iop2_12, int64_t sym2, const char *type2, double *v3, const int64_t *p3_1,
                      const int64_t *p3_2, int64_t iop3_12, const int64_t *p3_3, const int64_t *p3_4,
                      int64_t iop3_34, int64_t sym3, const char *type3, double fact1, double fact2) {
    Ten a = ten(p1_1, p1_2, ZORB, ZORB, iop1_12, 1, sym1, (double *)v1);
    Ten b = ten(p2_1, p2_2, ZORB, ZORB, iop2_12, 1, sym2, (double *)v2);
    Ten c = ten(p3_1, p3_2, p3_3, p3_4, iop3_12, iop3_34, sym3, v3);
    char t1[5], t2[5], t3[5];
    type4(type1, 2, t1);
    type4(type2, 2, t2);
    t1[2] = t2[2] = '+';
    t1[3] = t2[3] = '-';
    type4(type3, 4, t3);
    return engine(a, t1, b, t2, c, t3, fact1, fact2);
}

// Fortran binding: the reference's dispatcher STOPs on a failed check
// (src/libsrint/vv2v_dpd_444.f90:150-200); this one prints the library's
// message and ends the program with status 1, so a Fortran caller never
// continues with V3 untouched.  vv2v_dpd_444_ierr_ returns the code instead.
static int vv2v_dpd_444_f(const double *v1, const int64_t *p1_1, const int64_t *p1_2, const int64_t *iop1_12,
                          const int64_t *p1_3, const int64_t *p1_4, const int64_t *iop1_34, const int64_t *sym1,
                          const char *type1, const double *v2, const int64_t *p2_1, const int64_t *p2_2,
                          const int64_t *iop2_12, const int64_t *p2_3, const int64_t *p2_4, const int64_t *iop2_34,
                          const int64_t *sym2, const char *type2, double *v3, const int64_t *p3_1,
                          const int64_t *p3_2, const int64_t *iop3_12, const int64_t *p3_3, const int64_t *p3_4,
                          const int64_t *iop3_34, const int64_t *sym3, const char *type3, const double *fact1,
                          const double *fact2, size_t len_type1, size_t len_type2, size_t len_type3) {
    char t1[5], t2[5], t3[5];
    type4(type1, len_type1 < 4 ? (int)len_type1 : 4, t1);
    type4(type2, len_type2 < 4 ? (int)len_type2 : 4, t2);
    type4(type3, len_type3 < 4 ? (int)len_type3 : 4, t3);
    return cpsd_vv2v_dpd_444(v1, p1_1, p1_2, *iop1_12, p1_3, p1_4, *iop1_34, *sym1, t1, v2, p2_1, p2_2, *iop2_12,
                             p2_3, p2_4, *iop2_34, *sym2, t2, v3, p3_1, p3_2, *iop3_12, p3_3, p3_4, *iop3_34, *sym3,
                             t3, *fact1, *fact2);
}

void vv2v_dpd_444_ierr_(const double *v1, const int64_t *p1_1, const int64_t *p1_2, const int64_t *iop1_12,
                        const int64_t *p1_3, const int64_t *p1_4, const int64_t *iop1_34, const int64_t *sym1,
                        const char *type1, const double *v2, const int64_t *p2_1, const int64_t *p2_2,
                        const int64_t *iop2_12, const int64_t *p2_3, const int64_t *p2_4, const int64_t *iop2_34,
                        const int64_t *sym2, const char *type2, double *v3, const int64_t *p3_1,
                        const int64_t *p3_2, const int64_t *iop3_12, const int64_t *p3_3, const int64_t *p3_4,
                        const int64_t *iop3_34, const int64_t *sym3, const char *type3, const double *fact1,
                        const double *fact2, int64_t *ierr, size_t len_type1, size_t len_type2,
                        size_t len_type3) {
    *ierr = vv2v_dpd_444_f(v1, p1_1, p1_2, iop1_12, p1_3, p1_4, iop1_34, sym1, type1, v2, p2_1, p2_2, iop2_12, p2_3,
                           p2_4, iop2_34, sym2, type2, v3, p3_1, p3_2, iop3_12, p3_3, p3_4, iop3_34, sym3, type3,
                           fact1, fact2, len_type1, len_type2, len_type3);
}

void vv2v_dpd_444_(const double *v1, const int64_t *p1_1, const int64_t *p1_2, const int64_t *iop1_12,
                   const int64_t *p1_3, const int64_t *p1_4, const int64_t *iop1_34, const int64_t *sym1,
                   const char *type1, const double *v2, const int64_t *p2_1, const int64_t *p2_2,
                   const int64_t *iop2_12, const int64_t *p2_3, const int64_t *p2_4, const int64_t *iop2_34,
                   const int64_t *sym2, const char *type2, double *v3, const int64_t *p3_1, const int64_t *p3_2,
                   const int64_t *iop3_12, const int64_t *p3_3, const int64_t *p3_4, const int64_t *iop3_34,
                   const int64_t *sym3, const char *type3, const double *fact1, const double *fact2,
                   size_t len_type1, size_t len_type2, size_t len_type3) {
    int rc = vv2v_dpd_444_f(v1, p1_1, p1_2, iop1_12, p1_3, p1_4, iop1_34, sym1, type1, v2, p2_1, p2_2, iop2_12, p2_3,
                            p2_4, iop2_34, sym2, type2, v3, p3_1, p3_2, iop3_12, p3_3, p3_4, iop3_34, sym3, type3, fact1,
                            fact2, len_type1, len_type2, len_type3);
    if (rc != CPSD_OK) {
        fprintf(stderr, "ERROR: vv2v_dpd_444: %s (code %d)\n", last_error().c_str(), rc);
        fflush(stderr);
        exit(1);
    }
}

int cpsd_opt_init(cpsd_opt *t, const int64_t *popp, const int64_t *popq, const int64_t *popr, const int64_t *pops,
                  int64_t ioppq, int64_t ioprs, int64_t sym, double *dev_arr) {
    memcpy(t->popp, popp, sizeof t->popp);
    memcpy(t->popq, popq, sizeof t->popq);
    memcpy(t->popr, popr, sizeof t->popr);
    memcpy(t->pops, pops, sizeof t->pops);
    t->ioppq = ioppq;
    t->ioprs = ioprs;
    t->sym = sym;
    t->len = idsymsoc(sym, popp, popq, ioppq, popr, pops, ioprs);
    t->arr = dev_arr;
    return CPSD_OK;
}

static int xform(const cpsd_opt *in, cpsd_opt *out, int op0, int op1, i64 t0, i64 t1) {
    CPSD_TRY(need_init());
    const PairMapPlan *pm;
    Desc d;
    CPSD_TRY(plan_pairmap(desc_of(in), op0, op1, t0, t1, &d, &pm));
    Desc o = desc_of(out);
    if (o.key() != d.key()) return set_error(CPSD_ELAYOUT, "output descriptor does not match the transform");
    return launch_pairmap(pm, in->arr, out->arr, 1.0, 0.0);
}
int cpsd_iexpso(const cpsd_opt *in, cpsd_opt *out, int64_t e0, int64_t e1) {
    return xform(in, out, e0 ? PAIR_EXPAND : PAIR_ID, e1 ? PAIR_EXPAND : PAIR_ID, 1, 1);
}
int cpsd_icompso(const cpsd_opt *in, cpsd_opt *out, int64_t c0, int64_t c1) {
    return xform(in, out, c0 != 1 ? PAIR_COMPRESS : PAIR_ID, c1 != 1 ? PAIR_COMPRESS : PAIR_ID, c0, c1);
}
int cpsd_isymtrso(const cpsd_opt *in, cpsd_opt *out, int64_t s0, int64_t s1) {
    return xform(in, out, s0 ? PAIR_SWAP : PAIR_ID, s1 ? PAIR_SWAP : PAIR_ID, 1, 1);
}

int cpsd_debug_contract_plan(const cpsd_opt *v1, const char *t1, const cpsd_opt *v2, const char *t2,
                             const cpsd_opt *v3, const char *t3, int64_t nb, int64_t sA, int64_t sB, int64_t sC,
                             const void **tasks, int64_t *ntasks, const void **segs, int64_t *nsegs,
                             const void **tiles, int64_t *ntiles, int64_t *tile_bm, int64_t *tile_bn) {
    CPSD_TRY(need_init());
    Batch b;
    b.nb = nb;
    b.strideA = sA;
    b.strideB = sB;
    b.strideC = sC;
    const ContractPlan *p;
    CPSD_TRY(plan_contract(desc_of(v1), t1, desc_of(v2), t2, desc_of(v3), t3, b, &p));
    *tasks = p->h_tasks.data();
    *ntasks = (int64_t)p->h_tasks.size();
    *segs = p->h_segs.data();
    *nsegs = (int64_t)p->h_segs.size();
    *tiles = p->h_tiles.data();
    *ntiles = (int64_t)p->h_tiles.size();
    *tile_bm = TILE_BM[p->cfg];
    *tile_bn = TILE_BN[p->cfg];
    return CPSD_OK;
}

int cpsd_contract_records(double *ms, double *flops, int64_t *shape, int64_t maxrec, int64_t *nrec) {
    return contract_records(ms, flops, shape, maxrec, nrec);
}

int cpsd_debug_narrow_plan(const cpsd_opt *v1, const char *t1, const cpsd_opt *v2, const char *t2,
                           const cpsd_opt *v3, const char *t3, int64_t nb, int64_t sA, int64_t sB, int64_t sC,
                           const void **items, int64_t *nitems, const void **reds, int64_t *nreds, int64_t *flags) {
    CPSD_TRY(need_init());
    Batch b;
    b.nb = nb;
    b.strideA = sA;
    b.strideB = sB;
    b.strideC = sC;
    const ContractPlan *p;
    CPSD_TRY(plan_contract(desc_of(v1), t1, desc_of(v2), t2, desc_of(v3), t3, b, &p));
    const NarrowPlan *np = nullptr;
    if (!p->empty) CPSD_TRY(plan_narrow(p, &np));
    *items = np ? np->items.data() : nullptr;
    *nitems = np ? (int64_t)np->items.size() : 0;
    *reds = np ? np->reds.data() : nullptr;
    *nreds = np ? (int64_t)np->reds.size() : 0;
    flags[0] = np ? 1 : 0;
    flags[1] = np && np->swap ? 1 : 0;
    flags[2] = np && np->longk ? 1 : 0;
    flags[3] = np ? np->nparts : 0;
    flags[4] = np ? np->kc : 0;
    return CPSD_OK;
}

int cpsd_debug_rowdot_plan(const cpsd_opt *v1, const char *t1, const cpsd_opt *v2, const char *t2,
                           const cpsd_opt *v3, const char *t3, int64_t nb, int64_t sA, int64_t sB, int64_t sC,
                           const void **items, int64_t *nitems, const void **tasks, const void **segs,
                           int64_t *flags) {
    CPSD_TRY(need_init());
    Batch b;
    b.nb = nb;
    b.strideA = sA;
    b.strideB = sB;
    b.strideC = sC;
    const ContractPlan *p;
    CPSD_TRY(plan_contract(desc_of(v1), t1, desc_of(v2), t2, desc_of(v3), t3, b, &p));
    const RowDotPlan *rp = nullptr;
    if (!p->empty) CPSD_TRY(plan_rowdot(p, &rp));
    *items = rp ? rp->items.data() : nullptr;
    *nitems = rp ? (int64_t)rp->items.size() : 0;
    *tasks = rp ? rp->tasks.data() : nullptr;
    *segs = rp ? rp->segs.data() : nullptr;
    flags[0] = rp ? 1 : 0;
    flags[1] = rp && rp->swap ? 1 : 0;
    flags[2] = rp ? rp->kq : 0;
    flags[3] = rp ? rp->nc : 0;
    return CPSD_OK;
}

int cpsd_debug_shortk_plan(const cpsd_opt *v1, const char *t1, const cpsd_opt *v2, const char *t2,
                           const cpsd_opt *v3, const char *t3, int64_t nb, int64_t sA, int64_t sB, int64_t sC,
                           const void **items, int64_t *nitems, int64_t *flags) {
    CPSD_TRY(need_init());
    Batch b;
    b.nb = nb;
    b.strideA = sA;
    b.strideB = sB;
    b.strideC = sC;
    const ContractPlan *p;
    CPSD_TRY(plan_contract(desc_of(v1), t1, desc_of(v2), t2, desc_of(v3), t3, b, &p));
    const ShortKPlan *sp = nullptr;
    if (!p->empty) CPSD_TRY(plan_shortk(p, &sp));
    *items = sp ? sp->items.data() : nullptr;
    *nitems = sp ? (int64_t)sp->items.size() : 0;
    flags[0] = sp ? 1 : 0;
    flags[1] = sp && sp->fm ? 1 : 0;
    flags[2] = sp ? sp->bs : 0;
    flags[3] = sp ? sp->kmax : 0;
    return CPSD_OK;
}

int cpsd_debug_ozaki_plan(const cpsd_opt *v1, const char *t1, const cpsd_opt *v2, const char *t2,
                          const cpsd_opt *v3, const char *t3, int64_t nb, int64_t sA, int64_t sB, int64_t sC,
                          int digits, const void **tables, int64_t *sizes) {
    CPSD_TRY(need_init());
    if (digits < 3 || digits > 7) return set_error(CPSD_EARG, "digits must be 3..7");
    Batch b;
    b.nb = nb;
    b.strideA = sA;
    b.strideB = sB;
    b.strideC = sC;
    const ContractPlan *p;
    CPSD_TRY(plan_contract(desc_of(v1), t1, desc_of(v2), t2, desc_of(v3), t3, b, &p));
    const OzPlan *oz = nullptr;
    if (!p->empty) CPSD_TRY(plan_ozaki(p, digits, &oz));
    for (int i = 0; i < 22; i++) {
        tables[i] = nullptr;
        sizes[i] = 0;
    }
    if (!oz) return CPSD_OK;
    const void *t[13] = {oz->groups.data(), oz->tiles.data(), oz->ajobs.data(), oz->bjobs.data(),
                         oz->aroff.data(),  oz->akoff.data(), oz->broff.data(), oz->bkoff.data(),
                         oz->crow.data(),   oz->ccol.data(),  oz->mcombo.data(), oz->ncombo.data(),
                         oz->kcombo.data()};
    const int64_t n[13] = {(int64_t)oz->groups.size(), (int64_t)oz->tiles.size(), (int64_t)oz->ajobs.size(),
                           (int64_t)oz->bjobs.size(),  (int64_t)oz->aroff.size(), (int64_t)oz->akoff.size(),
                           (int64_t)oz->broff.size(),  (int64_t)oz->bkoff.size(), (int64_t)oz->crow.size(),
                           (int64_t)oz->ccol.size(),   (int64_t)oz->mcombo.size(), (int64_t)oz->ncombo.size(),
                           (int64_t)oz->kcombo.size()};
    for (int i = 0; i < 13; i++) {
        tables[i] = t[i];
        sizes[i] = n[i];
    }
    sizes[13] = oz->adig;
    sizes[14] = oz->bdig;
    sizes[15] = oz->nea;
    sizes[16] = oz->neb;
    sizes[17] = oz->kt_chunk;
    sizes[18] = oz->kt_max;
    sizes[19] = oz->BN;
    tables[20] = oz->astage.data();
    sizes[20] = (int64_t)oz->astage.size();
    tables[21] = oz->bstage.data();
    sizes[21] = (int64_t)oz->bstage.size();
    return CPSD_OK;
}

int cpsd_debug_pairmap_plan(const cpsd_opt *in, int64_t op0, int64_t op1, int64_t tgt0, int64_t tgt1,
                            const void **blocks, int64_t *nblocks, const void **idx, const void **sgn, int64_t *nidx,
                            int64_t *lterms, int64_t *rterms) {
    CPSD_TRY(need_init());
    const PairMapPlan *p;
    Desc d;
    CPSD_TRY(plan_pairmap(desc_of(in), (int)op0, (int)op1, tgt0, tgt1, &d, &p));
    *blocks = p->h_blocks.data();
    *nblocks = (int64_t)p->h_blocks.size();
    *idx = p->h_idx.data();
    *sgn = p->h_sgn.data();
    *nidx = (int64_t)p->h_idx.size();
    *lterms = p->lterms;
    *rterms = p->rterms;
    return CPSD_OK;
}

#define WRAP4(nm, fn)                                                                                           \
    int cpsd_##nm(const cpsd_opt *v1, const cpsd_opt *v2, cpsd_opt *v3, double fact, const char *t1,              \
                  const char *t2, const char *t3, int64_t anti) {                                                \
        CPSD_TRY(need_init());                                                                                   \
        Ten a = ten_of(v1), b = ten_of(v2), c = ten_of(v3);                                                      \
        return fn(a, b, c, fact, t1, t2, t3, anti);                                                              \
    }
#define WRAP3(nm, fn)                                                                                            \
    int cpsd_##nm(const cpsd_opt *v1, const cpsd_opt *v2, cpsd_opt *v3, double fact, const char *t1,              \
                  const char *t2, const char *t3) {                                                              \
        CPSD_TRY(need_init());                                                                                   \
        Ten a = ten_of(v1), b = ten_of(v2), c = ten_of(v3);                                                      \
        return fn(a, b, c, fact, t1, t2, t3);                                                                    \
    }
WRAP4(vv2v_444, w444)
WRAP4(vv2v_424, w424)
WRAP4(vv2v_224, w224)
WRAP3(vv2v_442, w442)
WRAP3(vv2v_422, w422)
WRAP3(vv2v_222, w222)

#define KER(nm)                                                                                                  \
    int cpsd_##nm(cpsd_opt *out, const cpsd_opt *a, const cpsd_opt *b, double fact) {                            \
        CPSD_TRY(need_init());                                                                                   \
        Ten o = ten_of(out), x = ten_of(a), y = ten_of(b);                                                       \
        return k_##nm(o, x, y, fact);                                                                            \
    }
KER(c1_r1iabj)
KER(c1_r1Fae)
KER(c1_r1Fmi)
KER(c1_r2abci)
KER(c1_r2ijka)
KER(c2_r1abci)
KER(c2_r1ijka)
KER(c2_r2Wmbej)
KER(c2_r2Wmnij)
KER(c2_r2abcd)
KER(c2_r2Fae)
KER(c2_r2Fmi)
KER(Fmi_r2abij)
KER(Fae_r2abij)
KER(Fmi_r1ijka)
KER(Fae_r1abci)
KER(Wkbij_r2ijka)
KER(Wkbij_r2abci)
KER(Wmbej_r2abij)
KER(Wmbej_r1abci)
KER(Wmbej_r1ijka)
KER(Wmnij_r1ijka)
KER(Wmnij_r2abij)
KER(Wkbij_r1iabj)
KER(Wabdj_r1abcd)
KER(Wkbij_r1Uklij)
KER(Fme_r1abij)
KER(c1_r2Fme)
KER(c1d_l1Wibaj)
KER(c1d_l1fab)
KER(c1d_l1fij)
KER(Fae_r1fia)
KER(Fmi_r1fia)
KER(Wkbij_r2Fkc)
KER(Wlkjd_r1abij)

}  // extern "C"
