// Host planner: turns a DPD contraction (three descriptors + letter specs)
// into a grouped GEMM over irrep blocks, and layout transforms into
// separable pair maps.  Plans are cached and their tables live on the
// device for the lifetime of the library.
//
// The index semantics are those of vv2v_dpd_444 and its siblings
// (src/libsrint/vv2v_dpd_444.f90:55-233, vv2v_dpd_444_d.f90:120-529):
// letters shared by V1,V3 form the M index, by V2,V3 the N index, by V1,V2
// the contracted K index; an intact packed pair (iop 0 / 2, same letters
// and iop in both operands) is one composite index, which reproduces the
// reference's fast path, and every other letter is addressed by stride,
// which reproduces its fallback.
#include <mutex>
#include <algorithm>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <string>

#include "runtime.hpp"

namespace cpsd {

namespace {

template <class T>
int upload(const std::vector<T> &v, T **d) {
    *d = nullptr;
    if (v.empty()) return CPSD_OK;
    CPSD_TRY(cuda_check(cudaMalloc(d, sizeof(T) * v.size()), "cudaMalloc(plan)"));
    // on the library stream: the kernels that read the tables are queued
    // behind the copy on the same stream (a legacy-stream cudaMemcpy from
    // pageable memory may still be in flight when it returns)
    return cuda_check(cudaMemcpyAsync(*d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, stream()),
                      "upload plan");
}

bool is_zorb(const i64 *p) {
    if (p[0] != 1) return false;
    for (int i = 1; i < 8; i++)
        if (p[i]) return false;
    return true;
}

struct Unit {
    int nlet;
    int let[2];
    int iop;
    bool in[3];
    int slot[3];  // slot (single letter) or pair index (packed)
    int cls;      // 0 M, 1 N, 2 K
};

}  // namespace

int ContractPlan::upload() {
    if (uploaded.load(std::memory_order_acquire)) return CPSD_OK;
    std::lock_guard<std::mutex> lock(upload_mutex());
    if (uploaded.load(std::memory_order_relaxed)) return CPSD_OK;
    CPSD_TRY(cpsd::upload(h_tasks, &d_tasks));
    CPSD_TRY(cpsd::upload(h_segs, &d_segs));
    CPSD_TRY(cpsd::upload(h_tiles, &d_tiles));
    CPSD_TRY(cpsd::upload(h_reduce, &d_reduce));
    // the tables may next be read by kernels on another thread's stream
    CPSD_TRY(cuda_check(cudaStreamSynchronize(stream()), "plan upload"));
    uploaded.store(true, std::memory_order_release);
    return CPSD_OK;
}
int PairMapPlan::upload() {
    if (uploaded.load(std::memory_order_acquire)) return CPSD_OK;
    std::lock_guard<std::mutex> lock(upload_mutex());
    if (uploaded.load(std::memory_order_relaxed)) return CPSD_OK;
    CPSD_TRY(cpsd::upload(h_blocks, &d_blocks));
    CPSD_TRY(cpsd::upload(h_idx, &d_idx));
    CPSD_TRY(cpsd::upload(h_sgn, &d_sgn));
    if (tiled) CPSD_TRY(cpsd::upload(h_tstart, &d_tstart));
    // the tables may next be read by kernels on another thread's stream
    CPSD_TRY(cuda_check(cudaStreamSynchronize(stream()), "plan upload"));
    uploaded.store(true, std::memory_order_release);
    return CPSD_OK;
}
int EnergyPlan::upload() {
    if (uploaded.load(std::memory_order_acquire)) return CPSD_OK;
    std::lock_guard<std::mutex> lock(upload_mutex());
    if (uploaded.load(std::memory_order_relaxed)) return CPSD_OK;
    CPSD_TRY(cpsd::upload(h_blk, &d_blk));
    CPSD_TRY(cpsd::upload(h_lidx, &d_lidx));
    CPSD_TRY(cpsd::upload(h_ridx, &d_ridx));
    // the tables may next be read by kernels on another thread's stream
    CPSD_TRY(cuda_check(cudaStreamSynchronize(stream()), "plan upload"));
    uploaded.store(true, std::memory_order_release);
    return CPSD_OK;
}

// Tile shape, tiles and split-K groups of a plan whose tasks and segments
// are built: the shape with the least estimated time counting the padded
// tensor-pipe work (FP64 ~35 TFLOP/s) and the operand re-reads (~6 TB/s),
// or force_cfg when it is >= 0; split-K so that small outputs with long K
// still fill the GPU
void finish_plan(ContractPlan *plan, std::vector<TaskDev> tasks, std::vector<SegDev> dsegs, int force_cfg) {
    int cfg = 0;
    double best = 1e300;
    for (int c = 0; c < 4; c++) {
        if (force_cfg >= 0 && c != force_cfg) continue;
        double fl = 0, by = 0;
        for (auto &tk : tasks) {
            double mt = (double)((tk.M + TILE_BM[c] - 1) / TILE_BM[c]), nt = (double)((tk.N + TILE_BN[c] - 1) / TILE_BN[c]);
            fl += 2.0 * mt * TILE_BM[c] * nt * TILE_BN[c] * (double)tk.Ktot;
            by += 8.0 * (double)tk.Ktot * ((double)tk.M * nt + (double)tk.N * mt);
        }
        double t = fl / 35e12 + by / 6e12;
        if (t < best * 0.999) {
            best = t;
            cfg = c;
        }
    }
    const i64 TBM = TILE_BM[cfg], TBN = TILE_BN[cfg];
    plan->cfg = cfg;
    // tiles, with split-K so that small outputs with long K still fill the GPU
    std::vector<TileDev> tiles;
    std::vector<int> red;
    i64 mn_tiles = 0;
    for (auto &tk : tasks) mn_tiles += ((tk.M + TBM - 1) / TBM) * ((tk.N + TBN - 1) / TBN);
    const i64 target = 4 * 148;
    i64 part = 0;
    for (int ti = 0; ti < (int)tasks.size(); ti++) {
        const TaskDev &tk = tasks[ti];
        i64 mt = (tk.M + TBM - 1) / TBM, nt = (tk.N + TBN - 1) / TBN;
        i64 want = (mn_tiles >= target) ? 1 : (target + mn_tiles - 1) / mn_tiles;
        i64 maxsplit = std::max<i64>(1, tk.Ktot / 256);
        i64 ns = std::min(want, maxsplit);
        if (ns > 64) ns = 64;
        for (i64 a = 0; a < mt; a++)
            for (i64 b = 0; b < nt; b++) {
                if (ns > 1) {
                    red.push_back(ti);
                    red.push_back((int)a);
                    red.push_back((int)b);
                    red.push_back((int)part);
                    red.push_back((int)ns);
                }
                for (i64 s = 0; s < ns; s++) {
                    TileDev t{};
                    t.task = ti;
                    t.mt = (int)a;
                    t.nt = (int)b;
                    t.nsplit = (int)ns;
                    t.k_lo = tk.Ktot * s / ns;
                    t.k_hi = tk.Ktot * (s + 1) / ns;
                    t.part = ns > 1 ? part + s : -1;
                    tiles.push_back(t);
                }
                if (ns > 1) part += ns;
            }
    }
    plan->ntasks = (int)tasks.size();
    plan->nsegs = (int)dsegs.size();
    plan->ntiles = (int)tiles.size();
    plan->nparts = part;
    plan->nreduce = (int)red.size() / 5;
    plan->empty = tiles.empty();
    plan->h_tasks = std::move(tasks);
    plan->h_segs = std::move(dsegs);
    plan->h_tiles = std::move(tiles);
    plan->h_reduce = std::move(red);
}

int plan_contract(const Desc &d1, const char *t1, const Desc &d2, const char *t2, const Desc &d3,
                  const char *t3, const Batch &batch, const ContractPlan **out) {
    static std::mutex m;
    std::lock_guard<std::mutex> lock(m);
    static std::map<std::string, std::unique_ptr<ContractPlan>> cache;
    std::string key = d1.key() + t1 + d2.key() + t2 + d3.key() + t3 + "#" + std::to_string(batch.nb) + "," +
                      std::to_string(batch.strideA) + "," + std::to_string(batch.strideB) + "," +
                      std::to_string(batch.strideC) + "#" + std::to_string(ctx().nirrep);
    auto it = cache.find(key);
    if (it != cache.end()) {
        *out = it->second.get();
        return CPSD_OK;
    }
    const Desc *D[3] = {&d1, &d2, &d3};
    const char *T[3] = {t1, t2, t3};
    char letters[8];
    int nlet = 0;
    int lslot[3][4];
    for (int t = 0; t < 3; t++)
        for (int s = 0; s < 4; s++) {
            char ch = T[t][s];
            if (ch == '.' || ch == '+' || ch == '-' || ch == '=') {
                if (!is_zorb(D[t]->pop[s]))
                    return set_error(CPSD_ELAYOUT, std::string("dummy slot without zorb population in ") + T[t]);
                lslot[t][s] = -1;
                continue;
            }
            int id = -1;
            for (int k = 0; k < nlet; k++)
                if (letters[k] == ch) id = k;
            if (id < 0) {
                if (nlet >= 6) return set_error(CPSD_EARG, "more than 6 distinct indices");
                id = nlet;
                letters[nlet++] = ch;
            }
            lslot[t][s] = id;
        }
    int where[6][3];
    for (int k = 0; k < nlet; k++) {
        int cnt = 0;
        for (int t = 0; t < 3; t++) {
            where[k][t] = -1;
            for (int s = 0; s < 4; s++)
                if (lslot[t][s] == k) {
                    if (where[k][t] >= 0) return set_error(CPSD_EARG, "index repeated inside one tensor");
                    where[k][t] = s;
                }
            if (where[k][t] >= 0) cnt++;
        }
        if (cnt != 2)
            return set_error(CPSD_EARG, std::string("index '") + letters[k] + "' must appear in exactly two tensors: " +
                                            t1 + "*" + t2 + "->" + t3);
        int ta = -1, tb = -1;
        for (int t = 0; t < 3; t++)
            if (where[k][t] >= 0) (ta < 0 ? ta : tb) = t;
        if (memcmp(D[ta]->pop[where[k][ta]], D[tb]->pop[where[k][tb]], sizeof(D[0]->pop[0])) != 0)
            return set_error(CPSD_ELAYOUT, std::string("orbital populations of index '") + letters[k] + "' differ");
    }
    // Units: a pair whose two letters stay together (same order, same iop)
    // in both tensors that carry it is one composite index running over all
    // pairs of its pair irrep, in the DPD order (the reference's direct-GEMM
    // fast path); packed pairs must be intact; every other letter is its
    // own unit.
    Unit U[8];
    int nu = 0;
    int lunit[6];
    for (int k = 0; k < nlet; k++) lunit[k] = -1;
    for (int t = 0; t < 3; t++)
        for (int p = 0; p < 2; p++) {
            i64 iop = D[t]->iop[p];
            int a = lslot[t][2 * p], b = lslot[t][2 * p + 1];
            if (a < 0 || b < 0) {
                if (iop != 1) return set_error(CPSD_ELAYOUT, "packed pair with a dummy index");
                continue;
            }
            if (lunit[a] >= 0 && lunit[a] == lunit[b] && U[lunit[a]].nlet == 2) continue;
            bool ok = false;
            for (int u = 0; u < 3; u++) {
                if (u == t) continue;
                for (int q = 0; q < 2; q++)
                    if (lslot[u][2 * q] == a && lslot[u][2 * q + 1] == b && D[u]->iop[q] == iop) ok = true;
            }
            if (!ok) {
                if (iop == 1) continue;
                return set_error(CPSD_ELAYOUT, std::string("packed pair not intact (expand to iop=1 first): ") + t1 +
                                                   "*" + t2 + "->" + t3);
            }
            U[nu] = Unit{2, {a, b}, (int)iop, {}, {}, 0};
            lunit[a] = lunit[b] = nu++;
        }
    for (int k = 0; k < nlet; k++) {
        if (lunit[k] >= 0) continue;
        U[nu] = Unit{1, {k, -1}, 1, {}, {}, 0};
        lunit[k] = nu++;
    }
    for (int u = 0; u < nu; u++) {
        int k = U[u].let[0];
        for (int t = 0; t < 3; t++) {
            U[u].in[t] = where[k][t] >= 0;
            U[u].slot[t] = (U[u].nlet == 2) ? where[k][t] / 2 : where[k][t];
        }
        U[u].cls = (U[u].in[0] && U[u].in[2]) ? 0 : (U[u].in[1] && U[u].in[2]) ? 1 : 2;
        if (U[u].nlet == 2)
            for (int t = 0; t < 3; t++)
                if (U[u].in[t]) {
                    int p = U[u].slot[t];
                    if (lslot[t][2 * p] != U[u].let[0] || lslot[t][2 * p + 1] != U[u].let[1])
                        return set_error(CPSD_ELAYOUT, "packed pair appears in a different order");
                }
    }
    int cm[MAXU + 1], cn[MAXU + 1], ck[MAXU + 1];
    int nm = 0, nn = 0, nk = 0;
    for (int u = 0; u < nu; u++) {
        int c = U[u].cls;
        if ((c == 0 && nm >= MAXU) || (c == 1 && nn >= MAXU) || (c == 2 && nk >= MAXU))
            return set_error(CPSD_EARG, "too many indices in one class");
        if (c == 0) cm[nm++] = u;
        else if (c == 1) cn[nn++] = u;
        else ck[nk++] = u;
    }
    // a batch of independent operand copies (e.g. the roots of one irrep)
    // becomes one more M index (first operand batched) or N index (second)
    bool batched = batch.nb > 1;
    bool batchM = batched && batch.strideA != 0;
    bool batchN = batched && !batchM;
    if (batchM && batch.strideB != 0) return set_error(CPSD_EARG, "only one operand may be batched");
    if ((batchM && nm >= MAXU) || (batchN && nn >= MAXU)) return set_error(CPSD_EARG, "no room for the batch index");

    // enumerate irrep assignments (depth-first with symmetry pruning)
    struct Seg {
        std::string okey, mkey, nkey, kkey;
        i64 ext[8];
        i64 base[3];
        i64 st[3][8];
    };
    std::vector<Seg> segs;
    i64 nir = ctx().nirrep;
    i64 uir[8];  // irrep of each unit: letter irrep, or pair irrep of a pair unit
    // units of each tensor for pruning: a tensor can be checked once all its units are set
    int last_u[3] = {-1, -1, -1};
    for (int t = 0; t < 3; t++)
        for (int u = 0; u < nu; u++)
            if (U[u].in[t]) last_u[t] = u;
    std::function<void(int)> rec = [&](int k) {
        if (k == nu) {
            Seg sg;
            for (int u = 0; u < nu; u++) {
                if (U[u].nlet == 2) {
                    int t0 = U[u].in[0] ? 0 : 1;
                    int p = U[u].slot[t0];
                    sg.ext[u] = (p == 0) ? D[t0]->nleft(uir[u]) : D[t0]->nright(uir[u]);
                } else {
                    int kk = U[u].let[0];
                    int t0 = where[kk][0] >= 0 ? 0 : 1;
                    sg.ext[u] = D[t0]->pop[where[kk][t0]][uir[u] - 1];
                }
                if (sg.ext[u] == 0) return;
            }
            for (int t = 0; t < 3; t++) {
                const Desc &d = *D[t];
                i64 PI[2], sub[2], h[4];
                bool whole[2];
                for (int p = 0; p < 2; p++) {
                    int a = lslot[t][2 * p], b = lslot[t][2 * p + 1];
                    whole[p] = a >= 0 && b >= 0 && lunit[a] == lunit[b] && U[lunit[a]].nlet == 2;
                    if (whole[p]) {
                        PI[p] = uir[lunit[a]];
                        sub[p] = 0;
                        h[2 * p] = h[2 * p + 1] = 1;
                    } else {
                        h[2 * p] = a < 0 ? 1 : uir[lunit[a]];
                        h[2 * p + 1] = b < 0 ? 1 : uir[lunit[b]];
                        PI[p] = dp(h[2 * p], h[2 * p + 1]);
                        sub[p] = isymoffso(h[2 * p + 1], PI[p], d.pop[2 * p], d.pop[2 * p + 1], d.iop[p]) - 1;
                    }
                }
                const i64 nl = d.nleft(PI[0]);
                sg.base[t] = d.block_base(PI[1]) + sub[1] * nl + sub[0];
                const i64 st4[4] = {1, whole[0] ? 0 : d.pop[0][h[0] - 1], nl, whole[1] ? 0 : nl * d.pop[2][h[2] - 1]};
                for (int u = 0; u < nu; u++) {
                    if (!U[u].in[t]) {
                        sg.st[t][u] = 0;
                        continue;
                    }
                    sg.st[t][u] = (U[u].nlet == 2) ? (U[u].slot[t] == 0 ? 1 : nl) : st4[U[u].slot[t]];
                }
            }
            sg.okey.clear();
            for (int u = 0; u < nu; u++) {
                const char c = (char)('0' + uir[u]);
                if (U[u].cls != 2) sg.okey += c;
                (U[u].cls == 0 ? sg.mkey : U[u].cls == 1 ? sg.nkey : sg.kkey) += c;
            }
            segs.push_back(sg);
            return;
        }
        for (i64 hh = 1; hh <= nir; hh++) {
            uir[k] = hh;
            bool ok = true;
            for (int t = 0; t < 3 && ok; t++) {
                if (last_u[t] != k) continue;
                i64 prod = 1;
                for (int u = 0; u < nu; u++)
                    if (U[u].in[t]) prod = dp(prod, uir[u]);
                if (prod != D[t]->sym) ok = false;
            }
            if (ok) rec(k + 1);
        }
    };
    // tensors whose letters are all dummies must still match their irrep
    for (int t = 0; t < 3; t++)
        if (last_u[t] < 0 && D[t]->sym != 1) {
            *out = nullptr;
            return set_error(CPSD_EARG, "scalar tensor with non-totally-symmetric irrep");
        }
    rec(0);

    // group segments into tasks by output irreps
    std::stable_sort(segs.begin(), segs.end(), [](const Seg &a, const Seg &b) { return a.okey < b.okey; });
    std::vector<TaskDev> tasks;
    std::vector<SegDev> dsegs;
    auto plan = std::make_unique<ContractPlan>();
    for (size_t i = 0; i < segs.size();) {
        size_t j = i;
        while (j < segs.size() && segs[j].okey == segs[i].okey) j++;
        const Seg &s0 = segs[i];
        TaskDev tk{};
        tk.nm = nm + (batchM ? 1 : 0);
        tk.nn = nn + (batchN ? 1 : 0);
        tk.M = 1;
        tk.N = 1;
        for (int a = 0; a < nm; a++) {
            tk.mExt[a] = s0.ext[cm[a]];
            tk.mSC[a] = s0.st[2][cm[a]];
            tk.M *= tk.mExt[a];
        }
        for (int a = 0; a < nn; a++) {
            tk.nExt[a] = s0.ext[cn[a]];
            tk.nSC[a] = s0.st[2][cn[a]];
            tk.N *= tk.nExt[a];
        }
        if (batchM) {
            tk.mExt[nm] = batch.nb;
            tk.mSC[nm] = batch.strideC;
            tk.M *= batch.nb;
        }
        if (batchN) {
            tk.nExt[nn] = batch.nb;
            tk.nSC[nn] = batch.strideC;
            tk.N *= batch.nb;
        }
        tk.baseC = s0.base[2];
        tk.seg0 = (int)dsegs.size();
        tk.Ktot = 0;
        for (size_t q = i; q < j; q++) {
            const Seg &s = segs[q];
            SegDev sd{};
            sd.baseA = s.base[0];
            sd.baseB = s.base[1];
            sd.nk = nk;
            sd.K = 1;
            for (int a = 0; a < nm; a++) sd.mSA[a] = s.st[0][cm[a]];
            for (int a = 0; a < nn; a++) sd.nSB[a] = s.st[1][cn[a]];
            if (batchM) sd.mSA[nm] = batch.strideA;
            if (batchN) sd.nSB[nn] = batch.strideB;
            for (int a = 0; a < nk; a++) {
                sd.kExt[a] = s.ext[ck[a]];
                sd.kSA[a] = s.st[0][ck[a]];
                sd.kSB[a] = s.st[1][ck[a]];
                sd.K *= sd.kExt[a];
            }
            if (sd.K == 0) continue;
            sd.aMfast = (nm > 0 && sd.mSA[0] == 1) ? 1 : 0;
            sd.bKfast = (nk > 0 && sd.kSB[0] == 1) ? 1 : 0;
            sd.kstart = tk.Ktot;
            tk.Ktot += sd.K;
            dsegs.push_back(sd);
            plan->seg_kkey.push_back(s.kkey);
        }
        tk.nseg = (int)dsegs.size() - tk.seg0;
        if (tk.M > 0 && tk.N > 0 && tk.nseg > 0) {
            tasks.push_back(tk);
            plan->task_mkey.push_back(s0.mkey);
            plan->task_nkey.push_back(s0.nkey);
            plan->flops += 2.0 * (double)tk.M * (double)tk.N * (double)tk.Ktot;
        } else {
            dsegs.resize(tk.seg0);
            plan->seg_kkey.resize(tk.seg0);
        }
        i = j;
    }
    finish_plan(plan.get(), std::move(tasks), std::move(dsegs));
    *out = plan.get();
    cache[key] = std::move(plan);
    return CPSD_OK;
}

// A strided GEMM as a one-task plan: C[m + n ldc + r sC] += A[m + k lda]
// B[k + n ldb + r sB] for m < M, n < N, k < K and r < nb copies of B and C
// (the panels of the out-of-core particle ladder)
int plan_gemm(i64 M, i64 N, i64 K, i64 lda, i64 ldb, i64 ldc, i64 nb, i64 sB, i64 sC, const ContractPlan **out) {
    static std::mutex m;
    std::lock_guard<std::mutex> lock(m);
    static std::map<std::string, std::unique_ptr<ContractPlan>> cache;
    const std::string key = std::to_string(M) + "," + std::to_string(N) + "," + std::to_string(K) + "," +
                            std::to_string(lda) + "," + std::to_string(ldb) + "," + std::to_string(ldc) + "," +
                            std::to_string(nb) + "," + std::to_string(sB) + "," + std::to_string(sC);
    auto it = cache.find(key);
    if (it != cache.end()) {
        *out = it->second.get();
        return CPSD_OK;
    }
    if (M <= 0 || N <= 0 || K <= 0 || nb <= 0) return set_error(CPSD_EARG, "plan_gemm: empty GEMM");
    TaskDev tk{};
    tk.nm = 1;
    tk.mExt[0] = M;
    tk.mSC[0] = 1;
    tk.nn = nb > 1 ? 2 : 1;
    tk.nExt[0] = N;
    tk.nSC[0] = ldc;
    tk.nExt[1] = nb;
    tk.nSC[1] = sC;
    tk.M = M;
    tk.N = N * nb;
    tk.Ktot = K;
    tk.seg0 = 0;
    tk.nseg = 1;
    SegDev sd{};
    sd.nk = 1;
    sd.K = K;
    sd.mSA[0] = 1;
    sd.nSB[0] = ldb;
    sd.nSB[1] = sB;
    sd.kExt[0] = K;
    sd.kSA[0] = lda;
    sd.kSB[0] = 1;
    sd.aMfast = 1;
    sd.bKfast = 1;
    auto plan = std::make_unique<ContractPlan>();
    plan->flops = 2.0 * (double)M * (double)N * (double)nb * (double)K;
    finish_plan(plan.get(), {tk}, {sd});
    *out = plan.get();
    cache[key] = std::move(plan);
    return CPSD_OK;
}

// ------------------------------------------------------------ pair maps
std::vector<PairEl> pair_list(const i64 *pp, const i64 *pq, i64 iop, i64 irr) {
    std::vector<PairEl> v;
    for (i64 iq = 1; iq <= ctx().nirrep; iq++) {
        i64 ip = dp(iq, irr);
        if (iop != 1 && ip > iq) continue;
        for (i64 q = 0; q < pq[iq - 1]; q++) {
            i64 pmax = pp[ip - 1];
            if (iop == 0 && ip == iq) pmax = q;
            if (iop == 2 && ip == iq) pmax = q + 1;
            for (i64 p = 0; p < pmax; p++) v.push_back({ip, p, iq, q});
        }
    }
    return v;
}
namespace {
// offset of (ip,p,iq,q) inside the pair space of a pair with pops/iop; -1
// if structurally zero; sign for packed partner
i64 pair_off(const i64 *pp, const i64 *pq, i64 iop, i64 ip, i64 p, i64 iq, i64 q, double *sgn) {
    i64 irr = dp(ip, iq);
    *sgn = 1.0;
    if (iop != 1 && (ip > iq || (ip == iq && p > q))) {
        std::swap(ip, iq);
        std::swap(p, q);
        *sgn = (iop == 0) ? -1.0 : 1.0;
    }
    if (iop == 1 || ip < iq) return isymoffso(iq, irr, pp, pq, iop) - 1 + q * pp[ip - 1] + p;
    if (iop == 0) {
        if (p == q) return -1;
        return isymoffso(iq, irr, pp, pq, 0) - 1 + q * (q - 1) / 2 + p;
    }
    return isymoffso(iq, irr, pp, pq, 2) - 1 + q * (q + 1) / 2 + p;
}
}  // namespace

// op per pair: PAIR_ID (copy), PAIR_EXPAND (packed -> iop 1),
// PAIR_COMPRESS (iop 1 -> target iop), PAIR_ANTI (out(p,q)=in(p,q)-in(q,p)),
// PAIR_ANTI_COMPRESS (packed out = in(p,q)-in(q,p)), PAIR_SWAP (out(q,p)=in(p,q))
int plan_pairmap(const Desc &din, int op0, int op1, i64 target_iop0, i64 target_iop1, Desc *dout_ret,
                 const PairMapPlan **out) {
    static std::mutex m;
    std::lock_guard<std::mutex> lock(m);
    static std::map<std::string, std::unique_ptr<PairMapPlan>> cache;
    Desc dout = din;
    int ops[2] = {op0, op1};
    i64 tgt[2] = {target_iop0, target_iop1};
    for (int k = 0; k < 2; k++) {
        switch (ops[k]) {
        case PAIR_ID:
            break;
        case PAIR_EXPAND:
            dout.iop[k] = 1;
            break;
        case PAIR_COMPRESS:
        case PAIR_ANTI_COMPRESS:
            if (din.iop[k] != 1) return set_error(CPSD_EARG, "compress needs a full (iop 1) pair");
            dout.iop[k] = tgt[k];
            break;
        case PAIR_ANTI:
        case PAIR_SWAP:
            if (din.iop[k] != 1) return set_error(CPSD_EARG, "swap/antisymmetrise needs a full (iop 1) pair");
            if (ops[k] == PAIR_SWAP) std::swap(dout.pop[2 * k], dout.pop[2 * k + 1]);
            else if (memcmp(din.pop[2 * k], din.pop[2 * k + 1], sizeof din.pop[0]) != 0)
                return set_error(CPSD_ELAYOUT, "antisymmetrised pair with different populations");
            break;
        default:
            return set_error(CPSD_EARG, "bad pair op");
        }
    }
    *dout_ret = dout;
    std::string key = din.key() + "|" + std::to_string(op0) + std::to_string(op1) + std::to_string(target_iop0) +
                      std::to_string(target_iop1) + "#" + std::to_string(ctx().nirrep);
    auto it = cache.find(key);
    if (it != cache.end()) {
        *out = it->second.get();
        return CPSD_OK;
    }
    auto plan = std::make_unique<PairMapPlan>();
    int nterm[2];
    for (int k = 0; k < 2; k++) nterm[k] = (ops[k] == PAIR_ANTI || ops[k] == PAIR_ANTI_COMPRESS) ? 2 : 1;
    plan->lterms = nterm[0];
    plan->rterms = nterm[1];
    std::vector<PMBlockDev> blocks;
    std::vector<long long> idx;
    std::vector<double> sgn;
    i64 start = 0;
    for (i64 R = 1; R <= ctx().nirrep; R++) {
        i64 L = dp(R, din.sym);
        for (int k = 0; k < 2; k++) (void)k;
        PMBlockDev b{};
        b.outBase = dout.block_base(R);
        b.nlo = dout.nleft(L);
        b.nro = dout.nright(R);
        b.inBase = din.block_base(R);
        b.nli = din.nleft(L);
        b.start = start;
        if (b.nlo * b.nro == 0) continue;
        for (int k = 0; k < 2; k++) {
            i64 irr = (k == 0) ? L : R;
            auto pl = pair_list(dout.pop[2 * k], dout.pop[2 * k + 1], dout.iop[k], irr);
            (k == 0 ? b.lmap : b.rmap) = (i64)idx.size();
            for (auto &e : pl) {
                for (int t = 0; t < nterm[k]; t++) {
                    i64 ip = e.ip, p = e.p, iq = e.iq, q = e.q;
                    double s = 1.0;
                    if (ops[k] == PAIR_SWAP) {
                        std::swap(ip, iq);
                        std::swap(p, q);
                    }
                    if (t == 1) {  // second antisymmetriser term: -in(q,p)
                        std::swap(ip, iq);
                        std::swap(p, q);
                        s = -1.0;
                    }
                    double ps;
                    i64 o = pair_off(din.pop[2 * k], din.pop[2 * k + 1], din.iop[k], ip, p, iq, q, &ps);
                    idx.push_back(o);
                    sgn.push_back(o < 0 ? 0.0 : s * ps);
                }
            }
        }
        blocks.push_back(b);
        start += b.nlo * b.nro;
    }
    plan->nblocks = (int)blocks.size();
    plan->total = start;
    // column tiling pays when most elements sit in blocks of at least 256
    // rows: each tile reads its rows' map entries once for 8 columns
    {
        i64 tall = 0, nt = 0;
        for (const PMBlockDev &b : blocks) {
            if (b.nlo >= 256) tall += b.nlo * b.nro;
            plan->h_tstart.push_back(nt);
            nt += ((b.nlo + 255) / 256) * ((b.nro + 7) / 8);
        }
        plan->ntiles = nt;
        plan->tiled = start > 0 && tall >= start * 9 / 10;
        if (!plan->tiled) plan->h_tstart.clear();
    }
    plan->h_blocks = std::move(blocks);
    plan->h_idx = std::move(idx);
    plan->h_sgn = std::move(sgn);
    *out = plan.get();
    cache[key] = std::move(plan);
    return CPSD_OK;
}

// ----------------------------------------------------------- energies
int plan_energy(const Desc &d, const char *kinds, const EnergyPlan **out) {
    static std::mutex m;
    std::lock_guard<std::mutex> lock(m);
    static std::map<std::string, std::unique_ptr<EnergyPlan>> cache;
    std::string key = d.key() + kinds + "#" + std::to_string(ctx().nirrep);
    auto it = cache.find(key);
    if (it != cache.end()) {
        *out = it->second.get();
        return CPSD_OK;
    }
    // eorb layout: occupied irreps then virtual irreps (resortEorb / seperateEorb)
    // slot populations identify the spaces: kinds[k] in 'o','v','z'
    const i64 *popo = nullptr, *popv = nullptr;
    for (int k = 0; k < 4; k++) {
        if (kinds[k] == 'o') popo = d.pop[k];
        if (kinds[k] == 'v') popv = d.pop[k];
    }
    if (!popo || !popv) return set_error(CPSD_EARG, "energy plan needs occupied and virtual slots");
    i64 ooff[9] = {0}, voff[9] = {0};
    for (i64 h = 0; h < ctx().nirrep; h++) ooff[h + 1] = ooff[h] + popo[h];
    voff[0] = ooff[ctx().nirrep];
    for (i64 h = 0; h < ctx().nirrep; h++) voff[h + 1] = voff[h] + popv[h];
    auto eidx = [&](char kind, i64 irr, i64 i) -> i64 {
        if (kind == 'o') return ooff[irr - 1] + i;
        if (kind == 'v') return voff[irr - 1] + i;
        return -1;
    };
    auto plan = std::make_unique<EnergyPlan>();
    std::vector<i64> blk, lidx, ridx;
    i64 off = 0;
    for (i64 R = 1; R <= ctx().nirrep; R++) {
        i64 L = dp(R, d.sym);
        auto lp = pair_list(d.pop[0], d.pop[1], d.iop[0], L);
        auto rp = pair_list(d.pop[2], d.pop[3], d.iop[1], R);
        if (lp.empty() || rp.empty()) continue;
        blk.push_back(off);
        blk.push_back((i64)lp.size());
        blk.push_back((i64)rp.size());
        blk.push_back((i64)lidx.size() / 2);
        blk.push_back((i64)ridx.size() / 2);
        for (auto &e : lp) {
            lidx.push_back(eidx(kinds[0], e.ip, e.p));
            lidx.push_back(eidx(kinds[1], e.iq, e.q));
        }
        for (auto &e : rp) {
            ridx.push_back(eidx(kinds[2], e.ip, e.p));
            ridx.push_back(eidx(kinds[3], e.iq, e.q));
        }
        off += (i64)lp.size() * (i64)rp.size();
    }
    plan->n = off;
    plan->nblocks = (int)blk.size() / 5;
    plan->h_blk = std::move(blk);
    plan->h_lidx = std::move(lidx);
    plan->h_ridx = std::move(ridx);
    *out = plan.get();
    cache[key] = std::move(plan);
    return CPSD_OK;
}

}  // namespace cpsd
