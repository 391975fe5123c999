// Host planner of the sliced-integer contraction path: regroups the tasks
// of a ContractPlan into dense GEMMs and builds the gather / scatter offset
// tables of the digit kernels (ozaki.cu).
//
// For a fixed irrep combination of the contracted units, every M-index
// combination pairs with every N-index combination (symmetry fixes the
// product irreps of the M and N units), so the tasks sharing a list of
// contracted combinations tile a dense block matrix C_g = A_g B_g.  The
// addresses are not separable across combinations (the DPD block offsets
// and strides depend on the irreps of letters of both indices), hence the
// per-combination tables: element (r, k) of A_g is at
// roff[r][kcombo(k)] + koff[k][rcombo(r)], and C likewise.
#include <mutex>
#include <algorithm>
#include <map>
#include <memory>

#include "ozaki.cuh"

namespace cpsd {

namespace {

i64 decode(i64 x, int n, const i64 *ext, const i64 *st) {
    i64 off = 0;
    for (int u = 0; u < n; u++) {
        off += (x % ext[u]) * st[u];
        x /= ext[u];
    }
    return off;
}

uint64_t fnv(uint64_t h, const void *p, size_t n) {
    const unsigned char *c = (const unsigned char *)p;
    for (size_t i = 0; i < n; i++) {
        h ^= c[i];
        h *= 1099511628211ull;
    }
    return h;
}

template <class T>
int upload_vec(const std::vector<T> &v, const T **d) {
    *d = nullptr;
    if (v.empty()) return CPSD_OK;
    T *p = nullptr;
    CPSD_TRY(cuda_check(cudaMalloc(&p, sizeof(T) * v.size()), "cudaMalloc(digit plan)"));
    *d = p;
    return cuda_check(cudaMemcpyAsync(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, stream()),
                      "upload digit plan");
}

i64 roundup(i64 x, i64 m) { return (x + m - 1) / m * m; }

}  // namespace

int OzPlan::upload() {
    if (uploaded.load(std::memory_order_acquire)) return CPSD_OK;
    std::lock_guard<std::mutex> lock(upload_mutex());
    if (uploaded.load(std::memory_order_relaxed)) return CPSD_OK;
    CPSD_TRY(upload_vec(tiles, &dev.tiles));
    CPSD_TRY(upload_vec(groups, &dev.groups));
    CPSD_TRY(upload_vec(crow, &dev.crow));
    CPSD_TRY(upload_vec(ccol, &dev.ccol));
    CPSD_TRY(upload_vec(mcombo, &dev.mcombo));
    CPSD_TRY(upload_vec(ncombo, &dev.ncombo));
    dev.ntiles = (int)tiles.size();
    const int *kc = nullptr;
    CPSD_TRY(upload_vec(kcombo, &kc));
    CPSD_TRY(upload_vec(ajobs, &adev.jobs));
    CPSD_TRY(upload_vec(aroff, &adev.roff));
    CPSD_TRY(upload_vec(akoff, &adev.koff));
    adev.njobs = (int)ajobs.size();
    adev.kt_max = kt_max;
    adev.nexpo = nea;
    bdev.kt_max = kt_max;
    bdev.nexpo = neb;
    adev.rcombo = dev.mcombo;
    adev.kcombo = kc;
    CPSD_TRY(upload_vec(bjobs, &bdev.jobs));
    CPSD_TRY(upload_vec(broff, &bdev.roff));
    CPSD_TRY(upload_vec(bkoff, &bdev.koff));
    bdev.njobs = (int)bjobs.size();
    bdev.rcombo = dev.ncombo;
    bdev.kcombo = kc;
    CPSD_TRY(upload_vec(astage, &adev.stage));
    CPSD_TRY(upload_vec(bstage, &bdev.stage));
    // the tables may next be read by kernels on another thread's stream
    CPSD_TRY(cuda_check(cudaStreamSynchronize(stream()), "plan upload"));
    uploaded.store(true, std::memory_order_release);
    return CPSD_OK;
}

int plan_ozaki(const ContractPlan *cp, int S, const OzPlan **out) {
    static std::mutex m;
    std::lock_guard<std::mutex> lock(m);
    static std::map<std::pair<const ContractPlan *, int>, std::unique_ptr<OzPlan>> cache;
    *out = nullptr;
    auto key = std::make_pair(cp, S);
    auto it = cache.find(key);
    if (it != cache.end()) {
        *out = it->second.get();
        return CPSD_OK;
    }
    auto P = std::make_unique<OzPlan>();
    OzPlan &p = *P;
    p.S = S;
    p.BN = oz_tile_n(S);
    p.flops = cp->flops;
    const int BN = p.BN;
    bool ok = !cp->empty && cp->task_mkey.size() == cp->h_tasks.size() && cp->seg_kkey.size() == cp->h_segs.size();
    // group the tasks by their (sorted) list of contracted combinations
    struct Grp {
        std::vector<std::string> kkeys;
        std::vector<std::string> mkeys, nkeys;
        std::map<std::pair<int, int>, int> task;  // (M comb, N comb) -> task
    };
    std::vector<Grp> grps;
    std::map<std::string, int> gidx;
    for (size_t ti = 0; ok && ti < cp->h_tasks.size(); ti++) {
        const TaskDev &tk = cp->h_tasks[ti];
        std::vector<std::string> kk;
        for (int q = 0; q < tk.nseg; q++) kk.push_back(cp->seg_kkey[tk.seg0 + q]);
        std::sort(kk.begin(), kk.end());
        std::string gk;
        for (auto &s : kk) gk += s + "|";
        auto gi = gidx.find(gk);
        int g;
        if (gi == gidx.end()) {
            g = (int)grps.size();
            gidx[gk] = g;
            grps.push_back(Grp{kk, {}, {}, {}});
        } else {
            g = gi->second;
        }
        Grp &G = grps[g];
        auto find_or_add = [](std::vector<std::string> &v, const std::string &s) {
            auto f = std::find(v.begin(), v.end(), s);
            if (f != v.end()) return (int)(f - v.begin());
            v.push_back(s);
            return (int)v.size() - 1;
        };
        int i = find_or_add(G.mkeys, cp->task_mkey[ti]);
        int l = find_or_add(G.nkeys, cp->task_nkey[ti]);
        if (G.task.count({i, l})) ok = false;
        G.task[{i, l}] = (int)ti;
    }
    for (auto &G : grps)
        if (G.task.size() != G.mkeys.size() * G.nkeys.size()) ok = false;  // not a full block matrix
    if (!ok) {
        cache[key] = nullptr;
        return CPSD_OK;
    }
    const i64 kmax = (i64)(2147483647ll / ((i64)S * 127 * 127));
    p.kt_chunk = (int)std::max<i64>(1, kmax / 64);
    double padded = 0.0;
    for (auto &G : grps) {
        const int nI = (int)G.mkeys.size(), nL = (int)G.nkeys.size(), nJ = (int)G.kkeys.size();
        // segment of task t for contracted combination j
        auto seg_of = [&](int t, int j) -> const SegDev & {
            const TaskDev &tk = cp->h_tasks[t];
            for (int q = 0; q < tk.nseg; q++)
                if (cp->seg_kkey[tk.seg0 + q] == G.kkeys[j]) return cp->h_segs[tk.seg0 + q];
            return cp->h_segs[tk.seg0];  // unreachable: every task of the group has all combinations
        };
        std::vector<i64> mstart(nI + 1, 0), nstart(nL + 1, 0), kstart(nJ + 1, 0);
        for (int i = 0; i < nI; i++) mstart[i + 1] = mstart[i] + cp->h_tasks[G.task.at({i, 0})].M;
        for (int l = 0; l < nL; l++) nstart[l + 1] = nstart[l] + cp->h_tasks[G.task.at({0, l})].N;
        for (int j = 0; j < nJ; j++) kstart[j + 1] = kstart[j] + seg_of(G.task.at({0, 0}), j).K;
        OzGroup og{};
        og.M = mstart[nI];
        og.N = nstart[nL];
        og.K = kstart[nJ];
        const i64 Mpad = roundup(og.M, 128), Npad = roundup(og.N, BN), Kpad = roundup(og.K, 64);
        og.KT = (int)(Kpad / 64);
        og.nI = nI;
        og.nL = nL;
        og.aoff = p.adig;
        og.boff = p.bdig;
        og.eaoff = p.nea;
        og.eboff = p.neb;
        og.moff = (i64)p.mcombo.size();
        og.noff = (i64)p.ncombo.size();
        og.crowoff = (i64)p.crow.size();
        og.ccoloff = (i64)p.ccol.size();
        const i64 kcoff = (i64)p.kcombo.size();
        const i64 aroff0 = (i64)p.aroff.size(), akoff0 = (i64)p.akoff.size();
        const i64 broff0 = (i64)p.broff.size(), bkoff0 = (i64)p.bkoff.size();
        p.aroff.resize(aroff0 + og.M * nJ);
        p.akoff.resize(akoff0 + og.K * nI);
        p.broff.resize(broff0 + og.N * nJ);
        p.bkoff.resize(bkoff0 + og.K * nL);
        p.crow.resize(og.crowoff + og.M * nL);
        p.ccol.resize(og.ccoloff + og.N * nI);
        for (int i = 0; i < nI; i++)
            for (i64 ml = 0; ml < mstart[i + 1] - mstart[i]; ml++) p.mcombo.push_back(i);
        for (int l = 0; l < nL; l++)
            for (i64 nl = 0; nl < nstart[l + 1] - nstart[l]; nl++) p.ncombo.push_back(l);
        for (int j = 0; j < nJ; j++)
            for (i64 kl = 0; kl < kstart[j + 1] - kstart[j]; kl++) p.kcombo.push_back(j);
        // A: rows M, contracted K (segments of any task with that M combination)
        for (int i = 0; i < nI; i++) {
            const TaskDev &tk = cp->h_tasks[G.task.at({i, 0})];
            for (int j = 0; j < nJ; j++) {
                const SegDev &sg = seg_of(G.task.at({i, 0}), j);
                for (i64 ml = 0; ml < tk.M; ml++)
                    p.aroff[aroff0 + (mstart[i] + ml) * nJ + j] = sg.baseA + decode(ml, tk.nm, tk.mExt, sg.mSA);
                for (i64 kl = 0; kl < sg.K; kl++)
                    p.akoff[akoff0 + (kstart[j] + kl) * nI + i] = decode(kl, sg.nk, sg.kExt, sg.kSA);
            }
        }
        // B: rows N
        for (int l = 0; l < nL; l++) {
            const TaskDev &tk = cp->h_tasks[G.task.at({0, l})];
            for (int j = 0; j < nJ; j++) {
                const SegDev &sg = seg_of(G.task.at({0, l}), j);
                for (i64 nl = 0; nl < tk.N; nl++)
                    p.broff[broff0 + (nstart[l] + nl) * nJ + j] = sg.baseB + decode(nl, tk.nn, tk.nExt, sg.nSB);
                for (i64 kl = 0; kl < sg.K; kl++)
                    p.bkoff[bkoff0 + (kstart[j] + kl) * nL + l] = decode(kl, sg.nk, sg.kExt, sg.kSB);
            }
        }
        // C: the task of each (M, N) combination pair
        for (int i = 0; i < nI; i++)
            for (int l = 0; l < nL; l++) {
                const TaskDev &tk = cp->h_tasks[G.task.at({i, l})];
                for (i64 ml = 0; ml < tk.M; ml++)
                    p.crow[og.crowoff + (mstart[i] + ml) * nL + l] = tk.baseC + decode(ml, tk.nm, tk.mExt, tk.mSC);
                for (i64 nl = 0; nl < tk.N; nl++)
                    p.ccol[og.ccoloff + (nstart[l] + nl) * nI + i] = decode(nl, tk.nn, tk.nExt, tk.nSC);
            }
        // affine descriptors of the K stages (per row combination) and of the
        // row tiles: most tiles of a large group sit inside one DPD block,
        // whose offsets step by constant strides
        auto stage_table = [&](const std::vector<i64> &koff, i64 koff0, int nrc, std::vector<OzStage> &out) {
            const i64 soff = (i64)out.size();
            out.resize(soff + (i64)og.KT * nrc);
            for (int kt = 0; kt < og.KT; kt++) {
                const i64 k0 = (i64)kt * 64, k1 = std::min<i64>(og.K, k0 + 64);
                const int j = p.kcombo[kcoff + k0];
                for (int rc = 0; rc < nrc; rc++) {
                    OzStage &st = out[soff + (i64)kt * nrc + rc];
                    st = OzStage{koff[koff0 + k0 * nrc + rc], 0, j, 1};
                    if (k1 - k0 > 1) st.sk = koff[koff0 + (k0 + 1) * nrc + rc] - st.ko0;
                    for (i64 k = k0; k < k1 && st.ok; k++)
                        if (p.kcombo[kcoff + k] != j || koff[koff0 + k * nrc + rc] != st.ko0 + (k - k0) * st.sk)
                            st.ok = 0;
                }
            }
            return soff;
        };
        auto job_affine = [](OzSliceJob &jb, const std::vector<i64> &roff, const std::vector<int> &combo, int RT) {
            const i64 r0 = (i64)jb.rt * RT, r1 = std::min<i64>(jb.R, r0 + RT);
            jb.rc = combo[jb.rcoff + r0];
            const i64 *ro = roff.data() + jb.roff;
            const i64 sr = r1 - r0 > 1 ? ro[(r0 + 1) * jb.nJ] - ro[r0 * jb.nJ] : 0;
            for (i64 r = r0; r < r1; r++) {
                if (combo[jb.rcoff + r] != jb.rc) return;
                for (int j = 0; j < jb.nJ; j++)
                    if (ro[r * jb.nJ + j] != ro[r0 * jb.nJ + j] + (r - r0) * sr) return;
            }
            jb.affine = 1;
            jb.sr = sr;
        };
        const i64 asoff = og.K > 0 ? stage_table(p.akoff, akoff0, nI, p.astage) : 0;
        const i64 bsoff = og.K > 0 ? stage_table(p.bkoff, bkoff0, nL, p.bstage) : 0;
        for (i64 rt = 0; rt < Mpad / 128; rt++) {
            OzSliceJob jb{og.M, og.K, og.KT, (int)rt, nJ, nI, aroff0, akoff0, og.moff, kcoff, og.eaoff, og.aoff};
            jb.soff = asoff;
            if (og.K > 0) job_affine(jb, p.aroff, p.mcombo, 128);
            p.ajobs.push_back(jb);
        }
        for (i64 rt = 0; rt < Npad / BN; rt++) {
            OzSliceJob jb{og.N, og.K, og.KT, (int)rt, nJ, nL, broff0, bkoff0, og.noff, kcoff, og.eboff, og.boff};
            jb.soff = bsoff;
            if (og.K > 0) job_affine(jb, p.broff, p.ncombo, BN);
            p.bjobs.push_back(jb);
        }
        for (i64 mt = 0; mt < Mpad / 128; mt++)
            for (i64 nt = 0; nt < Npad / BN; nt++)
                p.tiles.push_back(OzTile{(int)p.groups.size(), (int)mt, (int)nt, 0});
        p.adig += (i64)S * Mpad * Kpad;
        p.bdig += (i64)S * Npad * Kpad;
        p.nea += Mpad;
        p.neb += Npad;
        p.kt_max = std::max(p.kt_max, og.KT);
        p.kmin = p.groups.empty() ? og.K : std::min(p.kmin, og.K);
        padded += 2.0 * (double)Mpad * (double)Npad * (double)Kpad;
        p.groups.push_back(og);
    }
    p.pad_eff = padded > 0 ? p.flops / padded : 0.0;
    // signatures of the digit layouts: equal signatures read the same
    // elements of the source into the same digits
    uint64_t h = 1469598103934665603ull;
    h = fnv(h, &S, sizeof S);
    for (auto &j : p.ajobs) h = fnv(h, &j, sizeof j);
    h = fnv(h, p.aroff.data(), p.aroff.size() * sizeof(i64));
    h = fnv(h, p.akoff.data(), p.akoff.size() * sizeof(i64));
    h = fnv(h, p.mcombo.data(), p.mcombo.size() * sizeof(int));
    h = fnv(h, p.kcombo.data(), p.kcombo.size() * sizeof(int));
    p.ahash = h;
    h = 1469598103934665603ull ^ 0x9e3779b97f4a7c15ull;
    h = fnv(h, &S, sizeof S);
    h = fnv(h, &BN, sizeof BN);
    for (auto &j : p.bjobs) h = fnv(h, &j, sizeof j);
    h = fnv(h, p.broff.data(), p.broff.size() * sizeof(i64));
    h = fnv(h, p.bkoff.data(), p.bkoff.size() * sizeof(i64));
    h = fnv(h, p.ncombo.data(), p.ncombo.size() * sizeof(int));
    h = fnv(h, p.kcombo.data(), p.kcombo.size() * sizeof(int));
    p.bhash = h;
    *out = P.get();
    cache[key] = std::move(P);
    return CPSD_OK;
}

}  // namespace cpsd
