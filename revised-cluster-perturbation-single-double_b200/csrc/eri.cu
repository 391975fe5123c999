// The spin-free DPD integral lists as a linear function of the spatial
// two-electron integrals (pq|rs), and its adjoint.
//
// With every spin-free orbital k of the DPD lists given by its spatial
// orbital mo[k] and spin sp[k] (the lists' orbital order: occupied orbitals
// of irreps 1..n, then virtual ones), an element of a list is
//   <PQ||RS> = [sp_P = sp_R, sp_Q = sp_S] (P R|Q S) - [sp_P = sp_S, sp_Q = sp_R] (P S|Q R)
// with the list's slots mapped to P, Q, R, S (iabj(b,i,a,j) = <ia||bj>, the
// others <p1 p2||p3 p4> in slot order), the antisymmetrised integrals the
// reference reads from its input files (src/pyscf2cc/py2cc.py writes them
// from PySCF's MO integrals).  The forward map fills the lists from a dense
// (pq|rs) array; the adjoint accumulates d/d(pq|rs) of sum_e g(e) list(e)
// into a dense array (one atomic add per term, so the summation order and
// the last bits vary from run to run).  The dense array is nmo^4 doubles,
// indexed ((p nmo + r) nmo + q) nmo + s for (pr|qs).
#include <map>
#include <memory>
#include <mutex>
#include <string>

#include "drivers.hpp"

namespace cpsd {

namespace {

struct EriListPlan {
    i64 n = 0;
    int nblocks = 0;
    int4 perm{0, 1, 2, 3};
    i64 *d_blk = nullptr;  // per block: base, nl, nr, left pair offset, right pair offset
    int2 *d_lp = nullptr;  // global orbital indices of the slots of each left pair
    int2 *d_rp = nullptr;
};

__device__ __forceinline__ void eri_element(const i64 *__restrict__ blk, int nblocks, const int2 *__restrict__ lp,
                                            const int2 *__restrict__ rp, i64 e, int o[4]) {
    int b = 0, hi = nblocks - 1;  // last block starting at or before e
    while (b < hi) {
        const int mid = (b + hi + 1) >> 1;
        if (blk[5 * mid] <= e) b = mid;
        else hi = mid - 1;
    }
    const i64 *B = blk + 5 * b;
    const i64 loc = e - B[0], r = loc / B[1], l = loc - r * B[1];
    const int2 x = lp[B[3] + l], y = rp[B[4] + r];
    o[0] = x.x;
    o[1] = x.y;
    o[2] = y.x;
    o[3] = y.y;
}

__device__ __forceinline__ i64 eri_at(int nmo, int p, int r, int q, int s) {
    return (((i64)p * nmo + r) * nmo + q) * nmo + s;
}

__global__ void k_eri_forward(const i64 *__restrict__ blk, int nblocks, i64 n, const int2 *__restrict__ lp,
                              const int2 *__restrict__ rp, int4 perm, const int *__restrict__ mo,
                              const int *__restrict__ sp, int nmo, const double *__restrict__ eri,
                              double *__restrict__ out) {
    for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (i64)gridDim.x * blockDim.x) {
        int o[4];
        eri_element(blk, nblocks, lp, rp, e, o);
        const int P = o[perm.x], Q = o[perm.y], R = o[perm.z], S = o[perm.w];
        double v = 0.0;
        if (sp[P] == sp[R] && sp[Q] == sp[S]) v += eri[eri_at(nmo, mo[P], mo[R], mo[Q], mo[S])];
        if (sp[P] == sp[S] && sp[Q] == sp[R]) v -= eri[eri_at(nmo, mo[P], mo[S], mo[Q], mo[R])];
        out[e] = v;
    }
}

__global__ void k_eri_adjoint(const i64 *__restrict__ blk, int nblocks, i64 n, const int2 *__restrict__ lp,
                              const int2 *__restrict__ rp, int4 perm, const int *__restrict__ mo,
                              const int *__restrict__ sp, int nmo, const double *__restrict__ g,
                              double *__restrict__ geri) {
    for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (i64)gridDim.x * blockDim.x) {
        const double ge = g[e];
        if (ge == 0.0) continue;
        int o[4];
        eri_element(blk, nblocks, lp, rp, e, o);
        const int P = o[perm.x], Q = o[perm.y], R = o[perm.z], S = o[perm.w];
        if (sp[P] == sp[R] && sp[Q] == sp[S]) atomicAdd(geri + eri_at(nmo, mo[P], mo[R], mo[Q], mo[S]), ge);
        if (sp[P] == sp[S] && sp[Q] == sp[R]) atomicAdd(geri + eri_at(nmo, mo[P], mo[S], mo[Q], mo[R]), -ge);
    }
}

template <class T>
int upload_vec(const std::vector<T> &v, T **d) {
    *d = nullptr;
    if (v.empty()) return CPSD_OK;
    CPSD_TRY(cuda_check(cudaMalloc(d, sizeof(T) * v.size()), "cudaMalloc(eri plan)"));
    return cuda_check(cudaMemcpyAsync(*d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, stream()),
                      "upload eri plan");
}

// the six lists: slot kinds, iops and the slot -> <PQ||RS> map
// (allocate_mem.f90:14-44; iabj(b,i,a,j) = <ia||bj>)
struct ListKind {
    const char *kind;
    int iop0, iop1;
    int4 perm;
};
const ListKind kLists[6] = {{"oooo", 0, 0, {0, 1, 2, 3}}, {"ooov", 0, 1, {0, 1, 2, 3}},
                            {"vvoo", 0, 0, {0, 1, 2, 3}}, {"vovo", 1, 1, {1, 2, 0, 3}},
                            {"vvvo", 0, 1, {0, 1, 2, 3}}, {"vvvv", 0, 0, {0, 1, 2, 3}}};

int plan_eri_list(const Sys &S, int which, const EriListPlan **out) {
    static std::mutex m;
    std::lock_guard<std::mutex> lock(m);
    static std::map<std::string, std::unique_ptr<EriListPlan>> cache;
    std::string key = std::to_string(which) + "#" + std::to_string(ctx().nirrep);
    for (int h = 0; h < 8; h++) key += "," + std::to_string(S.popo[h]) + "," + std::to_string(S.popv[h]);
    auto it = cache.find(key);
    if (it != cache.end()) {
        *out = it->second.get();
        return CPSD_OK;
    }
    const ListKind &lk = kLists[which];
    i64 ooff[9] = {0}, voff[9] = {0};
    for (i64 h = 0; h < 8; h++) ooff[h + 1] = ooff[h] + S.popo[h];
    voff[0] = ooff[8];
    for (i64 h = 0; h < 8; h++) voff[h + 1] = voff[h] + S.popv[h];
    auto pops = [&](int k) { return lk.kind[k] == 'o' ? S.popo : S.popv; };
    auto glob = [&](int k, i64 irr, i64 i) { return (int)((lk.kind[k] == 'o' ? ooff[irr - 1] : voff[irr - 1]) + i); };
    auto plan = std::make_unique<EriListPlan>();
    plan->perm = lk.perm;
    std::vector<i64> blk;
    std::vector<int2> lp, rp;
    i64 off = 0;
    for (i64 R = 1; R <= S.nirrep; R++) {
        const auto l = pair_list(pops(0), pops(1), lk.iop0, R);  // sym 1: left irrep = right irrep
        const auto r = pair_list(pops(2), pops(3), lk.iop1, R);
        if (l.empty() || r.empty()) continue;
        blk.insert(blk.end(), {off, (i64)l.size(), (i64)r.size(), (i64)lp.size(), (i64)rp.size()});
        for (const PairEl &e : l) lp.push_back(make_int2(glob(0, e.ip, e.p), glob(1, e.iq, e.q)));
        for (const PairEl &e : r) rp.push_back(make_int2(glob(2, e.ip, e.p), glob(3, e.iq, e.q)));
        off += (i64)l.size() * (i64)r.size();
    }
    plan->n = off;
    plan->nblocks = (int)(blk.size() / 5);
    CPSD_TRY(upload_vec(blk, &plan->d_blk));
    CPSD_TRY(upload_vec(lp, &plan->d_lp));
    CPSD_TRY(upload_vec(rp, &plan->d_rp));
    CPSD_TRY(cuda_check(cudaStreamSynchronize(stream()), "eri plan upload"));
    *out = plan.get();
    cache[key] = std::move(plan);
    return CPSD_OK;
}

int grid_of(i64 n) {
    const i64 g = (n + 255) / 256;
    return (int)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

// device copies of the orbital map, checked against nmo
int upload_map(const Sys &S, const int64_t *orb_mo, const int64_t *orb_spin, int64_t nmo, int **dmo, int **dsp) {
    i64 norb = 0;
    for (int h = 0; h < 8; h++) norb += S.popo[h] + S.popv[h];
    if (nmo <= 0 || nmo > 46340) return set_error(CPSD_EARG, "nmo out of range");
    std::vector<int> mo((size_t)norb), sp((size_t)norb);
    for (i64 k = 0; k < norb; k++) {
        if (orb_mo[k] < 0 || orb_mo[k] >= nmo || (orb_spin[k] != 0 && orb_spin[k] != 1))
            return set_error(CPSD_EARG, "orbital map entry out of range");
        mo[(size_t)k] = (int)orb_mo[k];
        sp[(size_t)k] = (int)orb_spin[k];
    }
    CPSD_TRY(scratch(norb, dmo));
    CPSD_TRY(scratch(norb, dsp));
    CPSD_TRY(cuda_check(cudaMemcpyAsync(*dmo, mo.data(), sizeof(int) * mo.size(), cudaMemcpyHostToDevice, stream()),
                        "orbital map"));
    CPSD_TRY(cuda_check(cudaMemcpyAsync(*dsp, sp.data(), sizeof(int) * sp.size(), cudaMemcpyHostToDevice, stream()),
                        "orbital map"));
    // the host vectors go out of scope: wait for the copies
    return cuda_check(cudaStreamSynchronize(stream()), "orbital map");
}

}  // namespace
}  // namespace cpsd

using namespace cpsd;

extern "C" {

int cpsd_eri_lists(const cpsd_system *s, const int64_t *orb_mo, const int64_t *orb_spin, int64_t nmo,
                   const double *eri_dev, const cpsd_integrals *lists) {
    Sys S;
    CPSD_TRY(make_sys(s, &S));
    if (!eri_dev || !lists || !orb_mo || !orb_spin) return set_error(CPSD_EARG, "null argument");
    ScratchScope sc;
    int *mo, *sp;
    CPSD_TRY(upload_map(S, orb_mo, orb_spin, nmo, &mo, &sp));
    const double *outs[6] = {lists->ijkl, lists->ijka, lists->abij, lists->iabj, lists->abci, lists->abcd};
    for (int w = 0; w < 6; w++) {
        if (!outs[w]) continue;
        const EriListPlan *p;
        CPSD_TRY(plan_eri_list(S, w, &p));
        if (p->n == 0) continue;
        k_eri_forward<<<grid_of(p->n), 256, 0, stream()>>>(p->d_blk, p->nblocks, p->n, p->d_lp, p->d_rp, p->perm, mo,
                                                           sp, (int)nmo, eri_dev, (double *)outs[w]);
        count_launch();
        CPSD_TRY(cuda_check(cudaGetLastError(), "k_eri_forward"));
    }
    return cuda_check(cudaStreamSynchronize(stream()), "eri lists");
}

int cpsd_eri_adjoint(const cpsd_system *s, const int64_t *orb_mo, const int64_t *orb_spin, int64_t nmo,
                     const cpsd_integrals *grads, double *geri_dev) {
    Sys S;
    CPSD_TRY(make_sys(s, &S));
    if (!geri_dev || !grads || !orb_mo || !orb_spin) return set_error(CPSD_EARG, "null argument");
    ScratchScope sc;
    int *mo, *sp;
    CPSD_TRY(upload_map(S, orb_mo, orb_spin, nmo, &mo, &sp));
    const double *gs[6] = {grads->ijkl, grads->ijka, grads->abij, grads->iabj, grads->abci, grads->abcd};
    for (int w = 0; w < 6; w++) {
        if (!gs[w]) continue;
        const EriListPlan *p;
        CPSD_TRY(plan_eri_list(S, w, &p));
        if (p->n == 0) continue;
        k_eri_adjoint<<<grid_of(p->n), 256, 0, stream()>>>(p->d_blk, p->nblocks, p->n, p->d_lp, p->d_rp, p->perm, mo,
                                                           sp, (int)nmo, gs[w], geri_dev);
        count_launch();
        CPSD_TRY(cuda_check(cudaGetLastError(), "k_eri_adjoint"));
    }
    return cuda_check(cudaStreamSynchronize(stream()), "eri adjoint");
}

}  // extern "C"
