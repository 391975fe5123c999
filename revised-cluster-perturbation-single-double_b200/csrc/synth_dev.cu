// Synthetic spin-free integrals built on the device: the same definitions
// and layouts as synth.c (see there), for molecules whose integral tensors
// are too large to assemble on the host in reasonable time.  Input
// preparation only; not on any timed path.
//
//   (pr|qs) = sum_P L[P][p][r] L[P][q][s]: per aux irrep h one DGEMM
//   E_h = L_h^T L_h over the ordered MO pairs (p,r) of pair irrep h;
//   <pq||rs> = (pr|qs) d(sp,sr) d(sq,ss) - (ps|qr) d(sp,ss) d(sq,sr),
//   written element by element into the DPD blocks (one thread per element).
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

typedef int64_t i64;

namespace {

struct EriTables {
    const double *E[8];  // E_h, npairs_h x npairs_h, column-major
    i64 np[8];
    const int *pidx;     // nmo x nmo: index of the ordered pair (p,r) in its irrep block
    const int *pirr;     // nmo x nmo: pair irrep - 1
    int nmo;
};

__device__ __forceinline__ double eri(const EriTables &T, int p, int r, int q, int s) {
    const int a = p * T.nmo + r, b = q * T.nmo + s;
    const int h = T.pirr[a];
    if (h != T.pirr[b]) return 0.0;
    return T.E[h][(i64)T.pidx[a] + (i64)T.pidx[b] * T.np[h]];
}

// Lh[k + j naux_h] = L[aux_k][p_j][r_j]
__global__ void k_gather(const double *__restrict__ L, int nmo, const int *__restrict__ aux, int naux_h,
                         const int *__restrict__ pr, i64 npairs, double *__restrict__ Lh) {
    const i64 n = (i64)naux_h * npairs;
    for (i64 g = (i64)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (i64)gridDim.x * blockDim.x) {
        const i64 j = g / naux_h, k = g - j * naux_h;
        Lh[g] = L[(i64)aux[k] * nmo * nmo + pr[j]];
    }
}

// one DPD tensor (sym 1): blocks (base, nl, nr, left pair offset, right
// pair offset); pairs as (mo0, spin0, mo1, spin1); perm maps the slots to
// the positions of <pq||rs>
__global__ void k_fill(const i64 *__restrict__ blk, int nblocks, i64 n, const int4 *__restrict__ lp,
                       const int4 *__restrict__ rp, int4 perm, EriTables T, double *__restrict__ out) {
    for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (i64)gridDim.x * blockDim.x) {
        int b = 0, hi = nblocks - 1;
        while (b < hi) {
            const int mid = (b + hi + 1) >> 1;
            if (blk[5 * mid] <= e) b = mid;
            else hi = mid - 1;
        }
        const i64 *B = blk + 5 * b;
        const i64 loc = e - B[0], r = loc / B[1], l = loc - r * B[1];
        const int4 x = lp[B[3] + l], y = rp[B[4] + r];
        const int mo[4] = {x.x, x.z, y.x, y.z}, sp[4] = {x.y, x.w, y.y, y.w};
        const int P = perm.x, Q = perm.y, R = perm.z, S = perm.w;
        double v = 0.0;
        if (sp[P] == sp[R] && sp[Q] == sp[S]) v += eri(T, mo[P], mo[R], mo[Q], mo[S]);
        if (sp[P] == sp[S] && sp[Q] == sp[R]) v -= eri(T, mo[P], mo[S], mo[Q], mo[R]);
        out[e] = v;
    }
}

struct Orbs {  // spin-free orbitals of one space, per irrep: (mo, spin)
    std::vector<int> mo[8], sp[8];
};

int grid_for(i64 n) {
    i64 g = (n + 255) / 256;
    return (int)(g < 1 ? 1 : (g > 148 * 32 ? 148 * 32 : g));
}

}  // namespace

extern "C" {

/* Builds the requested DPD integral tensors (device pointers, NULL to skip)
 * of the synthetic molecule defined as in cpsd_synth_build; L_dev is the
 * naux x nmo x nmo factor on the device, the other arrays are host arrays.
 * Runs on `stream`; returns 0, or -1 (bad argument) / -2 (CUDA or cuBLAS
 * failure, e.g. not enough device memory for the pair blocks). */
int cpsd_synth_build_device(i64 nmo, i64 nirrep, const i64 *dirprd, const i64 *mo_irrep, i64 nocc_a, i64 nocc_b,
                            i64 naux, const i64 *aux_irrep, const double *L_dev, double *ijkl, double *ijka,
                            double *abij, double *iabj, double *abci, double *abcd, void *stream) {
    if (nmo <= 0 || nirrep < 1 || nirrep > 8 || naux <= 0 || !L_dev) return -1;
    cudaStream_t st = (cudaStream_t)stream;
    auto dp = [&](i64 a, i64 b) { return dirprd[(b - 1) * 8 + (a - 1)]; };
    // spin-free orbitals: per irrep the alpha orbitals, then the beta ones
    Orbs occ, vir;
    i64 popo[8] = {0}, popv[8] = {0};
    for (i64 h = 1; h <= nirrep; h++)
        for (int spin = 0; spin < 2; spin++) {
            const i64 nocc = spin == 0 ? nocc_a : nocc_b;
            for (i64 m = 0; m < nmo; m++)
                if (mo_irrep[m] == h) {
                    Orbs &o = m < nocc ? occ : vir;
                    o.mo[h - 1].push_back((int)m);
                    o.sp[h - 1].push_back(spin);
                }
        }
    for (int h = 0; h < nirrep; h++) {
        popo[h] = (i64)occ.mo[h].size();
        popv[h] = (i64)vir.mo[h].size();
    }
    // ordered MO pairs of each pair irrep; aux functions of each irrep
    std::vector<int> pidx((size_t)(nmo * nmo)), pirr((size_t)(nmo * nmo));
    std::vector<std::vector<int>> prs((size_t)nirrep), aux((size_t)nirrep);
    for (i64 p = 0; p < nmo; p++)
        for (i64 r = 0; r < nmo; r++) {
            const i64 h = dp(mo_irrep[p], mo_irrep[r]);
            pirr[(size_t)(p * nmo + r)] = (int)(h - 1);
            pidx[(size_t)(p * nmo + r)] = (int)prs[(size_t)(h - 1)].size();
            prs[(size_t)(h - 1)].push_back((int)(p * nmo + r));
        }
    for (i64 P = 0; P < naux; P++) aux[(size_t)(aux_irrep[P] - 1)].push_back((int)P);
    int rc = 0;
    cublasHandle_t hb = nullptr;
    std::vector<void *> dev;  // every device allocation, freed at the end
    auto dalloc = [&](size_t bytes) -> void * {
        void *p = nullptr;
        if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) return nullptr;
        dev.push_back(p);
        return p;
    };
    auto upload = [&](const void *h, size_t bytes) -> void * {
        void *p = dalloc(bytes);
        if (p && bytes && cudaMemcpyAsync(p, h, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) return nullptr;
        return p;
    };
    EriTables T;
    memset(&T, 0, sizeof T);
    T.nmo = (int)nmo;
    do {
        if (cublasCreate(&hb) != CUBLAS_STATUS_SUCCESS || cublasSetStream(hb, st) != CUBLAS_STATUS_SUCCESS) {
            rc = -2;
            break;
        }
        T.pidx = (const int *)upload(pidx.data(), sizeof(int) * pidx.size());
        T.pirr = (const int *)upload(pirr.data(), sizeof(int) * pirr.size());
        if (!T.pidx || !T.pirr) { rc = -2; break; }
        for (int h = 0; h < nirrep && rc == 0; h++) {
            const i64 np = (i64)prs[(size_t)h].size(), na = (i64)aux[(size_t)h].size();
            T.np[h] = np;
            double *E = (double *)dalloc(sizeof(double) * (size_t)(np * np));
            if (!E) { rc = -2; break; }
            T.E[h] = E;
            if (na == 0) {
                if (cudaMemsetAsync(E, 0, sizeof(double) * (size_t)(np * np), st) != cudaSuccess) rc = -2;
                continue;
            }
            const int *dpr = (const int *)upload(prs[(size_t)h].data(), sizeof(int) * (size_t)np);
            const int *dax = (const int *)upload(aux[(size_t)h].data(), sizeof(int) * (size_t)na);
            double *Lh = (double *)dalloc(sizeof(double) * (size_t)(na * np));
            if (!dpr || !dax || !Lh) { rc = -2; break; }
            k_gather<<<grid_for(na * np), 256, 0, st>>>(L_dev, (int)nmo, dax, (int)na, dpr, np, Lh);
            const double one = 1.0, zero = 0.0;
            if (cublasDgemm(hb, CUBLAS_OP_T, CUBLAS_OP_N, (int)np, (int)np, (int)na, &one, Lh, (int)na, Lh, (int)na,
                            &zero, E, (int)np) != CUBLAS_STATUS_SUCCESS)
                rc = -2;
        }
        if (rc) break;
        struct Want {
            double *out;
            const char *kind;
            int iop0, iop1;
            int4 perm;
        };
        const Want want[6] = {{ijkl, "oooo", 0, 0, {0, 1, 2, 3}}, {ijka, "ooov", 0, 1, {0, 1, 2, 3}},
                              {abij, "vvoo", 0, 0, {0, 1, 2, 3}}, {iabj, "vovo", 1, 1, {1, 2, 0, 3}},
                              {abci, "vvvo", 0, 1, {0, 1, 2, 3}}, {abcd, "vvvv", 0, 0, {0, 1, 2, 3}}};
        for (const Want &w : want) {
            if (!w.out) continue;
            const Orbs *sl[4];
            const i64 *pops[4];
            for (int k = 0; k < 4; k++) {
                sl[k] = w.kind[k] == 'o' ? &occ : &vir;
                pops[k] = w.kind[k] == 'o' ? popo : popv;
            }
            // the DPD pair order of synth.c / irpdso: sub-blocks by the
            // second index's irrep, left index fastest, p<q packing (iop 0)
            auto pairs = [&](int s0, int s1, int iop, i64 irr, std::vector<int4> &out) {
                for (i64 iq = 1; iq <= nirrep; iq++) {
                    const i64 ip = dp(iq, irr);
                    if (iop != 1 && ip > iq) continue;
                    for (i64 q = 0; q < pops[s1][iq - 1]; q++) {
                        const i64 pmax = (iop == 0 && ip == iq) ? q : pops[s0][ip - 1];
                        for (i64 p = 0; p < pmax; p++)
                            out.push_back(make_int4(sl[s0]->mo[ip - 1][(size_t)p], sl[s0]->sp[ip - 1][(size_t)p],
                                                    sl[s1]->mo[iq - 1][(size_t)q], sl[s1]->sp[iq - 1][(size_t)q]));
                    }
                }
            };
            std::vector<i64> blk;
            std::vector<int4> lp, rp;
            i64 off = 0;
            for (i64 R = 1; R <= nirrep; R++) {
                const size_t l0 = lp.size(), r0 = rp.size();
                pairs(0, 1, w.iop0, R, lp);
                pairs(2, 3, w.iop1, R, rp);
                const i64 nl = (i64)(lp.size() - l0), nr = (i64)(rp.size() - r0);
                if (nl * nr == 0) continue;
                blk.insert(blk.end(), {off, nl, nr, (i64)l0, (i64)r0});
                off += nl * nr;
            }
            if (off == 0) continue;
            const i64 *dblk = (const i64 *)upload(blk.data(), sizeof(i64) * blk.size());
            const int4 *dlp = (const int4 *)upload(lp.data(), sizeof(int4) * lp.size());
            const int4 *drp = (const int4 *)upload(rp.data(), sizeof(int4) * rp.size());
            if (!dblk || !dlp || !drp) { rc = -2; break; }
            k_fill<<<grid_for(off), 256, 0, st>>>(dblk, (int)(blk.size() / 5), off, dlp, drp, w.perm, T, w.out);
        }
        if (rc == 0 && (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)) rc = -2;
    } while (0);
    cudaStreamSynchronize(st);
    for (void *p : dev) cudaFree(p);
    if (hb) cublasDestroy(hb);
    return rc;
}

}  // extern "C"
