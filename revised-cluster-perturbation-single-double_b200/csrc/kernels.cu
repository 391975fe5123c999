// Device kernels of the DPD engine besides the contraction (contract.cu):
//  * k_pairmap  separable layout transforms (expand / compress /
//               antisymmetrise / swap of index pairs);
//  * k_energy   orbital-energy differences and denominators;
//  * BLAS-1     scale, axpy, deterministic (optionally compensated) dot.
#include <algorithm>
#include <cstdio>

#include "runtime.hpp"

namespace cpsd {

namespace {

// Each CTA covers PM_TILE consecutive output elements of one copy: thread t
// handles e0 + t + PM_T j (j < PM_PER), so the stores of a warp stay
// coalesced; the block, column r and row l of its first element come from
// one search and one division, the later ones by stepping l (a division
// again only at a block boundary or in blocks narrower than PM_T rows).
constexpr int PM_T = 256, PM_PER = 8, PM_TILE = PM_T * PM_PER;

__device__ __forceinline__ int pm_block(const PMBlockDev *__restrict__ blocks, int nblocks, i64 e) {
    int b = 0, hi = nblocks - 1;  // last block starting at or before e
    while (b < hi) {
        const int mid = (b + hi + 1) >> 1;
        if (blocks[mid].start <= e) b = mid;
        else hi = mid - 1;
    }
    return b;
}

__global__ void __launch_bounds__(PM_T) k_pairmap(const PMBlockDev *__restrict__ blocks, int nblocks, i64 total,
                                                  const long long *__restrict__ idx, const double *__restrict__ sgn,
                                                  int lt, int rt, const double *__restrict__ in0,
                                                  double *__restrict__ out0, double alpha, double beta, i64 nb,
                                                  i64 sin, i64 sout) {
    const i64 tiles = (total + PM_TILE - 1) / PM_TILE;
    for (i64 tile = blockIdx.x; tile < tiles * nb; tile += gridDim.x) {
        const i64 cpy = tile / tiles;
        const i64 e0 = (tile - cpy * tiles) * PM_TILE + threadIdx.x;
        if (e0 >= total) continue;
        const double *in = in0 + cpy * sin;
        double *out = out0 + cpy * sout;
        int b = pm_block(blocks, nblocks, e0);
        PMBlockDev B = blocks[b];
        i64 next = b + 1 < nblocks ? blocks[b + 1].start : total;
        i64 r = (e0 - B.start) / B.nlo, l = (e0 - B.start) - r * B.nlo;
        for (int j = 0; j < PM_PER; j++) {
            const i64 e = e0 + (i64)j * PM_T;
            if (e >= total) break;
            if (j > 0) {
                if (e >= next) {
                    while (e >= next) {
                        b++;
                        next = b + 1 < nblocks ? blocks[b + 1].start : total;
                    }
                    B = blocks[b];
                    r = (e - B.start) / B.nlo;
                    l = (e - B.start) - r * B.nlo;
                } else {
                    l += PM_T;
                    if (l >= B.nlo) {
                        if (B.nlo >= PM_T) {
                            l -= B.nlo;
                            r++;
                        } else {
                            r = (e - B.start) / B.nlo;
                            l = (e - B.start) - r * B.nlo;
                        }
                    }
                }
            }
            double v = 0.0;
            for (int tr = 0; tr < rt; tr++) {
                const i64 ri = idx[B.rmap + r * rt + tr];
                if (ri < 0) continue;
                const double sr = sgn[B.rmap + r * rt + tr];
                for (int tq = 0; tq < lt; tq++) {
                    const i64 li = idx[B.lmap + l * lt + tq];
                    if (li < 0) continue;
                    v += sr * sgn[B.lmap + l * lt + tq] * in[B.inBase + ri * B.nli + li];
                }
            }
            const i64 o = B.outBase + r * B.nlo + l;
            out[o] = (beta == 0.0) ? alpha * v : beta * out[o] + alpha * v;
        }
    }
}

// The same map over tiles of 256 rows x 8 columns of one block (plans whose
// elements sit mostly in blocks of at least 256 rows): thread t takes row
// l = 256 tl + t, reads its row map entries once, then issues the input
// loads of the tile's 8 columns together and stores them (coalesced along
// the rows).  Same sums in the same order as k_pairmap.
template <int LT, int RT>
__global__ void __launch_bounds__(PM_T) k_pairmap_cols(const PMBlockDev *__restrict__ blocks, int nblocks,
                                                       const i64 *__restrict__ tstart, i64 ntiles,
                                                       const long long *__restrict__ idx,
                                                       const double *__restrict__ sgn,
                                                       const double *__restrict__ in0, double *__restrict__ out0,
                                                       double alpha, double beta, i64 nb, i64 sin, i64 sout) {
    constexpr int NC = 8;
    for (i64 tile = blockIdx.x; tile < ntiles * nb; tile += gridDim.x) {
        const i64 cpy = tile / ntiles, t = tile - cpy * ntiles;
        int b = 0, hi = nblocks - 1;  // last block whose tiles start at or before t
        while (b < hi) {
            const int mid = (b + hi + 1) >> 1;
            if (tstart[mid] <= t) b = mid;
            else hi = mid - 1;
        }
        const PMBlockDev B = blocks[b];
        const i64 ntl = (B.nlo + PM_T - 1) / PM_T, loc = t - tstart[b];
        const i64 r0 = (loc / ntl) * NC, l = (loc % ntl) * PM_T + threadIdx.x;
        if (l >= B.nlo) continue;
        const double *in = in0 + cpy * sin;
        double *out = out0 + cpy * sout;
        long long li[LT];
        double sl[LT];
#pragma unroll
        for (int tq = 0; tq < LT; tq++) {
            li[tq] = idx[B.lmap + l * LT + tq];
            sl[tq] = sgn[B.lmap + l * LT + tq];
        }
        const int nc = (int)min((i64)NC, B.nro - r0);
        double v[NC];
#pragma unroll
        for (int c = 0; c < NC; c++) {
            v[c] = 0.0;
            if (c < nc)
#pragma unroll
                for (int tr = 0; tr < RT; tr++) {
                    const i64 ri = idx[B.rmap + (r0 + c) * RT + tr];
                    if (ri < 0) continue;
                    const double sr = sgn[B.rmap + (r0 + c) * RT + tr];
#pragma unroll
                    for (int tq = 0; tq < LT; tq++)
                        if (li[tq] >= 0) v[c] += sr * sl[tq] * in[B.inBase + ri * B.nli + li[tq]];
                }
        }
#pragma unroll
        for (int c = 0; c < NC; c++)
            if (c < nc) {
                const i64 o = B.outBase + (r0 + c) * B.nlo + l;
                out[o] = (beta == 0.0) ? alpha * v[c] : beta * out[o] + alpha * v[c];
            }
    }
}

__global__ void k_energy(const i64 *__restrict__ blk, int nblocks, i64 n, const i64 *__restrict__ lidx,
                         const i64 *__restrict__ ridx, const double *__restrict__ eorb, int mode,
                         const double *__restrict__ in0, double *__restrict__ out0, const double *__restrict__ w0v,
                         i64 nb, i64 sin, i64 sout) {
    for (i64 g = (i64)blockIdx.x * blockDim.x + threadIdx.x; g < n * nb; g += (i64)gridDim.x * blockDim.x) {
        i64 cpy = g / n, e = g - cpy * n;
        const double *in = in0 ? in0 + cpy * sin : nullptr;
        double *out = out0 + cpy * sout;
        double w0 = w0v ? w0v[cpy] : 0.0;
        int b = 0, hi = nblocks - 1;  // last block starting at or before e
        while (b < hi) {
            const int mid = (b + hi + 1) >> 1;
            if (blk[5 * mid] <= e) b = mid;
            else hi = mid - 1;
        }
        const i64 *B = blk + 5 * b;
        i64 loc = e - B[0];
        i64 r = loc / B[1], l = loc - r * B[1];
        i64 ia = lidx[2 * (B[3] + l)], ib = lidx[2 * (B[3] + l) + 1];
        i64 ii = ridx[2 * (B[4] + r)], ij = ridx[2 * (B[4] + r) + 1];
        double v;
        if (ii < 0) {  // 2-index (a,i): left pair holds a (vir) and i (occ)
            double ea = eorb[ia], ei = eorb[ib];
            if (mode == 0) v = ea - ei;
            else if (mode == 3) v = in[e] / (ei - ea);
            else if (mode == 5) v = ei - ea;  // the divisor of mode 3
            else v = (ea - ei) * in[e];       // mode 4
        } else {
            double ea = eorb[ia], eb = eorb[ib], ei = eorb[ii], ej = eorb[ij];
            if (mode == 0) v = ea + eb - ei - ej;
            else if (mode == 1) v = in[e] / ((ea + eb - ei - ej) - w0);
            else if (mode == 4) v = (ea + eb - ei - ej) * in[e];
            else if (mode == 5) v = ei + ej - ea - eb;  // the divisor of mode 2
            else if (mode == 6) v = in[e] * (1.0 / (w0 - (ea + eb - ei - ej)));
            else v = in[e] / (ei + ej - ea - eb);       // mode 2
        }
        out[e] = v;
    }
}

// Adjoint of the orbital-energy differences: with weights w = alpha x y on
// the elements of a DPD tensor, the derivative of sum_e w(e) e(pq,rs) with
// e(ab,ij) = ea+eb-ei-ej (e(a,i) = ea-ei) is, per orbital, the signed sum of
// the weights of the elements that carry it.  Per-pair sums first (rows:
// thread per left pair, columns: warp per right pair), then one signed
// atomic per pair orbital.
__global__ void k_energy_rows(const i64 *__restrict__ blk, const double *__restrict__ x,
                              const double *__restrict__ y, double alpha, double *__restrict__ rsum) {
    const i64 *B = blk + 5 * blockIdx.y;
    for (i64 l = (i64)blockIdx.x * blockDim.x + threadIdx.x; l < B[1]; l += (i64)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (i64 r = 0; r < B[2]; r++) {
            const i64 e = B[0] + r * B[1] + l;
            acc += y ? x[e] * y[e] : x[e];
        }
        rsum[B[3] + l] = alpha * acc;
    }
}

__global__ void k_energy_cols(const i64 *__restrict__ blk, const double *__restrict__ x,
                              const double *__restrict__ y, double alpha, double *__restrict__ csum) {
    const i64 *B = blk + 5 * blockIdx.y;
    const int lane = threadIdx.x & 31;
    const i64 nw = (i64)gridDim.x * (blockDim.x >> 5);
    for (i64 r = (i64)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < B[2]; r += nw) {
        double acc = 0.0;
        for (i64 l = lane; l < B[1]; l += 32) {
            const i64 e = B[0] + r * B[1] + l;
            acc += y ? x[e] * y[e] : x[e];
        }
        for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) csum[B[4] + r] = alpha * acc;
    }
}

// orbital k receives +sum for a virtual, -sum for an occupied orbital
// (Eorb holds the occupied orbitals first: index < nocc)
__global__ void k_energy_scatter(const i64 *__restrict__ lidx, i64 nl, const i64 *__restrict__ ridx, i64 nr,
                                 const double *__restrict__ rsum, const double *__restrict__ csum, i64 nocc,
                                 double *__restrict__ gorb) {
    for (i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x; k < nl + nr; k += (i64)gridDim.x * blockDim.x) {
        const bool left = k < nl;
        const i64 q = left ? k : k - nl;
        const double v = left ? rsum[q] : csum[q];
        const i64 *ix = left ? lidx + 2 * q : ridx + 2 * q;
        for (int t = 0; t < 2; t++)
            if (ix[t] >= 0) atomicAdd(gorb + ix[t], ix[t] < nocc ? -v : v);
    }
}

__global__ void k_scale(double *x, i64 n, double beta) {
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
        x[i] = (beta == 0.0) ? 0.0 : beta * x[i];
}
__global__ void k_axpy(i64 n, double a, const double *__restrict__ x, double *__restrict__ y) {
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
        y[i] += a * x[i];
}
// y_c += sgn * a[c] * x_c for each copy c (scalars resident on the device)
__global__ void k_axpy_dev(i64 n, const double *__restrict__ a, double sgn, const double *__restrict__ x,
                           double *__restrict__ y, i64 nb, i64 sx, i64 sy) {
    for (i64 g = (i64)blockIdx.x * blockDim.x + threadIdx.x; g < n * nb; g += (i64)gridDim.x * blockDim.x) {
        i64 c = g / n, i = g - c * n;
        y[c * sy + i] += sgn * a[c] * x[c * sx + i];
    }
}

constexpr int DOT_BLOCKS = 296;
__global__ void __launch_bounds__(256) k_dot_partial(const double *__restrict__ x, const double *__restrict__ y,
                                                     i64 n, double *__restrict__ part) {
    __shared__ double s[256];
    double a = 0.0;
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
        a = fma(x[i], y[i], a);
    s[threadIdx.x] = a;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}
// fixed-order final sum; Neumaier compensation when requested
__global__ void k_dot_final(const double *__restrict__ part, int np, double *out, int comp) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0, c = 0.0;
    for (int i = 0; i < np; i++) {
        double v = part[i];
        if (comp) {
            double t = s + v;
            if (fabs(s) >= fabs(v)) c += (s - t) + v;
            else c += (v - t) + s;
            s = t;
        } else {
            s += v;
        }
    }
    *out = s + c;
}

int grid_for(i64 n, int threads = 256) {
    i64 g = (n + threads - 1) / threads;
    if (g > 148 * 16) g = 148 * 16;
    if (g < 1) g = 1;
    return (int)g;
}
}  // namespace

int launch_pairmap(const PairMapPlan *p, const double *in, double *out, double alpha, double beta, i64 nb,
                   i64 in_stride, i64 out_stride) {
    if (p->total == 0 || nb <= 0) return CPSD_OK;
    CPSD_TRY(const_cast<PairMapPlan *>(p)->upload());
    cudaEvent_t end;
    CPSD_TRY(timing_begin(0.0, p->total, nb, p->lterms * p->rterms, 40, &end));
    const i64 tiles = (p->total + PM_TILE - 1) / PM_TILE * nb;
    if (p->tiled) {
        const unsigned grid = (unsigned)std::min<i64>(p->ntiles * nb, 148 * 16);
        if (p->lterms == 1 && p->rterms == 1)
            k_pairmap_cols<1, 1><<<grid, PM_T, 0, stream()>>>(p->d_blocks, p->nblocks, p->d_tstart, p->ntiles,
                                                              p->d_idx, p->d_sgn, in, out, alpha, beta, nb,
                                                              in_stride, out_stride);
        else if (p->lterms == 2 && p->rterms == 1)
            k_pairmap_cols<2, 1><<<grid, PM_T, 0, stream()>>>(p->d_blocks, p->nblocks, p->d_tstart, p->ntiles,
                                                              p->d_idx, p->d_sgn, in, out, alpha, beta, nb,
                                                              in_stride, out_stride);
        else if (p->lterms == 1)
            k_pairmap_cols<1, 2><<<grid, PM_T, 0, stream()>>>(p->d_blocks, p->nblocks, p->d_tstart, p->ntiles,
                                                              p->d_idx, p->d_sgn, in, out, alpha, beta, nb,
                                                              in_stride, out_stride);
        else
            k_pairmap_cols<2, 2><<<grid, PM_T, 0, stream()>>>(p->d_blocks, p->nblocks, p->d_tstart, p->ntiles,
                                                              p->d_idx, p->d_sgn, in, out, alpha, beta, nb,
                                                              in_stride, out_stride);
    } else {
        k_pairmap<<<(unsigned)std::min<i64>(tiles, 148 * 16), PM_T, 0, stream()>>>(
            p->d_blocks, p->nblocks, p->total, p->d_idx, p->d_sgn, p->lterms, p->rterms, in, out, alpha, beta, nb,
            in_stride, out_stride);
    }
    count_launch();
    CPSD_TRY(cuda_check(cudaGetLastError(), "k_pairmap"));
    return timing_end(end);
}

int launch_scale(double *x, i64 n, double beta) {
    if (n <= 0 || beta == 1.0) return CPSD_OK;
    if (beta == 0.0) return cuda_check(cudaMemsetAsync(x, 0, sizeof(double) * (size_t)n, stream()), "memset");
    k_scale<<<grid_for(n), 256, 0, stream()>>>(x, n, beta);
    count_launch();
    return cuda_check(cudaGetLastError(), "k_scale");
}

int launch_axpy(i64 n, double a, const double *x, double *y) {
    if (n <= 0) return CPSD_OK;
    k_axpy<<<grid_for(n), 256, 0, stream()>>>(n, a, x, y);
    count_launch();
    return cuda_check(cudaGetLastError(), "k_axpy");
}

int launch_axpy_dev(i64 n, const double *a_dev, double sgn, const double *x, double *y, i64 nb, i64 sx, i64 sy) {
    if (n <= 0 || nb <= 0) return CPSD_OK;
    k_axpy_dev<<<grid_for(n * nb), 256, 0, stream()>>>(n, a_dev, sgn, x, y, nb, sx, sy);
    count_launch();
    return cuda_check(cudaGetLastError(), "k_axpy_dev");
}

int launch_copy(double *y, const double *x, i64 n) {
    if (n <= 0) return CPSD_OK;
    return cuda_check(cudaMemcpyAsync(y, x, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, stream()),
                      "copy");
}

int launch_dot(const double *x, const double *y, i64 n, double *dev_out, bool compensated) {
    ScratchScope scope;
    double *part;
    CPSD_TRY(scratch(DOT_BLOCKS, &part));
    k_dot_partial<<<DOT_BLOCKS, 256, 0, stream()>>>(x, y, n, part);
    k_dot_final<<<1, 32, 0, stream()>>>(part, DOT_BLOCKS, dev_out, compensated ? 1 : 0);
    count_launch(2);
    return cuda_check(cudaGetLastError(), "k_dot");
}

int launch_energy(const EnergyPlan *p, int mode, const double *eorb, const double *in, double *out,
                  const double *w0_dev, i64 nb, i64 in_stride, i64 out_stride) {
    if (p->n == 0 || nb <= 0) return CPSD_OK;
    CPSD_TRY(const_cast<EnergyPlan *>(p)->upload());
    k_energy<<<grid_for(p->n * nb), 256, 0, stream()>>>(p->d_blk, p->nblocks, p->n, p->d_lidx, p->d_ridx, eorb,
                                                        mode, in, out, w0_dev, nb, in_stride, out_stride);
    count_launch();
    return cuda_check(cudaGetLastError(), "k_energy");
}

int launch_energy_adjoint(const EnergyPlan *p, const double *x, const double *y, double alpha, i64 nocc,
                          double *gorb) {
    if (p->n == 0) return CPSD_OK;
    CPSD_TRY(const_cast<EnergyPlan *>(p)->upload());
    const i64 nl = (i64)p->h_lidx.size() / 2, nr = (i64)p->h_ridx.size() / 2;
    i64 maxl = 1, maxr = 1;
    for (int b = 0; b < p->nblocks; b++) {
        maxl = std::max(maxl, p->h_blk[5 * b + 1]);
        maxr = std::max(maxr, p->h_blk[5 * b + 2]);
    }
    ScratchScope sc;
    double *rsum, *csum;
    CPSD_TRY(scratch(nl, &rsum));
    CPSD_TRY(scratch(nr, &csum));
    dim3 gr((unsigned)std::min<i64>((maxl + 255) / 256, 148), (unsigned)p->nblocks);
    dim3 gc((unsigned)std::min<i64>((maxr + 7) / 8, 296), (unsigned)p->nblocks);
    k_energy_rows<<<gr, 256, 0, stream()>>>(p->d_blk, x, y, alpha, rsum);
    k_energy_cols<<<gc, 256, 0, stream()>>>(p->d_blk, x, y, alpha, csum);
    k_energy_scatter<<<grid_for(nl + nr), 256, 0, stream()>>>(p->d_lidx, nl, p->d_ridx, nr, rsum, csum, nocc, gorb);
    count_launch();
    count_launch();
    count_launch();
    return cuda_check(cudaGetLastError(), "k_energy adjoint");
}

}  // namespace cpsd
