// Device kernels of the DPD engine (sm_100a):
//  * k_contract      grouped FP64 GEMM over irrep blocks, gather prologue /
//                    scatter epilogue from the planner's stride tables;
//  * k_splitk_reduce deterministic split-K reduction;
//  * k_pairmap       separable layout transforms (expand / compress /
//                    antisymmetrise / swap of index pairs);
//  * k_energy        orbital-energy differences and denominators;
//  * BLAS-1          scale, axpy, copy, deterministic (optionally
//                    compensated) dot product.
#include <cstdio>
#include <vector>

#include "runtime.hpp"

namespace cpsd {

namespace {
constexpr int BM = 64, BN = 64, BK = 16, NT = 256;
static_assert(BM * BK == 4 * NT && BN * BK == 4 * NT, "tile loads assume 4 elements per thread");

__device__ __forceinline__ i64 decode1(i64 x, int n, const i64 *ext, const i64 *st) {
    i64 off = 0;
    for (int u = 0; u < n; u++) {
        i64 e = ext[u];
        i64 q = x / e;
        off += (x - q * e) * st[u];
        x = q;
    }
    return off;
}
__device__ __forceinline__ void decode2(i64 x, int n, const i64 *ext, const i64 *s1, const i64 *s2, i64 *o1,
                                        i64 *o2) {
    i64 a = 0, b = 0;
    for (int u = 0; u < n; u++) {
        i64 e = ext[u];
        i64 q = x / e;
        i64 r = x - q * e;
        a += r * s1[u];
        b += r * s2[u];
        x = q;
    }
    *o1 = a;
    *o2 = b;
}

__global__ void __launch_bounds__(NT) k_contract(const double *__restrict__ A, const double *__restrict__ B,
                                                 double *__restrict__ C, const TaskDev *__restrict__ tasks,
                                                 const SegDev *__restrict__ segs, const TileDev *__restrict__ tiles,
                                                 double alpha, double *__restrict__ partial) {
    __shared__ double As[BK][BM];
    __shared__ double Bs[BK][BN];
    __shared__ i64 offM[BM], offN[BN], offKA[BK], offKB[BK];
    __shared__ TaskDev tk;
    __shared__ SegDev sg;
    const int tid = threadIdx.x;
    const TileDev tl = tiles[blockIdx.x];
    if (tid == 0) tk = tasks[tl.task];
    __syncthreads();
    const i64 m0 = (i64)tl.mt * BM, n0 = (i64)tl.nt * BN;
    const int tx = tid & 15, ty = tid >> 4;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.0;
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
        for (i64 k0 = kb; k0 < ke; k0 += BK) {
            __syncthreads();
            if (tid < BK) {
                i64 k = k0 + tid;
                if (k < ke) {
                    decode2(k, sg.nk, sg.kExt, sg.kSA, sg.kSB, &offKA[tid], &offKB[tid]);
                } else {
                    offKA[tid] = -1;
                    offKB[tid] = -1;
                }
            }
            __syncthreads();
#pragma unroll
            for (int i = 0; i < 4; i++) {
                int m, k;
                if (sg.aMfast) {
                    m = tid & (BM - 1);
                    k = (tid >> 6) + 4 * i;
                } else {
                    k = tid & (BK - 1);
                    m = (tid >> 4) + 16 * i;
                }
                i64 om = offM[m], ok = offKA[k];
                As[k][m] = (om >= 0 && ok >= 0) ? __ldg(A + om + ok) : 0.0;
                int n, k2;
                if (sg.bKfast) {
                    k2 = tid & (BK - 1);
                    n = (tid >> 4) + 16 * i;
                } else {
                    n = tid & (BN - 1);
                    k2 = (tid >> 6) + 4 * i;
                }
                i64 on = offN[n], ok2 = offKB[k2];
                Bs[k2][n] = (on >= 0 && ok2 >= 0) ? __ldg(B + on + ok2) : 0.0;
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < BK; k++) {
                double a[4], b[4];
#pragma unroll
                for (int i = 0; i < 4; i++) a[i] = As[k][ty * 4 + i];
#pragma unroll
                for (int j = 0; j < 4; j++) b[j] = Bs[k][tx * 4 + j];
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int j = 0; j < 4; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
            }
        }
    }
    __syncthreads();
    if (tl.part >= 0) {
        double *P = partial + (size_t)tl.part * (BM * BN);
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) P[(ty * 4 + i) * BN + tx * 4 + j] = acc[i][j];
        return;
    }
    if (tid < BM) {
        i64 m = m0 + tid;
        offM[tid] = (m < tk.M) ? decode1(m, tk.nm, tk.mExt, tk.mSC) : -1;
    } else if (tid < BM + BN) {
        i64 n = n0 + tid - BM;
        offN[tid - BM] = (n < tk.N) ? decode1(n, tk.nn, tk.nExt, tk.nSC) : -1;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; i++) {
        i64 om = offM[ty * 4 + i];
        if (om < 0) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            i64 on = offN[tx * 4 + j];
            if (on < 0) continue;
            double *c = C + tk.baseC + om + on;
            *c += alpha * acc[i][j];
        }
    }
}

// sum the split-K partial tiles of one output tile in a fixed order
__global__ void __launch_bounds__(NT) k_splitk_reduce(const int *__restrict__ red, const TaskDev *__restrict__ tasks,
                                                      const double *__restrict__ partial, double *__restrict__ C,
                                                      double alpha) {
    const int *r = red + 5 * blockIdx.x;
    const TaskDev &tk = tasks[r[0]];
    const i64 m0 = (i64)r[1] * BM, n0 = (i64)r[2] * BN;
    const i64 p0 = r[3];
    const int ns = r[4];
    __shared__ i64 offM[BM], offN[BN];
    int tid = threadIdx.x;
    if (tid < BM) {
        i64 m = m0 + tid;
        offM[tid] = (m < tk.M) ? decode1(m, tk.nm, tk.mExt, tk.mSC) : -1;
    } else if (tid < BM + BN) {
        i64 n = n0 + tid - BM;
        offN[tid - BM] = (n < tk.N) ? decode1(n, tk.nn, tk.nExt, tk.nSC) : -1;
    }
    __syncthreads();
    for (int e = tid; e < BM * BN; e += NT) {
        int mi = e / BN, ni = e % BN;
        i64 om = offM[mi], on = offN[ni];
        if (om < 0 || on < 0) continue;
        double s = 0.0;
        for (int q = 0; q < ns; q++) s += partial[(size_t)(p0 + q) * (BM * BN) + e];
        C[tk.baseC + om + on] += alpha * s;
    }
}

__global__ void k_pairmap(const PMBlockDev *__restrict__ blocks, int nblocks, i64 total,
                          const long long *__restrict__ idx, const double *__restrict__ sgn, int lt, int rt,
                          const double *__restrict__ in0, double *__restrict__ out0, double alpha, double beta,
                          i64 nb, i64 sin, i64 sout) {
    for (i64 g = (i64)blockIdx.x * blockDim.x + threadIdx.x; g < total * nb; g += (i64)gridDim.x * blockDim.x) {
        i64 cpy = g / total, e = g - cpy * total;
        const double *in = in0 + cpy * sin;
        double *out = out0 + cpy * sout;
        int b = 0;
        while (b + 1 < nblocks && blocks[b + 1].start <= e) b++;
        const PMBlockDev &B = blocks[b];
        i64 loc = e - B.start;
        i64 r = loc / B.nlo, l = loc - r * B.nlo;
        double v = 0.0;
        for (int tr = 0; tr < rt; tr++) {
            i64 ri = idx[B.rmap + r * rt + tr];
            if (ri < 0) continue;
            double sr = sgn[B.rmap + r * rt + tr];
            for (int tq = 0; tq < lt; tq++) {
                i64 li = idx[B.lmap + l * lt + tq];
                if (li < 0) continue;
                v += sr * sgn[B.lmap + l * lt + tq] * in[B.inBase + ri * B.nli + li];
            }
        }
        i64 o = B.outBase + r * B.nlo + l;
        out[o] = (beta == 0.0) ? alpha * v : beta * out[o] + alpha * v;
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
        int b = 0;
        while (b + 1 < nblocks && blk[5 * (b + 1)] <= e) b++;
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
            else v = (ea - ei) * in[e];  // mode 4
        } else {
            double ea = eorb[ia], eb = eorb[ib], ei = eorb[ii], ej = eorb[ij];
            if (mode == 0) v = ea + eb - ei - ej;
            else if (mode == 1) v = in[e] / ((ea + eb - ei - ej) - w0);
            else v = in[e] / (ei + ej - ea - eb);  // mode 2
        }
        out[e] = v;
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
__global__ void k_copy(double *__restrict__ y, const double *__restrict__ x, i64 n) {
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) y[i] = x[i];
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

// optional CUDA-event timing of every k_contract launch (on its stream)
namespace {
struct Timing {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    size_t used = 0;
    std::vector<double> flops;
};
Timing &timing() {
    static Timing t;
    return t;
}
}  // namespace

int contract_timing(int enable) {
    timing().on = enable != 0;
    return CPSD_OK;
}

int contract_time(double *ms, int64_t *launches, double *flops, int reset) {
    Timing &t = timing();
    double tot = 0.0, fl = 0.0;
    for (size_t i = 0; i + 1 < t.used; i += 2) {
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
    }
    return CPSD_OK;
}

static int timing_event(cudaEvent_t *e) {
    Timing &t = timing();
    if (t.used == t.pool.size()) {
        cudaEvent_t ev;
        CPSD_TRY(cuda_check(cudaEventCreate(&ev), "event create"));
        t.pool.push_back(ev);
    }
    *e = t.pool[t.used++];
    return CPSD_OK;
}

int launch_contract(const ContractPlan *p, const double *A, const double *B, double *C, double alpha) {
    if (p->empty) return CPSD_OK;
    CPSD_TRY(const_cast<ContractPlan *>(p)->upload());
    double *part = nullptr;
    ScratchScope scope;
    if (p->nparts > 0) CPSD_TRY(scratch(p->nparts * BM * BN, &part));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (timing().on) {
        CPSD_TRY(timing_event(&e0));
        CPSD_TRY(timing_event(&e1));
        timing().flops.push_back(p->flops);
        CPSD_TRY(cuda_check(cudaEventRecord(e0, stream()), "event record"));
    }
    k_contract<<<p->ntiles, NT, 0, stream()>>>(A, B, C, p->d_tasks, p->d_segs, p->d_tiles, alpha, part);
    count_launch();
    ctx().flops += p->flops;
    if (e1) CPSD_TRY(cuda_check(cudaEventRecord(e1, stream()), "event record"));
    if (p->nreduce > 0) {
        k_splitk_reduce<<<p->nreduce, NT, 0, stream()>>>(p->d_reduce, p->d_tasks, part, C, alpha);
        count_launch();
    }
    return cuda_check(cudaGetLastError(), "k_contract");
}

int launch_pairmap(const PairMapPlan *p, const double *in, double *out, double alpha, double beta, i64 nb,
                   i64 in_stride, i64 out_stride) {
    if (p->total == 0 || nb <= 0) return CPSD_OK;
    CPSD_TRY(const_cast<PairMapPlan *>(p)->upload());
    k_pairmap<<<grid_for(p->total * nb), 256, 0, stream()>>>(p->d_blocks, p->nblocks, p->total, p->d_idx, p->d_sgn,
                                                             p->lterms, p->rterms, in, out, alpha, beta, nb,
                                                             in_stride, out_stride);
    count_launch();
    return cuda_check(cudaGetLastError(), "k_pairmap");
}

int launch_scale(double *x, i64 n, double beta) {
    if (n <= 0 || beta == 1.0) return CPSD_OK;
    if (beta == 0.0) {
        return cuda_check(cudaMemsetAsync(x, 0, sizeof(double) * (size_t)n, stream()), "memset");
    }
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

// y_c += sgn * a[c] * x_c for each copy c (scalars resident on the device)
__global__ void k_axpy_dev(i64 n, const double *__restrict__ a, double sgn, const double *__restrict__ x,
                           double *__restrict__ y, i64 nb, i64 sx, i64 sy) {
    for (i64 g = (i64)blockIdx.x * blockDim.x + threadIdx.x; g < n * nb; g += (i64)gridDim.x * blockDim.x) {
        i64 c = g / n, i = g - c * n;
        y[c * sy + i] += sgn * a[c] * x[c * sx + i];
    }
}
int launch_axpy_dev(i64 n, const double *a_dev, double sgn, const double *x, double *y, i64 nb, i64 sx, i64 sy) {
    if (n <= 0 || nb <= 0) return CPSD_OK;
    k_axpy_dev<<<grid_for(n * nb), 256, 0, stream()>>>(n, a_dev, sgn, x, y, nb, sx, sy);
    count_launch();
    return cuda_check(cudaGetLastError(), "k_axpy_dev");
}

}  // namespace cpsd
