// Device-resident Davidson (src/lib_cc/mod_davidson.f90:40-728) and DIIS
// (src/libsrint/dosodiis2_d.f:1-119, dodiis.f, minv.f) for the small CIS /
// R1 spaces: one CTA owns the whole subspace logic, so an iteration costs
// one step launch + the batched sigma contraction + one Ritz-matrix update.
#include "solvers.cuh"

namespace cpsd {

namespace {
constexpr int DT = 512;  // threads of the single-CTA solver kernels

__device__ double block_sum(double v, double *sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int i = 0; i < DT / 32; i++) r += sh[i];
        sh[DT / 32] = r;
    }
    __syncthreads();
    double r = sh[DT / 32];
    __syncthreads();
    return r;
}

__device__ double block_dot(const double *x, const double *y, int n, double *sh) {
    double a = 0.0;
    for (int k = threadIdx.x; k < n; k += DT) a = fma(x[k], y[k], a);
    return block_sum(a, sh);
}

// value of the first element of largest magnitude (BLAS idamax semantics)
__device__ double block_amax(const double *x, int n, double *sh, int *shi) {
    double best = -1.0;
    int bi = 0x7fffffff;
    for (int k = threadIdx.x; k < n; k += DT) {
        double a = fabs(x[k]);
        if (a > best) {
            best = a;
            bi = k;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        double ob = __shfl_down_sync(0xffffffffu, best, o);
        int oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
            best = ob;
            bi = oi;
        }
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
        sh[w] = best;
        shi[w] = bi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = -1.0;
        int ii = 0x7fffffff;
        for (int i = 0; i < DT / 32; i++)
            if (sh[i] > b || (sh[i] == b && shi[i] < ii)) {
                b = sh[i];
                ii = shi[i];
            }
        shi[DT / 32] = ii;
    }
    __syncthreads();
    int idx = shi[DT / 32];
    __syncthreads();
    return (idx < n) ? x[idx] : 0.0;
}

// out[r] = x_r . y_r for the nr vector pairs x_r = x + r n, y_r = y + r n,
// each summed in block_dot's order (strided per-thread sums, warp
// shuffle-down, warp totals in warp order), with two barriers for all r
__device__ void block_dots(const double *x, const double *y, int n, int nr, double *red, double *out) {
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    for (int r = 0; r < nr; r++) {
        double a = 0.0;
        for (int k = threadIdx.x; k < n; k += DT) a = fma(x[(size_t)r * n + k], y[(size_t)r * n + k], a);
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if (l == 0) red[r * (DT / 32) + w] = a;
    }
    __syncthreads();
    if (threadIdx.x < nr) {
        double s = 0.0;
        for (int i = 0; i < DT / 32; i++) s += red[threadIdx.x * (DT / 32) + i];
        out[threadIdx.x] = s;
    }
    __syncthreads();
}

// out[r] = block_amax of x_r = x + r n for r < nr (value of the first
// element of largest magnitude), with two barriers for all r
__device__ void block_amaxs(const double *x, int n, int nr, double *redv, int *redi, double *out) {
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    for (int r = 0; r < nr; r++) {
        double best = -1.0;
        int bi = 0x7fffffff;
        for (int k = threadIdx.x; k < n; k += DT) {
            const double a = fabs(x[(size_t)r * n + k]);
            if (a > best) {
                best = a;
                bi = k;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_down_sync(0xffffffffu, best, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ob > best || (ob == best && oi < bi)) {
                best = ob;
                bi = oi;
            }
        }
        if (l == 0) {
            redv[r * (DT / 32) + w] = best;
            redi[r * (DT / 32) + w] = bi;
        }
    }
    __syncthreads();
    if (threadIdx.x < nr) {
        const int r = threadIdx.x;
        double bv = -1.0;
        int ii = 0x7fffffff;
        for (int i = 0; i < DT / 32; i++)
            if (redv[r * (DT / 32) + i] > bv || (redv[r * (DT / 32) + i] == bv && redi[r * (DT / 32) + i] < ii)) {
                bv = redv[r * (DT / 32) + i];
                ii = redi[r * (DT / 32) + i];
            }
        out[r] = (ii < n) ? x[(size_t)r * n + ii] : 0.0;
    }
    __syncthreads();
}

// dot product of two length-n vectors by one warp (result in every lane)
__device__ double warp_dot(const double *x, const double *y, int n) {
    const int lane = threadIdx.x & 31;
    double a = 0.0;
#pragma unroll 4
    for (int k = lane; k < n; k += 32) a = fma(x[k], y[k], a);
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    return a;
}

// Cyclic Jacobi on the symmetric n x n matrix S (row-major, ld DAV_MAXD,
// zero outside n x n) by the whole block; eigenvectors accumulate in the
// columns of V.  Classic threshold (Golub & Van Loan, Alg. 8.5.3): an
// element below 1e-17 sqrt(|a_pp a_qq|) is negligible and set to zero; a
// sweep without rotations ends the iteration.  The n(n-1)/2 rotations of a
// sweep run as n-1 rounds of n/2 disjoint rotations (round-robin pairing,
// n padded to even), each round one parallel update of S and V.  The
// iteration ends at the first round whose matrix has no element above the
// threshold: the rounds left of that sweep and the sweep without rotations
// would change no diagonal element and no column of V.  The
// rotation of a pair is
//   t = sgn(d b) |b| / (|d| + hypot(d, b)),  d = a_qq - a_pp, b = 2 a_pq,
//   c = 1 / sqrt(1 + t^2),  s = t c
// (the smaller root of t^2 + 2 tau t - 1 = 0, tau = d / b, written with one
// division), evaluated next to the threshold test.
__device__ void block_jacobi(double *S, double *V, int n) {
    __shared__ double cs[DAV_MAXD], sn[DAV_MAXD];
    __shared__ int pp[DAV_MAXD / 2], qq[DAV_MAXD / 2];
    const int tid = threadIdx.x;
    const int m = (n + 1) & ~1, half = m / 2;
    for (int e = tid; e < DAV_MAXD * DAV_MAXD; e += DT) {
        int i = e / DAV_MAXD, j = e % DAV_MAXD;
        V[e] = (i == j && i < m) ? 1.0 : 0.0;
    }
    __syncthreads();
    bool done = m <= 1;
    for (int sweep = 0; sweep < 50 && !done; sweep++) {
        for (int r = 0; r < m - 1; r++) {
            // does any element of the matrix still call for a rotation?
            // (asked by warps 1.., beside warp 0's rotation parameters)
            bool above = false;
            for (int e = tid - 32; e >= 0 && e < n * n; e += DT - 32) {
                const int p = e / n, q = e - p * n;
                if (p < q) {
                    const double apq = S[p * DAV_MAXD + q];
                    above |= !(fabs(apq) <= 1.0e-17 * sqrt(fabs(S[p * DAV_MAXD + p]) * fabs(S[q * DAV_MAXD + q])) ||
                               apq == 0.0);
                }
            }
            if (tid < half) {  // pair k of round r: (m-1, r) and (r+k, r-k) mod m-1
                int a, b;
                if (tid == 0) {
                    a = r;
                    b = m - 1;
                } else {
                    a = (r + tid) % (m - 1);
                    b = (r - tid + (m - 1)) % (m - 1);
                }
                int p = min(a, b), q = max(a, b);
                double apq = S[p * DAV_MAXD + q];
                double app = S[p * DAV_MAXD + p], aqq = S[q * DAV_MAXD + q];
                const double d = aqq - app, b2 = 2.0 * apq;
                double t = fabs(b2) / (fabs(d) + hypot(d, b2));
                if (d != 0.0 && ((d > 0.0) != (b2 > 0.0))) t = -t;
                const double ct = rsqrt(1.0 + t * t);
                double c = 1.0, s = 0.0;
                if (!(fabs(apq) <= 1.0e-17 * sqrt(fabs(app) * fabs(aqq)) || apq == 0.0)) {
                    c = ct;
                    s = t * ct;
                }
                pp[tid] = p;
                qq[tid] = q;
                cs[tid] = c;
                sn[tid] = s;
            }
            if (!__syncthreads_or(above)) {
                done = true;
                break;
            }
            // S <- J^T S J on the 2x2 blocks of (pair k rows, pair l columns)
            // by the first half of the block, V <- V J by the second
            for (int idx = tid; tid < DT / 2 && idx < half * half; idx += DT / 2) {
                const int k = idx / half, l = idx % half;
                const int pk = pp[k], qk = qq[k], pl = pp[l], ql = qq[l];
                const double ck = cs[k], sk = sn[k], cl = cs[l], sl = sn[l];
                double b00 = S[pk * DAV_MAXD + pl], b01 = S[pk * DAV_MAXD + ql];
                double b10 = S[qk * DAV_MAXD + pl], b11 = S[qk * DAV_MAXD + ql];
                double t00 = cl * b00 - sl * b01, t01 = sl * b00 + cl * b01;
                double t10 = cl * b10 - sl * b11, t11 = sl * b10 + cl * b11;
                double n00 = ck * t00 - sk * t10, n01 = ck * t01 - sk * t11;
                double n10 = sk * t00 + ck * t10, n11 = sk * t01 + ck * t11;
                if (k == l) n01 = n10 = 0.0;  // annihilated (or negligible) element
                S[pk * DAV_MAXD + pl] = n00;
                S[pk * DAV_MAXD + ql] = n01;
                S[qk * DAV_MAXD + pl] = n10;
                S[qk * DAV_MAXD + ql] = n11;
            }
            for (int idx = tid - DT / 2; idx >= 0 && idx < m * half; idx += DT / 2) {
                const int i = idx / half, l = idx % half;
                const int pl = pp[l], ql = qq[l];
                const double cl = cs[l], sl = sn[l];
                double vp = V[i * DAV_MAXD + pl], vq = V[i * DAV_MAXD + ql];
                V[i * DAV_MAXD + pl] = cl * vp - sl * vq;
                V[i * DAV_MAXD + ql] = sl * vp + cl * vq;
            }
            __syncthreads();
        }
    }
    __syncthreads();
}

// ------------------------------------------------ general real eigenproblem
// Eigenvalues and right eigenvectors of a general real n x n matrix (n <= 32)
// by one warp, in the form LAPACK's dgeev('N', 'V') returns them to the
// reference's Davidson (src/lib_cc/mod_davidson.f90:185-186): wr / wi the
// eigenvalues, a complex pair at (k, k + 1) with wi[k] > 0 first; column k
// of V the eigenvector of a real eigenvalue, columns k and k + 1 the real and
// imaginary parts of the eigenvector of wr[k] + i wi[k]; every eigenvector
// of unit 2-norm with its largest component real.  Method (Golub & Van Loan,
// Matrix Computations, 4th ed., sections 7.4-7.5 and 7.6.4):
//   1. Householder reduction to upper Hessenberg form, H = Z^T A Z;
//   2. Francis double-shift QR sweeps on the active window [l, hi] to real
//      Schur form T, Z accumulated; a subdiagonal element at most eps times
//      its two diagonal neighbours deflates; sweeps 10 and 20 of a window
//      use the ad-hoc exceptional shift of the LAPACK/EISPACK QR codes;
//      a 2 x 2 block with real eigenvalues is rotated to triangular form;
//   3. eigenvectors of T by back substitution (lane e solves for eigenvalue
//      e, complex arithmetic for a pair), then V = Z X and normalisation.
// Lane i owns row i or column i of every update; every lane walks the same
// control flow (deflation tests, shifts and reflectors are computed from
// shared values by all lanes alike).  H, Z and X are row-major with leading
// dimension GL (odd, so that a lane per row hits distinct banks); H is
// destroyed, Z and X are scratch, V (leading dimension DAV_MAXD, may alias
// Z) receives the vectors.  Returns the number of QR sweeps, or -1 when a
// window did not converge within 30 max(10, n) sweeps.
constexpr int GL = DAV_MAXD + 1;

__device__ __forceinline__ double warp_allsum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_allmax(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

struct cplx {
    double re, im;
};
__device__ __forceinline__ cplx cmul(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ cplx csub(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
// a / b by Smith's scaling (R. L. Smith, CACM 5 (1962) 435); |b| >= tiny
__device__ cplx cdiv(cplx a, cplx b, double tiny) {
    if (fabs(b.re) + fabs(b.im) < tiny) b = {tiny, 0.0};
    if (fabs(b.re) >= fabs(b.im)) {
        const double r = b.im / b.re, d = b.re + b.im * r;
        return {(a.re + a.im * r) / d, (a.im - a.re * r) / d};
    }
    const double r = b.re / b.im, d = b.im + b.re * r;
    return {(a.re * r + a.im) / d, (a.im * r - a.re) / d};
}

// x of the 2 x 2 system [[t00 - lam, t01], [t10, t11 - lam]] x = -rhs
// (Cramer's rule with the determinant kept away from zero)
__device__ void solve2(double t00, double t01, double t10, double t11, cplx lam, cplx r0, cplx r1, double tiny,
                       cplx *x0, cplx *x1) {
    const cplx a = {t00 - lam.re, -lam.im}, d = {t11 - lam.re, -lam.im};
    const cplx det = csub(cmul(a, d), {t01 * t10, 0.0});
    const cplx b0 = {-r0.re, -r0.im}, b1 = {-r1.re, -r1.im};
    *x0 = cdiv(csub(cmul(b0, d), {t01 * b1.re, t01 * b1.im}), det, tiny);
    *x1 = cdiv(csub(cmul(a, b1), {t10 * b0.re, t10 * b0.im}), det, tiny);
}

__device__ int warp_geev(double *H, double *Z, double *X, double *V, double *wr, double *wi, int n) {
    const int lane = threadIdx.x & 31;
    const double eps = 2.220446049250313e-16;
    for (int i = 0; i < n; i++)
        if (lane < n) Z[i * GL + lane] = (i == lane) ? 1.0 : 0.0;
    __syncwarp();
    // ---- 1. Hessenberg form: reflector k zeroes column k below row k + 1
    for (int k = 0; k + 2 < n; k++) {
        const double xi = (lane > k && lane < n) ? H[lane * GL + k] : 0.0;
        const double tail2 = warp_allsum(lane > k + 1 ? xi * xi : 0.0);
        if (tail2 == 0.0) continue;  // column already reduced (same on every lane)
        const double x0 = H[(k + 1) * GL + k];
        const double alpha = -copysign(sqrt(tail2 + x0 * x0), x0);
        const double beta = 1.0 / (alpha * (alpha - x0));  // 2 / v^T v
        if (lane < n) X[lane] = (lane == k + 1) ? x0 - alpha : (lane > k + 1 ? xi : 0.0);
        __syncwarp();
        if (lane >= k && lane < n) {  // H <- P H, lane = column
            double s = 0.0;
            for (int i = k + 1; i < n; i++) s += X[i] * H[i * GL + lane];
            s *= beta;
            for (int i = k + 1; i < n; i++) H[i * GL + lane] -= s * X[i];
            if (lane == k) {
                H[(k + 1) * GL + k] = alpha;
                for (int i = k + 2; i < n; i++) H[i * GL + k] = 0.0;
            }
        }
        __syncwarp();
        if (lane < n) {  // H <- H P and Z <- Z P, lane = row
            double s = 0.0, t = 0.0;
            for (int j = k + 1; j < n; j++) {
                s += H[lane * GL + j] * X[j];
                t += Z[lane * GL + j] * X[j];
            }
            s *= beta;
            t *= beta;
            for (int j = k + 1; j < n; j++) {
                H[lane * GL + j] -= s * X[j];
                Z[lane * GL + j] -= t * X[j];
            }
        }
        __syncwarp();
    }
    // 1-norm of H: the scale of the deflation test when both diagonal
    // neighbours vanish
    double cn = 0.0;
    if (lane < n)
        for (int i = 0; i < n; i++) cn += fabs(H[i * GL + lane]);
    const double anorm = warp_allmax(cn);
    const double tiny = fmax(eps * anorm, 1.0e-300);
    // ---- 2. real Schur form
    const int maxits = 30 * max(10, n);
    int hi = n - 1, its = 0, sweeps = 0;
    while (hi >= 0) {
        int l = hi;
        for (; l > 0; l--) {
            double s = fabs(H[(l - 1) * GL + l - 1]) + fabs(H[l * GL + l]);
            if (s == 0.0) s = anorm;
            if (fabs(H[l * GL + l - 1]) <= eps * s) break;
        }
        __syncwarp();
        if (l > 0 && lane == 0) H[l * GL + l - 1] = 0.0;
        __syncwarp();
        if (l == hi) {  // 1 x 1 block
            if (lane == 0) {
                wr[hi] = H[hi * GL + hi];
                wi[hi] = 0.0;
            }
            hi--;
            its = 0;
            continue;
        }
        if (l == hi - 1) {  // 2 x 2 block
            const int m = hi - 1;
            const double a = H[m * GL + m], b = H[m * GL + hi], c = H[hi * GL + m], d = H[hi * GL + hi];
            const double p = 0.5 * (a - d), disc = p * p + b * c;
            if (disc >= 0.0) {
                // real pair: rotate by G = [cs -sn; sn cs] whose first column
                // is the eigenvector (z, c) of lam1 = d + z
                const double z = p + copysign(sqrt(disc), p);
                const double lam1 = d + z, lam2 = (z != 0.0) ? d - (b * c) / z : lam1;
                const double r = hypot(z, c), cs = z / r, sn = c / r;
                if (lane >= m && lane < n) {
                    const double hm = H[m * GL + lane], hh = H[hi * GL + lane];
                    H[m * GL + lane] = cs * hm + sn * hh;
                    H[hi * GL + lane] = -sn * hm + cs * hh;
                }
                __syncwarp();
                if (lane < n) {
                    if (lane <= hi) {
                        const double hm = H[lane * GL + m], hh = H[lane * GL + hi];
                        H[lane * GL + m] = cs * hm + sn * hh;
                        H[lane * GL + hi] = -sn * hm + cs * hh;
                    }
                    const double zm = Z[lane * GL + m], zh = Z[lane * GL + hi];
                    Z[lane * GL + m] = cs * zm + sn * zh;
                    Z[lane * GL + hi] = -sn * zm + cs * zh;
                }
                __syncwarp();
                if (lane == 0) {
                    H[hi * GL + m] = 0.0;
                    H[m * GL + m] = lam1;
                    H[hi * GL + hi] = lam2;
                    wr[m] = lam1;
                    wr[hi] = lam2;
                    wi[m] = wi[hi] = 0.0;
                }
            } else if (lane == 0) {  // complex pair: the block stays
                wr[m] = wr[hi] = 0.5 * (a + d);
                wi[m] = sqrt(-disc);
                wi[hi] = -wi[m];
            }
            __syncwarp();
            hi -= 2;
            its = 0;
            continue;
        }
        if (its >= maxits) return -1;
        its++;
        sweeps++;
        double h11, h12, h21, h22;  // the shifts are the eigenvalues of [h11 h12; h21 h22]
        if (its == 10 || its == 20) {
            const double s = (its == 10) ? fabs(H[(l + 1) * GL + l]) + fabs(H[(l + 2) * GL + l + 1])
                                         : fabs(H[hi * GL + hi - 1]) + fabs(H[(hi - 1) * GL + hi - 2]);
            h11 = 0.75 * s + ((its == 10) ? H[l * GL + l] : H[hi * GL + hi]);
            h12 = -0.4375 * s;
            h21 = s;
            h22 = h11;
        } else {
            h11 = H[(hi - 1) * GL + hi - 1];
            h12 = H[(hi - 1) * GL + hi];
            h21 = H[hi * GL + hi - 1];
            h22 = H[hi * GL + hi];
        }
        const double tr = h11 + h22, det = h11 * h22 - h12 * h21;
        // first column of (H - s1)(H - s2) in the window
        const double hll = H[l * GL + l], h1l = H[(l + 1) * GL + l];
        double x = hll * hll + H[l * GL + l + 1] * h1l - tr * hll + det;
        double y = h1l * (hll + H[(l + 1) * GL + l + 1] - tr);
        double z = h1l * H[(l + 2) * GL + l + 1];
        for (int k = l; k <= hi - 1; k++) {
            const bool three = k < hi - 1;  // reflector length 3, else 2
            if (!three) z = 0.0;
            const double t2 = y * y + z * z;
            if (t2 != 0.0) {
                const double alpha = -copysign(sqrt(x * x + t2), x);
                const double beta = 1.0 / (alpha * (alpha - x));
                const double v0 = x - alpha, v1 = y, v2 = z;
                const int q = max(l, k - 1);
                if (lane >= q && lane < n) {  // rows k.. of columns q..n-1
                    double a0 = H[k * GL + lane], a1 = H[(k + 1) * GL + lane];
                    double a2 = three ? H[(k + 2) * GL + lane] : 0.0;
                    const double s = beta * (v0 * a0 + v1 * a1 + v2 * a2);
                    a0 -= s * v0;
                    a1 -= s * v1;
                    a2 -= s * v2;
                    if (lane == k - 1) {  // the bulge column: exactly (alpha, 0, 0)
                        a0 = alpha;
                        a1 = a2 = 0.0;
                    }
                    H[k * GL + lane] = a0;
                    H[(k + 1) * GL + lane] = a1;
                    if (three) H[(k + 2) * GL + lane] = a2;
                }
                __syncwarp();
                if (lane < n) {  // columns k.. of rows 0..min(k+3, hi); Z all rows
                    if (lane <= min(k + 3, hi)) {
                        const double a0 = H[lane * GL + k], a1 = H[lane * GL + k + 1];
                        const double a2 = three ? H[lane * GL + k + 2] : 0.0;
                        const double s = beta * (a0 * v0 + a1 * v1 + a2 * v2);
                        H[lane * GL + k] = a0 - s * v0;
                        H[lane * GL + k + 1] = a1 - s * v1;
                        if (three) H[lane * GL + k + 2] = a2 - s * v2;
                    }
                    const double c0 = Z[lane * GL + k], c1 = Z[lane * GL + k + 1];
                    const double c2 = three ? Z[lane * GL + k + 2] : 0.0;
                    const double s = beta * (c0 * v0 + c1 * v1 + c2 * v2);
                    Z[lane * GL + k] = c0 - s * v0;
                    Z[lane * GL + k + 1] = c1 - s * v1;
                    if (three) Z[lane * GL + k + 2] = c2 - s * v2;
                }
                __syncwarp();
            }
            if (three) {
                x = H[(k + 1) * GL + k];
                y = H[(k + 2) * GL + k];
                z = (k < hi - 2) ? H[(k + 3) * GL + k] : 0.0;
            }
        }
    }
    __syncwarp();
    // ---- 3. eigenvectors of T (lane e: eigenvalue e; a pair by its first lane)
    if (lane < n && wi[lane] >= 0.0) {
        const int e = lane;
        const cplx lam = {wr[e], wi[e]};
        const bool pair = wi[e] > 0.0;
        const int top = pair ? e + 1 : e;  // last nonzero row of x
        for (int i = top + 1; i < n; i++) {
            X[i * GL + e] = 0.0;
            if (pair) X[i * GL + e + 1] = 0.0;
        }
        // x[i] kept as (X[i][e], X[i][e+1]) for a pair, X[i][e] otherwise
        if (pair) {
            // eigenvector of the block [a b; c d] for lam: (lam - d, c) or
            // (b, lam - a), whichever is longer
            const double a = H[e * GL + e], b = H[e * GL + e + 1], c = H[(e + 1) * GL + e], d = H[(e + 1) * GL + e + 1];
            const cplx u0 = {lam.re - d, lam.im}, w1 = {lam.re - a, lam.im};
            const double nu = u0.re * u0.re + u0.im * u0.im + c * c, nw = b * b + w1.re * w1.re + w1.im * w1.im;
            const cplx x0 = (nu >= nw) ? u0 : cplx{b, 0.0}, x1 = (nu >= nw) ? cplx{c, 0.0} : w1;
            X[e * GL + e] = x0.re;
            X[e * GL + e + 1] = x0.im;
            X[(e + 1) * GL + e] = x1.re;
            X[(e + 1) * GL + e + 1] = x1.im;
        } else {
            X[e * GL + e] = 1.0;
        }
        auto xval = [&](int j) -> cplx {
            return pair ? cplx{X[j * GL + e], X[j * GL + e + 1]} : cplx{X[j * GL + e], 0.0};
        };
        auto rowsum = [&](int i, int j0) -> cplx {  // sum_{j >= j0} T[i][j] x[j]
            cplx r = {0.0, 0.0};
            for (int j = j0; j <= top; j++) {
                const cplx xj = xval(j);
                r.re += H[i * GL + j] * xj.re;
                r.im += H[i * GL + j] * xj.im;
            }
            return r;
        };
        for (int i = e - 1; i >= 0;) {
            if (i > 0 && H[i * GL + i - 1] != 0.0) {  // rows i-1, i: a 2 x 2 block
                const cplx r0 = rowsum(i - 1, i + 1), r1 = rowsum(i, i + 1);
                cplx x0, x1;
                solve2(H[(i - 1) * GL + i - 1], H[(i - 1) * GL + i], H[i * GL + i - 1], H[i * GL + i], lam, r0, r1,
                       tiny, &x0, &x1);
                X[(i - 1) * GL + e] = x0.re;
                X[i * GL + e] = x1.re;
                if (pair) {
                    X[(i - 1) * GL + e + 1] = x0.im;
                    X[i * GL + e + 1] = x1.im;
                }
                i -= 2;
            } else {
                const cplx r = rowsum(i, i + 1);
                const cplx xi = cdiv({-r.re, -r.im}, {H[i * GL + i] - lam.re, -lam.im}, tiny);
                X[i * GL + e] = xi.re;
                if (pair) X[i * GL + e + 1] = xi.im;
                i -= 1;
            }
        }
    }
    __syncwarp();
    // V = Z X into H (T is no longer read); lane e: column e
    if (lane < n) {
        const int top = (wi[lane] > 0.0) ? lane + 1 : lane;
        for (int i = 0; i < n; i++) {
            double s = 0.0;
            for (int j = 0; j <= top; j++) s += Z[i * GL + j] * X[j * GL + lane];
            H[i * GL + lane] = s;
        }
    }
    __syncwarp();
    // unit 2-norm, largest component real (a pair: by its first lane)
    if (lane < n && wi[lane] >= 0.0) {
        const int e = lane;
        if (wi[e] == 0.0) {
            double s = 0.0;
            for (int i = 0; i < n; i++) s += H[i * GL + e] * H[i * GL + e];
            const double f = 1.0 / sqrt(s);
            for (int i = 0; i < n; i++) H[i * GL + e] *= f;
        } else {
            double s = 0.0, best = -1.0;
            int kb = 0;
            for (int i = 0; i < n; i++) {
                const double m2 = H[i * GL + e] * H[i * GL + e] + H[i * GL + e + 1] * H[i * GL + e + 1];
                s += m2;
                if (m2 > best) {
                    best = m2;
                    kb = i;
                }
            }
            // multiply by conj(v_kb) / (|v_kb| |v|)
            const double mk = sqrt(best), f = 1.0 / (sqrt(s) * mk);
            const double cr = H[kb * GL + e] * f, ci = H[kb * GL + e + 1] * f;
            for (int i = 0; i < n; i++) {
                const double re = H[i * GL + e], im = H[i * GL + e + 1];
                H[i * GL + e] = re * cr + im * ci;
                H[i * GL + e + 1] = im * cr - re * ci;
            }
            H[kb * GL + e + 1] = 0.0;
        }
    }
    __syncwarp();
    // each column to unit norm where it is off by more than 1e-10, as the
    // reference does with the real and imaginary parts it keeps
    // (mod_davidson.f90:211-217); copy out with V's leading dimension
    if (lane < n) {
        double s = 0.0;
        for (int i = 0; i < n; i++) s += H[i * GL + lane] * H[i * GL + lane];
        const double t = sqrt(s), f = (fabs(t - 1.0) > 1.0e-10) ? 1.0 / t : 1.0;
        for (int i = 0; i < DAV_MAXD; i++) V[i * DAV_MAXD + lane] = (i < n) ? H[i * GL + lane] * f : 0.0;
    } else {
        for (int i = 0; i < DAV_MAXD; i++) V[i * DAV_MAXD + lane] = 0.0;
    }
    __syncwarp();
    return sweeps;
}

// Schmidt_2D (mod_davidson.f90:642-680) on the dim columns (length len <= 32)
// of `in`, by one warp: lane k holds row k; modified Gram-Schmidt in the
// reference's order
__device__ void warp_schmidt_2d(const double *in, double *out, int len, int dim) {
    const int lane = threadIdx.x & 31;
    for (int i = 0; i < dim; i++)
        if (lane < len) out[i * len + lane] = in[i * len + lane];
    __syncwarp();
    for (int i = 1; i < dim; i++) {
        double x = (lane < len) ? out[i * len + lane] : 0.0;
        for (int j = 0; j < i; j++) {
            double y = (lane < len) ? out[j * len + lane] : 0.0;
            double ov = x * y;
            for (int o = 16; o > 0; o >>= 1) ov += __shfl_xor_sync(0xffffffffu, ov, o);
            x += -ov * y;
        }
        double nrm = x * x;
        for (int o = 16; o > 0; o >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
        nrm = sqrt(nrm);
        if (lane < len) out[i * len + lane] = x * (1.0 / nrm);
        __syncwarp();
    }
}

__global__ void __launch_bounds__(DT) k_dav_init(DavState *st, DavBuffers b) {
    DavState &s = *st;
    const int n = s.dimA, D = s.D, nr = s.nroot;
    for (int e = threadIdx.x >> 5; e < nr * nr; e += DT / 32) {
        const int i = e / nr, j = e % nr;
        double v = warp_dot(b.fileEV + (size_t)j * (n + 1) + 1, b.AB[0] + (size_t)i * n, n);
        if ((threadIdx.x & 31) == 0) s.Abar[j + i * D] = v;
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < nr; i++) {
            s.eigenVal[i] = b.fileEV[(size_t)i * (n + 1)];
            for (int k = 0; k < D; k++) s.vecNeed[k + i * D] = (k == i) ? 1.0 : 0.0;
        }
        s.iterations = 1;
        s.dimIter = nr;
        s.dimFree = D - nr;
        s.dim_exceed = 0;
        s.cur = 0;
        s.done = 0;
        s.converged = 0;
    }
}

__global__ void __launch_bounds__(DT) k_dav_step(DavState *st, DavBuffers b) {
    __shared__ double S[DAV_MAXD * GL], V[DAV_MAXD * GL], X[DAV_MAXD * GL], ovl[DAV_MAXD];
    __shared__ double sh[DT / 32 + 1];
    DavState &s = *st;
    const int tid = threadIdx.x;
    const int D = s.D, n = s.dimA, nroot = s.nroot;
    if (s.done) return;
    if (s.iterations > s.maxcyc) {
        if (tid == 0) {
            s.done = 1;
            if (b.mailbox) {
                b.mailbox[0] = 0;
                __threadfence_system();
            }
        }
        return;
    }
    int dimIter = s.dimIter, cur = s.cur, dimFree = s.dimFree;
    const int dim_exceed = s.dim_exceed;
    // ---- step 3: eigenpairs of Abar, dgeev in the reference
    // (mod_davidson.f90:185-219).  Abar = B^T A B is symmetric when A is
    // (spin-flip CIS with real integrals); when it is symmetric to 1e-12 of
    // its largest element, the parallel Jacobi on 0.5 (Abar + Abar^T) gives
    // dgeev's eigenpairs (to rounding) fastest; otherwise one warp solves
    // the general problem (warp_geev: real parts of the eigenvalues, real
    // and imaginary parts of complex eigenvectors as dgeev returns them,
    // complex values counted as the reference's imaginary-eigenvalue warning)
    __shared__ double vR[DAV_MAXD], vI[DAV_MAXD];
    __shared__ int lw[DAV_MAXD], general;
    if (tid < 32) {
        double am = 0.0, ad = 0.0;
        if (tid < dimIter)
            for (int i = 0; i < dimIter; i++) {
                const double aij = s.Abar[i + tid * D], aji = s.Abar[tid + i * D];
                am = fmax(am, fabs(aij));
                ad = fmax(ad, fabs(aij - aji));
            }
        am = warp_allmax(am);
        ad = warp_allmax(ad);
        if (tid == 0) general = ad > 1.0e-12 * am;
    }
    __syncthreads();
    if (!general) {
        for (int e = tid; e < DAV_MAXD * DAV_MAXD; e += DT) {
            int i = e / DAV_MAXD, j = e % DAV_MAXD;
            S[e] = (i < dimIter && j < dimIter) ? 0.5 * (s.Abar[i + j * D] + s.Abar[j + i * D]) : 0.0;
        }
        __syncthreads();
        block_jacobi(S, V, dimIter);
        if (tid < dimIter) vR[tid] = S[tid * DAV_MAXD + tid];
    } else {
        for (int e = tid; e < dimIter * dimIter; e += DT) {
            const int i = e / dimIter, j = e % dimIter;
            S[i * GL + j] = s.Abar[i + j * D];
        }
        __syncthreads();
        if (tid < 32) {
            const int sw = warp_geev(S, V, X, V, vR, vI, dimIter);
            if (tid == 0) {
                s.nonsym_steps++;
                if (sw < 0) s.eig_fail = 1;
                for (int i = 0; i < dimIter; i++)
                    if (fabs(vI[i]) > 1.0e-10) s.warn_imag++;
            }
        }
    }
    __syncthreads();
    if (s.eig_fail) {  // the QR iteration did not converge: stop the solver
        if (tid == 0) {
            s.done = 1;
            if (b.mailbox) {
                b.mailbox[0] = 0;
                __threadfence_system();
            }
        }
        return;
    }
    // eigenvalues, their order and the chosen roots, worked out in shared
    // memory (vecR(i, k) = V[i][k] for i < dimIter, zero below) and then
    // published to the state
    for (int e = tid; e < D * dimIter; e += DT) {
        int i = e % D, k = e / D;
        s.vecR[i + k * D] = (i < dimIter) ? V[i * DAV_MAXD + k] : 0.0;
    }
    __syncthreads();
    if (tid == 0) {
        // sort (mod_davidson.f90:620-640)
        for (int i = 0; i < dimIter; i++) lw[i] = i + 1;
        for (int i = 0; i < dimIter - 1; i++)
            for (int j = i + 1; j < dimIter; j++)
                if (vR[lw[j] - 1] < vR[lw[i] - 1]) {
                    int t = lw[j];
                    lw[j] = lw[i];
                    lw[i] = t;
                }
        // root tracking by largest component (mod_davidson.f90:227-251),
        // searched over the positions not yet given to a root: the
        // reference also searches the assigned ones and, when one of them
        // wins, gives one eigenvector to two roots, whose collapse then
        // orthonormalises a repeated vector (division by zero); wherever the
        // reference assigns distinct vectors the choice is the same
        if (!s.lowest) {
            for (int iroot = 1; iroot <= nroot; iroot++) {
                double t1 = 0.0;
                int i = iroot;
                for (int j = iroot; j <= dimIter; j++) {
                    double t2 = fabs(V[(iroot - 1) * DAV_MAXD + (lw[j - 1] - 1)]);
                    if (t2 > t1) {
                        t1 = t2;
                        i = j;
                    }
                }
                int idx = lw[i - 1];
                for (int j = 1; j <= i - iroot; j++) lw[i - j] = lw[i - j - 1];
                lw[iroot - 1] = idx;
            }
        }
    }
    __syncthreads();
    if (tid < dimIter) {
        s.valR[tid] = vR[tid];
        s.lowestE[tid] = lw[tid];
    }
    if (tid < nroot) s.eigenVal[tid] = vR[lw[tid] - 1];
    for (int e = tid; e < nroot * D; e += DT) {
        const int ir = e / D, k = e % D;
        s.vecNeed[k + ir * D] = (k < dimIter) ? V[k * DAV_MAXD + (lw[ir] - 1)] : 0.0;
    }
    __syncthreads();
    // ---- collapse when the subspace was full (mod_davidson.f90:266-325)
    if (dim_exceed) {
        const int nd = s.ndimIter;
        for (int e = tid; e < nd * dimIter; e += DT) {
            int k = e % dimIter, i = e / dimIter;
            s.oldE[k + i * dimIter] = s.vecR[k + (s.lowestE[i] - 1) * D];
        }
        __syncthreads();
        if (tid < 32) warp_schmidt_2d(s.oldE, s.newE, dimIter, nd);
        __syncthreads();
        const int nw = 1 - cur;
        for (int ir = 0; ir < nd; ir++)
            for (int k = tid; k < n; k += DT) {
                double a = 0.0, c = 0.0;
                for (int i = 0; i < dimIter; i++) {
                    double t = s.newE[i + ir * dimIter];
                    a += t * b.AB[cur][(size_t)i * n + k];
                    c += t * b.B[cur][(size_t)i * n + k];
                }
                b.AB[nw][(size_t)ir * n + k] = a;
                b.B[nw][(size_t)ir * n + k] = c;
            }
        __syncthreads();
        cur = nw;
        dimFree = s.ndimFree;
        dimIter = nd;
        for (int e = tid >> 5; e < dimIter * dimIter; e += DT / 32) {
            const int i = e / dimIter, j = e % dimIter;
            double v = warp_dot(b.AB[cur] + (size_t)i * n, b.B[cur] + (size_t)j * n, n);
            if ((tid & 31) == 0) s.Abar[j + i * D] = v;
        }
        __syncthreads();
    }
    // ---- steps 4-6.  The Ritz vector, residual, convergence test and
    // preconditioned vector of a root depend only on the subspace before this
    // step (the new vectors go to positions >= dimIter), so they are formed
    // for all roots at once in per-root slices of w0 / w1 (each reduction
    // summed in block_dot / block_amax order); only the Schmidt projections
    // and the insertion of the new vectors run root after root.
    __shared__ double rd[DAV_MAXD * (DT / 32)], rv[DAV_MAXD];
    __shared__ int ri[DAV_MAXD * (DT / 32)], cvd[DAV_MAXD];
    double *const W0 = b.w0, *const W1 = b.w1;
    if (dim_exceed) {
        for (int e = tid; e < nroot * n; e += DT) {
            const int ir = e / n, k = e - ir * n;
            W0[(size_t)ir * n + k] = b.AB[cur][(size_t)ir * n + k];
            W1[(size_t)ir * n + k] = b.B[cur][(size_t)ir * n + k];
        }
    } else {
        // one pass over the basis serves RB roots: element k of every basis
        // vector is loaded once and summed into each root in basis order
        // (coefficient vecNeed(i, root) = V[i][lw[root] - 1])
        constexpr int RB = 8;
        for (int r0 = 0; r0 < nroot; r0 += RB) {
            const int nr = min(RB, nroot - r0);
            int col[RB];
#pragma unroll
            for (int q = 0; q < RB; q++) col[q] = q < nr ? lw[r0 + q] - 1 : 0;
            for (int k = tid; k < n; k += DT) {
                double a[RB], c[RB];
#pragma unroll
                for (int q = 0; q < RB; q++) a[q] = c[q] = 0.0;
#pragma unroll 4
                for (int i = 0; i < dimIter; i++) {
                    const double x = b.AB[cur][(size_t)i * n + k], y = b.B[cur][(size_t)i * n + k];
#pragma unroll
                    for (int q = 0; q < RB; q++) {
                        const double t = V[i * DAV_MAXD + col[q]];
                        a[q] += t * x;
                        c[q] += t * y;
                    }
                }
#pragma unroll
                for (int q = 0; q < RB; q++)
                    if (q < nr) {
                        W0[(size_t)(r0 + q) * n + k] = a[q];
                        W1[(size_t)(r0 + q) * n + k] = c[q];
                    }
            }
        }
    }
    __syncthreads();
    block_dots(W1, W1, n, nroot, rd, rv);
    for (int e = tid; e < nroot * n; e += DT) {
        const int ir = e / n, k = e - ir * n;
        const double t = sqrt(rv[ir]), ev = s.eigenVal[ir];
        double q = W1[(size_t)ir * n + k], aq = W0[(size_t)ir * n + k];
        if (fabs(t - 1.0) > 1.0e-10) {
            q *= 1.0 / t;
            aq *= 1.0 / t;
        }
        b.fileEV[(size_t)ir * (n + 1) + 1 + k] = q;
        W1[(size_t)ir * n + k] = q;
        W0[(size_t)ir * n + k] = aq - ev * q;
    }
    if (tid < nroot) b.fileEV[(size_t)tid * (n + 1)] = s.eigenVal[tid];
    __syncthreads();
    block_amaxs(W0, n, nroot, rd, ri, rv);
    if (tid < nroot) {
        cvd[tid] = fabs(rv[tid]) < s.maxError ? 1 : 0;
        s.conv[tid] = cvd[tid];
    }
    __syncthreads();
    int nNew = 0, nconv = 0;
    for (int ir = 0; ir < nroot; ir++) nconv += cvd[ir];
    for (int e = tid; e < nroot * n; e += DT) {
        const int ir = e / n, k = e - ir * n;
        if (cvd[ir]) continue;
        double d = s.eigenVal[ir] - b.diag[k];
        if (fabs(d) < 1.0e-4) d = (d < 0.0) ? -1.0e-4 : 1.0e-4;
        W1[(size_t)ir * n + k] = W0[(size_t)ir * n + k] / d;
    }
    __syncthreads();
    // SchmidtS (mod_davidson.f90:682-727): normalise, then project
    block_dots(W1, W1, n, nroot, rd, rv);
    for (int e = tid; e < nroot * n; e += DT) {
        const int ir = e / n, k = e - ir * n;
        if (!cvd[ir]) W1[(size_t)ir * n + k] *= 1.0 / sqrt(rv[ir]);
    }
    __syncthreads();
    for (int ir = 0; ir < nroot; ir++) {
        if (cvd[ir] || dimFree == 0) continue;
        double *const w1 = W1 + (size_t)ir * n;
        // projections on the basis: classical Gram-Schmidt applied twice
        // (same result as the reference's sequential projections to
        // rounding, with all overlaps of a pass computed at once)
        const int nb = dimIter + nNew;
        for (int pass = 0; pass < 2; pass++) {
            for (int i = tid >> 5; i < nb; i += DT / 32) {
                double v = warp_dot(b.B[cur] + (size_t)i * n, w1, n);
                if ((tid & 31) == 0) ovl[i] = v;
            }
            __syncthreads();
            for (int k = tid; k < n; k += DT) {
                double x = w1[k];
#pragma unroll 8
                for (int i = 0; i < nb; i++) x += -ovl[i] * b.B[cur][(size_t)i * n + k];
                w1[k] = x;
            }
            __syncthreads();
        }
        const double nrm = sqrt(block_dot(w1, w1, n, sh));
        if (nrm < 1.0e-6) continue;
        const int pos = dimIter + nNew;
        for (int k = tid; k < n; k += DT) b.B[cur][(size_t)pos * n + k] = w1[k] * (1.0 / nrm);
        __syncthreads();
        dimFree--;
        nNew++;
    }
    if (tid == 0) {
        s.cur = cur;
        s.dimIter = dimIter;
        s.dimFree = dimFree;
        s.newpos = dimIter;
        s.nNew = nNew;
        if (nconv == nroot) {
            s.done = 1;
            s.converged = 1;
        } else {
            s.dim_exceed = 0;
            if (dimFree == 0) {
                s.dim_exceed = 1;
                s.ndimIter = D - s.dimDel;
                if (s.ndimIter < nroot) {
                    s.ndimIter = nroot;
                    s.ndimFree = D - s.ndimIter;
                } else {
                    s.ndimFree = s.dimDel;
                }
            }
        }
        if (b.mailbox) {
            b.mailbox[0] = s.done ? 0 : 1;
            __threadfence_system();
        }
    }
    // staged copies of the new basis vectors (zero beyond nNew) for a sigma
    // launch whose size does not depend on nNew
    if (b.W)
        for (int q = 0; q < nroot; q++)
            for (int k = tid; k < n; k += DT)
                b.W[(size_t)q * n + k] = q < nNew ? b.B[cur][(size_t)(dimIter + q) * n + k] : 0.0;
}

// Ritz-matrix update with the new vectors (mod_davidson.f90:460-496); with
// staged sigma vectors, AW[0..nNew) are first put in place in AB
__global__ void __launch_bounds__(DT) k_dav_abar(DavState *st, DavBuffers b) {
    DavState &s = *st;
    if (s.done) return;
    const int n = s.dimA, D = s.D, dimIter = s.dimIter, nNew = s.nNew, cur = s.cur;
    if (b.AW) {
        for (int q = 0; q < nNew; q++)
            for (int k = threadIdx.x; k < n; k += DT)
                b.AB[cur][(size_t)(dimIter + q) * n + k] = b.AW[(size_t)q * n + k];
        __syncthreads();
    }
    const double *B = b.B[cur], *AB = b.AB[cur];
    // new rows (i >= dimIter, j < dimIter) then new columns (j >= dimIter)
    const int nrow = nNew * dimIter, tot = nrow + nNew * (dimIter + nNew);
    for (int e = threadIdx.x >> 5; e < tot; e += DT / 32) {
        int i, j;
        if (e < nrow) {
            j = e / nNew;
            i = dimIter + e % nNew;
        } else {
            j = dimIter + (e - nrow) / (dimIter + nNew);
            i = (e - nrow) % (dimIter + nNew);
        }
        double v = warp_dot(B + (size_t)i * n, AB + (size_t)j * n, n);
        if ((threadIdx.x & 31) == 0) s.Abar[i + j * D] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        s.dimIter = dimIter + nNew;
        s.iterations++;
    }
}

// eigen test of the final roots (mod_davidson.f90:525-542): AR in w-buffer
__global__ void __launch_bounds__(DT) k_dav_final(DavState *st, DavBuffers b, const double *AR) {
    __shared__ double sh[DT / 32 + 1];
    __shared__ int shi[DT / 32 + 1];
    DavState &s = *st;
    const int n = s.dimA;
    double worst = 0.0;
    for (int ir = 0; ir < s.nroot; ir++) {
        const double *R = b.fileEV + (size_t)ir * (n + 1);
        double w = R[0];
        for (int k = threadIdx.x; k < n; k += DT) b.w0[k] = AR[(size_t)ir * n + k] - w * R[1 + k];
        __syncthreads();
        double e = fabs(block_amax(b.w0, n, sh, shi));
        if (e > worst) worst = e;
    }
    if (threadIdx.x == 0) s.max_resid = worst;
}

// ------------------------------------------------------------------- DIIS
// LINPACK dgefa / dgesl (as MINV, src/libsrint/minv.f, calls them) by one
// warp on a matrix in shared memory (n <= 32): lane i owns row i.  Pivot =
// first row of largest magnitude; every element sees the same operations in
// the same order as the sequential LINPACK loops.
__device__ void warp_dgefa(double *a, int lda, int n, int *ipvt) {
    const int i = threadIdx.x & 31;
    for (int k = 0; k < n - 1; k++) {
        double m = (i >= k && i < n) ? fabs(a[i + k * lda]) : -1.0;
        int l = (i >= k && i < n) ? i : 0x7fffffff;
        for (int o = 16; o > 0; o >>= 1) {
            double om = __shfl_xor_sync(0xffffffffu, m, o);
            int ol = __shfl_xor_sync(0xffffffffu, l, o);
            if (om > m || (om == m && ol < l)) {
                m = om;
                l = ol;
            }
        }
        if (i == 0) ipvt[k] = l;
        __syncwarp();
        if (a[l + k * lda] == 0.0) continue;
        if (l != k && i >= k && i < n) {  // swap rows l and k in columns >= k (lane i: column i)
            double t = a[l + i * lda];
            a[l + i * lda] = a[k + i * lda];
            a[k + i * lda] = t;
        }
        __syncwarp();
        const double t = -1.0 / a[k + k * lda];
        if (i > k && i < n) {
            double aik = a[i + k * lda] * t;
            a[i + k * lda] = aik;
            for (int j = k + 1; j < n; j++) a[i + j * lda] += a[k + j * lda] * aik;
        }
        __syncwarp();
    }
    if (i == 0) ipvt[n - 1] = n - 1;
    __syncwarp();
}
__device__ void warp_dgesl(const double *a, int lda, int n, const int *ipvt, double *bv) {
    const int i = threadIdx.x & 31;
    for (int k = 0; k < n - 1; k++) {
        const int l = ipvt[k];
        const double t = bv[l];
        __syncwarp();
        if (i == 0 && l != k) {
            bv[l] = bv[k];
            bv[k] = t;
        }
        __syncwarp();
        if (i > k && i < n) bv[i] += t * a[i + k * lda];
        __syncwarp();
    }
    for (int kb = 0; kb < n; kb++) {
        const int k = n - 1 - kb;
        if (i == 0) bv[k] /= a[k + k * lda];
        __syncwarp();
        const double t = -bv[k];
        if (i < k) bv[i] += t * a[i + k * lda];
        __syncwarp();
    }
}

// R -= (<L|R> / ||L||) L, the reference's orthogonalR2L (which divides by
// the norm, not its square)
__device__ void block_orth(double *R, const double *L, int n, double *sh) {
    // L.L and L.R in one pass and one reduction, each summed in
    // block_dot's order (strided per-thread sums, shuffle-down, warp totals
    // in warp order)
    __shared__ double red[2][DT / 32];
    double aa = 0.0, ab = 0.0;
    for (int k = threadIdx.x; k < n; k += DT) {
        const double l = L[k];
        aa = fma(l, l, aa);
        ab = fma(l, R[k], ab);
    }
    for (int o = 16; o > 0; o >>= 1) {
        aa += __shfl_down_sync(0xffffffffu, aa, o);
        ab += __shfl_down_sync(0xffffffffu, ab, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[0][w] = aa;
        red[1][w] = ab;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double t = 0.0;
        for (int i = 0; i < DT / 32; i++) t += red[threadIdx.x][i];
        sh[threadIdx.x] = t;
    }
    __syncthreads();
    double nrm = sqrt(sh[0]);
    double dot = sh[1];
    __syncthreads();
    double f = -dot / nrm;
    for (int k = threadIdx.x; k < n; k += DT) R[k] += f * L[k];
    __syncthreads();
}

__device__ void diis_extrapolate(DiisState &s, const DiisBuffers &b, double *vec, double *sh, int *shi, double *Bm,
                                 double *coef, double *aug, double *rhs, int *ipvt);

// R *= 1 / <R|V> (the left vector's normalisation to the right one,
// calEigenCISDoo.f90:99-104: a dscal by the reciprocal)
__device__ void block_unit_dot(double *R, const double *V, int n, double *sh) {
    const double d = 1.0 / block_dot(R, V, n, sh);
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += DT) R[k] *= d;
    __syncthreads();
}

// one step of the device-driven solver for root blockIdx.x (see solvers.cuh)
__global__ void __launch_bounds__(DT) k_solver_step(SolverArgs a) {
    __shared__ double sh[DT / 32 + 1];
    __shared__ int shi[DT / 32 + 1];
    __shared__ double Bm[DIIS_MAXDIM * DIIS_MAXDIM];
    __shared__ double coef[DIIS_MAXDIM + 1];
    __shared__ double aug[(DIIS_MAXDIM + 1) * (DIIS_MAXDIM + 1)], rhs[DIIS_MAXDIM + 1];
    __shared__ int ipvt[DIIS_MAXDIM + 1];
    const int r = blockIdx.x, tid = threadIdx.x, len = a.len;
    SolverState &ss = a.ss[r];
    if (!ss.active) return;
    const int iter = ss.iter + 1;
    double *pr = a.pr + (size_t)r * len, *R1 = a.R1 + (size_t)r * len;
    const double *cc = a.cc + (size_t)r * len, *S = a.S + (size_t)r * len;
    const double *L = a.L ? a.L + (size_t)r * len : nullptr;
    if (iter > 1) {  // pr = cc; pr += (-w0) R1; pr += sigma  (the reference's updates, in order)
        if (a.w0) {
            const double mw0 = -a.w0[r];
            for (int k = tid; k < len; k += DT) pr[k] = fma(mw0, R1[k], cc[k]) + S[k];
        } else {
            for (int k = tid; k < len; k += DT) pr[k] = cc[k] + S[k];
        }
        __syncthreads();
    }
    if (iter > 1 || !a.keep_first)
        for (int k = tid; k < len; k += DT) R1[k] = pr[k] / a.den[k];
    __syncthreads();
    const double *NV = a.nrmv ? a.nrmv + (size_t)r * len : nullptr;
    DiisState &ds = a.ds[r];
    DiisBuffers b;
    b.prev = a.db.prev + (size_t)r * a.sprev;
    b.err = a.db.err + (size_t)r * a.serr;
    b.amp = a.db.amp + (size_t)r * a.serr;
    if (L) block_orth(R1, L, len, sh);
    if (NV) block_unit_dot(R1, NV, len, sh);
    if (iter == 1) {
        for (int k = tid; k < len; k += DT) b.prev[k] = R1[k];
        if (tid == 0) {
            ds.idimr = 1;
            ds.ndimr = 1;
            ds.res = 1.0;
        }
    } else {
        diis_extrapolate(ds, b, R1, sh, shi, Bm, coef, aug, rhs, ipvt);
    }
    __syncthreads();
    if (L) block_orth(R1, L, len, sh);
    if (NV) block_unit_dot(R1, NV, len, sh);
    if (tid == 0) {
        const double res = ds.res;
        ss.iter = iter;
        ss.res = res;
        if ((iter > 1 && fabs(res) < a.tol) || iter > a.cyc) ss.active = 0;
        a.mailbox[r] = ss.active;
        __threadfence_system();
    }
}

__device__ void diis_extrapolate(DiisState &s, const DiisBuffers &b, double *vec, double *sh, int *shi, double *Bm,
                                 double *coef, double *aug, double *rhs, int *ipvt) {
    const int len = s.len, maxdim = s.maxdim, tid = threadIdx.x;
    const int id = s.idimr - 1;
    for (int k = tid; k < len; k += DT) {
        double p = b.prev[k];
        b.amp[(size_t)id * len + k] = p;
        double e = vec[k] - p;
        vec[k] = e;
        b.err[(size_t)id * len + k] = e;
    }
    __syncthreads();
    const int nd = s.ndimr;
    // only the row of the error vector stored now changes; the others are
    // kept in the state from earlier steps
    for (int j = tid >> 5; j < nd; j += DT / 32) {
        double x = warp_dot(b.err + (size_t)id * len, b.err + (size_t)j * len, len);
        if ((tid & 31) == 0) {
            s.Bm[id + j * DIIS_MAXDIM] = x;
            s.Bm[j + id * DIIS_MAXDIM] = x;
        }
    }
    __syncthreads();
    for (int e = tid; e < DIIS_MAXDIM * DIIS_MAXDIM; e += DT) Bm[e] = s.Bm[e];
    __syncthreads();
    if (tid < 32) {  // dodiis (src/libsrint/dodiis.f): bordered system with -1e-4
        const int n1 = nd + 1;
        for (int e = tid; e < n1 * n1; e += 32) {
            const int i = e % n1, j = e / n1;
            aug[e] = (i == 0 && j == 0) ? 0.0
                     : (i == 0 || j == 0) ? -1.0e-4
                                          : Bm[(i - 1) + (j - 1) * DIIS_MAXDIM];
        }
        if (tid < n1) rhs[tid] = (tid == 0) ? -1.0e-4 : 0.0;
        __syncwarp();
        warp_dgefa(aug, n1, n1, ipvt);
        warp_dgesl(aug, n1, n1, ipvt, rhs);
        if (tid < nd) coef[tid] = rhs[tid + 1];
    }
    __syncthreads();
    for (int k = tid; k < len; k += DT) {
        double v = 0.0;
        for (int i = 0; i < nd; i++) v += coef[i] * b.err[(size_t)i * len + k];
        vec[k] = v;
    }
    __syncthreads();
    double res = block_amax(vec, len, sh, shi);
    for (int k = tid; k < len; k += DT) {
        double v = vec[k];
        for (int i = 0; i < nd; i++) v += coef[i] * b.amp[(size_t)i * len + k];
        vec[k] = v;
        b.prev[k] = v;
    }
    if (tid == 0) {
        s.res = res;
        s.ndimr = (nd + 1 < maxdim) ? nd + 1 : maxdim;
        s.idimr = s.idimr + 1;
        if (s.idimr > maxdim) s.idimr = 1;
    }
}

// the general eigen-solve of the Davidson step on one given matrix
// (row-major, n <= DAV_MAXD), for verification against LAPACK
__global__ void __launch_bounds__(32) k_geev_probe(const double *A, int n, double *wr, double *wi, double *V,
                                                    int *sweeps) {
    __shared__ double H[DAV_MAXD * GL], Z[DAV_MAXD * GL], X[DAV_MAXD * GL], r[DAV_MAXD], im[DAV_MAXD];
    for (int e = threadIdx.x; e < n * n; e += 32) H[(e / n) * GL + e % n] = A[e];
    __syncwarp();
    const int sw = warp_geev(H, Z, X, Z, r, im, n);
    if (threadIdx.x < n) {
        wr[threadIdx.x] = r[threadIdx.x];
        wi[threadIdx.x] = im[threadIdx.x];
    }
    for (int e = threadIdx.x; e < n * n; e += 32) V[e] = Z[(e / n) * DAV_MAXD + e % n];
    if (threadIdx.x == 0) *sweeps = sw;
}

}  // namespace

int geev_probe(const double *A_dev, int n, double *wr, double *wi, double *V, int *sweeps) {
    if (n < 1 || n > DAV_MAXD) return set_error(CPSD_EARG, "geev: n must be 1..32");
    k_geev_probe<<<1, 32, 0, stream()>>>(A_dev, n, wr, wi, V, sweeps);
    count_launch();
    return cuda_check(cudaGetLastError(), "k_geev_probe");
}

int dav_init_launch(DavState *st, const DavBuffers &b) {
    k_dav_init<<<1, DT, 0, stream()>>>(st, b);
    count_launch();
    return cuda_check(cudaGetLastError(), "k_dav_init");
}
int dav_step_launch(DavState *st, const DavBuffers &b) {
    cudaEvent_t end;
    CPSD_TRY(timing_begin(0.0, 0, 0, 0, 30, &end));
    k_dav_step<<<1, DT, 0, stream()>>>(st, b);
    count_launch();
    CPSD_TRY(cuda_check(cudaGetLastError(), "k_dav_step"));
    return timing_end(end);
}
int dav_abar_launch(DavState *st, const DavBuffers &b) {
    cudaEvent_t end;
    CPSD_TRY(timing_begin(0.0, 0, 0, 0, 31, &end));
    k_dav_abar<<<1, DT, 0, stream()>>>(st, b);
    count_launch();
    CPSD_TRY(cuda_check(cudaGetLastError(), "k_dav_abar"));
    return timing_end(end);
}
int dav_final_launch(DavState *st, const DavBuffers &b) {
    // AR of the final roots was written to b.AB[0] by the caller
    k_dav_final<<<1, DT, 0, stream()>>>(st, b, b.AB[0]);
    count_launch();
    return cuda_check(cudaGetLastError(), "k_dav_final");
}
int solver_step_launch(const SolverArgs &a) {
    if (a.nb <= 0) return CPSD_OK;
    cudaEvent_t end;
    CPSD_TRY(timing_begin(0.0, a.nb, 0, 0, 32, &end));
    k_solver_step<<<a.nb, DT, 0, stream()>>>(a);
    count_launch();
    CPSD_TRY(cuda_check(cudaGetLastError(), "k_solver_step"));
    return timing_end(end);
}

}  // namespace cpsd
