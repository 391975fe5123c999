// Sliced-integer contraction on the 5th-generation tensor cores (sm_100a).
//
// A FP64 contraction C += alpha * A B is evaluated as an exact integer sum:
// every row of A (column of B) is scaled by a power of two 2^e so that its
// largest element is below 1 in magnitude, and each scaled value y is cut
// into S signed 7-bit digits q_t = trunc(128^(t+1) y - ...), so that
// a = 2^e sum_t q_t 128^-(t+1) up to 2^e 128^-S (Ozaki, Ogita, Oishi & Rump,
// "Error-free transformations of matrix multiplication by using fast
// routines of matrix multiplication", 2012; the integer form of Ootomo,
// Ozaki & Yokota 2024).  The digit products q_t(A) q_u(B) with t + u <= S - 1
// are summed exactly in int32 by tcgen05.mma kind::i8, one TMEM accumulator
// per diagonal d = t + u, and the epilogue combines the diagonals in FP64:
// C += alpha 2^(e_a + e_b) sum_d acc_d 128^-(d+2).  The truncation error is
// below (S + 1) K 128^-S max|a_row| max|b_col| per element.
//
// Operands are first gathered from their DPD layout into the digit tiles
// (k_oz_slice): per 128 (A) or BN (B) rows and 64 contracted indices, S
// canonical K-major tiles (8 x 16-byte core matrices, no swizzle) stored
// contiguously, so one bulk copy (cp.async.bulk) moves a whole pipeline
// stage.  One CTA computes one 128 x BN output tile (k_oz_gemm): a producer
// warp streams the stages through an mbarrier ring, one thread issues the
// MMAs, four warps read the accumulators back (tcgen05.ld) and scatter the
// FP64 result through the output offset tables.  Every wait is bounded: on
// a timeout the kernel records it in an error word and drains.
#include <atomic>
#include <cstdint>

#include "ozaki.cuh"

namespace cpsd {

namespace {

constexpr int OZ_BK = 64;             // contracted indices per stage (bytes of a digit row)
constexpr int OZ_THREADS = 192;       // 4 epilogue warps, 1 producer warp, 1 MMA warp
constexpr uint32_t OZ_SPIN = 1u << 20;  // poll limit of every mbarrier wait
constexpr int OZ_EXPO_NONE = (int)0x80808080;  // byte-filled "no element yet" (all-zero row)

// scale exponent of a row / column; an all-zero one has zero digits, any
// exponent does
__device__ __forceinline__ int oz_expo(int e) { return e == OZ_EXPO_NONE ? 0 : e; }

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// bounded wait for the phase with the given parity; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t i = 0; i < OZ_SPIN; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// K-major canonical layout without swizzle: core matrices of 8 rows x 16
// bytes (128 contiguous bytes), LBO = next core matrix along K, SBO = next
// group of 8 rows
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    return d;                // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor of kind::i8: s8 x s8 -> s32, both K-major, M = 128
__host__ __device__ constexpr uint32_t umma_idesc_i8(int n) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

template <int S, int BN>
struct OzCfg {
    static constexpr int A_STAGE = S * 128 * OZ_BK;  // bytes of the A digit tiles of one stage
    static constexpr int B_STAGE = S * BN * OZ_BK;
    static constexpr int STAGE = A_STAGE + B_STAGE;
    // stages in the ring: as many as fit in 220 KB (at most 4); the CTA's
    // dynamic shared memory is NST stages + 1 KB of alignment slack, within
    // the 227 KB a CTA may have
    static constexpr int NST = (220 * 1024) / STAGE >= 4 ? 4 : (220 * 1024) / STAGE;
    static constexpr int SMEM = NST * STAGE + 1024;
    static constexpr int NCOL_RAW = S * BN;
    static constexpr int NCOL = NCOL_RAW <= 32 ? 32 : NCOL_RAW <= 64 ? 64 : NCOL_RAW <= 128 ? 128 : NCOL_RAW <= 256 ? 256 : 512;
    static_assert(NST >= 2, "at least two pipeline stages");
    static_assert(SMEM <= 227 * 1024, "dynamic shared memory above the per-CTA limit");
    static_assert(NCOL_RAW <= 512, "accumulators exceed TMEM");
    static_assert(BN % 16 == 0 && BN <= 256 && 256 / BN >= 1, "MMA N: multiples of 16 up to 256");
};

// One output tile per CTA: 128 rows (TMEM lanes) x BN columns, S diagonal
// accumulators side by side in TMEM columns.
template <int S, int BN>
__global__ void __launch_bounds__(OZ_THREADS, 1)
    k_oz_gemm(const OzTile *__restrict__ tiles, const OzGroup *__restrict__ groups, const int8_t *__restrict__ Adig,
              const int8_t *__restrict__ Bdig, const int *__restrict__ ea, const int *__restrict__ eb,
              const i64 *__restrict__ crow, const i64 *__restrict__ ccol, const int *__restrict__ mcombo,
              const int *__restrict__ ncombo, double *__restrict__ C, double alpha, int kt0, int kt1,
              int *__restrict__ err) {
    using Cf = OzCfg<S, BN>;
    extern __shared__ __align__(1024) unsigned char oz_smem[];
    unsigned char *stages = (unsigned char *)(((uintptr_t)oz_smem + 1023) & ~(uintptr_t)1023);
    __shared__ __align__(8) uint64_t full[Cf::NST], empty[Cf::NST], done;
    __shared__ uint32_t tmem_base_sh;
    __shared__ int fail_sh;  // some wait of this CTA timed out
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const OzTile tl = tiles[blockIdx.x];
    const OzGroup g = groups[tl.g];
    const int KT = g.KT;
    const int kb = kt0, ke = kt1 < KT ? kt1 : KT;
    const int nk = ke > kb ? ke - kb : 0;  // groups with fewer K stages add nothing in later chunks

    if (warp == 5) {  // TMEM columns for the S accumulators
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"(Cf::NCOL)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < Cf::NST; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&done, 1);
        fail_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_sh;
    bool ok = true;
    int issued = 0;  // producer: stages whose bulk copies it started

    if (warp == 4) {
        if (lane == 0) {  // producer
            const int8_t *Ab = Adig + g.aoff + (size_t)tl.mt * KT * Cf::A_STAGE;
            const int8_t *Bb = Bdig + g.boff + (size_t)tl.nt * KT * Cf::B_STAGE;
            for (int i = 0; i < nk; i++, issued++) {
                const int s = i % Cf::NST, u = i / Cf::NST;
                if (u > 0 && !mbar_wait(&empty[s], (u - 1) & 1)) {
                    ok = false;
                    break;
                }
                unsigned char *sa = stages + (size_t)s * Cf::STAGE;
                mbar_expect_tx(&full[s], Cf::STAGE);
                bulk_g2s(sa, Ab + (size_t)(kb + i) * Cf::A_STAGE, Cf::A_STAGE, &full[s]);
                bulk_g2s(sa + Cf::A_STAGE, Bb + (size_t)(kb + i) * Cf::B_STAGE, Cf::B_STAGE, &full[s]);
            }
        }
    } else if (warp == 5) {
        if (lane == 0) {  // MMA issuer
            // The products A_t B_v (t + v < S) go to accumulator d = t + v at
            // TMEM columns d*BN.  For one t the B digit tiles v = v0..v0+nv-1
            // lie back to back in shared memory (one canonical tile of nv*BN
            // rows) and their accumulators back to back in TMEM, so one MMA
            // of N = nv*BN (at most 256) does them all: A_t is read from
            // shared memory once per MMA instead of once per digit pair.
            // Every accumulator is first written by t = 0 at the first stage
            // (no accumulation there), later MMAs accumulate.
            constexpr int VPER = 256 / BN;
            for (int i = 0; i < nk; i++) {
                const int s = i % Cf::NST, u = i / Cf::NST;
                if (!mbar_wait(&full[s], u & 1)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t sa = smem_u32(stages + (size_t)s * Cf::STAGE), sb = sa + Cf::A_STAGE;
#pragma unroll
                for (int kk = 0; kk < OZ_BK / 32; kk++)
#pragma unroll
                    for (int t = 0; t < S; t++)
#pragma unroll
                        for (int v0 = 0; v0 < S - t; v0 += VPER) {
                            const int nv = S - t - v0 < VPER ? S - t - v0 : VPER;
                            const uint64_t ad = umma_desc(sa + t * 128 * OZ_BK + kk * 256, 128, 8 * OZ_BK);
                            const uint64_t bd = umma_desc(sb + v0 * BN * OZ_BK + kk * 256, 128, 8 * OZ_BK);
                            const uint32_t acc = (i > 0 || kk > 0 || t > 0) ? 1u : 0u;
                            umma_i8(tmem + (uint32_t)((t + v0) * BN), ad, bd, umma_idesc_i8(nv * BN), acc);
                        }
                umma_commit(&empty[s]);  // frees the stage once these MMAs are done
            }
            umma_commit(&done);
        }
    } else {  // epilogue: warp w reads TMEM lanes 32w..32w+31 = tile rows
        // one lane waits so that the warp stays converged for tcgen05.ld
        int fin_l = 0;
        if (lane == 0) fin_l = mbar_wait(&done, 0) ? 1 : 0;
        const bool fin = __shfl_sync(0xffffffffu, fin_l, 0) != 0;
        tc_fence_after();
        const int r = warp * 32 + lane;
        const i64 m = (i64)tl.mt * 128 + r;
        const bool rowok = fin && m < g.M;
        const int mc = rowok ? mcombo[g.moff + m] : 0;
        const int e_a = rowok ? oz_expo(ea[g.eaoff + m]) : 0;
        const i64 *crow_m = crow + g.crowoff + (rowok ? m : 0) * g.nL;
        for (int c0 = 0; c0 < BN; c0 += 16) {
            double acc[16];
#pragma unroll
            for (int j = 0; j < 16; j++) acc[j] = 0.0;
            double w = 1.0 / 16384.0;  // 128^-(d+2), d = 0
#pragma unroll
            for (int d = 0; d < S; d++) {
                int32_t v[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(d * BN + c0), v);
#pragma unroll
                for (int j = 0; j < 16; j++) acc[j] += (double)v[j] * w;
                w *= 1.0 / 128.0;
            }
            if (!rowok || nk == 0) continue;
            // 8 columns at a time: all their index loads, then all their C
            // loads, then the stores, so that the latencies of a group
            // overlap instead of chaining output after output (every output
            // address is written once, and C never aliases the tables)
            const i64 nbase = (i64)tl.nt * BN + c0;
#pragma unroll
            for (int h = 0; h < 16; h += 8) {
                const int nj = (int)min((i64)8, g.N - (nbase + h));
                if (nj <= 0) break;
                int nc[8], ex[8];
#pragma unroll
                for (int j = 0; j < 8; j++)
                    if (j < nj) {
                        nc[j] = ncombo[g.noff + nbase + h + j];
                        ex[j] = eb[g.eboff + nbase + h + j];
                    }
                i64 addr[8];
#pragma unroll
                for (int j = 0; j < 8; j++)
                    if (j < nj) addr[j] = crow_m[nc[j]] + ccol[g.ccoloff + (nbase + h + j) * g.nI + mc];
                double cv[8];
#pragma unroll
                for (int j = 0; j < 8; j++)
                    if (j < nj) cv[j] = C[addr[j]];
#pragma unroll
                for (int j = 0; j < 8; j++)
                    if (j < nj) C[addr[j]] = cv[j] + alpha * ldexp(acc[h + j], e_a + oz_expo(ex[j]));
            }
        }
        if (!fin) ok = false;
    }
    if (!ok) {
        atomicExch(err, 1);
        atomicOr(&fail_sh, 1);
    }
    __syncthreads();
    if (fail_sh) {
        // drain before TMEM is freed and the CTA's shared memory is given
        // back: the producer waits out its bulk copies still in flight (only
        // the last NST stages can be: every earlier stage was consumed
        // before its slot was refilled), the MMA issuer waits for the
        // completion of every MMA it issued (its final commit); both waits
        // are bounded like the others
        if (warp == 4 && lane == 0)
            for (int i = issued > Cf::NST ? issued - Cf::NST : 0; i < issued; i++)
                mbar_wait(&full[i % Cf::NST], (i / Cf::NST) & 1);
        if (warp == 5 && lane == 0) mbar_wait(&done, 0);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 5) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cf::NCOL) : "memory");
    }
}

// Digit tiles of one operand side, in two fully parallel passes over the
// slicing jobs (one row tile of one group each).  Element (r, k) of a group
// lives at src[roff[r * nJ + kcombo[k]] + koff[k * nI + rcombo[r]]] (row r
// of irrep combination rcombo[r], contracted index k of combination
// kcombo[k]); on an affine job and stage (OzSliceJob) the address is a base
// plus row and column steps, with no table read per element.  Thread t of a
// block always handles row t mod RT of its tile, 16 contracted indices (one
// 16-byte row of a core matrix) at a time; a warp covers 32 consecutive
// rows, so for a fixed index its loads are one contiguous run when the rows
// are.
constexpr int OZ_EXPO_CHUNK = 16;  // most K stages per block of the exponent pass

// gather of one K stage of a job: base and column step when the stage is
// affine for the job
struct OzStageAddr {
    bool fast;
    i64 base, sk;
};
__device__ __forceinline__ OzStageAddr oz_stage_addr(const OzSliceJob &jb, const OzStage *__restrict__ stage,
                                                     const i64 *__restrict__ roff, int kt, i64 r0) {
    OzStageAddr a{false, 0, 0};
    if (jb.affine) {
        const OzStage st = stage[jb.soff + (i64)kt * jb.nI + jb.rc];
        if (st.ok) {
            a.fast = true;
            a.base = roff[jb.roff + r0 * jb.nJ + st.j] + st.ko0;
            a.sk = st.sk;
        }
    }
    return a;
}

// elements kst + kk .. kst + kk + 15 of one row (zero beyond K; kst = first
// index of the stage), all loads in flight
__device__ __forceinline__ void oz_load16(double (&x)[16], const OzSliceJob &jb, const OzStageAddr &sa,
                                          const double *__restrict__ src, const i64 *__restrict__ roff,
                                          const i64 *__restrict__ koff, const int *__restrict__ rcombo,
                                          const int *__restrict__ kcombo, i64 row, i64 r0, i64 kst, int kk) {
    const i64 k0 = kst + kk;
    if (sa.fast) {
        const double *p = src + (sa.base + (row - r0) * jb.sr + (i64)kk * sa.sk);
        if (k0 + 16 <= jb.K) {
#pragma unroll
            for (int q = 0; q < 16; q++) x[q] = __ldg(p + (i64)q * sa.sk);
        } else {
#pragma unroll
            for (int q = 0; q < 16; q++) x[q] = k0 + q < jb.K ? __ldg(p + (i64)q * sa.sk) : 0.0;
        }
        return;
    }
    const int rc = rcombo[jb.rcoff + row];
    const i64 *ro = roff + jb.roff + row * jb.nJ;
    i64 addr[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const i64 k = k0 + q;
        addr[q] = k < jb.K ? ro[kcombo[jb.kcoff + k]] + koff[jb.koff + k * jb.nI + rc] : -1;
    }
#pragma unroll
    for (int q = 0; q < 16; q++) x[q] = addr[q] >= 0 ? __ldg(src + addr[q]) : 0.0;
}

// pass 1: exponent e of every row maximum (|x| < 2^e) over `chunk` stages
// (grid.y), merged with atomicMax into expo, which holds OZ_EXPO_NONE on
// entry.  Each thread keeps the running maximum of its row in a register.
template <int RT>
__global__ void __launch_bounds__(256) k_oz_expo(const OzSliceJob *__restrict__ jobs,
                                                 const OzStage *__restrict__ stage, const double *__restrict__ src,
                                                 const i64 *__restrict__ roff, const i64 *__restrict__ koff,
                                                 const int *__restrict__ rcombo, const int *__restrict__ kcombo,
                                                 int chunk, int *__restrict__ expo) {
    const OzSliceJob jb = jobs[blockIdx.x];
    const int kt0 = blockIdx.y * chunk;
    if (kt0 >= jb.KT) return;
    const int kt1 = min(jb.KT, kt0 + chunk);
    constexpr int PER = 256 / RT;              // threads per row
    constexpr int NU = (OZ_BK / 16) / PER;     // 16-index units of a thread per stage
    __shared__ int rmax[RT];
    const int tid = threadIdx.x, r = tid % RT;
    for (int i = tid; i < RT; i += 256) rmax[i] = OZ_EXPO_NONE;
    __syncthreads();
    const i64 r0 = (i64)jb.rt * RT, row = r0 + r;
    double amax = 0.0;
    if (row < jb.R)
        for (int kt = kt0; kt < kt1; kt++) {
            const OzStageAddr sa = oz_stage_addr(jb, stage, roff, kt, r0);
            double x[NU][16];
#pragma unroll
            for (int u = 0; u < NU; u++)
                oz_load16(x[u], jb, sa, src, roff, koff, rcombo, kcombo, row, r0, (i64)kt * OZ_BK,
                          (tid / RT + u * PER) * 16);
#pragma unroll
            for (int u = 0; u < NU; u++)
#pragma unroll
                for (int q = 0; q < 16; q++) amax = fmax(amax, fabs(x[u][q]));
        }
    if (amax != 0.0) {
        int ex;
        frexp(amax, &ex);
        atomicMax(&rmax[r], ex);
    }
    __syncthreads();
    for (int i = tid; i < RT; i += 256)
        if (r0 + i < jb.R && rmax[i] != OZ_EXPO_NONE) atomicMax(&expo[jb.eoff + r0 + i], rmax[i]);
}

// pass 2: the S digit tiles of stage blockIdx.y, written as 16-byte rows of
// the core matrices; rows and columns beyond the group's extents get zero
// digits
template <int S, int RT>
__global__ void __launch_bounds__(256) k_oz_slice(const OzSliceJob *__restrict__ jobs,
                                                  const OzStage *__restrict__ stage, const double *__restrict__ src,
                                                  const i64 *__restrict__ roff, const i64 *__restrict__ koff,
                                                  const int *__restrict__ rcombo, const int *__restrict__ kcombo,
                                                  int8_t *__restrict__ dig, const int *__restrict__ expo) {
    const OzSliceJob jb = jobs[blockIdx.x];
    const int kt = blockIdx.y;
    if (kt >= jb.KT) return;
    constexpr int PER = 256 / RT, NU = (OZ_BK / 16) / PER;
    const int tid = threadIdx.x, r = tid % RT;
    const i64 r0 = (i64)jb.rt * RT, row = r0 + r;
    int8_t *tile = dig + jb.doff + ((size_t)jb.rt * jb.KT + kt) * (size_t)(S * RT * OZ_BK);
    uint32_t w[NU][S][4];
#pragma unroll
    for (int u = 0; u < NU; u++)
#pragma unroll
        for (int t = 0; t < S; t++) w[u][t][0] = w[u][t][1] = w[u][t][2] = w[u][t][3] = 0u;
    if (row < jb.R) {
        const OzStageAddr sa = oz_stage_addr(jb, stage, roff, kt, r0);
        double x[NU][16];
#pragma unroll
        for (int u = 0; u < NU; u++)
            oz_load16(x[u], jb, sa, src, roff, koff, rcombo, kcombo, row, r0, (i64)kt * OZ_BK,
                      (tid / RT + u * PER) * 16);
        // 2^-e in two finite factors: a row whose largest element is below
        // 2^-1022 has e < -1021 and 2^-e alone would overflow
        const int e = oz_expo(expo[jb.eoff + row]);
        const double sc1 = ldexp(1.0, -(e / 2)), sc2 = ldexp(1.0, -(e - e / 2));
#pragma unroll
        for (int u = 0; u < NU; u++)
#pragma unroll
            for (int q = 0; q < 16; q++) {
                double y = x[u][q] * sc1 * sc2;
#pragma unroll
                for (int t = 0; t < S; t++) {
                    y *= 128.0;
                    const double qd = trunc(y);
                    y -= qd;
                    w[u][t][q >> 2] |= ((uint32_t)(uint8_t)(int8_t)(int)qd) << (8 * (q & 3));
                }
            }
    }
#pragma unroll
    for (int u = 0; u < NU; u++) {
        const int k16 = tid / RT + u * PER;
        const size_t off = (size_t)(r >> 3) * (8 * OZ_BK) + (size_t)k16 * 128 + (size_t)(r & 7) * 16;
#pragma unroll
        for (int t = 0; t < S; t++)
            *reinterpret_cast<uint4 *>(tile + (size_t)t * RT * OZ_BK + off) =
                make_uint4(w[u][t][0], w[u][t][1], w[u][t][2], w[u][t][3]);
    }
}

template <int S, int BN>
int oz_gemm_launch(const OzDevPlan &p, const int8_t *Adig, const int8_t *Bdig, const int *ea, const int *eb,
                   double *C, double alpha, int kt0, int kt1, int *err) {
    using Cf = OzCfg<S, BN>;
    static std::atomic<bool> attr{false};
    if (!attr) {
        CPSD_TRY(cuda_check(cudaFuncSetAttribute(k_oz_gemm<S, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cf::SMEM),
                            "oz smem attr"));
        attr = true;
    }
    k_oz_gemm<S, BN><<<p.ntiles, OZ_THREADS, Cf::SMEM, stream()>>>(p.tiles, p.groups, Adig, Bdig, ea, eb, p.crow,
                                                                   p.ccol, p.mcombo, p.ncombo, C, alpha, kt0, kt1,
                                                                   err);
    count_launch();
    return cuda_check(cudaGetLastError(), "k_oz_gemm");
}

template <int S, int RT>
int oz_slice_launch(const OzSideDev &sd, const double *src, int8_t *dig, int *expo) {
    if (sd.njobs == 0) return CPSD_OK;
    CPSD_TRY(cuda_check(cudaMemsetAsync(expo, 0x80, sizeof(int) * (size_t)sd.nexpo, stream()), "clear exponents"));
    // stages per exponent block: up to OZ_EXPO_CHUNK, fewer while the grid
    // would not give every SM four blocks
    static const int sms = [] {
        int d = 0, n = 148;
        if (cudaGetDevice(&d) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d) != cudaSuccess)
            n = 148;
        return n;
    }();
    int chunk = OZ_EXPO_CHUNK;
    while (chunk > 1 && (i64)sd.njobs * ((sd.kt_max + chunk - 1) / chunk) < 4 * (i64)sms) chunk /= 2;
    const dim3 ge(sd.njobs, (sd.kt_max + chunk - 1) / chunk), gd(sd.njobs, sd.kt_max);
    k_oz_expo<RT><<<ge, 256, 0, stream()>>>(sd.jobs, sd.stage, src, sd.roff, sd.koff, sd.rcombo, sd.kcombo, chunk,
                                            expo);
    k_oz_slice<S, RT><<<gd, 256, 0, stream()>>>(sd.jobs, sd.stage, src, sd.roff, sd.koff, sd.rcombo, sd.kcombo, dig,
                                                expo);
    count_launch(2);
    return cuda_check(cudaGetLastError(), "k_oz_slice");
}

}  // namespace

int oz_slice(int S, int rows_per_tile, const OzSideDev &sd, const double *src, int8_t *dig, int *expo) {
#define OZ_SL(s)                                                                    \
    case s:                                                                         \
        return rows_per_tile == 128 ? oz_slice_launch<s, 128>(sd, src, dig, expo)  \
                                    : oz_slice_launch<s, 64>(sd, src, dig, expo);
    switch (S) {
        OZ_SL(3)
        OZ_SL(4)
        OZ_SL(5)
        OZ_SL(6)
        OZ_SL(7)
    default:
        return set_error(CPSD_EARG, "digit count must be 3..7");
    }
#undef OZ_SL
}

int oz_gemm(int S, const OzDevPlan &p, const int8_t *Adig, const int8_t *Bdig, const int *ea, const int *eb,
            double *C, double alpha, int kt0, int kt1, int *err) {
    switch (S) {
    case 3:
        return oz_gemm_launch<3, 128>(p, Adig, Bdig, ea, eb, C, alpha, kt0, kt1, err);
    case 4:
        return oz_gemm_launch<4, 128>(p, Adig, Bdig, ea, eb, C, alpha, kt0, kt1, err);
    case 5:
        return oz_gemm_launch<5, 64>(p, Adig, Bdig, ea, eb, C, alpha, kt0, kt1, err);
    case 6:
        return oz_gemm_launch<6, 64>(p, Adig, Bdig, ea, eb, C, alpha, kt0, kt1, err);
    case 7:
        return oz_gemm_launch<7, 64>(p, Adig, Bdig, ea, eb, C, alpha, kt0, kt1, err);
    default:
        return set_error(CPSD_EARG, "digit count must be 3..7");
    }
}

int oz_tile_n(int S) { return S <= 4 ? 128 : 64; }

}  // namespace cpsd
