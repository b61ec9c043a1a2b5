// Split-precision fused precession + coil contraction on sm_100a tensor cores.
//
// Math (one precession segment = a run of consecutive precession blocks):
//   phase in turns   theta(s,j) = theta0(s) + w(s) kappa_16(j) + sum_k b_k(s) kappa_k(j),  k = 0..15
//     b_0..15  : the 16 solid-harmonic basis values of spin s (FP64, resident)
//     w        : dw/(2 pi) (0 when dw is off),  kappa_16 = -t_j
//     theta0   : arg(m0)/(2 pi)
//     kappa_k  : -gamma * trapezoid integral of field column k from the segment
//                start to ADC sample j (FP64 prefix table)
//   M(s,j)   = |m0| 2^(t_j * r2(s)) * cis(2 pi theta)   (r2 = -log2(e)/T2)
//   S(j,c)   = sum_s M(s,j) csm(s,c)                      (no conjugation)
// This is the reference's phi = -2 pi gamma cumtrapz(dt, Bz) and
// Mxy = M0 exp(i phi - t/T2) (src/simulation/Bloch/BlochHighOrderSimulatitonMethod.jl:76-92)
// with the cumulative integral factored into per-spin x per-sample terms.
//
// Precision.  theta(s,j) is a small FP64 GEMM (samples x 16) * (16 x spins)
// on FP64 tensor-core MMAs (mma.sync m8n8k4.f64), its accumulator initialised
// with theta0 + w kappa_16.  One FP64 add of 1.5*2^20 leaves frac(theta) as a
// 32-bit fixed-point turn count in the low mantissa word: the mod-2pi range
// reduction, exact to 2^-32 turn.  cos/sin of 2 pi frac(theta) in [-pi, pi)
// and the decay come from the SFU (sin/cos/ex2.approx).  M and the
// sensitivities are split into FP16 hi + lo pairs after exact power-of-two
// scaling (per coil, and per segment for the amplitude), and the coil
// contraction runs as two kind::f16 tcgen05 MMAs per 16-deep K-step, each with
// N = 2 x columns: A_lo x [B_hi | B_lo] first, then A_hi x [B_hi | B_lo], so
// one accumulator generation (per 32-spin chunk) holds A.B_hi and A.B_lo side
// by side.  The drain adds the two halves in FP32 into a TMEM row accumulator
// and every WINDOW chunks promotes it into FP64 split-K partials; the final
// sum undoes the scaling exactly.
//
// Kernel organisation (one CTA per SM, persistent, slab-major work items of
// (time tile of 128 samples) x (range of 32-spin chunks)):
//   warps 0-7   phase: warp w computes the turn fractions of the 16 tile rows
//               32(w%4) + 16(w/4) .. +15 for each chunk (DMMA) and writes them
//               to TMEM in the m8n8 fragment layout (tcgen05.st.16x256b).
//   warps 8-15  magnetisation: the same 16 rows for warp w-8; read the turn
//               fractions, form M, split it into FP16 hi/lo and write the A
//               operand to TMEM; drain the accumulator.
//   warp 16     MMA issuer: tcgen05.mma.kind::f16, A in TMEM, B (the
//               sensitivities, pre-split) in shared memory; tcgen05.commit
//               releases shared-memory stages, A buffers and accumulators.
//   warp 17     loader: cp.async.bulk of each chunk's B operand and spin table.
// TMEM (512 columns for N <= 64 output columns): accumulators 2 x 2N, A
// operands 2 x 64, turn fractions 2 x 32, FP32 row accumulator N.
// Every wait is bounded: on time-out the kernel records the place in a device
// error word and returns without hanging the GPU.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_fp16.h>

#include "homs_common.cuh"
#include "homs_split.cuh"

namespace homs {

namespace split {

constexpr int TM = 128;          // samples per tile (UMMA M)
constexpr int KC = 32;           // spins per chunk
constexpr int KSTEPS = 4;        // (2*KC real K values) / 16 per f16 MMA
constexpr int MAX_STAGE = 6;     // shared-memory stages of B operand + spin table
constexpr int NTERM = 16;        // phase GEMM depth (DMMA K): the 16 basis terms
constexpr int PREFIX_STRIDE = 24;  // doubles per prefix row: kappa_0..kappa_16, t at PREFIX_T
constexpr int PREFIX_T = 20;
constexpr int GROUP_COILS = 32;  // coils per kernel pass (N <= 64 output columns)
// Warp roles: 8 phase warps and 8 magnetisation warps (2 of each per TMEM
// lane quarter, paired by the 16 rows they share), MMA issuer, loader.
constexpr int NPHASE_WARPS = 8;
constexpr int NMAG_WARPS = 8;
constexpr int MMA_WARP = 16;
constexpr int LOAD_WARP = 17;
constexpr int THREADS = 576;
constexpr uint32_t TMEM_COLS = 512;
constexpr long long WAIT_BUDGET = 4000000000LL;  // cycles (~2 s)
// FLUSH chunks (8 MMAs each) form one FP32 TMEM accumulator generation: the
// tensor core's accumulator add is not round-to-nearest, and its error is
// systematic and grows with |D| and with the number of MMAs per generation
// (two chunks per generation raised the signal NRMSE from 4.6e-7 to 5.2e-7 on
// the 3D workload for a 1% gain, so each chunk keeps its own).
// The drain adds generations (round to nearest, FP32) in a TMEM row
// accumulator and promotes it to the FP64 partials every WINDOW chunks.
constexpr int FLUSH = 1;
constexpr int WINDOW = 32;  // a multiple of FLUSH

// TMEM column map for N output columns (N <= 64).
__host__ __device__ constexpr uint32_t d_col(int n, int buf) { return (uint32_t)(buf * 2 * n); }
__host__ __device__ constexpr uint32_t a_col(int n, int buf) { return (uint32_t)(4 * n + buf * 64); }
__host__ __device__ constexpr uint32_t t_col(int n, int tb) { return (uint32_t)(4 * n + 128 + tb * 32); }
__host__ __device__ constexpr uint32_t acc_col(int n) { return (uint32_t)(4 * n + 192); }

// B operand of one chunk: KSTEPS slabs of 2N rows ([B_hi | B_lo]) x 16 f16,
// no-swizzle K-major (core matrices of 8 rows x 16 bytes).
__host__ __device__ constexpr int b_bytes(int n) { return KSTEPS * 2 * n * 32; }

// Spin table of a chunk, in doubles: basis term k (0..15) of local spin s at
// ((k/4)*KC + s)*4 + k%4, so that one DMMA B fragment (k = 4ks + tq, spin
// base + gq) is 32 consecutive doubles; then theta0 = arg(m0)/(2 pi) and
// dw/(2 pi) per spin, and one packed float2 (-log2(e)/T2, log2|m0|) per spin.
__host__ __device__ inline int tab_index(int k, int s) { return (((k >> 2) * KC + s) << 2) + (k & 3); }
constexpr int TAB_THETA0 = NTERM * KC;
constexpr int TAB_DW = TAB_THETA0 + KC;
constexpr int TAB_PACK = TAB_DW + KC;
constexpr int SPIN_BYTES = (TAB_PACK + KC) * 8;

// Smallest e with 2^e >= x for a non-negative double given by its bits (0 for 0).
__host__ __device__ inline int pow2_ceil_exp(unsigned long long bits) {
    if (bits == 0) return 0;
    int e = (int)((bits >> 52) & 0x7FF) - 1023;
    if (bits & 0xFFFFFFFFFFFFFull) e += 1;
    return e;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_budget(uint64_t *bar, uint32_t parity, long long budget) {
    if (mbar_try(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try(bar, parity)) {
        if (clock64() - t0 > budget) return false;
    }
    return true;
}
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    return mbar_wait_budget(bar, parity, WAIT_BUDGET);
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_mma_f16(uint32_t d, uint32_t a, uint64_t bdesc, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d),
        "r"(a), "l"(bdesc), "r"(idesc), "r"(accum)
        : "memory");
}
// FP64 tensor-core MMA, 8x8x4: c += a * b in the m8n8k4 fragment layouts
// (a: row groupID, col threadID_in_group; b: row threadID_in_group, col
// groupID; c: row groupID, cols 2*threadID_in_group + {0,1}).
__device__ __forceinline__ void dmma_8x8x4(double &c0, double &c1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
        : "+d"(c0), "+d"(c1)
        : "d"(a), "d"(b));
}
__device__ __forceinline__ float ex2_approx(float x) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float sin_approx(float x) {
    float r;
    asm("sin.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float cos_approx(float x) {
    float r;
    asm("cos.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// 16 TMEM lanes x 8r columns (r = 2 or 4 repetitions): thread t writes lanes
// t/4 (v[4i], v[4i+1]) and t/4+8 (v[4i+2], v[4i+3]), columns 8i + 2*(t%4) + {0,1}.
__device__ __forceinline__ void tmem_st_16x256b_x2(uint32_t taddr, const uint32_t *v) {
    asm volatile("tcgen05.st.sync.aligned.16x256b.x2.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
                 : "memory");
}
__device__ __forceinline__ void tmem_st_16x256b_x4(uint32_t taddr, const uint32_t *v) {
    asm volatile(
        "tcgen05.st.sync.aligned.16x256b.x4.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16};" ::"r"(taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
        "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
        : "memory");
}
__device__ __forceinline__ void tmem_ld_16x256b_x4(uint32_t taddr, uint32_t *v) {
    asm volatile(
        "tcgen05.ld.sync.aligned.16x256b.x4.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr)
        : "memory");
}
// 32 TMEM lanes (thread <-> lane) x 8 or 16 consecutive columns.
__device__ __forceinline__ void tmem_ld_32x32b_x8(uint32_t taddr, float *v) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr)
                 : "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld_32x32b_x16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_st_32x32b_x8(uint32_t taddr, const float *v) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7])
                 : "memory");
}
__device__ __forceinline__ void tmem_st_32x32b_x16(uint32_t taddr, const float *v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16};" ::"r"(taddr),
        "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]), "f"(v[8]), "f"(v[9]),
        "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15])
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// No-swizzle K-major shared-memory matrix descriptor: core matrices of
// 8 rows x 16 bytes, K-direction core stride (LBO) 128 B, row-group stride
// (SBO) 256 B, descriptor version 1.
__device__ __forceinline__ uint64_t bdesc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(256 >> 4) << 32) |
           (1ull << 46);
}

// Work items of one launch.  The (tile x chunk) grid is cut into `slabs`
// ranges of chunks; item i is slab z = i / tiles of tile i % tiles, and CTA b
// takes items b, b + G, b + 2G, ...  The CTAs running at any one time thus
// read the chunks of two or three consecutive slabs, which stay in L2 for
// every tile that needs them.  Item (tile, z) owns partial slot z.
struct KernelArgs {
    const double *prefix;      // [rows][PREFIX_STRIDE]
    const uint8_t *b_operand;  // [nchunks][b_bytes]
    const double *spin_table;  // [nchunks][SPIN_BYTES / 8]
    const unsigned long long *amp_max;  // bits of max |m0| over the segment's spins
    double *partial;           // [tiles][slabs][TM][N], FP64 split-K partials
    unsigned int *err;
    int64_t nsamples;
    int n_chunks;
    int tiles;
    int slabs;
    int nstage;  // shared-memory stages of B operand + spin table
};

struct Item {
    int tile, z, c0, c1;
};
__device__ __forceinline__ Item item_of(const KernelArgs &a, int i) {
    Item it;
    it.z = i / a.tiles;
    it.tile = i - it.z * a.tiles;
    it.c0 = (int)((int64_t)a.n_chunks * it.z / a.slabs);
    it.c1 = (int)((int64_t)a.n_chunks * (it.z + 1) / a.slabs);
    return it;
}

// The phase accumulator starts at TURN_BIAS + theta0 + w kappa_16: with
// |theta| < 2^18, every partial sum stays in [2^20, 2^21), where the FP64
// spacing is 2^-32, so the low mantissa word of the result is frac(theta)
// * 2^32 (the mod-2pi range reduction) and each DMMA add rounds at 2^-33 turn.
constexpr double TURN_BIAS = 1572864.0;  // 1.5 * 2^20
__device__ __forceinline__ uint32_t turn_fraction(double biased_th) { return (uint32_t)__double2loint(biased_th); }

// A operand words of one spin-sample: M = 2^(tj r2 + l2) cis(2 pi u / 2^32),
// split into FP16 hi + lo, each packed as (re low half, im high half).
__device__ __forceinline__ void magnetisation(uint32_t u, float tj, float r2, float l2, uint32_t &hi, uint32_t &lo) {
    const float x = (float)(int32_t)u * 1.4629180792671596e-09f;  // 2 pi / 2^32, x in [-pi, pi)
    const float a = ex2_approx(fmaf(tj, r2, l2));
    const float mre = a * cos_approx(x), mim = a * sin_approx(x);
    const __half2 h = __floats2half2_rn(mre, mim);
    const float2 hf = __half22float2(h);
    const __half2 l = __floats2half2_rn(mre - hf.x, mim - hf.y);
    hi = *reinterpret_cast<const uint32_t *>(&h);
    lo = *reinterpret_cast<const uint32_t *>(&l);
}

template <int N>
__global__ void __launch_bounds__(THREADS, 1) split_precession_kernel(KernelArgs args) {
    constexpr int BB = b_bytes(N);
    constexpr int HALF = N / 2;  // accumulator columns drained per magnetisation thread
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    const int NSTAGE = args.nstage;
    uint8_t *sB = smem;                                             // NSTAGE * BB
    double *sSpin = reinterpret_cast<double *>(sB + NSTAGE * BB);  // NSTAGE * SPIN_BYTES
    uint64_t *bars = reinterpret_cast<uint64_t *>(reinterpret_cast<uint8_t *>(sSpin) + NSTAGE * SPIN_BYTES);
    uint64_t *full = bars;                    // [NSTAGE] loader -> consumers (tx)
    uint64_t *empty = bars + MAX_STAGE;       // [NSTAGE] MMA commit -> loader
    uint64_t *a_full = bars + 2 * MAX_STAGE;  // [2] magnetisation warps -> MMA
    uint64_t *a_empty = a_full + 2;           // [2] MMA commit -> magnetisation warps
    uint64_t *d_full = a_empty + 2;           // [2] MMA commit -> drain
    uint64_t *d_empty = d_full + 2;           // [2] drain -> MMA
    uint64_t *t_full = d_empty + 2;           // [8 row groups][2] phase warp -> magnetisation warp
    uint64_t *t_empty = t_full + 16;          // [8 row groups][2] magnetisation warp -> phase warp
    uint64_t *done = t_empty + 16;            // [1] final MMA commit
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int i = 0; i < NSTAGE; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&a_full[i], NMAG_WARPS);  // one elected arrive per magnetisation warp
            mbar_init(&a_empty[i], 1);
            mbar_init(&d_full[i], 1);
            mbar_init(&d_empty[i], NMAG_WARPS);
        }
        for (int i = 0; i < 16; ++i) {
            mbar_init(&t_full[i], 1);
            mbar_init(&t_empty[i], 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == MMA_WARP) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    const int n_items = args.tiles * args.slabs;
    const int G = (int)gridDim.x;
    const int gq = lane >> 2, tq = lane & 3;
    bool dead = false;

    if (warp == LOAD_WARP) {
        if (lane == 0) {
            int stage = 0;
            uint32_t eph = 1;  // parity of empty[stage] that frees it (the first pass is free)
            for (int i = blockIdx.x; i < n_items && !dead; i += G) {
                const Item it = item_of(args, i);
                for (int c = it.c0; c < it.c1; ++c) {
                    if (!mbar_wait(&empty[stage], eph)) {
                        atomicOr(args.err, 1u);
                        dead = true;
                        break;
                    }
                    mbar_expect_tx(&full[stage], (uint32_t)(BB + SPIN_BYTES));
                    bulk_g2s(sB + (size_t)stage * BB, args.b_operand + (size_t)c * BB, (uint32_t)BB, &full[stage]);
                    bulk_g2s(reinterpret_cast<uint8_t *>(sSpin) + (size_t)stage * SPIN_BYTES,
                             reinterpret_cast<const uint8_t *>(args.spin_table) + (size_t)c * SPIN_BYTES,
                             (uint32_t)SPIN_BYTES, &full[stage]);
                    if (++stage == NSTAGE) {
                        stage = 0;
                        eph ^= 1u;
                    }
                }
            }
        }
        __syncwarp();
    } else if (warp == MMA_WARP) {
        if (lane == 0) {
            // kind::f16: D f32 (bit 4), A and B f16 (format 0), both K-major; N = 2N columns.
            constexpr uint32_t idesc = (1u << 4) | ((uint32_t)((2 * N) >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
            int g = 0;    // chunks issued; chunk g uses A buffer g % 2
            int gen = 0;  // accumulator generations issued; generation gen uses accumulator gen % 2
            int stage = 0;
            uint32_t fph = 0;  // parity of full[stage] for chunk g
            for (int i = blockIdx.x; i < n_items && !dead; i += G) {
                const Item it = item_of(args, i);
                for (int c = it.c0; c < it.c1; ++c, ++g) {
                    const int buf = g & 1, dbuf = gen & 1;
                    const int ci = c - it.c0;
                    const bool gen_first = (ci % FLUSH) == 0;
                    const bool gen_last = (ci % FLUSH) == FLUSH - 1 || c + 1 == it.c1;
                    if (gen_first && !mbar_wait(&d_empty[dbuf], (uint32_t)(((gen >> 1) + 1) & 1))) {
                        atomicOr(args.err, 2u);
                        dead = true;
                        break;
                    }
                    if (!mbar_wait(&full[stage], fph) || !mbar_wait(&a_full[buf], (uint32_t)((g >> 1) & 1))) {
                        atomicOr(args.err, 4u);
                        dead = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t dcol = tmem + d_col(N, dbuf);
                    const uint32_t acol = tmem + a_col(N, buf);
                    const uint32_t sbase = smem_u32(sB + (size_t)stage * BB);
                    // The small lo pass goes first, while D is small, then the hi pass.
#pragma unroll
                    for (int ks = 0; ks < KSTEPS; ++ks)
                        tc_mma_f16(dcol, acol + 32u + (uint32_t)ks * 8u, bdesc(sbase + (uint32_t)(ks * 2 * N * 32)),
                                   idesc, (gen_first && ks == 0) ? 0u : 1u);
#pragma unroll
                    for (int ks = 0; ks < KSTEPS; ++ks)
                        tc_mma_f16(dcol, acol + (uint32_t)ks * 8u, bdesc(sbase + (uint32_t)(ks * 2 * N * 32)), idesc,
                                   1u);
                    tc_commit(&empty[stage]);
                    tc_commit(&a_empty[buf]);
                    if (gen_last) {
                        tc_commit(&d_full[dbuf]);
                        ++gen;
                    }
                    if (++stage == NSTAGE) {
                        stage = 0;
                        fph ^= 1u;
                    }
                }
            }
            // Drain: wait for every issued MMA before TMEM is released.
            tc_commit(done);
            if (!mbar_wait(done, 0)) atomicOr(args.err, 8u);
        }
        __syncwarp();
    } else if (warp < NPHASE_WARPS) {
        // Phase warp w: turn fractions of tile rows 32q + 16p .. +15 (q = w % 4,
        // p = w / 4): 2 x 4 DMMA 8x8 tiles per chunk, K = 16, accumulators
        // initialised with TURN_BIAS + theta0 + w kappa_16; written to TMEM
        // columns t_col(tb) + spin of those rows.
        const int q = warp & 3, p = warp >> 2;
        const int grp = q * 2 + p;  // row group shared with magnetisation warp 8 + warp
        const uint32_t t_lane = (uint32_t)(q * 32 + p * 16) << 16;
        int stage = 0, tb = 0;
        uint32_t fph = 0, tk = 0;  // parities of full[stage] and of this use of turn buffer tb
        for (int i = blockIdx.x; i < n_items && !dead; i += G) {
            const Item it = item_of(args, i);
            // A fragments: kappa[row 32q + 16p + 8mt + gq][k = 4ks + tq], and kappa_16 of the row.
            double ka[2][4], k16[2];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                int64_t j = (int64_t)it.tile * TM + q * 32 + p * 16 + mt * 8 + gq;
                if (j >= args.nsamples) j = args.nsamples - 1;
                const double *pr = args.prefix + (size_t)j * PREFIX_STRIDE;
#pragma unroll
                for (int ks = 0; ks < 4; ++ks) ka[mt][ks] = pr[4 * ks + tq];
                k16[mt] = pr[16];
            }
            for (int c = it.c0; c < it.c1; ++c) {
                bool ok = mbar_wait(&full[stage], fph);
                ok = ok && mbar_wait(&t_empty[grp * 2 + tb], tk ^ 1u);
                __syncwarp();
                if (!__all_sync(0xffffffffu, ok)) {
                    if (lane == 0) atomicOr(args.err, 128u);
                    dead = true;
                    break;
                }
                tc_fence_after();
                const double *tab = sSpin + (size_t)stage * (SPIN_BYTES / 8);
                const uint32_t tcol = tmem + t_col(N, tb) + t_lane;
                // Two spin groups at a time: 4 independent accumulator chains,
                // k-step outermost.
#pragma unroll
                for (int np = 0; np < 2; ++np) {
                    double bf[2][4], th[2][2][2];
#pragma unroll
                    for (int n2 = 0; n2 < 2; ++n2) {
                        const int nt = 2 * np + n2;
#pragma unroll
                        for (int ks = 0; ks < 4; ++ks) bf[n2][ks] = tab[tab_index(4 * ks + tq, 8 * nt + gq)];
                        const double2 t0 = *reinterpret_cast<const double2 *>(tab + TAB_THETA0 + 8 * nt + 2 * tq);
                        const double2 dw = *reinterpret_cast<const double2 *>(tab + TAB_DW + 8 * nt + 2 * tq);
                        const double b0 = t0.x + TURN_BIAS, b1 = t0.y + TURN_BIAS;
#pragma unroll
                        for (int mt = 0; mt < 2; ++mt) {
                            th[n2][mt][0] = fma(dw.x, k16[mt], b0);
                            th[n2][mt][1] = fma(dw.y, k16[mt], b1);
                        }
                    }
#pragma unroll
                    for (int ks = 0; ks < 4; ++ks)
#pragma unroll
                        for (int n2 = 0; n2 < 2; ++n2)
#pragma unroll
                            for (int mt = 0; mt < 2; ++mt)
                                dmma_8x8x4(th[n2][mt][0], th[n2][mt][1], ka[mt][ks], bf[n2][ks]);
                    // Spin groups 2np, 2np+1: 16x256b.x2 register order [4 n2 + 2 mt + i].
                    uint32_t v[8];
#pragma unroll
                    for (int n2 = 0; n2 < 2; ++n2)
#pragma unroll
                        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                            for (int ii = 0; ii < 2; ++ii) v[4 * n2 + 2 * mt + ii] = turn_fraction(th[n2][mt][ii]);
                    tmem_st_16x256b_x2(tcol + (uint32_t)(16 * np), v);
                }
                tmem_wait_st();
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&t_full[grp * 2 + tb]);
                if (++stage == NSTAGE) {
                    stage = 0;
                    fph ^= 1u;
                }
                if (++tb == 2) {
                    tb = 0;
                    tk ^= 1u;
                }
            }
        }
    } else {
        // Magnetisation warp w: TMEM lane quarter q = w % 4, half h: tile rows
        // 32q + 16h .. +15 (the rows of phase warp w - 8) and all 32 spins of
        // each chunk.  For the accumulator drain it takes thread <-> tile row
        // 32q + lane and output columns [h N/2, (h+1) N/2).
        const int q = warp & 3, h = (warp - NPHASE_WARPS) >> 2;
        const int grp = q * 2 + h;
        const uint32_t q_lane = (uint32_t)(q * 32) << 16;
        const uint32_t m_lane = (uint32_t)(q * 32 + h * 16) << 16;
        const int row = q * 32 + lane;
        // Amplitude scale of the segment: M is formed as M / 2^eA (|M| <= 1).
        const float l2off = (float)pow2_ceil_exp(*args.amp_max);
        int g = 0;    // chunks produced by this CTA
        int gen = 0;  // accumulator generations completed
        int stage = 0, tb = 0;
        uint32_t tk = 0;
        int pend = -1;  // accumulator generation waiting to be drained
        double *pend_dst = nullptr;
        bool pend_wfirst = false, pend_promote = false, pend_pfirst = false;
        // Drain: add the generation's two halves (A.B_hi, A.B_lo) into the
        // FP32 row accumulator in TMEM; every WINDOW chunks, and at the end of
        // an item, add the accumulator into the FP64 split-K partial instead.
        auto drain = [&]() -> bool {
            const int buf = pend & 1;
            const bool ok = mbar_wait(&d_full[buf], (uint32_t)((pend >> 1) & 1));
            __syncwarp();
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) atomicOr(args.err, 32u);
                return false;
            }
            tc_fence_after();
            const uint32_t dsrc = tmem + q_lane + d_col(N, buf) + (uint32_t)(h * HALF);
            const uint32_t asrc = tmem + q_lane + acc_col(N) + (uint32_t)(h * HALF);
#pragma unroll
            for (int cb = 0; cb < HALF; cb += 16) {
                constexpr int W0 = HALF >= 16 ? 16 : 8;
                const int w = (HALF - cb) >= 16 ? 16 : 8;
                (void)W0;
                float d1[16], d2[16], ac[16];
                if (w == 16) {
                    tmem_ld_32x32b_x16(dsrc + (uint32_t)cb, d1);
                    tmem_ld_32x32b_x16(dsrc + (uint32_t)(N + cb), d2);
                    if (!pend_wfirst) tmem_ld_32x32b_x16(asrc + (uint32_t)cb, ac);
                } else {
                    tmem_ld_32x32b_x8(dsrc + (uint32_t)cb, d1);
                    tmem_ld_32x32b_x8(dsrc + (uint32_t)(N + cb), d2);
                    if (!pend_wfirst) tmem_ld_32x32b_x8(asrc + (uint32_t)cb, ac);
                }
                tmem_wait_ld();
                if (cb + 16 >= HALF) {
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&d_empty[buf]);
                }
#pragma unroll
                for (int e = 0; e < 16; ++e)
                    if (e < w) d1[e] = pend_wfirst ? d1[e] + d2[e] : (d1[e] + d2[e]) + ac[e];
                if (pend_promote) {
                    double *d = pend_dst + cb;
#pragma unroll
                    for (int e = 0; e < 16; e += 2) {
                        if (e < w) {
                            double2 o = pend_pfirst ? make_double2(0.0, 0.0) : *reinterpret_cast<double2 *>(d + e);
                            o.x += (double)d1[e];
                            o.y += (double)d1[e + 1];
                            *reinterpret_cast<double2 *>(d + e) = o;
                        }
                    }
                } else if (w == 16) {
                    tmem_st_32x32b_x16(asrc + (uint32_t)cb, d1);
                } else {
                    tmem_st_32x32b_x8(asrc + (uint32_t)cb, d1);
                }
            }
            pend = -1;
            return true;
        };
        for (int i = blockIdx.x; i < n_items && !dead; i += G) {
            const Item it = item_of(args, i);
            double *dst_piece =
                args.partial + (((size_t)it.tile * args.slabs + it.z) * TM + row) * (size_t)N + h * HALF;
            float tj[2];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                int64_t j = (int64_t)it.tile * TM + q * 32 + h * 16 + mt * 8 + gq;
                if (j >= args.nsamples) j = args.nsamples - 1;
                tj[mt] = (float)args.prefix[(size_t)j * PREFIX_STRIDE + PREFIX_T];
            }
            for (int c = it.c0; c < it.c1; ++c) {
                const int buf = g & 1;
                bool ok = mbar_wait(&t_full[grp * 2 + tb], tk);
                ok = ok && mbar_wait(&a_empty[buf], (uint32_t)(((g >> 1) + 1) & 1));
                __syncwarp();
                if (!__all_sync(0xffffffffu, ok)) {
                    if (lane == 0) atomicOr(args.err, 16u);
                    dead = true;
                    break;
                }
                tc_fence_after();
                // Turn fractions of rows 16h + 8mt + gq, spins 8nt + 2tq + i:
                // 16x256b.x4 register order [4 nt + 2 mt + i].
                uint32_t tu[16];
                tmem_ld_16x256b_x4(tmem + t_col(N, tb) + m_lane, tu);
                tmem_wait_ld();
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&t_empty[grp * 2 + tb]);
                const double *tab = sSpin + (size_t)stage * (SPIN_BYTES / 8);
                const uint32_t acol = tmem + a_col(N, buf) + m_lane;
#pragma unroll
                for (int np = 0; np < 2; ++np) {
                    // Spin groups 2np, 2np+1: 16x256b.x2 register order [4 n2 + 2 mt + i].
                    uint32_t hi[8], lo[8];
#pragma unroll
                    for (int n2 = 0; n2 < 2; ++n2) {
                        // This thread's spins of group nt: 8nt + 2tq + i.
                        const int nt = 2 * np + n2;
                        const float4 rl = *reinterpret_cast<const float4 *>(tab + TAB_PACK + 8 * nt + 2 * tq);
                        const float r2v[2] = {rl.x, rl.z};
                        const float l2v[2] = {rl.y - l2off, rl.w - l2off};
#pragma unroll
                        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                            for (int ii = 0; ii < 2; ++ii) {
                                const int e = 4 * n2 + 2 * mt + ii;
                                magnetisation(tu[4 * nt + 2 * mt + ii], tj[mt], r2v[ii], l2v[ii], hi[e], lo[e]);
                            }
                    }
                    tmem_st_16x256b_x2(acol + (uint32_t)(16 * np), hi);
                    tmem_st_16x256b_x2(acol + 32u + (uint32_t)(16 * np), lo);
                }
                tmem_wait_st();
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&a_full[buf]);
                // The previous generation has had a whole chunk of time to
                // finish: drain it now.
                if (pend >= 0 && !drain()) {
                    dead = true;
                    break;
                }
                const int ci = c - it.c0;
                if ((ci % FLUSH) == FLUSH - 1 || c + 1 == it.c1) {
                    const int gstart = ci - ci % FLUSH;  // first chunk of this generation
                    pend = gen++;
                    pend_dst = dst_piece;
                    pend_wfirst = (gstart % WINDOW) == 0;
                    pend_promote = (ci % WINDOW) == WINDOW - 1 || c + 1 == it.c1;
                    pend_pfirst = gstart < WINDOW;
                }
                ++g;
                if (++stage == NSTAGE) stage = 0;
                if (++tb == 2) {
                    tb = 0;
                    tk ^= 1u;
                }
            }
            if (dead) break;
            if (pend >= 0 && !drain()) {
                dead = true;
                break;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == MMA_WARP) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// Sum the split-K partials of each (sample, column) in slab order (FP64),
// undo the power-of-two scaling of the operands and write complex samples:
// column n < ncg is Re S(j, coil0 + n), ncg <= n < 2 ncg is Im.
template <typename T>
__global__ void __launch_bounds__(256) split_finalize_kernel(const double *partial, int64_t nsamples, int32_t ncg,
                                                             int n_cols, int slabs, const int *coil_exp,
                                                             const unsigned long long *amp_max, cplx<T> *sig,
                                                             int64_t ldsig) {
    // A block sums FIN_ROWS rows x n_cols columns of one time tile over the
    // slabs (each slab's rows are contiguous: coalesced reads), in slab order,
    // then writes every coil's samples of those rows from shared memory.
    constexpr int FIN_ROWS = 32, PER = FIN_ROWS * 64 / 256;
    __shared__ double sacc[FIN_ROWS * 64];
    const int ea = pow2_ceil_exp(*amp_max);
    const int64_t tiles = (nsamples + TM - 1) / TM;
    const int64_t units = tiles * (TM / FIN_ROWS);
    const int elems = FIN_ROWS * n_cols;  // n_cols <= 64
    for (int64_t u = blockIdx.x; u < units; u += gridDim.x) {
        const int64_t tile = u / (TM / FIN_ROWS);
        const int r0 = (int)(u % (TM / FIN_ROWS)) * FIN_ROWS;
        double acc[PER];
#pragma unroll
        for (int k = 0; k < PER; ++k) acc[k] = 0.0;
        for (int z = 0; z < slabs; ++z) {
            const double *src = partial + (((size_t)tile * slabs + z) * TM + r0) * (size_t)n_cols;
#pragma unroll
            for (int k = 0; k < PER; ++k) {
                const int e = threadIdx.x + k * 256;
                if (e < elems) acc[k] += src[e];
            }
        }
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int e = threadIdx.x + k * 256;
            if (e < elems) sacc[e] = acc[k];
        }
        __syncthreads();
        for (int q = threadIdx.x; q < FIN_ROWS * ncg; q += blockDim.x) {
            const int c = q / FIN_ROWS, row = q % FIN_ROWS;
            const int64_t j = tile * TM + r0 + row;
            if (j < nsamples) {
                const int e = coil_exp[c] + ea;
                sig[j + (int64_t)c * ldsig] =
                    cplx<T>{T(ldexp(sacc[row * n_cols + c], e)), T(ldexp(sacc[row * n_cols + ncg + c], e))};
            }
        }
        __syncthreads();
    }
}

// Per-spin 16-term basis (FP64), CPU expression order
// (src/simulation/Bloch/BlochHighOrderSimulatitonMethod.jl:54-68).
__global__ void basis_kernel(const double *x, const double *y, const double *z, int64_t ns, double *basis) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < ns; s += (int64_t)gridDim.x * blockDim.x) {
        const double X = x[s], Y = y[s], Z = z[s];
        const double x2 = X * X, y2 = Y * Y, z2 = Z * Z;
        const double r2 = (x2 + y2) + z2;
        double *b = basis + s * 16;
        b[0] = 1.0;
        b[1] = X;
        b[2] = Y;
        b[3] = Z;
        b[4] = X * Y;
        b[5] = Z * Y;
        b[6] = 3.0 * z2 - r2;
        b[7] = X * Z;
        b[8] = x2 - y2;
        b[9] = (3.0 * Y) * x2 - (y2 * Y);
        b[10] = (X * Z) * Y;
        b[11] = (5.0 * z2 - r2) * Y;
        b[12] = 5.0 * (z2 * Z) - (3.0 * Z) * r2;
        b[13] = (5.0 * z2 - r2) * X;
        b[14] = x2 * Z - y2 * Z;
        b[15] = (x2 * X) - (3.0 * X) * y2;
    }
}


// Largest |Re| or |Im| of each coil's sensitivity (bits of a non-negative
// double, combined with an unsigned max).
// Per coil: the largest |Re| or |Im| of its sensitivities, as the bits of a
// non-negative double (which order like the values).  Each block reduces a
// range of whole spin rows in shared memory first (blockDim a multiple of nc
// when nc <= 256, so a thread always sees the same coil), then merges one
// value per coil into `mx`.
__global__ void coil_max_kernel(const cplx<double> *csm_rows, int64_t ns, int32_t nc, unsigned long long *mx) {
    extern __shared__ unsigned long long smax[];  // nc entries
    for (int c = threadIdx.x; c < nc; c += blockDim.x) smax[c] = 0ull;
    __syncthreads();
    const int64_t rows_per_block = (ns + gridDim.x - 1) / gridDim.x;
    const int64_t i0 = min(ns, rows_per_block * blockIdx.x) * nc, i1 = min(ns, rows_per_block * (blockIdx.x + 1)) * nc;
    if ((int)blockDim.x % nc == 0) {
        unsigned long long local = 0ull;
        for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
            const cplx<double> v = csm_rows[i];
            local = max(local, (unsigned long long)__double_as_longlong(fmax(fabs(v.re), fabs(v.im))));
        }
        atomicMax(&smax[threadIdx.x % nc], local);
    } else {
        for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
            const cplx<double> v = csm_rows[i];
            atomicMax(&smax[i % nc], (unsigned long long)__double_as_longlong(fmax(fabs(v.re), fabs(v.im))));
        }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < nc; c += blockDim.x)
        if (smax[c]) atomicMax(&mx[c], smax[c]);
}

__global__ void coil_exp_kernel(const unsigned long long *mx, int32_t nc, int *coil_exp) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x)
        coil_exp[c] = pow2_ceil_exp(mx[c]);
}

// Sensitivities -> FP16 hi/lo B operand, per coil group of GROUP_COILS coils,
// scaled by 2^-e(coil) so that every entry is at most 1 in magnitude.  Real
// K index k = 2 s + comp of local spin s:
//   B[n][k] = (n < ncg ? Re c(s,n) : Im c(s,n-ncg))   for comp = 0 (re of M),
//   B[n][k] = (n < ncg ? -Im c(s,n) : Re c(s,n-ncg))  for comp = 1 (im of M);
// rows 0..N-1 of each K-step slab hold the hi parts, rows N..2N-1 the lo parts.
__global__ void b_operand_kernel(const cplx<double> *csm_rows, int64_t ns, int32_t nc, int n_cols, int64_t nchunks,
                                 int ngroups, const int *coil_exp, __half *out) {
    // One thread per 16-byte core-matrix row: operand row nn (hi rows
    // 0..n_cols-1, lo rows n_cols..2 n_cols-1) of K-step ks, K-half kb (8
    // consecutive K = 4 spins x (re, im)).
    const int64_t total = (int64_t)ngroups * nchunks * KSTEPS * (2 * n_cols) * 2;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = i;
        const int kb = (int)(r & 1);
        r >>= 1;
        const int nn = (int)(r % (2 * n_cols));
        r /= 2 * n_cols;
        const int ks = (int)(r % KSTEPS);
        const int64_t gc = r / KSTEPS;  // group * nchunks + chunk
        const int grp = (int)(gc / nchunks);
        const int64_t chunk = gc % nchunks;
        const bool lopart = nn >= n_cols;
        const int n = lopart ? nn - n_cols : nn;
        const int coil0 = grp * GROUP_COILS;
        const int ncg = min(GROUP_COILS, nc - coil0);
        const bool live = n < 2 * ncg;
        const int coil = coil0 + (n < ncg ? n : n - ncg);
        const int e = live ? coil_exp[coil] : 0;
        __align__(16) __half row[8];
#pragma unroll
        for (int j = 0; j < 8; j += 2) {
            const int k = 16 * ks + 8 * kb + j;  // even: this spin's (re, im) pair is K = k, k + 1
            const int64_t sp = chunk * KC + (k >> 1);
            double v0 = 0.0, v1 = 0.0;
            if (live && sp < ns) {
                const cplx<double> cv = csm_rows[sp * nc + coil];
                // Column n < ncg holds Re S: (re, -im); column ncg + n holds Im S: (im, re).
                v0 = ldexp(n < ncg ? cv.re : cv.im, -e);
                v1 = ldexp(n < ncg ? -cv.im : cv.re, -e);
            }
            const __half h0 = __double2half(v0), h1 = __double2half(v1);
            row[j] = lopart ? __double2half(v0 - (double)__half2float(h0)) : h0;
            row[j + 1] = lopart ? __double2half(v1 - (double)__half2float(h1)) : h1;
        }
        uint8_t *base = reinterpret_cast<uint8_t *>(out) + (size_t)gc * b_bytes(n_cols) + (size_t)ks * 2 * n_cols * 32;
        const size_t off = (size_t)(nn / 8) * 256 + (size_t)kb * 128 + (size_t)(nn % 8) * 16;
        *reinterpret_cast<uint4 *>(base + off) = *reinterpret_cast<const uint4 *>(row);
    }
}

// Spin table of a segment, from the state at its start (layout of
// tab_index per chunk): the 16 basis terms, theta0 = arg(m0)/(2 pi), dw/(2 pi)
// (0 if dw is off in precession) and the packed float2 (-log2(e)/T2,
// log2|m0|).  Also records the largest |m0| (amplitude scale of the FP16
// operand) and checks the phase range: |theta| must stay below 2^18 turns for
// the fixed-point reduction (error bit 64 otherwise).
__global__ void spin_table_kernel(const double *basis, const double *dw, const double *T2, const cplx<double> *xy,
                                  int64_t ns, int64_t nchunks, uint32_t method, const double *colmax,
                                  unsigned int *err, unsigned long long *amp_max, double *table) {
    const int64_t total = nchunks * KC;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < total;
         s += (int64_t)gridDim.x * blockDim.x) {
        double *t = table + (s / KC) * (SPIN_BYTES / 8);
        const int sl = (int)(s % KC);
        double row[17];
        for (int k = 0; k < 17; ++k) row[k] = 0.0;
        double theta0 = 0.0;
        float2 rl = make_float2(0.0f, -INFINITY);
        unsigned long long amp = 0ull;
        if (s < ns) {
            for (int k = 0; k < 16; ++k) row[k] = basis[s * 16 + k];
            row[16] = (method & HOMS_DW_PRECESSION) ? dw[s] / (2.0 * 3.141592653589793) : 0.0;
            const cplx<double> m0 = xy[s];
            const double mag = hypot(m0.re, m0.im);
            theta0 = atan2(m0.im, m0.re) / (2.0 * 3.141592653589793);
            double bound = fabs(theta0);
            for (int k = 0; k < 17; ++k) bound += fabs(row[k]) * colmax[k];
            if (!(bound < 262144.0)) atomicOr(err, 64u);
            rl.x = (float)(-1.4426950408889634 / T2[s]);
            rl.y = mag > 0.0 ? (float)log2(mag) : -INFINITY;
            amp = (unsigned long long)__double_as_longlong(mag);
        }
        // One atomic per warp for the amplitude maximum (bits of non-negative doubles order like the values).
        const unsigned active = __activemask();
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long other = __shfl_xor_sync(active, amp, o);
            if ((active >> ((threadIdx.x & 31) ^ o)) & 1u) amp = max(amp, other);
        }
        if ((threadIdx.x & 31) == __ffs(active) - 1 && amp) atomicMax(amp_max, amp);
        for (int k = 0; k < NTERM; ++k) t[tab_index(k, sl)] = row[k];
        t[TAB_THETA0 + sl] = theta0;
        t[TAB_DW + sl] = row[16];
        *reinterpret_cast<float2 *>(&t[TAB_PACK + sl]) = rl;
    }
}

// Prefix table of one segment.  Blocks 0..16: column k, a deterministic
// chunked scan of the trapezoid sums (f(n)+f(n+1)) dt(n), written at every
// ADC node (row = sample index) and at the end node (row nsamples), plus the
// column's largest |value| at row nsamples+1.  Block 17: elapsed time t
// (entry PREFIX_T) and the constant columns 17 (= 1) and 18, 19 (= 0).
__global__ void prefix_kernel(const double *dt, const double *const *src, const uint8_t *adc, const int32_t *rank,
                              int64_t rank_base, int64_t n_lo, int64_t n_hi, int64_t nsamples, double gamma,
                              double *prefix) {
    __shared__ double part[256];
    const int col = blockIdx.x;
    const double *f = col < 17 ? src[col] : reinterpret_cast<const double *>(1);  // nullptr: zero; 1: constant one
    const bool one = f == reinterpret_cast<const double *>(1);
    const bool zero = f == nullptr;
    const double scale = col < 16 ? -gamma * 0.5 : (col == 16 ? -0.5 : 0.5);
    const int out_col = col < 17 ? col : PREFIX_T;
    const int64_t nint = n_hi - n_lo;
    const int64_t per = (nint + blockDim.x - 1) / blockDim.x;
    const int64_t i0 = min(nint, per * threadIdx.x), i1 = min(nint, i0 + per);
    double local = 0.0;
    for (int64_t i = i0; i < i1; ++i) {
        const int64_t n = n_lo + i;
        const double term = zero ? 0.0 : (one ? 2.0 : (f[n] + f[n + 1])) * dt[n];
        local += term;
    }
    part[threadIdx.x] = local;
    __syncthreads();
    if (threadIdx.x == 0) {
        double run = 0.0;
        for (int i = 0; i < (int)blockDim.x; ++i) {
            const double v = part[i];
            part[i] = run;
            run += v;
        }
    }
    __syncthreads();
    double cum = part[threadIdx.x];
    double peak = 0.0;
    for (int64_t i = i0; i < i1; ++i) {
        const int64_t n = n_lo + i;
        const double term = zero ? 0.0 : (one ? 2.0 : (f[n] + f[n + 1])) * dt[n];
        cum += term;
        peak = fmax(peak, fabs(scale * cum));
        if (adc[n + 1]) {
            double *pr = prefix + (size_t)(rank[n + 1] - rank_base) * PREFIX_STRIDE;
            pr[out_col] = scale * cum;
            if (col == 17) {
                pr[17] = 1.0;
                pr[18] = 0.0;
                pr[19] = 0.0;
            }
        }
        if (n + 1 == n_hi) {
            double *pr = prefix + (size_t)nsamples * PREFIX_STRIDE;
            pr[out_col] = scale * cum;
            if (col == 17) {
                pr[17] = 1.0;
                pr[18] = 0.0;
                pr[19] = 0.0;
            }
        }
    }
    if (nint == 0 && threadIdx.x == 0) {
        double *pr = prefix + (size_t)nsamples * PREFIX_STRIDE;
        pr[out_col] = 0.0;
        if (col == 17) {
            pr[17] = 1.0;
            pr[18] = 0.0;
            pr[19] = 0.0;
        }
    }
    // Largest |kappa| of the column (row nsamples+1) for the phase-range check.
    __syncthreads();
    part[threadIdx.x] = peak;
    __syncthreads();
    if (threadIdx.x == 0 && col < 17) {
        double mx = 0.0;
        for (int i = 0; i < (int)blockDim.x; ++i) mx = fmax(mx, part[i]);
        prefix[(size_t)(nsamples + 1) * PREFIX_STRIDE + col] = mx;
    }
}

// Final state of a segment in FP64: Mxy = |m0| e^{-T/T2} cis(2 pi theta_end),
// Mz = Mz e^{-T/T1} + rho (1 - e^{-T/T1}).
__global__ void state_update_kernel(const double *table, const double *endrow, const double *T1, const double *T2,
                                    const double *rho, int64_t ns, cplx<double> *xy, double *mz) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < ns; s += (int64_t)gridDim.x * blockDim.x) {
        const double *t = table + (s / KC) * (SPIN_BYTES / 8);
        const int sl = (int)(s % KC);
        double th = fma(t[TAB_DW + sl], endrow[16], t[TAB_THETA0 + sl]);
        for (int k = 0; k < NTERM; ++k) th = fma(t[tab_index(k, sl)], endrow[k], th);
        const double T = endrow[PREFIX_T];
        const cplx<double> m0 = xy[s];
        const double mag = hypot(m0.re, m0.im);
        const double f = th - rint(th);
        double sn, cs;
        sincospi(2.0 * f, &sn, &cs);
        const double e2 = exp(-T / T2[s]);
        xy[s] = cplx<double>{mag * e2 * cs, mag * e2 * sn};
        const double e1 = exp(-T / T1[s]);
        mz[s] = mz[s] * e1 + rho[s] * (1.0 - e1);
    }
}

inline int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32)); }


// Self-test of the bounded-wait path: one thread waits, with `budget`
// cycles, on an mbarrier that nothing arrives at; when the wait runs out it
// records code 256 in the error word and returns, as the split kernel's
// waits do.
__global__ void wait_selftest_kernel(unsigned int *err, long long budget) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        if (!mbar_wait_budget(&bar, 0u, budget)) atomicOr(err, 256u);
    }
}

}  // namespace split

using namespace split;

cudaError_t wait_selftest(unsigned int *err, long long budget_cycles, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(unsigned int), stream);
    if (e != cudaSuccess) return e;
    wait_selftest_kernel<<<1, 32, 0, stream>>>(err, budget_cycles);
    return cudaGetLastError();
}

SplitResident::~SplitResident() {
    for (void *p : {spin_table, prefix, tvec, partial, amp, err})
        if (p) cudaFree(p);
    if (!phantom_view)
        for (void *p : {basis, b_operand, coil_exp})
            if (p) cudaFree(p);
}

// Forget shared phantom operands (owned elsewhere) so that they are rebuilt.
static void split_detach(SplitResident &r) {
    if (!r.phantom_view) return;
    r.basis = r.b_operand = r.coil_exp = nullptr;
    r.basis_bytes = r.b_bytes = r.coil_exp_bytes = 0;
    r.phantom_view = false;
}

static cudaError_t grow(void *&p, size_t &have, size_t need) {
    if (need <= have && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    have = 0;
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(need, 256));
    if (e == cudaSuccess) have = std::max<size_t>(need, 256);
    return e;
}

cudaError_t split_prepare(SplitResident &r, int64_t ns, int32_t nc, const void *x, const void *y, const void *z,
                          const void *dw, const void *csm_rows, bool is_f64, cudaStream_t stream, std::string *err) {
    (void)dw;
    if (!is_f64) {
        *err =
            "split mode takes FP64 phantom and sequence arrays: FP32 positions alone carry phase errors above the "
            "split path's error budget";
        return cudaSuccess;
    }
    split_detach(r);
    const int ngroups = (nc + GROUP_COILS - 1) / GROUP_COILS;
    const int ncg_max = std::min<int32_t>(nc, GROUP_COILS);
    const int n_cols = std::max(16, ((2 * ncg_max + 15) / 16) * 16);
    r.ns = ns;
    r.nc = nc;
    r.n_mma = n_cols;
    r.ngroups = ngroups;
    const int64_t nchunks = (ns + KC - 1) / KC;
    r.ns_pad = nchunks * KC;
    cudaError_t e;
    if ((e = grow(r.basis, r.basis_bytes, sizeof(double) * 16 * (size_t)ns)) != cudaSuccess) return e;
    if ((e = grow(r.b_operand, r.b_bytes, (size_t)b_bytes(n_cols) * (size_t)nchunks * ngroups)) != cudaSuccess)
        return e;
    // Per-coil scale exponents, preceded by the per-coil maxima they come from.
    if ((e = grow(r.coil_exp, r.coil_exp_bytes, (sizeof(unsigned long long) + sizeof(int)) * (size_t)nc)) !=
        cudaSuccess)
        return e;
    if (!r.amp) {
        if ((e = cudaMalloc(&r.amp, sizeof(unsigned long long))) != cudaSuccess) return e;
    }
    if (!r.err) {
        if ((e = cudaMalloc(&r.err, sizeof(unsigned int))) != cudaSuccess) return e;
    }
    unsigned long long *cmax = reinterpret_cast<unsigned long long *>(r.coil_exp);
    int *cexp = reinterpret_cast<int *>(cmax + nc);
    basis_kernel<<<grid_for(ns), 256, 0, stream>>>((const double *)x, (const double *)y, (const double *)z, ns,
                                                   (double *)r.basis);
    if ((e = cudaMemsetAsync(cmax, 0, sizeof(unsigned long long) * (size_t)nc, stream)) != cudaSuccess) return e;
    {
        const int threads = nc <= 256 ? nc * (256 / nc) : 256;
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(ns, 148 * 8));
        const size_t smem = sizeof(unsigned long long) * (size_t)nc;
        if (smem > 48 * 1024) {
            *err = "split mode: more coils than the sensitivity-scale reduction supports (6144)";
            return cudaSuccess;
        }
        coil_max_kernel<<<blocks, threads, smem, stream>>>((const cplx<double> *)csm_rows, ns, nc, cmax);
    }
    coil_exp_kernel<<<1, 128, 0, stream>>>(cmax, nc, cexp);
    const int64_t total = (int64_t)ngroups * nchunks * KSTEPS * 2 * n_cols * 2;
    b_operand_kernel<<<grid_for(total), 256, 0, stream>>>((const cplx<double> *)csm_rows, ns, nc, n_cols, nchunks,
                                                          ngroups, cexp, (__half *)r.b_operand);
    return cudaGetLastError();
}

// Shared memory: 1 KB alignment slack, NSTAGE x (B operand + spin table), the barriers.
constexpr size_t SMEM_LIMIT = 227 * 1024;
constexpr size_t SMEM_FIXED = 1024 + 512;

static int kernel_stages(int n_cols) {
    const size_t per = (size_t)b_bytes(n_cols) + SPIN_BYTES;
    return (int)std::min<size_t>(MAX_STAGE, (SMEM_LIMIT - SMEM_FIXED) / per);
}

static size_t kernel_smem(int n_cols) {
    return SMEM_FIXED + (size_t)kernel_stages(n_cols) * (b_bytes(n_cols) + SPIN_BYTES);
}

// Number of chunk slabs per tile: the smallest that keeps the busiest CTA's
// work (items x (chunks per item + an allowance for the per-item start-up))
// within reach of the best split.
static int choose_slabs(int64_t tiles, int64_t nchunks, int64_t G) {
    int best = 1;
    double best_cost = 1e300;
    const int64_t zmax = std::min<int64_t>(nchunks, 4096);
    for (int64_t z = 1; z <= zmax; ++z) {
        const int64_t per_cta = (tiles * z + G - 1) / G;
        const double cost = (double)per_cta * (double)((nchunks + z - 1) / z + 2);
        if (cost < best_cost * 0.995) {
            best_cost = cost;
            best = (int)z;
        }
    }
    return best;
}

template <int N>
static cudaError_t launch_precession(const KernelArgs &ka, unsigned grid, size_t smem, cudaStream_t stream) {
    cudaError_t e = allow_max_dynamic_smem((const void *)split_precession_kernel<N>);
    if (e != cudaSuccess) return e;
    split_precession_kernel<N><<<grid, THREADS, smem, stream>>>(ka);
    return cudaGetLastError();
}

static cudaError_t launch_precession(int n_cols, const KernelArgs &ka, unsigned grid, size_t smem,
                                     cudaStream_t stream) {
    switch (n_cols) {
        case 16: return launch_precession<16>(ka, grid, smem, stream);
        case 32: return launch_precession<32>(ka, grid, smem, stream);
        case 48: return launch_precession<48>(ka, grid, smem, stream);
        case 64: return launch_precession<64>(ka, grid, smem, stream);
        default: return cudaErrorInvalidValue;
    }
}

// One precession segment.
static cudaError_t split_segment(SplitResident &r, const SplitRunArgs &a, int64_t n_lo, int64_t n_hi,
                                 int64_t sample0, int64_t nsamples, cudaStream_t stream, std::string *err) {
    cudaError_t e;
    const int64_t nchunks = r.ns_pad / KC;
    const int64_t tiles = (nsamples + TM - 1) / TM;
    if (!a.grank || !a.src_dev) {
        *err = "internal: split segment without its ADC rank and column tables";
        return cudaSuccess;
    }
    const uint32_t m = a.method;
    const size_t prefix_rows = (size_t)std::max<int64_t>(tiles * TM, nsamples + 2);
    if ((e = grow(r.prefix, r.prefix_bytes, prefix_rows * PREFIX_STRIDE * sizeof(double))) != cudaSuccess) return e;
    if ((e = grow(r.spin_table, r.spin_bytes, (size_t)nchunks * SPIN_BYTES)) != cudaSuccess) return e;
    // The segment's samples are the global ADC indices sample0 .. sample0 + nsamples - 1.
    prefix_kernel<<<18, 256, 0, stream>>>((const double *)a.dt, reinterpret_cast<const double *const *>(a.src_dev),
                                          (const uint8_t *)a.adc, a.grank, sample0, n_lo, n_hi, nsamples, a.gamma,
                                          (double *)r.prefix);
    if ((e = cudaMemsetAsync(r.amp, 0, sizeof(unsigned long long), stream)) != cudaSuccess) return e;
    spin_table_kernel<<<grid_for(r.ns_pad), 256, 0, stream>>>(
        (const double *)r.basis, (const double *)a.dw, (const double *)a.T2, (const cplx<double> *)a.xy, r.ns, nchunks,
        m, (const double *)r.prefix + (size_t)(nsamples + 1) * PREFIX_STRIDE, (unsigned int *)r.err,
        (unsigned long long *)r.amp, (double *)r.spin_table);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (nsamples > 0) {
        int dev = 0, nsm = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        const int slabs = choose_slabs(tiles, nchunks, nsm);
        const int64_t n_items = tiles * slabs;
        if (tiles > INT32_MAX / slabs || nchunks > INT32_MAX) {
            *err = "split mode: segment too large for one launch";
            return cudaSuccess;
        }
        const int64_t G = std::min<int64_t>(nsm, n_items);
        const size_t pbytes = sizeof(double) * (size_t)tiles * slabs * TM * r.n_mma;
        if ((e = grow(r.partial, r.partial_bytes, pbytes)) != cudaSuccess) return e;
        const size_t smem = kernel_smem(r.n_mma);
        const int *cexp = reinterpret_cast<const int *>(reinterpret_cast<const unsigned long long *>(r.coil_exp) + r.nc);
        KernelArgs ka;
        ka.prefix = (const double *)r.prefix;
        ka.spin_table = (const double *)r.spin_table;
        ka.amp_max = (const unsigned long long *)r.amp;
        ka.partial = (double *)r.partial;
        ka.err = (unsigned int *)r.err;
        ka.nsamples = nsamples;
        ka.n_chunks = (int)nchunks;
        ka.tiles = (int)tiles;
        ka.slabs = slabs;
        ka.nstage = kernel_stages(r.n_mma);
        const unsigned ev_flags = a.capture ? cudaEventRecordExternal : cudaEventRecordDefault;
        if (a.ev_start) cudaEventRecordWithFlags(a.ev_start, stream, ev_flags);
        // One pass per group of GROUP_COILS coils.
        for (int grp = 0; grp < r.ngroups; ++grp) {
            const int coil0 = grp * GROUP_COILS;
            const int ncg = std::min<int>(GROUP_COILS, r.nc - coil0);
            ka.b_operand = (const uint8_t *)r.b_operand + (size_t)grp * nchunks * b_bytes(r.n_mma);
            e = launch_precession(r.n_mma, ka, (unsigned)G, smem, stream);
            if (a.ev_stop && grp + 1 == r.ngroups) cudaEventRecordWithFlags(a.ev_stop, stream, ev_flags);
            if (a.launches) *a.launches += 2;
            if (e != cudaSuccess) return e;
            const int fin_blocks = (int)std::min<int64_t>(tiles * (TM / 32), 148 * 8);
            if (a.sizeof_T == 8)
                split_finalize_kernel<double><<<fin_blocks, 256, 0, stream>>>(
                    (const double *)r.partial, nsamples, ncg, r.n_mma, slabs, cexp + coil0,
                    (const unsigned long long *)r.amp, (cplx<double> *)a.sig + sample0 + (int64_t)coil0 * a.nadc,
                    a.nadc);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
    }
    if (a.launches) *a.launches += 3;
    state_update_kernel<<<grid_for(r.ns), 256, 0, stream>>>(
        (const double *)r.spin_table, (const double *)r.prefix + (size_t)nsamples * PREFIX_STRIDE, (const double *)a.T1,
        (const double *)a.T2, (const double *)a.rho, r.ns, (cplx<double> *)a.xy, (double *)a.mz);
    return cudaGetLastError();
}

cudaError_t split_attach(SplitResident &r, const SplitResident &src) {
    if (&r == &src) return cudaSuccess;
    if (!r.phantom_view) {
        for (void **p : {&r.basis, &r.b_operand, &r.coil_exp}) {
            if (*p) cudaFree(*p);
            *p = nullptr;
        }
    }
    r.basis = src.basis;
    r.b_operand = src.b_operand;
    r.coil_exp = src.coil_exp;
    r.basis_bytes = src.basis_bytes;
    r.b_bytes = src.b_bytes;
    r.coil_exp_bytes = src.coil_exp_bytes;
    r.ns = src.ns;
    r.ns_pad = src.ns_pad;
    r.nc = src.nc;
    r.n_mma = src.n_mma;
    r.ngroups = src.ngroups;
    r.phantom_view = true;
    cudaError_t e;
    if (!r.amp && (e = cudaMalloc(&r.amp, sizeof(unsigned long long))) != cudaSuccess) return e;
    if (!r.err && (e = cudaMalloc(&r.err, sizeof(unsigned int))) != cudaSuccess) return e;
    return cudaSuccess;
}

void split_column_sources(uint32_t m, const void *const h[16], const void *gx, const void *gy, const void *gz,
                          const void *out[17]) {
    out[0] = (m & HOMS_HO0) ? h[0] : nullptr;
    for (int k = 1; k <= 3; ++k) out[k] = (m & HOMS_HO1) ? h[k] : (k == 1 ? gx : k == 2 ? gy : gz);
    for (int k = 4; k <= 8; ++k) out[k] = (m & HOMS_HO2) ? h[k] : nullptr;
    for (int k = 9; k <= 15; ++k) out[k] = (m & HOMS_HO3) ? h[k] : nullptr;
    out[16] = (m & HOMS_DW_PRECESSION) ? reinterpret_cast<const void *>(1) : nullptr;
}

cudaError_t split_reset_error(SplitResident &r, cudaStream_t stream) {
    return cudaMemsetAsync(r.err, 0, sizeof(unsigned int), stream);
}

cudaError_t split_run_segment(SplitResident &r, const SplitRunArgs &a, int64_t n_lo, int64_t n_hi, int64_t sample0,
                              int64_t nsamples, cudaStream_t stream, std::string *err) {
    return split_segment(r, a, n_lo, n_hi, sample0, nsamples, stream, err);
}

cudaError_t split_check(SplitResident &r, cudaStream_t stream, std::string *err) {
    unsigned int h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, r.err, sizeof(h), cudaMemcpyDeviceToHost, stream);
    if (e != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
    if (h & 64u)
        *err = "split mode: the accumulated phase of a precession segment exceeds 2^18 turns";
    else if (h != 0)
        *err = "split kernel: a bounded device wait timed out (code " + std::to_string(h) + ")";
    return cudaSuccess;
}

}  // namespace homs
