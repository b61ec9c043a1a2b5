// Split-precision fused precession + coil contraction on sm_100a tensor cores.
//
// Math (one precession segment = a run of consecutive precession blocks):
//   phase in turns   theta(s,j) = sum_k b_k(s) * kappa_k(j),  k = 0..19
//     b_0..15  : the 16 solid-harmonic basis values of spin s (FP64, resident)
//     b_16     : dw/(2 pi)               kappa_16 = -t_j
//     b_17     : theta0 = arg(m0)/(2 pi) kappa_17 = 1
//     kappa_k  : -gamma * trapezoid integral of field column k from the segment
//                start to ADC sample j (FP64 prefix table, k < 16)
//   M(s,j)   = |m0| 2^(t_j * r2(s)) * cis(2 pi theta)   (r2 = -log2(e)/T2)
//   S(j,c)   = sum_s M(s,j) csm(s,c)                      (no conjugation)
// This is the reference's phi = -2 pi gamma cumtrapz(dt, Bz) and
// Mxy = M0 exp(i phi - t/T2) (src/simulation/Bloch/BlochHighOrderSimulatitonMethod.jl:76-92)
// with the cumulative integral factored into per-spin x per-sample terms.
//
// Precision: theta(s,j) is a small FP64 GEMM (samples x 20) * (20 x spins),
// computed with FP64 tensor-core MMAs (mma.sync m8n8k4.f64).  One FP64 add of
// 1.5*2^20 leaves frac(theta) as a 32-bit fixed-point turn count in the low
// mantissa word (the mod-2pi range reduction, exact to 2^-32 turn).  A
// quadrant select plus float32 polynomials (coefficients fitted by
// fit_sincos.py) give cos/sin; the decay is one ex2.approx.  M is split into
// TF32 hi + lo and the coil contraction runs as three TF32 tcgen05 MMAs per
// K-step (hi*lo and lo*hi first, hi*hi last) with FP32 accumulation in TMEM,
// one accumulator generation per 32-spin chunk, drained through an FP32
// shared-memory accumulator into FP64 split-K partials.
//
// Kernel organisation (one CTA per SM, persistent, stream-K over
// (time tile of 128 samples) x (chunk of 32 spins) units):
//   warps 0-15 producers: warp w owns TMEM lane quarter w%4 (32 sample rows)
//              and 8 spins (w/4) of each chunk; DMMA gives the phases in the
//              m8n8 accumulator layout, which tcgen05.st.16x256b writes to
//              TMEM rows unchanged (A operand).  The same warps drain the
//              TMEM accumulator (tcgen05.ld.32x32b, thread <-> sample row).
//   warp 16    MMA issuer: tcgen05.mma.kind::tf32 with A in TMEM, B (the
//              sensitivities, pre-split) in shared memory; tcgen05.commit
//              releases shared-memory stages, A stages and accumulators.
//   warp 17    loader: cp.async.bulk of each chunk's B operand and spin table.
// Every wait is bounded: on time-out the kernel records the place in a device
// error word and returns without hanging the GPU.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "homs_common.cuh"
#include "homs_split.cuh"

namespace homs {

namespace split {

constexpr int TM = 128;          // samples per tile (UMMA M)
constexpr int KC = 32;           // spins per chunk
constexpr int KSTEPS = 8;        // (2*KC real K values) / 8 per tf32 MMA
constexpr int MAX_STAGE = 4;     // shared-memory stages (fewer for wide N)
constexpr int NTERM = 20;        // phase GEMM depth: 16 basis + dw + theta0 + 2 zero
constexpr int SPIN_ROWS = 21;    // k-major spin table rows per chunk: b_0..b_19, packed (r2, log2|m0|)
constexpr int SPIN_PACK = 20;
constexpr int SPIN_BYTES = SPIN_ROWS * KC * 8;
constexpr int PREFIX_STRIDE = 24;  // doubles per prefix row: kappa_0..kappa_19, t, pad
constexpr int PREFIX_T = 20;
constexpr int NPROD_WARPS = 16;  // 4 per TMEM lane quarter
constexpr int MMA_WARP = 16;
constexpr int LOAD_WARP = 17;
constexpr int THREADS = 576;
constexpr uint32_t TMEM_COLS = 512;
constexpr uint32_t A_COL0 = 256;
constexpr long long WAIT_BUDGET = 4000000000LL;  // cycles (~2 s)
// Chunks accumulated in one FP32 TMEM generation before it is drained.  The
// tensor core's accumulator add is not round-to-nearest: its error is
// systematic and grows with |D| and with the number of MMAs per generation,
// so each 32-spin chunk gets its own generation.
constexpr int FLUSH = 1;
// Chunks summed (round to nearest, FP32) in shared memory before promotion to
// the FP64 partials, and the row padding of that accumulator (bank spread).
constexpr int WINDOW = 32;
constexpr int ACC_PAD = 4;

// Sine/cosine coefficients on [-pi/4, pi/4] (see fit_sincos.py).
constexpr float S1 = -0.16666650772094727f, S2 = 0.00833197869360447f, S3 = -0.00019495606829877943f;
constexpr float C1 = -0.5f, C2 = 0.04166662320494652f, C3 = -0.0013886763481423259f, C4 = 2.439039235468954e-05f;

__host__ __device__ inline int b_bytes(int n_mma) { return 2 * KSTEPS * n_mma * 32; }

// K order of a chunk's A/B operands: the producer warp for spins 8P..8P+7
// writes 16 columns 16P + j, where column j holds spin 8P + 2*((j%8)/2) +
// j/8 (re for even j, im for odd j) -- the column order of
// tcgen05.st.16x256b.x2 applied to the m8n8 accumulator fragments.
__host__ __device__ inline void k_to_spin(int k, int &s_local, int &imag) {
    const int P = k >> 4, r = k & 15;
    s_local = 8 * P + 2 * ((r & 7) >> 1) + (r >> 3);
    imag = r & 1;
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
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    if (mbar_try(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try(bar, parity)) {
        if (clock64() - t0 > WAIT_BUDGET) return false;
    }
    return true;
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
__device__ __forceinline__ void tc_mma_tf32(uint32_t d, uint32_t a, uint64_t bdesc, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d),
        "r"(a), "l"(bdesc), "r"(idesc), "r"(accum)
        : "memory");
}
// FP64 tensor-core MMA, 8x8x4: c += a * b in the m8n8k4 fragment layouts
// (a: row groupID, col threadID_in_group; b: row threadID_in_group, col
// groupID; c: row groupID, cols 2*threadID_in_group + {0,1}).
__device__ __forceinline__ void dmma_8x8x4(double &c0, double &c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}
// Round to TF32 (10 stored mantissa bits), nearest with ties away from zero:
// add half of the 13 dropped bits to the magnitude, then clear them.
__device__ __forceinline__ uint32_t tf32_rna(float x) { return (__float_as_uint(x) + 0x1000u) & 0xFFFFE000u; }
__device__ __forceinline__ float ex2_approx(float x) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// 16 TMEM lanes x 16 columns: thread t writes lanes t/4 and t/4+8, columns
// 2*(t%4)+{0,1} (v[0..3]) and 8+2*(t%4)+{0,1} (v[4..7]).
__device__ __forceinline__ void tmem_st_16x256b_x2(uint32_t taddr, const uint32_t *v) {
    asm volatile("tcgen05.st.sync.aligned.16x256b.x2.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
                 : "memory");
}
__device__ __forceinline__ void tmem_ld_x4(uint32_t taddr, float *v) {
    uint32_t r[4];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(taddr)
                 : "memory");
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = __uint_as_float(r[i]);
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

struct KernelArgs {
    const double *prefix;      // [rows][PREFIX_STRIDE]
    const uint8_t *b_operand;  // [nchunks][b_bytes]
    const double *spin_table;  // [nchunks][SPIN_ROWS][KC]
    double *partial;           // [tiles][maxp][TM][n_mma], FP64 split-K partials
    unsigned int *err;
    int64_t nsamples;
    int64_t n_chunks;
    int64_t tiles;
    int maxp;
    int n_mma;
    int nstage;
};

__device__ __forceinline__ int64_t cta_of(int64_t L, int64_t G, int64_t W) { return ((L + 1) * G - 1) / W; }

// M(s,j) for one spin given the FP64 turn count; returns (re, im).
__device__ __forceinline__ void magnetisation(double th, float tj, float r2, float l2m0, float &mre, float &mim) {
    const double g = th + 1572864.0;  // 1.5 * 2^20: frac(th) * 2^32 lands in the low word
    const uint32_t u = (uint32_t)__double2loint(g);
    const uint32_t v = u + 0x20000000u;
    const uint32_t q = v >> 30;
    const int32_t rr = (int32_t)(v & 0x3FFFFFFFu) - 0x20000000;
    const float x = (float)rr * 1.4629180792671596e-09f;  // 2 pi / 2^32
    const float x2 = x * x;
    const float sp = fmaf(x * x2, fmaf(x2, fmaf(x2, S3, S2), S1), x);
    const float cp = fmaf(x2, fmaf(x2, fmaf(x2, fmaf(x2, C4, C3), C2), C1), 1.0f);
    // cis(x + q*pi/2): swap for odd q, negate cos for q in {1,2}, sin for q in {2,3}.
    const bool swap = (q & 1u) != 0;
    const uint32_t cbits = __float_as_uint(swap ? sp : cp) ^ ((((q + 1u) >> 1) & 1u) << 31);
    const uint32_t sbits = __float_as_uint(swap ? cp : sp) ^ ((q >> 1) << 31);
    const float c = __uint_as_float(cbits), s = __uint_as_float(sbits);
    const float a = ex2_approx(fmaf(tj, r2, l2m0));
    mre = a * c;
    mim = a * s;
}

__global__ void __launch_bounds__(THREADS, 1) split_precession_kernel(KernelArgs args) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    const int n_mma = args.n_mma;
    const int NSTAGE = args.nstage;
    const int BB = b_bytes(n_mma);
    uint8_t *sB = smem;                                             // NSTAGE * BB
    double *sSpin = reinterpret_cast<double *>(sB + NSTAGE * BB);  // NSTAGE * SPIN_BYTES
    float *accf = reinterpret_cast<float *>(reinterpret_cast<uint8_t *>(sSpin) + NSTAGE * SPIN_BYTES);  // TM x (n_mma+pad)
    uint64_t *bars = reinterpret_cast<uint64_t *>(accf + (size_t)TM * (n_mma + ACC_PAD));
    uint64_t *full = bars;                    // [NSTAGE] loader -> consumers (tx)
    uint64_t *empty = bars + MAX_STAGE;       // [NSTAGE] MMA commit -> loader
    uint64_t *a_full = bars + 2 * MAX_STAGE;  // [2] producers -> MMA
    uint64_t *a_empty = a_full + 2;           // [2] MMA commit -> producers
    uint64_t *d_full = a_empty + 2;           // [2] MMA commit -> drain
    uint64_t *d_empty = d_full + 2;           // [2] drain -> MMA
    uint64_t *done = d_empty + 2;             // [1] final MMA commit
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int i = 0; i < NSTAGE; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&a_full[i], NPROD_WARPS * 32);
            mbar_init(&a_empty[i], 1);
            mbar_init(&d_full[i], 1);
            mbar_init(&d_empty[i], NPROD_WARPS * 32);
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

    const int64_t G = gridDim.x;
    const int64_t W = args.tiles * args.n_chunks;
    const int64_t u0 = W * (int64_t)blockIdx.x / G, u1 = W * ((int64_t)blockIdx.x + 1) / G;
    bool dead = false;

    if (warp == LOAD_WARP) {
        if (lane == 0) {
            int64_t g = 0;
            for (int64_t u = u0; u < u1 && !dead; ++u, ++g) {
                const int64_t chunk = u % args.n_chunks;
                const int stage = (int)(g % NSTAGE);
                if (!mbar_wait(&empty[stage], (uint32_t)(((g / NSTAGE) + 1) & 1))) {
                    atomicOr(args.err, 1u);
                    dead = true;
                    break;
                }
                mbar_expect_tx(&full[stage], (uint32_t)(BB + SPIN_BYTES));
                bulk_g2s(sB + (size_t)stage * BB, args.b_operand + (size_t)chunk * BB, (uint32_t)BB, &full[stage]);
                bulk_g2s(reinterpret_cast<uint8_t *>(sSpin) + (size_t)stage * SPIN_BYTES,
                         reinterpret_cast<const uint8_t *>(args.spin_table) + (size_t)chunk * SPIN_BYTES,
                         (uint32_t)SPIN_BYTES, &full[stage]);
            }
        }
        __syncwarp();
    } else if (warp == MMA_WARP) {
        if (lane == 0) {
            const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n_mma >> 3) << 17) |
                                   ((uint32_t)(TM >> 4) << 24);
            int64_t g = 0, grp = 0;
            int64_t u = u0;
            while (u < u1 && !dead) {
                const int64_t k0 = u % args.n_chunks;
                const int64_t k1 = min(args.n_chunks, k0 + (u1 - u));
                int dbuf = 0;
                uint32_t dcol = 0;
                for (int64_t k = k0; k < k1; ++k, ++g) {
                    const bool gstart = ((k - k0) % FLUSH) == 0;
                    if (gstart) {
                        dbuf = (int)(grp & 1);
                        if (!mbar_wait(&d_empty[dbuf], (uint32_t)(((grp >> 1) + 1) & 1))) {
                            atomicOr(args.err, 2u);
                            dead = true;
                            break;
                        }
                        tc_fence_after();
                        dcol = tmem + (uint32_t)(dbuf * n_mma);
                    }
                    const int stage = (int)(g % NSTAGE);
                    const int as = (int)(g & 1);
                    if (!mbar_wait(&full[stage], (uint32_t)((g / NSTAGE) & 1)) ||
                        !mbar_wait(&a_full[as], (uint32_t)((g >> 1) & 1))) {
                        atomicOr(args.err, 4u);
                        dead = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sbase = smem_u32(sB + (size_t)stage * BB);
                    const uint32_t a_hi = tmem + A_COL0 + (uint32_t)as * 128u;
                    const uint32_t a_lo = a_hi + 64u;
                    // The accumulator add of each MMA rounds relative to |D|,
                    // so the two small cross-term passes (hi*lo, lo*hi) go
                    // first, while D is small, and hi*hi last.
#pragma unroll
                    for (int ks = 0; ks < KSTEPS; ++ks) {
                        const uint64_t bhi = bdesc(sbase + (uint32_t)(ks * n_mma * 32));
                        const uint64_t blo = bdesc(sbase + (uint32_t)((KSTEPS + ks) * n_mma * 32));
                        const uint32_t first = (gstart && ks == 0) ? 0u : 1u;
                        tc_mma_tf32(dcol, a_hi + ks * 8, blo, idesc, first);
                        tc_mma_tf32(dcol, a_lo + ks * 8, bhi, idesc, 1u);
                    }
#pragma unroll
                    for (int ks = 0; ks < KSTEPS; ++ks) {
                        const uint64_t bhi = bdesc(sbase + (uint32_t)(ks * n_mma * 32));
                        tc_mma_tf32(dcol, a_hi + ks * 8, bhi, idesc, 1u);
                    }
                    tc_commit(&empty[stage]);
                    tc_commit(&a_empty[as]);
                    if ((k - k0) % FLUSH == FLUSH - 1 || k + 1 == k1) {
                        tc_commit(&d_full[dbuf]);
                        ++grp;
                    }
                }
                if (dead) break;
                u += k1 - k0;
            }
            // Drain: wait for every issued MMA before TMEM is released.
            tc_commit(done);
            if (!mbar_wait(done, 0)) atomicOr(args.err, 8u);
        }
        __syncwarp();
    } else {
        // Producers.  Warp w: lane quarter Q (tile rows 32Q..32Q+31), spin
        // group P (8 spins of each chunk).  DMMA fragment coordinates:
        // gq = groupID (row / spin of a fragment), tq = threadID_in_group.
        const int Q = warp & 3, P = warp >> 2;
        const int gq = lane >> 2, tq = lane & 3;
        const uint32_t lane_base = (uint32_t)(Q * 32) << 16;
        // Accumulator drain: thread <-> tile row (32x32b), columns [P*ncol, (P+1)*ncol).
        const int row = Q * 32 + lane;
        const int ncol = n_mma / 4;
        float *arow = accf + (size_t)row * (n_mma + ACC_PAD) + P * ncol;
        int64_t g = 0, grp = 0;
        int64_t u = u0;
        // Two-level drain of each chunk's accumulator generation: the FP32
        // TMEM result is added (round to nearest) into this thread's FP32 row
        // accumulator in shared memory; every WINDOW chunks, and at the end of
        // a piece, that row is promoted into the FP64 split-K partial.
        int64_t pend_grp = -1;
        double *pend_dst = nullptr;
        bool pend_wfirst = false, pend_promote = false, pend_pfirst = false;
        auto drain = [&]() -> bool {
            const int dbuf = (int)(pend_grp & 1);
            const bool ok = mbar_wait(&d_full[dbuf], (uint32_t)((pend_grp >> 1) & 1));
            __syncwarp();
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) atomicOr(args.err, 32u);
                return false;
            }
            tc_fence_after();
            for (int cc = 0; cc < ncol; cc += 4) {
                float v[4];
                tmem_ld_x4(tmem + lane_base + (uint32_t)(dbuf * n_mma + P * ncol + cc), v);
                tmem_wait_ld();
                float4 a = pend_wfirst ? make_float4(0.f, 0.f, 0.f, 0.f) : *reinterpret_cast<float4 *>(arow + cc);
                a.x += v[0];
                a.y += v[1];
                a.z += v[2];
                a.w += v[3];
                *reinterpret_cast<float4 *>(arow + cc) = a;
            }
            tc_fence_before();
            mbar_arrive(&d_empty[dbuf]);
            if (pend_promote) {
                for (int cc = 0; cc < ncol; cc += 2) {
                    const float2 a = *reinterpret_cast<const float2 *>(arow + cc);
                    double2 *d = reinterpret_cast<double2 *>(pend_dst + cc);
                    double2 o = pend_pfirst ? make_double2(0.0, 0.0) : *d;
                    o.x += (double)a.x;
                    o.y += (double)a.y;
                    *d = o;
                }
            }
            pend_grp = -1;
            return true;
        };
        while (u < u1 && !dead) {
            const int64_t tile = u / args.n_chunks;
            const int64_t k0 = u % args.n_chunks;
            const int64_t k1 = min(args.n_chunks, k0 + (u1 - u));
            const int slot = (int)(blockIdx.x - cta_of(tile * args.n_chunks, G, W));
            double *dst_piece =
                args.partial + (((size_t)tile * args.maxp + slot) * TM + row) * (size_t)n_mma + P * ncol;
            // A fragments of the phase GEMM: kappa[row 32Q + 8mt + gq][k = 4ks + tq].
            double ka[4][5];
            float tj[4];
#pragma unroll
            for (int mt = 0; mt < 4; ++mt) {
                int64_t j = tile * TM + Q * 32 + mt * 8 + gq;
                if (j >= args.nsamples) j = args.nsamples - 1;
                const double *pr = args.prefix + (size_t)j * PREFIX_STRIDE;
#pragma unroll
                for (int ks = 0; ks < 5; ++ks) ka[mt][ks] = pr[4 * ks + tq];
                tj[mt] = (float)pr[PREFIX_T];
            }
            for (int64_t k = k0; k < k1; ++k, ++g) {
                const int stage = (int)(g % NSTAGE);
                const int as = (int)(g & 1);
                bool ok = mbar_wait(&full[stage], (uint32_t)((g / NSTAGE) & 1));
                ok = ok && mbar_wait(&a_empty[as], (uint32_t)(((g >> 1) + 1) & 1));
                __syncwarp();
                if (!__all_sync(0xffffffffu, ok)) {
                    if (lane == 0) atomicOr(args.err, 16u);
                    dead = true;
                    break;
                }
                tc_fence_after();
                const double *tab = sSpin + (size_t)stage * (SPIN_BYTES / 8);
                // B fragments: b[k = 4ks + tq][spin 8P + gq].
                double bf[5];
#pragma unroll
                for (int ks = 0; ks < 5; ++ks) bf[ks] = tab[(4 * ks + tq) * KC + 8 * P + gq];
                double th[4][2];
#pragma unroll
                for (int mt = 0; mt < 4; ++mt) {
                    th[mt][0] = 0.0;
                    th[mt][1] = 0.0;
#pragma unroll
                    for (int ks = 0; ks < 5; ++ks) dmma_8x8x4(th[mt][0], th[mt][1], ka[mt][ks], bf[ks]);
                }
                // This thread's spins: 8P + 2tq + i.
                const float4 rl = *reinterpret_cast<const float4 *>(tab + SPIN_PACK * KC + 8 * P + 2 * tq);
                const float r2v[2] = {rl.x, rl.z};
                const float l2v[2] = {rl.y, rl.w};
                // 16x256b.x2 register order per pair of row tiles (mt, mt+1):
                // [i*4 + (mt&1)*2 + comp] for spin 2tq + i.
                uint32_t hi[2][8], lo[2][8];
#pragma unroll
                for (int mt = 0; mt < 4; ++mt) {
#pragma unroll
                    for (int i = 0; i < 2; ++i) {
                        float mre, mim;
                        magnetisation(th[mt][i], tj[mt], r2v[i], l2v[i], mre, mim);
                        const uint32_t hr = tf32_rna(mre), hm = tf32_rna(mim);
                        const int e = i * 4 + (mt & 1) * 2;
                        hi[mt >> 1][e] = hr;
                        hi[mt >> 1][e + 1] = hm;
                        lo[mt >> 1][e] = tf32_rna(mre - __uint_as_float(hr));
                        lo[mt >> 1][e + 1] = tf32_rna(mim - __uint_as_float(hm));
                    }
                }
                const uint32_t a_col = tmem + A_COL0 + (uint32_t)as * 128u + (uint32_t)P * 16u;
                tmem_st_16x256b_x2(a_col + lane_base, hi[0]);
                tmem_st_16x256b_x2(a_col + lane_base + (16u << 16), hi[1]);
                tmem_st_16x256b_x2(a_col + 64u + lane_base, lo[0]);
                tmem_st_16x256b_x2(a_col + 64u + lane_base + (16u << 16), lo[1]);
                tmem_wait_st();
                tc_fence_before();
                mbar_arrive(&a_full[as]);
                // The previous generation has had a whole chunk of producer
                // time to finish: drain it now.
                if (pend_grp >= 0 && !drain()) {
                    dead = true;
                    break;
                }
                if ((k - k0) % FLUSH == FLUSH - 1 || k + 1 == k1) {
                    const int64_t i = k - k0;
                    pend_grp = grp++;
                    pend_dst = dst_piece;
                    pend_wfirst = (i % WINDOW) == 0;
                    pend_promote = (i % WINDOW) == WINDOW - 1 || k + 1 == k1;
                    pend_pfirst = i < WINDOW;
                }
            }
            if (dead) break;
            if (pend_grp >= 0 && !drain()) {
                dead = true;
                break;
            }
            u += k1 - k0;
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == MMA_WARP) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// Sum split-K partials of each (sample, column) in piece order (FP64) and
// write complex samples: column n < nc is Re S(j, n), nc <= n < 2nc is Im.
template <typename T>
__global__ void split_finalize_kernel(const double *partial, int64_t nsamples, int32_t nc, int n_mma, int maxp,
                                      int64_t n_chunks, int64_t G, int64_t W, cplx<T> *sig, int64_t ldsig) {
    const int64_t total = nsamples * nc;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = i % nsamples;
        const int32_t c = (int32_t)(i / nsamples);
        const int64_t tile = j / TM;
        const int row = (int)(j % TM);
        const int64_t first = cta_of(tile * n_chunks, G, W);
        const int64_t last = cta_of((tile + 1) * n_chunks - 1, G, W);
        const int np = (int)(last - first + 1);
        double re = 0.0, im = 0.0;
        for (int p = 0; p < np; ++p) {
            const double *src = partial + (((size_t)tile * maxp + p) * TM + row) * (size_t)n_mma;
            re += src[c];
            im += src[nc + c];
        }
        sig[j + (int64_t)c * ldsig] = cplx<T>{T(re), T(im)};
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

// Sensitivities -> TF32 hi/lo B operand in the no-swizzle K-major layout, K
// permuted as k_to_spin.  With real K index kk of spin s:
//   B[n][kk] = (n < nc ? Re c(s,n) : Im c(s,n-nc))   for the re column,
//   B[n][kk] = (n < nc ? -Im c(s,n) : Re c(s,n-nc))  for the im column.
__global__ void b_operand_kernel(const cplx<double> *csm_rows, int64_t ns, int32_t nc, int n_mma, int64_t nchunks,
                                 float *out) {
    const int64_t per_chunk = (int64_t)KSTEPS * n_mma * 8;
    const int64_t total = nchunks * per_chunk;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t chunk = i / per_chunk;
        int64_t r = i % per_chunk;
        const int ks = (int)(r / (n_mma * 8));
        r %= (n_mma * 8);
        const int n = (int)(r / 8), kk = (int)(r % 8);
        int s_local, imrow;
        k_to_spin(ks * 8 + kk, s_local, imrow);
        const int64_t s = chunk * KC + s_local;
        double v = 0.0;
        if (s < ns && n < 2 * nc) {
            const cplx<double> c = csm_rows[s * nc + (n < nc ? n : n - nc)];
            if (n < nc) v = imrow ? -c.im : c.re;
            else v = imrow ? c.re : c.im;
        }
        const float vf = (float)v;
        const uint32_t hb = tf32_rna(vf);
        // lo carries what the TF32 hi misses of the FP64 value.
        const uint32_t lb = tf32_rna((float)(v - (double)__uint_as_float(hb)));
        const size_t off = (size_t)(n / 8) * 256 + (size_t)(kk / 4) * 128 + (size_t)(n % 8) * 16 + (size_t)(kk % 4) * 4;
        uint8_t *base = reinterpret_cast<uint8_t *>(out) + (size_t)chunk * b_bytes(n_mma);
        *reinterpret_cast<uint32_t *>(base + (size_t)ks * n_mma * 32 + off) = hb;
        *reinterpret_cast<uint32_t *>(base + (size_t)(KSTEPS + ks) * n_mma * 32 + off) = lb;
    }
}

// Spin table of a segment, from the state at its start (k-major per chunk):
// rows 0..15 basis, 16 dw/(2 pi) (0 if dw is off in precession),
// 17 theta0 = arg(m0)/(2 pi), 18..19 zero, 20 packed float2
// (-log2(e)/T2, log2|m0|).  Also checks the phase range: |theta| must stay
// below 2^18 turns for the fixed-point reduction (error bit 64 otherwise).
__global__ void spin_table_kernel(const double *basis, const double *dw, const double *T2, const cplx<double> *xy,
                                  int64_t ns, int64_t nchunks, uint32_t method, const double *colmax,
                                  unsigned int *err, double *table) {
    const int64_t total = nchunks * KC;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < total;
         s += (int64_t)gridDim.x * blockDim.x) {
        double *t = table + (s / KC) * (SPIN_ROWS * KC) + (s % KC);
        if (s < ns) {
            for (int k = 0; k < 16; ++k) t[k * KC] = basis[s * 16 + k];
            t[16 * KC] = (method & HOMS_DW_PRECESSION) ? dw[s] / (2.0 * 3.141592653589793) : 0.0;
            const cplx<double> m0 = xy[s];
            const double mag = hypot(m0.re, m0.im);
            t[17 * KC] = atan2(m0.im, m0.re) / (2.0 * 3.141592653589793);
            double bound = fabs(t[17 * KC]);
            for (int k = 0; k < 17; ++k) bound += fabs(t[k * KC]) * colmax[k];
            if (!(bound < 262144.0)) atomicOr(err, 64u);
            float2 rl;
            rl.x = (float)(-1.4426950408889634 / T2[s]);
            rl.y = mag > 0.0 ? (float)log2(mag) : -INFINITY;
            *reinterpret_cast<float2 *>(&t[SPIN_PACK * KC]) = rl;
        } else {
            for (int k = 0; k < 18; ++k) t[k * KC] = 0.0;
            *reinterpret_cast<float2 *>(&t[SPIN_PACK * KC]) = make_float2(0.0f, -INFINITY);
        }
        t[18 * KC] = 0.0;
        t[19 * KC] = 0.0;
    }
}

// Prefix table of one segment.  Blocks 0..16: column k, a deterministic
// chunked scan of the trapezoid sums (f(n)+f(n+1)) dt(n), written at every
// ADC node (row = sample index) and at the end node (row nsamples), plus the
// column's largest |value| at row nsamples+1.  Block 17: elapsed time t
// (entry PREFIX_T) and the constant columns 17 (= 1) and 18, 19 (= 0).
__global__ void prefix_kernel(const double *dt, const double *const *src, const uint8_t *adc, const int32_t *rank,
                              int64_t n_lo, int64_t n_hi, int64_t nsamples, double gamma, double *prefix) {
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
            double *pr = prefix + (size_t)rank[n + 1] * PREFIX_STRIDE;
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
        const double *t = table + (s / KC) * (SPIN_ROWS * KC) + (s % KC);
        double th = t[17 * KC];
        for (int k = 0; k < 17; ++k) th = fma(t[k * KC], endrow[k], th);
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

}  // namespace split

using namespace split;

SplitResident::~SplitResident() {
    for (void *p : {basis, b_operand, spin_table, prefix, tvec, partial, tile_map, err})
        if (p) cudaFree(p);
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
    const int n_mma = std::max(16, ((2 * nc + 15) / 16) * 16);
    if (n_mma > 128) {
        *err = "split mode supports at most 64 coils per run";
        return cudaSuccess;
    }
    r.ns = ns;
    r.nc = nc;
    r.n_mma = n_mma;
    const int64_t nchunks = (ns + KC - 1) / KC;
    r.ns_pad = nchunks * KC;
    cudaError_t e;
    if ((e = grow(r.basis, r.basis_bytes, sizeof(double) * 16 * (size_t)ns)) != cudaSuccess) return e;
    if ((e = grow(r.b_operand, r.b_bytes, (size_t)b_bytes(n_mma) * (size_t)nchunks)) != cudaSuccess) return e;
    if (!r.err) {
        if ((e = cudaMalloc(&r.err, sizeof(unsigned int))) != cudaSuccess) return e;
    }
    basis_kernel<<<grid_for(ns), 256, 0, stream>>>((const double *)x, (const double *)y, (const double *)z, ns,
                                                   (double *)r.basis);
    const int64_t total = nchunks * KSTEPS * n_mma * 8;
    b_operand_kernel<<<grid_for(total), 256, 0, stream>>>((const cplx<double> *)csm_rows, ns, nc, n_mma, nchunks,
                                                          (float *)r.b_operand);
    return cudaGetLastError();
}

static size_t acc_bytes(int n_mma) { return sizeof(float) * (size_t)TM * (n_mma + ACC_PAD); }

static int kernel_stages(int n_mma) {
    const size_t budget = 220 * 1024;
    const size_t per = (size_t)b_bytes(n_mma) + SPIN_BYTES;
    return (int)std::max<size_t>(2, std::min<size_t>(MAX_STAGE, (budget - 2048 - acc_bytes(n_mma)) / per));
}

static size_t kernel_smem(int n_mma) {
    return 1024 + (size_t)kernel_stages(n_mma) * (b_bytes(n_mma) + SPIN_BYTES) + acc_bytes(n_mma) + 32 * 8 + 64;
}

// One precession segment.
static cudaError_t split_segment(SplitResident &r, const SplitRunArgs &a, int64_t n_lo, int64_t n_hi,
                                 int64_t sample0, int64_t nsamples, cudaStream_t stream, std::string *err) {
    cudaError_t e;
    const int64_t nchunks = r.ns_pad / KC;
    const int64_t tiles = (nsamples + TM - 1) / TM;
    // ADC rank per node of the segment (host), uploaded with the column sources.
    std::vector<int32_t> rank((size_t)a.nt, 0);
    int64_t c = 0;
    for (int64_t n = n_lo + 1; n <= n_hi; ++n)
        if (a.adc_host[n]) rank[(size_t)n] = (int32_t)c++;
    if (c != nsamples) {
        *err = "internal: segment sample count mismatch";
        return cudaSuccess;
    }
    const size_t rank_bytes = (sizeof(int32_t) * (size_t)a.nt + 255) & ~size_t(255);  // keeps the pointer table aligned
    const size_t src_bytes = sizeof(void *) * 17;
    const size_t prefix_rows = (size_t)std::max<int64_t>(tiles * TM, nsamples + 2);
    if ((e = grow(r.prefix, r.prefix_bytes, prefix_rows * PREFIX_STRIDE * sizeof(double))) != cudaSuccess) return e;
    if ((e = grow(r.tvec, r.tvec_bytes, rank_bytes + src_bytes)) != cudaSuccess) return e;
    if ((e = grow(r.spin_table, r.spin_bytes, (size_t)nchunks * SPIN_BYTES)) != cudaSuccess) return e;
    const double *src[17];
    const uint32_t m = a.method;
    src[0] = (m & HOMS_HO0) ? (const double *)a.h[0] : nullptr;
    for (int k = 1; k <= 3; ++k)
        src[k] = (m & HOMS_HO1) ? (const double *)a.h[k] : (const double *)(k == 1 ? a.gx : k == 2 ? a.gy : a.gz);
    for (int k = 4; k <= 8; ++k) src[k] = (m & HOMS_HO2) ? (const double *)a.h[k] : nullptr;
    for (int k = 9; k <= 15; ++k) src[k] = (m & HOMS_HO3) ? (const double *)a.h[k] : nullptr;
    src[16] = (m & HOMS_DW_PRECESSION) ? reinterpret_cast<const double *>(1) : nullptr;
    uint8_t *tv = (uint8_t *)r.tvec;
    if ((e = cudaMemcpyAsync(tv, rank.data(), rank_bytes, cudaMemcpyHostToDevice, stream)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(tv + rank_bytes, src, src_bytes, cudaMemcpyHostToDevice, stream)) != cudaSuccess) return e;
    // The host arrays above are stack/vector memory: finish the copies before they go away.
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
    prefix_kernel<<<18, 256, 0, stream>>>((const double *)a.dt, reinterpret_cast<const double *const *>(tv + rank_bytes),
                                          (const uint8_t *)a.adc, reinterpret_cast<const int32_t *>(tv), n_lo, n_hi,
                                          nsamples, a.gamma, (double *)r.prefix);
    spin_table_kernel<<<grid_for(r.ns_pad), 256, 0, stream>>>(
        (const double *)r.basis, (const double *)a.dw, (const double *)a.T2, (const cplx<double> *)a.xy, r.ns, nchunks,
        m, (const double *)r.prefix + (size_t)(nsamples + 1) * PREFIX_STRIDE, (unsigned int *)r.err,
        (double *)r.spin_table);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (nsamples > 0) {
        int dev = 0, nsm = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        const int64_t W = tiles * nchunks;
        const int64_t G = std::min<int64_t>(nsm, W);
        int maxp = 1;
        for (int64_t t = 0; t < tiles; ++t) {
            const int64_t f = ((t * nchunks + 1) * G - 1) / W;
            const int64_t l = (((t + 1) * nchunks) * G - 1) / W;
            maxp = std::max<int>(maxp, (int)(l - f + 1));
        }
        const size_t pbytes = sizeof(double) * (size_t)tiles * maxp * TM * r.n_mma;
        if ((e = grow(r.partial, r.partial_bytes, pbytes)) != cudaSuccess) return e;
        const size_t smem = kernel_smem(r.n_mma);
        if ((e = cudaFuncSetAttribute(split_precession_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
            cudaSuccess)
            return e;
        KernelArgs ka;
        ka.prefix = (const double *)r.prefix;
        ka.b_operand = (const uint8_t *)r.b_operand;
        ka.spin_table = (const double *)r.spin_table;
        ka.partial = (double *)r.partial;
        ka.err = (unsigned int *)r.err;
        ka.nsamples = nsamples;
        ka.n_chunks = nchunks;
        ka.tiles = tiles;
        ka.maxp = maxp;
        ka.n_mma = r.n_mma;
        ka.nstage = kernel_stages(r.n_mma);
        if (a.ev_start) cudaEventRecord(a.ev_start, stream);
        split_precession_kernel<<<(unsigned)G, THREADS, smem, stream>>>(ka);
        if (a.ev_stop) cudaEventRecord(a.ev_stop, stream);
        if (a.launches) *a.launches += 2;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        const int64_t total = nsamples * r.nc;
        if (a.sizeof_T == 8)
            split_finalize_kernel<double><<<grid_for(total), 256, 0, stream>>>(
                (const double *)r.partial, nsamples, r.nc, r.n_mma, maxp, nchunks, G, W,
                (cplx<double> *)a.sig + sample0, a.nadc);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (a.launches) *a.launches += 3;
    state_update_kernel<<<grid_for(r.ns), 256, 0, stream>>>(
        (const double *)r.spin_table, (const double *)r.prefix + (size_t)nsamples * PREFIX_STRIDE, (const double *)a.T1,
        (const double *)a.T2, (const double *)a.rho, r.ns, (cplx<double> *)a.xy, (double *)a.mz);
    return cudaGetLastError();
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
