// Split-precision fused precession + coil contraction on sm_100a tensor cores,
// in exact integer arithmetic on the int8 tcgen05 pipe.
//
// Math (one precession segment = a run of consecutive precession blocks):
//   phase in turns   theta(s,j) = theta0(s) + kappa_0(j) + sum_k b_k(s) kappa_k(j)
//     k = 1..15 : the unnormalised solid-harmonic basis terms of spin s,
//                 kappa_k = -gamma * trapezoid integral of field column k from
//                 the segment start to ADC sample j
//     k = 16    : b_16 = dw/(2 pi),  kappa_16 = -t_j (0 when dw is off)
//     kappa_0   : the h0 term (basis value 1), theta0 = arg(m0)/(2 pi)
//   M(s,j)   = |m0| 2^(t_j * r2(s)) * cis(2 pi theta)   (r2 = -log2(e)/T2)
//   S(j,c)   = sum_s M(s,j) csm(s,c)                      (no conjugation)
// This is the reference's phi = -2 pi gamma cumtrapz(dt, Bz) and
// Mxy = M0 exp(i phi - t/T2) (src/simulation/Bloch/BlochHighOrderSimulatitonMethod.jl:76-92)
// with the cumulative integral factored into per-spin x per-sample terms.
//
// Phase, exactly.  Per field term k the coefficient is the integer
// B_k(s) = rint(b_k 2^38 / bmax_k) and the integral K_k(j) =
// rint(kappa_k bmax_k 2^26), so that B K 2^-64 = b kappa to 2^-27 turn
// (|K| <= 2^38 requires bmax_k * max|kappa_k| <= 2^12 turns, checked per
// segment).  Both are split into five balanced int8 digits (base 256); the
// digit products of equal weight 2^(8w) are summed exactly by int8 tcgen05
// MMAs (int32 accumulators), and the classes w = 3..7 form the 32-bit turn
// fraction: w >= 8 are whole turns (the mod-2pi reduction is the integer
// wraparound), w <= 1 lie below 2^-32 turn and w = 2 adds at most 12 units
// of 2^-32 turn (|S_2| <= 3 digit pairs x 16 terms x 2^14), so it is left
// out.  The turn fraction
//   u = sum_{w>=3} S_w 2^(8w-32) mod 2^32
// is exact up to the rounding of B and K and that 12 * 2^-32 turn.
//
// Trigonometry.  u is reduced to the nearest half turn in integers
// (|x| <= pi/2, which keeps the float scale of the angle from biasing the
// phase at the wrap), then sin/cos.approx and a sign (cis(x + h pi) =
// (-1)^h cis(x)); the decay is ex2.approx of a small argument.  |M| < 1 after
// a power-of-two scale per segment.
//
// Coil contraction, exactly.  M becomes a 30-bit integer (|M| < 2^30), four
// int8 digits: F = rint(M 2^22) gives three unsigned bytes (the top one offset
// by 64) and the rounding residual, scaled to [-127, 127] and rounded, the
// signed low byte; 30 bits keep spins of small amplitude (outside an excited
// slice, for instance) precise against a signal that cancels, and a spin of
// zero amplitude contributes exactly nothing.  The per-coil scaled
// sensitivities become integers of 23 bits (|c| <= 127 2^16), three balanced
// digits.  Eight int8 MMAs per 32-spin chunk accumulate the digit classes
// T5..T2 (weights 2^40..2^16 of the 2^53 full scale; lower classes lie below
// 2^-29 of it) in int32 TMEM for a whole work item (at most 256 chunks:
// |T| < 1.34e9 < 2^31), with no rounding at all.  At the end of an item its
// classes become one integer per output element, added (red.global.add.u64)
// into the tile's int64 accumulator: the slabs' sums are exact, so their order
// does not matter and a result is the same bit for bit on every run.  The
// finalize removes the offset of the top digit from the integer, then rounds
// once to FP64.
//
// Kernel organisation (one CTA per SM, persistent, slab-major work items of
// (time tile of 128 samples) x (range of 32-spin chunks)):
//   warps 0-15  magnetisation: warp w owns tile rows 32(w%4) .. +31 (its
//               TMEM lane quarter) and spins 8(w/4) .. +7 of every chunk:
//               reads the phase classes, forms the turn, M and its digits,
//               writes the coil MMA's A operand to TMEM; drains the coil
//               classes into the tile's int64 accumulator.
//   warp 16     coil MMA issuer: per chunk 8 coil MMAs (A in TMEM, B: the
//               chunk's sensitivity digits); one commit releases both the
//               shared-memory stage and the A buffer.
//   warp 17     loader: cp.async.bulk of each item's phase A tile and each
//               chunk's operands (non-multicast).
//   warp 18     phase MMA issuer: per chunk 3 phase MMAs (A: the tile's
//               integral digits in shared memory, B: the chunk's coefficient
//               digits), one chunk ahead of the magnetisation warps.
// The two issuers keep either chain of waits and MMAs off the other's
// critical path.  Issuing MMAs, commits and bulk copies costs issue slots of
// the issuing warp's scheduler (warp w runs on scheduler w % 4): each helper
// sits on its own scheduler, and scheduler 3 carries none.
// TMEM (512 columns): phase classes 160, coil A operand 64, coil classes 4N.
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
constexpr int NSLOT = 16;        // phase terms per spin: basis 1..15 and dw/(2 pi)
constexpr int PHASE_DIGITS = 5;  // base-256 digits of the phase integers
constexpr int PREFIX_STRIDE = 24;  // doubles per prefix row: kappa_0..kappa_16, t at PREFIX_T
constexpr int PREFIX_T = 20;
constexpr int GROUP_COILS = 32;  // coils per kernel pass (N <= 64 output columns)
constexpr int NMAG_WARPS = 16;
constexpr int MMA_WARP = 16;    // coil MMA issuer (allocates TMEM)
constexpr int LOAD_WARP = 17;
constexpr int PHASE_WARP = 18;  // phase MMA issuer
constexpr int THREADS = 608;
constexpr uint32_t TMEM_COLS = 512;
constexpr int MAX_STAGE = 6;
constexpr int MAX_ITEM_CHUNKS = 256;  // int32 coil classes stay below 2^31 over an item
// A spin adds less than 2^39 to an accumulator element (units of 2^16: digit
// values below 2^31 and 2^23, two products per output), so one int64 holds the
// sum over 2^24 spins.  Items go to accumulator slot (first chunk >> 18): at
// most 2^18 + MAX_ITEM_CHUNKS chunks, under 2^23 + 2^13 spins, per slot.
constexpr int ACC_SLOT_LOG2 = 18;
__host__ __device__ constexpr int acc_slots(int64_t n_chunks) {
    return (int)((n_chunks + (1 << ACC_SLOT_LOG2) - 1) >> ACC_SLOT_LOG2);
}
constexpr long long WAIT_BUDGET = 4000000000LL;  // cycles (~2 s)
constexpr double PHASE_RANGE_LIMIT = 4096.0;     // turns: bmax_k * max|kappa_k| per term and segment

// Phase MMAs: A' tiles [a4|a3], [a2|a1], [a0|0] (128 rows x 32 bytes each) and
// B' blocks of 32 spin rows per digit class w (classes 7..3 at TMEM columns
// (7 - w) * 32): MMA 1 covers w = 7..3 (N = 160), MMA 2 w = 6..3 (N = 128,
// columns 32..159), MMA 3 w = 4..3 (N = 64, columns 96..159).
constexpr int PH_N1 = 160, PH_N2 = 128, PH_N3 = 64;
constexpr int PH_CLASSES = 5;
constexpr int PH_OFF2 = PH_N1 * 32, PH_OFF3 = (PH_N1 + PH_N2) * 32;
constexpr int PHASE_B_BYTES = (PH_N1 + PH_N2 + PH_N3) * 32;  // per chunk
constexpr int PHASE_A_BYTES = 3 * TM * 32;                   // per tile
constexpr int PARAM_BYTES = 3 * KC * 4;                      // per chunk
// Coil B operand per chunk: 2 K-steps of 16 spins x (re, im) = 32 int8, each
// [c2 | c1 | c0] x N rows.
__host__ __device__ constexpr int coil_b_bytes(int n) { return 2 * 3 * n * 32; }

// TMEM columns.
constexpr uint32_t P_COL = 0;    // phase classes (160 columns)
constexpr uint32_t A_COL = 192;  // coil A: per K-step [d3 | d2 | d1 | d0], 8 columns each
constexpr uint32_t D_COL = 256;  // coil classes [T5 | T4 | T3 | T2], N columns each

// Canonical no-swizzle K-major layout of an operand with 32 bytes of K per
// row: core matrices of 8 rows x 16 bytes, K-direction stride 128 B, 8-row
// group stride 256 B.
__host__ __device__ inline int kmaj(int row, int kbyte) {
    return (row >> 3) * 256 + (kbyte >> 4) * 128 + (row & 7) * 16 + (kbyte & 15);
}

// Smallest e with 2^e >= x for a non-negative double given by its bits (0 for 0).
__host__ __device__ inline int pow2_ceil_exp(unsigned long long bits) {
    if (bits == 0) return 0;
    int e = (int)((bits >> 52) & 0x7FF) - 1023;
    if (bits & 0xFFFFFFFFFFFFFull) e += 1;
    return e;
}

// Balanced base-256 digit i of v (digits 0..n-2 in [-128, 127]; the top one
// takes the rest).
__host__ __device__ inline int balanced_digit(long long v, int i, int n) {
    for (int k = 0; k < i; ++k) {
        const long long d = ((v + 128) & 255) - 128;
        v = (v - d) >> 8;
    }
    if (i == n - 1) return (int)v;
    return (int)(((v + 128) & 255) - 128);
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
// The single-thread helpers' wait: try_wait with a suspend-time hint (fewer
// probes while waiting; a barrier probe takes issue slots from the other
// warps of the prober's scheduler); bounded like mbar_wait.
constexpr uint32_t SUSPEND_HINT_NS = 1000000u;
__device__ __forceinline__ bool mbar_try_hint(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(SUSPEND_HINT_NS)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_helper(uint64_t *bar, uint32_t parity) {
    if (mbar_try_hint(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_hint(bar, parity)) {
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
// int8 MMA, A and B from shared memory (descriptors).
__device__ __forceinline__ void tc_mma_i8_ss(uint32_t d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                             uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
        : "memory");
}
// int8 MMA, A in TMEM, B from shared memory.
__device__ __forceinline__ void tc_mma_i8_ts(uint32_t d, uint32_t a, uint64_t bdesc, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d),
        "r"(a), "l"(bdesc), "r"(idesc), "r"(accum)
        : "memory");
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
// Integer multiply-adds with the multiplier in a register (a kernel argument,
// so that the power-of-two shifts they implement issue on the FMA pipe
// rather than the busier integer ALU pipe): lo = a b + c, hi = hi32(a b) + c.
__device__ __forceinline__ uint32_t mad_lo(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t r;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
    return r;
}
__device__ __forceinline__ uint32_t mad_hi_s(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t r;
    asm("mad.hi.s32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
    return r;
}
__device__ __forceinline__ uint32_t mul_hi_u(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("mul.hi.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(sel));
    return r;
}

// 32 TMEM lanes (thread <-> lane) x 4 or 8 consecutive columns.
__device__ __forceinline__ void tmem_ld_x4(uint32_t taddr, uint32_t *v) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
                 : "r"(taddr)
                 : "memory");
}
__device__ __forceinline__ void tmem_ld_x8(uint32_t taddr, uint32_t *v) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr)
                 : "memory");
}
__device__ __forceinline__ void tmem_st_x4(uint32_t taddr, const uint32_t *v) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr), "r"(v[0]), "r"(v[1]),
                 "r"(v[2]), "r"(v[3])
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor of the canonical layout above (descriptor
// version 1, no swizzle).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(256 >> 4) << 32) |
           (1ull << 46);
}
// Instruction descriptor of kind::i8, M = 128, K-major A and B, int32 D:
// a_signed/b_signed select s8 (1) or u8 (0).
__host__ __device__ constexpr uint32_t idesc_i8(int n, bool a_signed, bool b_signed) {
    return (2u << 4) | ((a_signed ? 1u : 0u) << 7) | ((b_signed ? 1u : 0u) << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(TM >> 4) << 24);
}

// Work items.  A launch runs one or more jobs (a job: one precession
// segment and coil group of one simulation; several simulations' jobs share
// a launch in the server's rounds).  A job's (tile x chunk) grid is cut into
// `slabs` ranges of chunks; its item k is slab z = k / tiles of tile
// k % tiles, and the launch's items are the jobs' items one job after the
// other.  CTA b takes items b, b + G, b + 2G, ...  The CTAs running at any
// one time thus read the chunks of two or three consecutive slabs, which stay
// in L2 for every tile that needs them.  Item (tile, z) adds into its job's
// accumulator of that tile (spin-range slot of its first chunk).
constexpr int MAX_JOBS = SPLIT_MAX_JOBS;
struct KernelJob {
    const uint8_t *phase_a;    // [tiles][PHASE_A_BYTES]
    const uint8_t *phase_b;    // [nchunks][PHASE_B_BYTES]
    const uint8_t *coil_b;     // [nchunks][coil_b_bytes(N)] of this coil group
    const uint8_t *params;     // [nchunks][PARAM_BYTES]
    const uint32_t *rows;      // [tiles * TM][2]: base turn, elapsed time (float bits)
    unsigned long long *acc;   // [tiles][acc_slots(n_chunks)][N][TM] int64, zero before the launch
    unsigned int *err;         // the job's device error word
    int n_chunks, tiles, slabs;
    int item0;                 // launch index of the job's first item
};
struct KernelArgs {
    KernelJob job[MAX_JOBS];
    int n_jobs, n_items, nstage;
    uint32_t mul8, mul16, mul24;  // 2^8, 2^16, 2^24 (multipliers of mad_lo / mad_hi)
};

// The launch's job table (in shared memory) and item count.
struct Work {
    const KernelJob *jobs;
    int n_jobs, n_items;
};
struct Cursor {
    int i, c, c0, c1, tile, z, local, job;
    bool valid;
};
__device__ __forceinline__ void cursor_item(const Work &w, Cursor &cu) {
    cu.valid = cu.i < w.n_items;
    if (!cu.valid) return;
    while (cu.i >= w.jobs[cu.job].item0 + w.jobs[cu.job].tiles * w.jobs[cu.job].slabs) ++cu.job;
    const KernelJob &J = w.jobs[cu.job];
    const int k = cu.i - J.item0;
    cu.z = k / J.tiles;
    cu.tile = k - cu.z * J.tiles;
    cu.c0 = (int)((int64_t)J.n_chunks * cu.z / J.slabs);
    cu.c1 = (int)((int64_t)J.n_chunks * (cu.z + 1) / J.slabs);
    cu.c = cu.c0;
}
__device__ __forceinline__ Cursor cursor_start(const Work &w) {
    Cursor cu;
    cu.i = blockIdx.x;
    cu.local = 0;
    cu.job = 0;
    cursor_item(w, cu);
    return cu;
}
__device__ __forceinline__ void cursor_next(const Work &w, Cursor &cu) {
    if (++cu.c < cu.c1) return;
    cu.i += gridDim.x;
    ++cu.local;
    cursor_item(w, cu);
}
// A failed wait is reported in the error word of every job of the launch.
__device__ __forceinline__ void report(const Work &w, unsigned int code) {
    for (int j = 0; j < w.n_jobs; ++j) atomicOr(w.jobs[j].err, code);
}

constexpr float TWO_PI_2M24 = 3.7450702829239069e-07f;  // 2 pi / 2^24: one unit of the 23-bit half-turn angle
constexpr float MAGIC_1P5_2P23 = 12582912.0f;           // 1.5 * 2^23
// The angle is one FFMA, fb * TWO_PI_2M24 + ANGLE_OFFSET with fb = 2^23 + the
// 23-bit remainder; ANGLE_OFFSET is -1.5 * 2^23 * TWO_PI_2M24 rounded to float,
// so every angle carries the same offset angle_offset_error() (about 1e-7
// rad), which the finalize removes exactly by a rotation of the signal.
constexpr float ANGLE_OFFSET = -MAGIC_1P5_2P23 * TWO_PI_2M24;
inline __host__ __device__ double angle_offset_error() {
    return (double)ANGLE_OFFSET + (double)MAGIC_1P5_2P23 * (double)TWO_PI_2M24;
}
// Low magnetisation digit: rint(r * 2^30 (1 - 2^-7)) for the rounding residual
// |r| <= 2^-23 of the top three digits, so |digit| <= 127 without a clamp.
constexpr float LOW_DIGIT_SCALE = 1065353216.0f;  // 2^30 - 2^23

// Amplitude exponent of a segment: the smallest e with 2^e >= max|m0| (1 + 2^-19),
// so that |M| / 2^e stays below 1 - 2^-20 and the sin/cos/ex2 approximations
// (errors below 2^-20 relative) cannot carry |M 2^-e| to 1 or above.
__device__ __forceinline__ int amp_exp(unsigned long long bits) {
    if (bits == 0) return 0;
    const double v = __longlong_as_double((long long)bits) * (1.0 + 0x1p-19);
    return pow2_ceil_exp((unsigned long long)__double_as_longlong(v));
}

template <int N>
__global__ void __launch_bounds__(THREADS, 1) split_precession_kernel(const __grid_constant__ KernelArgs args) {
    constexpr int CB = coil_b_bytes(N);
    constexpr int STAGE_BYTES = CB + PHASE_B_BYTES + PARAM_BYTES;
    constexpr int NQ = N / 4;  // coil columns drained per magnetisation warp
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    const int NSTAGE = args.nstage;
    uint8_t *sA = smem;                                  // 2 x PHASE_A_BYTES
    uint8_t *sStage = smem + 2 * PHASE_A_BYTES;          // NSTAGE x STAGE_BYTES
    uint64_t *bars = reinterpret_cast<uint64_t *>(sStage + (size_t)NSTAGE * STAGE_BYTES);
    // empty[s]: the coil MMAs of the stage's chunk are complete, so both the
    // stage (-> loader) and the coil A buffer (-> magnetisation warps) are free.
    uint64_t *full = bars;                   // [NSTAGE] loader -> MMA issuers, magnetisation (tx)
    uint64_t *empty = bars + MAX_STAGE;      // [NSTAGE] coil MMA commit -> loader, magnetisation
    uint64_t *a_full_ph = empty + MAX_STAGE; // [2] loader -> phase issuer (phase A tile, tx)
    uint64_t *a_empty_ph = a_full_ph + 2;    // [2] last phase MMA of an item -> loader
    uint64_t *p_full = a_empty_ph + 2;       // phase MMA commit -> magnetisation
    uint64_t *p_empty = p_full + 1;          // magnetisation warps -> phase issuer
    uint64_t *a_full = p_empty + 1;          // magnetisation warps -> coil issuer (coil A written)
    uint64_t *d_full = a_full + 1;           // last coil MMA of an item -> drain
    uint64_t *d_empty = d_full + 1;          // drain (coil classes cleared) -> coil issuer
    uint64_t *done = d_empty + 1;            // [2] every MMA of the coil / phase issuer complete
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 2);
    KernelJob *sjobs = reinterpret_cast<KernelJob *>(done + 4);  // the launch's job table

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    {
        constexpr int WORDS = (int)(sizeof(KernelJob) / sizeof(unsigned long long));
        const unsigned long long *src = reinterpret_cast<const unsigned long long *>(args.job);
        for (int k = threadIdx.x; k < args.n_jobs * WORDS; k += blockDim.x)
            reinterpret_cast<unsigned long long *>(sjobs)[k] = src[k];
    }
    const Work W{sjobs, args.n_jobs, args.n_items};
    if (threadIdx.x == 0) {
        for (int i = 0; i < NSTAGE; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&a_full_ph[i], 1);
            mbar_init(&a_empty_ph[i], 1);
        }
        for (int i = 0; i < 2; ++i) mbar_init(&done[i], 1);
        mbar_init(p_full, 1);
        mbar_init(p_empty, NMAG_WARPS);
        mbar_init(a_full, NMAG_WARPS);
        mbar_init(d_empty, NMAG_WARPS);
        mbar_init(d_full, 1);
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
    bool dead = false;

    if (warp == LOAD_WARP) {
        if (lane == 0) {
            int stage = 0;
            uint32_t sph = 0;  // parity of the stage ring's current pass
            int issued[MAX_STAGE] = {0, 0, 0, 0, 0, 0};
            int issued_a[2] = {0, 0};
            for (Cursor cu = cursor_start(W); cu.valid && !dead; cu.i += gridDim.x, ++cu.local, cursor_item(W, cu)) {
                const int ib = cu.local & 1;
                if (!mbar_wait_helper(&a_empty_ph[ib], (uint32_t)(((cu.local >> 1) + 1) & 1))) {
                    report(W, 1u);
                    dead = true;
                    break;
                }
                mbar_expect_tx(&a_full_ph[ib], (uint32_t)PHASE_A_BYTES);
                const KernelJob &J = sjobs[cu.job];
                bulk_g2s(sA + ib * PHASE_A_BYTES, J.phase_a + (size_t)cu.tile * PHASE_A_BYTES, PHASE_A_BYTES,
                         &a_full_ph[ib]);
                ++issued_a[ib];
                for (int c = cu.c0; c < cu.c1; ++c) {
                    if (!mbar_wait_helper(&empty[stage], sph ^ 1u)) {
                        report(W, 1u);
                        dead = true;
                        break;
                    }
                    uint8_t *st = sStage + (size_t)stage * STAGE_BYTES;
                    mbar_expect_tx(&full[stage], (uint32_t)STAGE_BYTES);
                    bulk_g2s(st, J.coil_b + (size_t)c * CB, CB, &full[stage]);
                    bulk_g2s(st + CB, J.phase_b + (size_t)c * PHASE_B_BYTES, PHASE_B_BYTES, &full[stage]);
                    bulk_g2s(st + CB + PHASE_B_BYTES, J.params + (size_t)c * PARAM_BYTES, PARAM_BYTES, &full[stage]);
                    ++issued[stage];
                    if (++stage == NSTAGE) {
                        stage = 0;
                        sph ^= 1u;
                    }
                }
            }
            // Before the CTA leaves (also on the failure path), let every copy
            // this warp issued land: no bulk copy may still be writing into
            // shared memory when the CTA exits.
            for (int s = 0; s < NSTAGE; ++s)
                if (issued[s] > 0) (void)mbar_wait_budget(&full[s], (uint32_t)((issued[s] - 1) & 1), 100000000LL);
            for (int b = 0; b < 2; ++b)
                if (issued_a[b] > 0)
                    (void)mbar_wait_budget(&a_full_ph[b], (uint32_t)((issued_a[b] - 1) & 1), 100000000LL);
        }
        __syncwarp();
    } else if (warp == PHASE_WARP) {
        // Phase MMAs of every chunk: classes into TMEM columns P_COL, one chunk
        // ahead of the magnetisation warps.
        if (lane == 0) {
            constexpr uint32_t id_ph1 = idesc_i8(PH_N1, true, true);
            constexpr uint32_t id_ph2 = idesc_i8(PH_N2, true, true);
            constexpr uint32_t id_ph3 = idesc_i8(PH_N3, true, true);
            int stage = 0, gp = 0;
            uint32_t sph = 0;
            for (Cursor cp = cursor_start(W); cp.valid; ++gp) {
                const int ib = cp.local & 1;
                if (!mbar_wait_helper(&full[stage], sph) ||
                    (cp.c == cp.c0 && !mbar_wait_helper(&a_full_ph[ib], (uint32_t)((cp.local >> 1) & 1))) ||
                    !mbar_wait_helper(p_empty, (uint32_t)((gp + 1) & 1))) {
                    report(W, 2u);
                    break;
                }
                tc_fence_after();
                const uint32_t a0 = smem_u32(sA + ib * PHASE_A_BYTES);
                const uint32_t b0 = smem_u32(sStage + (size_t)stage * STAGE_BYTES + CB);
                tc_mma_i8_ss(tmem + P_COL, sdesc(a0), sdesc(b0), id_ph1, 0u);
                tc_mma_i8_ss(tmem + P_COL + 32u, sdesc(a0 + TM * 32), sdesc(b0 + PH_OFF2), id_ph2, 1u);
                tc_mma_i8_ss(tmem + P_COL + 96u, sdesc(a0 + 2 * TM * 32), sdesc(b0 + PH_OFF3), id_ph3, 1u);
                tc_commit(p_full);
                if (cp.c + 1 == cp.c1) tc_commit(&a_empty_ph[ib]);
                if (++stage == NSTAGE) {
                    stage = 0;
                    sph ^= 1u;
                }
                cursor_next(W, cp);
            }
            // Every issued MMA completes before TMEM is released.
            tc_commit(&done[1]);
            if (!mbar_wait(&done[1], 0)) report(W, 8u);
        }
        __syncwarp();
    } else if (warp == MMA_WARP) {
        // Coil MMAs of every chunk: digit classes into TMEM columns D_COL.
        if (lane == 0) {
            constexpr uint32_t id_c3 = idesc_i8(3 * N, false, true);
            constexpr uint32_t id_c2 = idesc_i8(2 * N, false, true);
            constexpr uint32_t id_c1 = idesc_i8(N, true, true);  // signed low digit of M
            int stage = 0, gc = 0;
            uint32_t sph = 0;
            for (Cursor cc = cursor_start(W); cc.valid; ++gc) {
                if (!mbar_wait_helper(&full[stage], sph) || !mbar_wait_helper(a_full, (uint32_t)(gc & 1)) ||
                    (cc.c == cc.c0 && !mbar_wait_helper(d_empty, (uint32_t)(cc.local & 1)))) {
                    report(W, 4u);
                    break;
                }
                tc_fence_after();
                const uint32_t b0 = smem_u32(sStage + (size_t)stage * STAGE_BYTES);
#pragma unroll
                for (int ks = 0; ks < 2; ++ks) {
                    const uint64_t bd = sdesc(b0 + (uint32_t)(ks * 3 * N * 32));
                    const uint32_t acol = tmem + A_COL + (uint32_t)(ks * 32);
                    tc_mma_i8_ts(tmem + D_COL, acol, bd, id_c3, 1u);                            // d3 x [c2|c1|c0]
                    tc_mma_i8_ts(tmem + D_COL + (uint32_t)N, acol + 8u, bd, id_c3, 1u);        // d2 x [c2|c1|c0]
                    tc_mma_i8_ts(tmem + D_COL + (uint32_t)(2 * N), acol + 16u, bd, id_c2, 1u);  // d1 x [c2|c1]
                    tc_mma_i8_ts(tmem + D_COL + (uint32_t)(3 * N), acol + 24u, bd, id_c1, 1u);  // d0 x [c2]
                }
                tc_commit(&empty[stage]);
                if (cc.c + 1 == cc.c1) tc_commit(d_full);
                if (++stage == NSTAGE) {
                    stage = 0;
                    sph ^= 1u;
                }
                cursor_next(W, cc);
            }
            // Every issued MMA completes before TMEM is released.
            tc_commit(&done[0]);
            if (!mbar_wait(&done[0], 0)) report(W, 8u);
        }
        __syncwarp();
    } else {
        // Magnetisation warp: lane quarter q (tile rows 32q + lane), spins 8cq .. 8cq+7.
        const int q = warp & 3, cq = warp >> 2;
        const uint32_t lq = (uint32_t)(q * 32) << 16;
        const int row = q * 32 + lane;
        const int ks = cq >> 1;
        // Amplitude scale of the segment: M is formed as M / 2^eA (log2|m0| - eA
        // comes with the spin parameters, so the ex2 argument stays small and
        // its float rounding near 2^-24 relative); the top digits carry M to
        // 2^-22 and the low digit the next 8 bits.
        // Clear the coil classes (completion 0 of d_empty releases the first item).
        {
            const uint32_t z[4] = {0u, 0u, 0u, 0u};
#pragma unroll
            for (int t = 0; t < 4; ++t)
#pragma unroll
                for (int cb = 0; cb < NQ; cb += 4)
                    tmem_st_x4(tmem + lq + D_COL + (uint32_t)(t * N + cq * NQ + cb), z);
            tmem_wait_st();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(d_empty);
        }
        const uint32_t m8 = args.mul8, m16 = args.mul16, m24 = args.mul24;
        const int n_items = W.n_items;
        int g = 0, stage = 0, prev_stage = 0;
        uint32_t sph = 0, prev_sph = 0;
        // Phase classes w = 7..3 (columns (7 - w) * 32) of this warp's 8 spins,
        // loaded for chunk g + 1 once chunk g's A operand is handed over.
        uint32_t pc[PH_CLASSES][8];
        auto wait_all = [&](uint64_t *bar, uint32_t parity) -> bool {
            const bool ok = mbar_wait(bar, parity);
            __syncwarp();
            return __all_sync(0xffffffffu, ok);
        };
        auto load_phase = [&](int gg) -> bool {
            if (!wait_all(p_full, (uint32_t)(gg & 1))) return false;
            tc_fence_after();
#pragma unroll
            for (int t = 0; t < PH_CLASSES; ++t) tmem_ld_x8(tmem + lq + P_COL + (uint32_t)(t * 32 + cq * 8), pc[t]);
            tmem_wait_ld();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(p_empty);
            return true;
        };
        Cursor cu = cursor_start(W);
        if (cu.valid && !load_phase(0)) {
            if (lane == 0) report(W, 16u);
            dead = true;
        }
        for (; cu.valid && !dead; cu.i += gridDim.x, ++cu.local, cursor_item(W, cu)) {
            const KernelJob &J = sjobs[cu.job];
            const uint32_t base = J.rows[2 * ((size_t)cu.tile * TM + row)];
            const float tj = __uint_as_float(J.rows[2 * ((size_t)cu.tile * TM + row) + 1]);
            for (int c = cu.c0; c < cu.c1; ++c, ++g) {
                if (!wait_all(&full[stage], sph)) {
                    if (lane == 0) report(W, 32u);
                    dead = true;
                    break;
                }
                // Spin parameters of this warp's 8 spins: turn of arg(m0), r2, log2|m0| - eA.
                const uint32_t *par =
                    reinterpret_cast<const uint32_t *>(sStage + (size_t)stage * STAGE_BYTES + CB + PHASE_B_BYTES);
                uint32_t th[8], r2b[8], l2b[8];
#pragma unroll
                for (int v = 0; v < 2; ++v) {
                    const uint4 a4 = *reinterpret_cast<const uint4 *>(par + cq * 8 + 4 * v);
                    const uint4 b4 = *reinterpret_cast<const uint4 *>(par + KC + cq * 8 + 4 * v);
                    const uint4 c4 = *reinterpret_cast<const uint4 *>(par + 2 * KC + cq * 8 + 4 * v);
                    th[4 * v] = a4.x, th[4 * v + 1] = a4.y, th[4 * v + 2] = a4.z, th[4 * v + 3] = a4.w;
                    r2b[4 * v] = b4.x, r2b[4 * v + 1] = b4.y, r2b[4 * v + 2] = b4.z, r2b[4 * v + 3] = b4.w;
                    l2b[4 * v] = c4.x, l2b[4 * v + 1] = c4.y, l2b[4 * v + 2] = c4.z, l2b[4 * v + 3] = c4.w;
                }
                const int cur_stage = stage;
                const uint32_t cur_sph = sph;
                if (++stage == NSTAGE) {
                    stage = 0;
                    sph ^= 1u;
                }
                uint32_t wd[4][4];  // digit planes d1, d2, d3 (+64), d0 of spins (2p, 2p+1)
                // In stages over the warp's 8 spins (8 independent operations per step
                // for the schedulers to interleave).
                // u = turn + 2^30 + 128: classes 7, 6, 5 shifted left by 24, 16, 8 bits,
                // class 4 as is, class 3 shifted right (arithmetic) by 8.
                uint32_t u[8];
                float x[8], e[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    uint32_t v = base + th[i] + pc[3][i];
                    v = mad_lo(pc[2][i], m8, v);
                    v = mad_lo(pc[1][i], m16, v);
                    v = mad_lo(pc[0][i], m24, v);
                    u[i] = mad_hi_s(pc[4][i], m24, v);
                }
                // Half-turn reduction: half h = u >> 31 (the sign of M), remainder
                // (u & (2^31 - 1)) - 2^30 to 23 bits (the +128 of u rounds it); the decay
                // argument t r2 + (log2|m0| - eA).
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const uint32_t fb = (mul_hi_u(u[i], m24) & 0x7FFFFFu) | 0x4B000000u;
                    x[i] = __fmaf_rn(__uint_as_float(fb), TWO_PI_2M24, ANGLE_OFFSET);
                    e[i] = fmaf(tj, __uint_as_float(r2b[i]), __uint_as_float(l2b[i]));
                }
                float re[8], im[8], a[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    re[i] = cos_approx(x[i]);
                    im[i] = sin_approx(x[i]);
                    a[i] = __uint_as_float(__float_as_uint(ex2_approx(e[i])) ^ (u[i] & 0x80000000u));
                }
                // 3 + rint(M 2^22) 2^-22 (|M| < 1, so the sum stays in [2, 4) where the
                // float grid is 2^-22): bits 0x40400000 + F for F = rint(M 2^22), bytes
                // 0, 1 the digits d1, d2 and byte 2 the top digit d3 + 64.  The residual
                // M - F 2^-22 (|.| <= 2^-23, exact before its one rounding) gives the
                // signed low digit, byte 0 of MAGIC + rint(residual LOW_DIGIT_SCALE).
                // A spin of zero amplitude gives zero digits (no offset but the top one's).
                uint32_t vre[8], vim[8], lre[8], lim[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const float hre = __fmaf_rn(a[i], re[i], 3.0f);
                    const float him = __fmaf_rn(a[i], im[i], 3.0f);
                    vre[i] = __float_as_uint(hre);
                    vim[i] = __float_as_uint(him);
                    const float rre = __fmaf_rn(a[i], re[i], __fsub_rn(3.0f, hre));
                    const float rim = __fmaf_rn(a[i], im[i], __fsub_rn(3.0f, him));
                    lre[i] = __float_as_uint(__fmaf_rn(rre, LOW_DIGIT_SCALE, MAGIC_1P5_2P23));
                    lim[i] = __float_as_uint(__fmaf_rn(rim, LOW_DIGIT_SCALE, MAGIC_1P5_2P23));
                }
                // K order of a word: (re, im) of spin 2pp, then of spin 2pp+1.
#pragma unroll
                for (int pp = 0; pp < 4; ++pp) {
                    const uint32_t p0 = prmt(vre[2 * pp], vim[2 * pp], 0x5140u), p1 = prmt(vre[2 * pp + 1], vim[2 * pp + 1], 0x5140u);
                    const uint32_t q0 = prmt(vre[2 * pp], vim[2 * pp], 0x6262u), q1 = prmt(vre[2 * pp + 1], vim[2 * pp + 1], 0x6262u);
                    const uint32_t r0 = prmt(lre[2 * pp], lim[2 * pp], 0x5140u), r1 = prmt(lre[2 * pp + 1], lim[2 * pp + 1], 0x5140u);
                    wd[0][pp] = prmt(p0, p1, 0x5410u);
                    wd[1][pp] = prmt(p0, p1, 0x7632u);
                    wd[2][pp] = prmt(q0, q1, 0x5410u);
                    wd[3][pp] = prmt(r0, r1, 0x5410u);
                }
                // Hand the A operand to the coil issuer (once the previous chunk's coil
                // MMAs, which read the buffer, are complete), then take the next
                // chunk's phase classes.
                if (g > 0 && !wait_all(&empty[prev_stage], prev_sph)) {
                    if (lane == 0) report(W, 128u);
                    dead = true;
                    break;
                }
                prev_stage = cur_stage;
                prev_sph = cur_sph;
                tc_fence_after();
                const uint32_t acol = tmem + lq + A_COL + (uint32_t)(ks * 32 + 4 * (cq & 1));
                tmem_st_x4(acol, wd[2]);        // d3 + 64
                tmem_st_x4(acol + 8u, wd[1]);   // d2
                tmem_st_x4(acol + 16u, wd[0]);  // d1
                tmem_st_x4(acol + 24u, wd[3]);  // d0
                tmem_wait_st();
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(a_full);
                const bool more = c + 1 < cu.c1 || cu.i + (int)gridDim.x < n_items;
                if (more && !load_phase(g + 1)) {
                    if (lane == 0) report(W, 16u);
                    dead = true;
                    break;
                }
            }
            if (dead) break;
            // Item end: the coil classes of this warp's rows and columns, one
            // integer per element, added into the tile's accumulator (the lanes'
            // rows are consecutive there), then cleared for the next item.
            if (!wait_all(d_full, (uint32_t)(cu.local & 1))) {
                if (lane == 0) report(W, 512u);
                dead = true;
                break;
            }
            tc_fence_after();
            unsigned long long *dst =
                J.acc + (((size_t)cu.tile * acc_slots(J.n_chunks) + (cu.c0 >> ACC_SLOT_LOG2)) * N + cq * NQ) * TM + row;
            const uint32_t z[4] = {0u, 0u, 0u, 0u};
#pragma unroll
            for (int cb = 0; cb < NQ; cb += 4) {
                uint32_t t5[4], t4[4], t3[4], t2[4];
                const uint32_t col = tmem + lq + D_COL + (uint32_t)(cq * NQ + cb);
                tmem_ld_x4(col, t5);
                tmem_ld_x4(col + (uint32_t)N, t4);
                tmem_ld_x4(col + (uint32_t)(2 * N), t3);
                tmem_ld_x4(col + (uint32_t)(3 * N), t2);
                tmem_wait_ld();
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    // classes in units of 2^16 (|sum| < 2^55 over an item: exact in int64)
                    const long long s = ((long long)(int32_t)t5[e] << 24) + ((long long)(int32_t)t4[e] << 16) +
                                        ((long long)(int32_t)t3[e] << 8) + (long long)(int32_t)t2[e];
                    atomicAdd(dst + (size_t)(cb + e) * TM, (unsigned long long)s);
                }
#pragma unroll
                for (int t = 0; t < 4; ++t) tmem_st_x4(col + (uint32_t)(t * N), z);
            }
            tmem_wait_st();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(d_empty);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == MMA_WARP) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// Per (sample, column): the accumulator's integer less the offset of the top
// magnetisation digit (64 * 2^24 times the column's sensitivity integers:
// colsum * 2^14 in the accumulator's units of 2^16), exact in int64 for one
// slot and rounded once to FP64 (several slots: each rounded, summed in slot
// order); then the rotation by -angle_offset_error() (the constant offset of
// the kernel's angles), the power-of-two scales of the operands undone, and
// complex samples written: column n < ncg is Re S(j, coil0 + n), ncg <= n <
// 2 ncg is Im.  The accumulator is left zero for the next launch.
template <typename T>
__global__ void __launch_bounds__(256) split_finalize_kernel(unsigned long long *acc, int64_t nsamples, int32_t ncg,
                                                             int n_cols, int nacc, const long long *colsum,
                                                             const int *coil_exp,
                                                             const unsigned long long *amp_max, cplx<T> *sig,
                                                             int64_t ldsig) {
    // A block takes FIN_ROWS rows x n_cols columns of one time tile (the
    // accumulator's rows are contiguous per column: coalesced), then writes
    // every coil's samples of those rows from shared memory.
    constexpr int FIN_ROWS = 32, PER = FIN_ROWS * 64 / 256;
    __shared__ double sacc[FIN_ROWS * 64];
    const int ea = amp_exp(*amp_max);
    double rs, rc;
    sincos(-angle_offset_error(), &rs, &rc);
    const int64_t tiles = (nsamples + TM - 1) / TM;
    const int64_t units = tiles * (TM / FIN_ROWS);
    const int elems = FIN_ROWS * n_cols;  // n_cols <= 64
    for (int64_t u = blockIdx.x; u < units; u += gridDim.x) {
        const int64_t tile = u / (TM / FIN_ROWS);
        const int r0 = (int)(u % (TM / FIN_ROWS)) * FIN_ROWS;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int e = threadIdx.x + k * 256;
            if (e < elems) {
                const int col = e / FIN_ROWS, row = e % FIN_ROWS;
                unsigned long long *src = acc + ((size_t)tile * nacc * n_cols + col) * TM + r0 + row;
                double v;
                if (nacc == 1) {
                    // at most 2^23 + 2^13 spins: |colsum| < 2^46, the offset and the
                    // difference fit in int64
                    v = (double)((long long)*src - colsum[col] * (1ll << 14));
                    *src = 0ull;
                } else {
                    // more spins: the offset in FP64 (colsum 2^14 can leave int64)
                    v = -ldexp((double)colsum[col], 14);
                    for (int z = 0; z < nacc; ++z) {
                        unsigned long long *p = src + (size_t)z * n_cols * TM;
                        v += (double)(long long)*p;
                        *p = 0ull;
                    }
                }
                sacc[col * FIN_ROWS + row] = v;
            }
        }
        __syncthreads();
        for (int q = threadIdx.x; q < FIN_ROWS * ncg; q += blockDim.x) {
            const int c = q / FIN_ROWS, row = q % FIN_ROWS;
            const int64_t j = tile * TM + r0 + row;
            if (j < nsamples) {
                // undo the scales: M's integers are M 2^(30 - e_A), the
                // sensitivities' c 2^(23 - e_c) 127/128, the accumulator's unit 2^16
                const int e = coil_exp[c] + ea - 37;
                const double re = sacc[c * FIN_ROWS + row], im = sacc[(ncg + c) * FIN_ROWS + row];
                sig[j + (int64_t)c * ldsig] =
                    cplx<T>{T(ldexp(re * rc - im * rs, e) * (128.0 / 127.0)), T(ldexp(re * rs + im * rc, e) * (128.0 / 127.0))};
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

// Coefficient of phase term `slot` of spin s: basis term slot + 1, or dw/(2 pi).
__device__ __forceinline__ double term_coef(const double *basis, const double *dw, int64_t s, int slot) {
    return slot < NSLOT - 1 ? basis[s * 16 + slot + 1] : dw[s] * (1.0 / (2.0 * 3.141592653589793));
}

// Largest |coefficient| of every phase term over the spins (bits of
// non-negative doubles, combined with an unsigned max).
__global__ void term_max_kernel(const double *basis, const double *dw, int64_t ns, unsigned long long *mx) {
    __shared__ unsigned long long smax[NSLOT];
    if (threadIdx.x < NSLOT) smax[threadIdx.x] = 0ull;
    __syncthreads();
    unsigned long long local[NSLOT];
#pragma unroll
    for (int k = 0; k < NSLOT; ++k) local[k] = 0ull;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < ns; s += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < NSLOT; ++k)
            local[k] = max(local[k], (unsigned long long)__double_as_longlong(fabs(term_coef(basis, dw, s, k))));
#pragma unroll
    for (int k = 0; k < NSLOT; ++k) atomicMax(&smax[k], local[k]);
    __syncthreads();
    if (threadIdx.x < NSLOT && smax[threadIdx.x]) atomicMax(&mx[threadIdx.x], smax[threadIdx.x]);
}

// Phase B operand of every chunk: per spin the five balanced digits of
// B_k = rint(b_k 2^38 / bmax_k) for the 16 terms (16 bytes per digit), placed
// as the B' rows of the three phase MMAs (class block w, spin s):
//   MMA 1: row (7 - w) 32 + s, K halves digits (w - 4, w - 3), w = 7..3
//   MMA 2: row (6 - w) 32 + s, K halves digits (w - 2, w - 1), w = 6..3
//   MMA 3: row (4 - w) 32 + s, K halves digits (w, none),      w = 4..3
// with zeros where the digit index is outside 0..4 and for padding spins.
__global__ void phase_b_kernel(const double *basis, const double *dw, int64_t ns, int64_t nchunks,
                               const unsigned long long *term_max, uint8_t *out) {
    const int64_t total = nchunks * KC;
    for (int64_t gs = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; gs < total;
         gs += (int64_t)gridDim.x * blockDim.x) {
        const int64_t chunk = gs / KC;
        const int s = (int)(gs % KC);
        uint32_t dig[PHASE_DIGITS][4];  // digit d of the 16 terms, 4 bytes per word
#pragma unroll
        for (int d = 0; d < PHASE_DIGITS; ++d)
#pragma unroll
            for (int w = 0; w < 4; ++w) dig[d][w] = 0u;
        if (gs < ns) {
            for (int k = 0; k < NSLOT; ++k) {
                const double bmax = __longlong_as_double((long long)term_max[k]);
                long long v = 0;
                if (bmax > 0.0) v = llrint(ldexp(term_coef(basis, dw, gs, k) / bmax, 38));
                for (int d = 0; d < PHASE_DIGITS; ++d) {
                    long long dd;
                    if (d < PHASE_DIGITS - 1) {
                        dd = ((v + 128) & 255) - 128;
                        v = (v - dd) >> 8;
                    } else {
                        dd = v;
                    }
                    dig[d][k >> 2] |= ((uint32_t)dd & 0xFFu) << (8 * (k & 3));
                }
            }
        }
        uint8_t *base = out + (size_t)chunk * PHASE_B_BYTES;
        auto put = [&](int off, int row, int kc, int d) {
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (d >= 0 && d < PHASE_DIGITS) v = make_uint4(dig[d][0], dig[d][1], dig[d][2], dig[d][3]);
            *reinterpret_cast<uint4 *>(base + off + kmaj(row, kc * 16)) = v;
        };
        for (int w = 7; w >= 3; --w) {
            put(0, (7 - w) * 32 + s, 0, w - 4);
            put(0, (7 - w) * 32 + s, 1, w - 3);
        }
        for (int w = 6; w >= 3; --w) {
            put(PH_OFF2, (6 - w) * 32 + s, 0, w - 2);
            put(PH_OFF2, (6 - w) * 32 + s, 1, w - 1);
        }
        for (int w = 4; w >= 3; --w) {
            put(PH_OFF3, (4 - w) * 32 + s, 0, w);
            put(PH_OFF3, (4 - w) * 32 + s, 1, -1);
        }
    }
}

// Largest |Re| or |Im| of each coil's sensitivities, as the bits of a
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

// Scale of a coil's sensitivities: 2^(23 - e_coil) 127/128, so that the
// integers stay within 127 2^16 and their top balanced digit within [-127,
// 127] (2^-23 relative precision; undone exactly by the finalize's 128/127).
__host__ __device__ inline double coil_scale(int e_coil) { return ldexp(127.0 / 128.0, 23 - e_coil); }

// Sensitivity integer of output column n (coil group coil0, ncg coils) for
// component comp of M (0: Re M, 1: Im M) of spin sp: Re S = sum Re M Re c -
// Im M Im c (column n < ncg), Im S = sum Re M Im c + Im M Re c (column ncg + n),
// each sensitivity times coil_scale.
__device__ __forceinline__ long long coil_int(const cplx<double> *csm_rows, int64_t ns, int32_t nc, int coil0,
                                              int ncg, const int *coil_exp, int n, int comp, int64_t sp) {
    if (sp >= ns || n >= 2 * ncg) return 0;
    const int coil = coil0 + (n < ncg ? n : n - ncg);
    const cplx<double> cv = csm_rows[sp * nc + coil];
    const double v = n < ncg ? (comp == 0 ? cv.re : -cv.im) : (comp == 0 ? cv.im : cv.re);
    return llrint(v * coil_scale(coil_exp[coil]));
}

// Coil B operand per coil group and chunk: K-step ks (spins 16 ks .. +15,
// K byte 2 s + comp), rows [c2 | c1 | c0] x n_cols of the balanced digits of
// the sensitivity integers.  One thread builds one 16-byte piece (one operand
// row, one half of the K-step: 8 spins x (re, im)).
__global__ void coil_b_kernel(const cplx<double> *csm_rows, int64_t ns, int32_t nc, int n_cols, int64_t nchunks,
                              int ngroups, const int *coil_exp, uint8_t *out) {
    const int rows = 3 * n_cols;
    const int64_t total = (int64_t)ngroups * nchunks * 2 * rows * 2;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = i;
        const int kc = (int)(r & 1);
        r >>= 1;
        const int row = (int)(r % rows);
        r /= rows;
        const int ks = (int)(r & 1);
        const int64_t gc = r >> 1;  // group * nchunks + chunk
        const int grp = (int)(gc / nchunks);
        const int64_t chunk = gc % nchunks;
        const int digit = 2 - row / n_cols;  // rows c2, c1, c0
        const int n = row % n_cols;
        const int coil0 = grp * GROUP_COILS;
        const int ncg = min(GROUP_COILS, nc - coil0);
        uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int b = 0; b < 16; ++b) {
            const int kbyte = kc * 16 + b;
            const int64_t sp = chunk * KC + ks * 16 + (kbyte >> 1);
            const long long v = coil_int(csm_rows, ns, nc, coil0, ncg, coil_exp, n, kbyte & 1, sp);
            const int d = balanced_digit(v, digit, 3);
            w[b >> 2] |= ((uint32_t)d & 0xFFu) << (8 * (b & 3));
        }
        uint8_t *base = out + (size_t)gc * coil_b_bytes(n_cols) + (size_t)ks * rows * 32;
        *reinterpret_cast<uint4 *>(base + kmaj(row, kc * 16)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// Per coil group and output column: the sum over all spins and both
// components of the sensitivity integers (exact int64; colsum zeroed first).
// A grid-stride pass over the spin-major rows (coalesced); each block sums
// into shared int64 counters, then adds them to colsum.  Integer sums do not
// depend on the order, so the result is exact and reproducible.
__global__ void colsum_kernel(const cplx<double> *csm_rows, int64_t ns, int32_t nc, int n_cols, const int *coil_exp,
                              unsigned long long *colsum) {
    extern __shared__ unsigned long long csum[];  // ngroups * n_cols
    const int ngroups = (nc + GROUP_COILS - 1) / GROUP_COILS;
    for (int i = threadIdx.x; i < ngroups * n_cols; i += blockDim.x) csum[i] = 0ull;
    __syncthreads();
    const int64_t total = ns * nc;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int coil = (int)(i % nc);
        const int grp = coil / GROUP_COILS, c = coil - grp * GROUP_COILS;
        const int ncg = min(GROUP_COILS, nc - grp * GROUP_COILS);
        const cplx<double> cv = csm_rows[i];
        const double sc = coil_scale(coil_exp[coil]);
        // the terms of coil_int: column c is Re c (Re M) + (-Im c) (Im M), column ncg + c is Im c + Re c
        const long long re = llrint(cv.re * sc), im = llrint(cv.im * sc), mim = llrint(-cv.im * sc);
        atomicAdd(&csum[grp * n_cols + c], (unsigned long long)(re + mim));
        atomicAdd(&csum[grp * n_cols + ncg + c], (unsigned long long)(im + re));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < ngroups * n_cols; i += blockDim.x)
        if (csum[i]) atomicAdd(&colsum[i], csum[i]);
}

// Per-segment spin parameters of every chunk, [turn of arg(m0) x 32 | r2 x 32
// | l2 x 32]: the initial phase as a 32-bit turn fraction, -log2(e)/T2 and
// log2|m0| (float; l2_shift_kernel then subtracts the segment's amplitude
// exponent); also the largest |m0| (amplitude scale of the segment).
__global__ void spin_params_kernel(const double *T2, const cplx<double> *xy, int64_t ns, int64_t nchunks,
                                   unsigned long long *amp_max, uint32_t *params) {
    const int64_t total = nchunks * KC;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < total;
         s += (int64_t)gridDim.x * blockDim.x) {
        uint32_t *p = params + (s / KC) * (PARAM_BYTES / 4);
        const int sl = (int)(s % KC);
        uint32_t th = 0u;
        float r2 = 0.0f, l2 = -INFINITY;
        unsigned long long amp = 0ull;
        if (s < ns) {
            const cplx<double> m0 = xy[s];
            const double mag = hypot(m0.re, m0.im);
            const double t0 = atan2(m0.im, m0.re) * (1.0 / (2.0 * 3.141592653589793));
            th = (uint32_t)(unsigned long long)llrint(ldexp(t0 - floor(t0), 32));
            r2 = (float)(-1.4426950408889634 / T2[s]);
            l2 = mag > 0.0 ? (float)log2(mag) : -INFINITY;
            amp = (unsigned long long)__double_as_longlong(mag);
        }
        // One atomic per warp for the amplitude maximum.
        const unsigned active = __activemask();
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long other = __shfl_xor_sync(active, amp, o);
            if ((active >> ((threadIdx.x & 31) ^ o)) & 1u) amp = max(amp, other);
        }
        if ((threadIdx.x & 31) == __ffs(active) - 1 && amp) atomicMax(amp_max, amp);
        p[sl] = th;
        p[KC + sl] = __float_as_uint(r2);
        p[2 * KC + sl] = __float_as_uint(l2);
    }
}

// log2|m0| - eA of every spin of the segment (eA = amp_exp of the largest
// |m0|), so that the magnetisation warps' ex2 argument t r2 + l2 stays small.
__global__ void l2_shift_kernel(uint32_t *params, int64_t nchunks, const unsigned long long *amp_max) {
    const float ea = (float)amp_exp(*amp_max);
    const int64_t total = nchunks * KC;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < total;
         s += (int64_t)gridDim.x * blockDim.x) {
        uint32_t *p = params + (s / KC) * (PARAM_BYTES / 4) + 2 * KC + (s % KC);
        *p = __float_as_uint(__uint_as_float(*p) - ea);
    }
}

// Prefix table of one segment, over blocks (column, part): columns 0..16 are
// kappa_k, the scaled running trapezoid sums (f(n)+f(n+1)) dt(n), written at
// every ADC node (row = sample index) and at the end node (row nsamples), with
// the column's largest |value| at row nsamples+1; column 17 is the elapsed
// time t (entry PREFIX_T) and the constant columns 17 (= 1) and 18, 19 (= 0).
// A column's intervals are cut into PREFIX_PARTS contiguous parts, and a
// part into one contiguous run per thread.  Every sum is taken in a fixed
// order (within a run, runs in thread order, parts in part order), so the
// table does not depend on timing.  Two launches: the part totals
// (prefix_part_kernel, into rows nsamples+2 ..), then the scan itself
// (prefix_kernel), each part starting from the sum of the parts before it.
constexpr int PREFIX_PARTS = 8;
constexpr int PREFIX_COLS = 18;
struct PrefixColumn {
    const double *f;
    bool one, zero;
    double scale;
    int out_col;
};
__device__ __forceinline__ PrefixColumn prefix_column(const double *const *src, int col, double gamma) {
    PrefixColumn c;
    c.f = col < 17 ? src[col] : reinterpret_cast<const double *>(1);  // nullptr: zero; 1: constant one
    c.one = c.f == reinterpret_cast<const double *>(1);
    c.zero = c.f == nullptr;
    c.scale = col < 16 ? -gamma * 0.5 : (col == 16 ? -0.5 : 0.5);
    c.out_col = col < 17 ? col : PREFIX_T;
    return c;
}
__device__ __forceinline__ double prefix_term(const PrefixColumn &c, const double *dt, int64_t n) {
    return c.zero ? 0.0 : (c.one ? 2.0 : (c.f[n] + c.f[n + 1])) * dt[n];
}
// This thread's run [i0, i1) of part `part` of nint intervals.
__device__ __forceinline__ void prefix_run(int64_t nint, int part, int64_t &i0, int64_t &i1) {
    const int64_t p0 = nint * part / PREFIX_PARTS, p1 = nint * (part + 1) / PREFIX_PARTS;
    const int64_t per = (p1 - p0 + blockDim.x - 1) / blockDim.x;
    i0 = min(p1, p0 + per * threadIdx.x);
    i1 = min(p1, i0 + per);
}
// Sum of the runs' values in thread order (thread 0), and each run's exclusive
// prefix in part[].
__device__ double block_exclusive(double *part, double local) {
    part[threadIdx.x] = local;
    __syncthreads();
    __shared__ double total;
    if (threadIdx.x == 0) {
        double run = 0.0;
        for (int i = 0; i < (int)blockDim.x; ++i) {
            const double v = part[i];
            part[i] = run;
            run += v;
        }
        total = run;
    }
    __syncthreads();
    return total;
}

__global__ void prefix_part_kernel(const double *dt, const double *const *src, int64_t n_lo, int64_t n_hi,
                                   int64_t nsamples, double gamma, double *prefix) {
    __shared__ double part[256];
    const int col = blockIdx.x, pt = blockIdx.y;
    const PrefixColumn c = prefix_column(src, col, gamma);
    int64_t i0, i1;
    prefix_run(n_hi - n_lo, pt, i0, i1);
    double local = 0.0;
    for (int64_t i = i0; i < i1; ++i) local += prefix_term(c, dt, n_lo + i);
    const double total = block_exclusive(part, local);
    if (threadIdx.x == 0) {
        prefix[(size_t)(nsamples + 2 + pt) * PREFIX_STRIDE + col] = total;
        if (pt == 0 && col < 17) prefix[(size_t)(nsamples + 1) * PREFIX_STRIDE + col] = 0.0;  // the maximum, below
    }
}

__global__ void prefix_kernel(const double *dt, const double *const *src, const uint8_t *adc, const int32_t *rank,
                              int64_t rank_base, int64_t n_lo, int64_t n_hi, int64_t nsamples, double gamma,
                              double *prefix) {
    __shared__ double part[256];
    const int col = blockIdx.x, pt = blockIdx.y;
    const PrefixColumn c = prefix_column(src, col, gamma);
    const int64_t nint = n_hi - n_lo;
    int64_t i0, i1;
    prefix_run(nint, pt, i0, i1);
    double carry = 0.0;
    for (int q = 0; q < pt; ++q) carry += prefix[(size_t)(nsamples + 2 + q) * PREFIX_STRIDE + col];
    double local = 0.0;
    for (int64_t i = i0; i < i1; ++i) local += prefix_term(c, dt, n_lo + i);
    block_exclusive(part, local);
    double cum = carry + part[threadIdx.x];
    double peak = 0.0;
    for (int64_t i = i0; i < i1; ++i) {
        const int64_t n = n_lo + i;
        cum += prefix_term(c, dt, n);
        peak = fmax(peak, fabs(c.scale * cum));
        if (adc[n + 1]) {
            double *pr = prefix + (size_t)(rank[n + 1] - rank_base) * PREFIX_STRIDE;
            pr[c.out_col] = c.scale * cum;
            if (col == 17) {
                pr[17] = 1.0;
                pr[18] = 0.0;
                pr[19] = 0.0;
            }
        }
        if (n + 1 == n_hi) {
            double *pr = prefix + (size_t)nsamples * PREFIX_STRIDE;
            pr[c.out_col] = c.scale * cum;
            if (col == 17) {
                pr[17] = 1.0;
                pr[18] = 0.0;
                pr[19] = 0.0;
            }
        }
    }
    if (nint == 0 && pt == 0 && threadIdx.x == 0) {
        double *pr = prefix + (size_t)nsamples * PREFIX_STRIDE;
        pr[c.out_col] = 0.0;
        if (col == 17) {
            pr[17] = 1.0;
            pr[18] = 0.0;
            pr[19] = 0.0;
        }
    }
    // Largest |kappa| of the column (row nsamples+1) for the phase-range check:
    // the block's maximum, then the parts' by an integer maximum of the bits
    // (the values are non-negative, so their bits order as they do).
    __syncthreads();
    part[threadIdx.x] = peak;
    __syncthreads();
    if (threadIdx.x == 0 && col < 17) {
        double mx = 0.0;
        for (int i = 0; i < (int)blockDim.x; ++i) mx = fmax(mx, part[i]);
        atomicMax(reinterpret_cast<unsigned long long *>(prefix + (size_t)(nsamples + 1) * PREFIX_STRIDE + col),
                  (unsigned long long)__double_as_longlong(mx));
    }
}

// Phase A operand of every tile of a segment and the per-sample rows: for
// sample j the integers K_k(j) = rint(kappa_k(j) bmax_k 2^26) of the 16 terms
// as five balanced digits, placed as the A' tiles [a4|a3], [a2|a1], [a0|0]
// (row j % 128 of tile j / 128), the base turn rint(frac(kappa_0) 2^32) +
// 2^30 + 128 (quarter-turn offset and the rounding of the 23-bit angle) and
// the elapsed time.  Rows past nsamples are zero.  Sets error bit 64 when a
// term's range bmax_k max|kappa_k| exceeds PHASE_RANGE_LIMIT turns.
__global__ void phase_a_kernel(const double *prefix, int64_t nsamples, int64_t nrows,
                               const unsigned long long *term_max, unsigned int *err, uint8_t *phase_a,
                               uint32_t *rows) {
    const double *kmax = prefix + (size_t)(nsamples + 1) * PREFIX_STRIDE;
    if (blockIdx.x == 0 && threadIdx.x < NSLOT) {
        const double bmax = __longlong_as_double((long long)term_max[threadIdx.x]);
        if (!(bmax * kmax[threadIdx.x + 1] <= PHASE_RANGE_LIMIT)) atomicOr(err, 64u);
    }
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nrows;
         j += (int64_t)gridDim.x * blockDim.x) {
        uint32_t dig[PHASE_DIGITS][4];
#pragma unroll
        for (int d = 0; d < PHASE_DIGITS; ++d)
#pragma unroll
            for (int w = 0; w < 4; ++w) dig[d][w] = 0u;
        uint32_t base = 0x40000080u;
        float tj = 0.0f;
        if (j < nsamples) {
            const double *pr = prefix + (size_t)j * PREFIX_STRIDE;
            for (int k = 0; k < NSLOT; ++k) {
                const double bmax = __longlong_as_double((long long)term_max[k]);
                // |K| <= 2^38 is checked above; clamp so a failed check cannot overflow
                const double kv = fmin(fmax(ldexp(pr[k + 1] * bmax, 26), -2.7e11), 2.7e11);
                long long v = llrint(kv);
                for (int d = 0; d < PHASE_DIGITS; ++d) {
                    long long dd;
                    if (d < PHASE_DIGITS - 1) {
                        dd = ((v + 128) & 255) - 128;
                        v = (v - dd) >> 8;
                    } else {
                        dd = v;
                    }
                    dig[d][k >> 2] |= ((uint32_t)dd & 0xFFu) << (8 * (k & 3));
                }
            }
            const double k0 = pr[0];
            base += (uint32_t)(unsigned long long)llrint(ldexp(k0 - floor(k0), 32));
            tj = (float)pr[PREFIX_T];
        }
        const int64_t tile = j / TM;
        const int r = (int)(j % TM);
        uint8_t *t = phase_a + (size_t)tile * PHASE_A_BYTES;
        auto put = [&](int m, int kc, int d) {
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (d >= 0) v = make_uint4(dig[d][0], dig[d][1], dig[d][2], dig[d][3]);
            *reinterpret_cast<uint4 *>(t + m * TM * 32 + kmaj(r, kc * 16)) = v;
        };
        put(0, 0, 4);
        put(0, 1, 3);
        put(1, 0, 2);
        put(1, 1, 1);
        put(2, 0, 0);
        put(2, 1, -1);
        rows[2 * j] = base;
        rows[2 * j + 1] = __float_as_uint(tj);
    }
}

// Final state of a segment in FP64: Mxy = |m0| e^{-T/T2} cis(2 pi theta_end),
// Mz = Mz e^{-T/T1} + rho (1 - e^{-T/T1}).
__global__ void state_update_kernel(const double *basis, const double *dw, const double *endrow, const double *T1,
                                    const double *T2, const double *rho, int64_t ns, cplx<double> *xy, double *mz) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < ns; s += (int64_t)gridDim.x * blockDim.x) {
        const cplx<double> m0 = xy[s];
        double th = fma(dw[s] * (1.0 / (2.0 * 3.141592653589793)), endrow[16],
                        atan2(m0.im, m0.re) * (1.0 / (2.0 * 3.141592653589793)));
        for (int k = 0; k < 16; ++k) th = fma(basis[s * 16 + k], endrow[k], th);
        const double T = endrow[PREFIX_T];
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

double split_bytes_per_spin(int32_t ncoils) {
    const int ngroups = (ncoils + GROUP_COILS - 1) / GROUP_COILS;
    const int ncg_max = std::min<int32_t>(ncoils, GROUP_COILS);
    const int n_cols = std::max(16, ((2 * ncg_max + 15) / 16) * 16);
    return 128.0 + (double)PHASE_B_BYTES / KC + (double)ngroups * coil_b_bytes(n_cols) / KC + PARAM_BYTES / KC;
}

SplitResident::~SplitResident() {
    for (void *p : {params, prefix, phase_a, rows, accum, amp, err})
        if (p) cudaFree(p);
    if (!phantom_view)
        for (void *p : {basis, phase_b, coil_b, colsum, term_max, coil_exp})
            if (p) cudaFree(p);
}

// Forget shared phantom operands (owned elsewhere) so that they are rebuilt.
static void split_detach(SplitResident &r) {
    if (!r.phantom_view) return;
    r.basis = r.phase_b = r.coil_b = r.colsum = r.term_max = r.coil_exp = nullptr;
    r.basis_bytes = r.phase_b_bytes = r.coil_b_bytes = r.colsum_bytes = r.term_max_bytes = r.coil_exp_bytes = 0;
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
    if ((e = grow(r.phase_b, r.phase_b_bytes, (size_t)PHASE_B_BYTES * (size_t)nchunks)) != cudaSuccess) return e;
    if ((e = grow(r.coil_b, r.coil_b_bytes, (size_t)coil_b_bytes(n_cols) * (size_t)nchunks * ngroups)) != cudaSuccess)
        return e;
    if ((e = grow(r.colsum, r.colsum_bytes, sizeof(long long) * (size_t)n_cols * ngroups)) != cudaSuccess) return e;
    if ((e = grow(r.term_max, r.term_max_bytes, sizeof(unsigned long long) * NSLOT)) != cudaSuccess) return e;
    // Per-coil scale exponents, preceded by the per-coil maxima they come from.
    if ((e = grow(r.coil_exp, r.coil_exp_bytes, (sizeof(unsigned long long) + sizeof(int)) * (size_t)nc)) !=
        cudaSuccess)
        return e;
    if (!r.amp && (e = cudaMalloc(&r.amp, sizeof(unsigned long long))) != cudaSuccess) return e;
    if (!r.err && (e = cudaMalloc(&r.err, sizeof(unsigned int))) != cudaSuccess) return e;
    unsigned long long *cmax = reinterpret_cast<unsigned long long *>(r.coil_exp);
    int *cexp = reinterpret_cast<int *>(cmax + nc);
    basis_kernel<<<grid_for(ns), 256, 0, stream>>>((const double *)x, (const double *)y, (const double *)z, ns,
                                                   (double *)r.basis);
    if ((e = cudaMemsetAsync(r.term_max, 0, sizeof(unsigned long long) * NSLOT, stream)) != cudaSuccess) return e;
    term_max_kernel<<<(int)std::max<int64_t>(1, std::min<int64_t>((ns + 255) / 256, 148 * 4)), 256, 0, stream>>>(
        (const double *)r.basis, (const double *)dw, ns, (unsigned long long *)r.term_max);
    phase_b_kernel<<<grid_for(r.ns_pad), 256, 0, stream>>>((const double *)r.basis, (const double *)dw, ns, nchunks,
                                                           (const unsigned long long *)r.term_max,
                                                           (uint8_t *)r.phase_b);
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
    const int64_t pieces = (int64_t)ngroups * nchunks * 2 * 3 * n_cols * 2;
    coil_b_kernel<<<grid_for(pieces), 256, 0, stream>>>((const cplx<double> *)csm_rows, ns, nc, n_cols, nchunks,
                                                        ngroups, cexp, (uint8_t *)r.coil_b);
    if ((e = cudaMemsetAsync(r.colsum, 0, sizeof(long long) * (size_t)n_cols * ngroups, stream)) != cudaSuccess)
        return e;
    if ((e = allow_max_dynamic_smem((const void *)colsum_kernel)) != cudaSuccess) return e;
    colsum_kernel<<<grid_for(ns * nc), 256, sizeof(unsigned long long) * (size_t)n_cols * ngroups, stream>>>(
        (const cplx<double> *)csm_rows, ns, nc, n_cols, cexp, (unsigned long long *)r.colsum);
    return cudaGetLastError();
}

// Shared memory: 1 KB alignment slack, two phase A tiles, NSTAGE stages, the barriers and the job table.
constexpr size_t SMEM_LIMIT = 227 * 1024;
constexpr size_t SMEM_FIXED = 1024 + 2 * PHASE_A_BYTES + 256 + MAX_JOBS * sizeof(KernelJob);

static size_t stage_bytes(int n_cols) { return (size_t)coil_b_bytes(n_cols) + PHASE_B_BYTES + PARAM_BYTES; }

static int kernel_stages(int n_cols) {
    return (int)std::min<size_t>(MAX_STAGE, (SMEM_LIMIT - SMEM_FIXED) / stage_bytes(n_cols));
}

static size_t kernel_smem(int n_cols) { return SMEM_FIXED + (size_t)kernel_stages(n_cols) * stage_bytes(n_cols); }

// Number of chunk slabs per tile: the smallest that keeps the busiest CTA's
// work (items x (chunks per item + an allowance for the per-item start-up))
// within reach of the best split, with at most MAX_ITEM_CHUNKS chunks per item.
static int choose_slabs(int64_t tiles, int64_t nchunks, int64_t G) {
    const int64_t zmin = std::max<int64_t>(1, (nchunks + MAX_ITEM_CHUNKS - 1) / MAX_ITEM_CHUNKS);
    int best = (int)zmin;
    double best_cost = 1e300;
    const int64_t zmax = std::max<int64_t>(zmin, std::min<int64_t>(nchunks, 4096));
    for (int64_t z = zmin; z <= zmax; ++z) {
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

static int sm_count() {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return nsm;
}

cudaError_t split_launch(const SplitJobDesc *jobs, int n_jobs, cudaStream_t stream) {
    if (n_jobs <= 0) return cudaSuccess;
    if (n_jobs > MAX_JOBS) return cudaErrorInvalidValue;
    const int n_mma = jobs[0].n_mma;
    KernelArgs ka;
    std::memset(&ka, 0, sizeof(ka));
    int64_t items = 0;
    for (int j = 0; j < n_jobs; ++j) {
        const SplitJobDesc &d = jobs[j];
        if (d.n_mma != n_mma) return cudaErrorInvalidValue;
        KernelJob &k = ka.job[j];
        k.phase_a = (const uint8_t *)d.phase_a;
        k.phase_b = (const uint8_t *)d.phase_b;
        k.coil_b = (const uint8_t *)d.coil_b;
        k.params = (const uint8_t *)d.params;
        k.rows = (const uint32_t *)d.rows;
        k.acc = (unsigned long long *)d.accum;
        k.err = d.err;
        k.n_chunks = d.n_chunks;
        k.tiles = d.tiles;
        k.slabs = d.slabs;
        k.item0 = (int)items;
        items += (int64_t)d.tiles * d.slabs;
    }
    if (items > INT32_MAX / 2) return cudaErrorInvalidValue;
    if (items == 0) return cudaSuccess;
    ka.n_jobs = n_jobs;
    ka.n_items = (int)items;
    ka.nstage = kernel_stages(n_mma);
    ka.mul8 = 1u << 8;
    ka.mul16 = 1u << 16;
    ka.mul24 = 1u << 24;
    const int64_t G = std::min<int64_t>(sm_count(), items);
    return launch_precession(n_mma, ka, (unsigned)G, kernel_smem(n_mma), stream);
}

// Prologue of one precession segment: the prefix table, the spin parameters
// and amplitude scale, the phase A tiles and the work-item split.
cudaError_t split_segment_begin(SplitResident &r, const SplitRunArgs &a, int64_t n_lo, int64_t n_hi, int64_t sample0,
                                int64_t nsamples, cudaStream_t stream, std::string *err, SplitSegment *seg) {
    cudaError_t e;
    const int64_t nchunks = r.ns_pad / KC;
    const int64_t tiles = (nsamples + TM - 1) / TM;
    if (!a.grank || !a.src_dev) {
        *err = "internal: split segment without its ADC rank and column tables";
        return cudaSuccess;
    }
    seg->nsamples = nsamples;
    seg->tiles = tiles;
    seg->nchunks = nchunks;
    seg->slabs = 0;
    const size_t prefix_rows = (size_t)std::max<int64_t>(tiles * TM, nsamples + 2 + PREFIX_PARTS);
    if ((e = grow(r.prefix, r.prefix_bytes, prefix_rows * PREFIX_STRIDE * sizeof(double))) != cudaSuccess) return e;
    if ((e = grow(r.params, r.params_bytes, (size_t)nchunks * PARAM_BYTES)) != cudaSuccess) return e;
    // The segment's samples are the global ADC indices sample0 .. sample0 + nsamples - 1.
    const dim3 pgrid(PREFIX_COLS, PREFIX_PARTS);
    prefix_part_kernel<<<pgrid, 256, 0, stream>>>((const double *)a.dt, reinterpret_cast<const double *const *>(a.src_dev),
                                                  n_lo, n_hi, nsamples, a.gamma, (double *)r.prefix);
    prefix_kernel<<<pgrid, 256, 0, stream>>>((const double *)a.dt, reinterpret_cast<const double *const *>(a.src_dev),
                                             (const uint8_t *)a.adc, a.grank, sample0, n_lo, n_hi, nsamples, a.gamma,
                                             (double *)r.prefix);
    if ((e = cudaMemsetAsync(r.amp, 0, sizeof(unsigned long long), stream)) != cudaSuccess) return e;
    spin_params_kernel<<<grid_for(r.ns_pad), 256, 0, stream>>>((const double *)a.T2, (const cplx<double> *)a.xy,
                                                               r.ns, nchunks, (unsigned long long *)r.amp,
                                                               (uint32_t *)r.params);
    l2_shift_kernel<<<grid_for(r.ns_pad), 256, 0, stream>>>((uint32_t *)r.params, nchunks,
                                                            (const unsigned long long *)r.amp);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (a.launches) *a.launches += 4;
    if (nsamples == 0) return cudaSuccess;
    if ((e = grow(r.phase_a, r.phase_a_bytes, (size_t)tiles * PHASE_A_BYTES)) != cudaSuccess) return e;
    if ((e = grow(r.rows, r.rows_bytes, (size_t)tiles * TM * 2 * sizeof(uint32_t))) != cudaSuccess) return e;
    phase_a_kernel<<<grid_for(tiles * TM), 256, 0, stream>>>((const double *)r.prefix, nsamples, tiles * TM,
                                                             (const unsigned long long *)r.term_max,
                                                             (unsigned int *)r.err, (uint8_t *)r.phase_a,
                                                             (uint32_t *)r.rows);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (a.launches) *a.launches += 1;
    const int slabs = choose_slabs(tiles, nchunks, sm_count());
    if (tiles > INT32_MAX / slabs || nchunks > INT32_MAX || slabs > nchunks) {
        *err = "split mode: segment too large for one launch";
        return cudaSuccess;
    }
    seg->slabs = slabs;
    seg->nacc = acc_slots(nchunks);
    // the coil accumulators start at zero (each group's finalize leaves them so)
    const size_t abytes = sizeof(unsigned long long) * (size_t)tiles * seg->nacc * TM * r.n_mma;
    if ((e = grow(r.accum, r.accum_bytes, abytes)) != cudaSuccess) return e;
    return cudaMemsetAsync(r.accum, 0, abytes, stream);
}

SplitJobDesc split_segment_job(const SplitResident &r, const SplitSegment &seg, int grp) {
    SplitJobDesc d;
    d.phase_a = r.phase_a;
    d.phase_b = r.phase_b;
    d.coil_b = (const uint8_t *)r.coil_b + (size_t)grp * seg.nchunks * coil_b_bytes(r.n_mma);
    d.params = r.params;
    d.rows = r.rows;
    d.accum = r.accum;
    d.err = (unsigned int *)r.err;
    d.n_chunks = (int32_t)seg.nchunks;
    d.tiles = (int32_t)seg.tiles;
    d.slabs = seg.slabs;
    d.n_mma = r.n_mma;
    return d;
}

cudaError_t split_segment_finalize(SplitResident &r, const SplitRunArgs &a, const SplitSegment &seg, int grp,
                                   int64_t sample0, cudaStream_t stream) {
    const int coil0 = grp * GROUP_COILS;
    const int ncg = std::min<int>(GROUP_COILS, r.nc - coil0);
    const int *cexp = reinterpret_cast<const int *>(reinterpret_cast<const unsigned long long *>(r.coil_exp) + r.nc);
    const int fin_blocks = (int)std::min<int64_t>(seg.tiles * (TM / 32), 148 * 8);
    if (a.sizeof_T == 8)
        split_finalize_kernel<double><<<fin_blocks, 256, 0, stream>>>(
            (unsigned long long *)r.accum, seg.nsamples, ncg, r.n_mma, seg.nacc,
            (const long long *)r.colsum + (size_t)grp * r.n_mma, cexp + coil0, (const unsigned long long *)r.amp,
            (cplx<double> *)a.sig + sample0 + (int64_t)coil0 * a.nadc, a.nadc);
    return cudaGetLastError();
}

cudaError_t split_segment_end(SplitResident &r, const SplitRunArgs &a, const SplitSegment &seg, cudaStream_t stream) {
    if (a.launches) *a.launches += 1;
    state_update_kernel<<<grid_for(r.ns), 256, 0, stream>>>(
        (const double *)r.basis, (const double *)a.dw, (const double *)r.prefix + (size_t)seg.nsamples * PREFIX_STRIDE,
        (const double *)a.T1, (const double *)a.T2, (const double *)a.rho, r.ns, (cplx<double> *)a.xy,
        (double *)a.mz);
    return cudaGetLastError();
}

cudaError_t split_attach(SplitResident &r, const SplitResident &src) {
    if (&r == &src) return cudaSuccess;
    if (!r.phantom_view) {
        for (void **p : {&r.basis, &r.phase_b, &r.coil_b, &r.colsum, &r.term_max, &r.coil_exp}) {
            if (*p) cudaFree(*p);
            *p = nullptr;
        }
    }
    r.basis = src.basis;
    r.phase_b = src.phase_b;
    r.coil_b = src.coil_b;
    r.colsum = src.colsum;
    r.term_max = src.term_max;
    r.coil_exp = src.coil_exp;
    r.basis_bytes = src.basis_bytes;
    r.phase_b_bytes = src.phase_b_bytes;
    r.coil_b_bytes = src.coil_b_bytes;
    r.colsum_bytes = src.colsum_bytes;
    r.term_max_bytes = src.term_max_bytes;
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

// One precession segment on its own: the prologue, per coil group one launch
// and its finalize, the state update.
cudaError_t split_run_segment(SplitResident &r, const SplitRunArgs &a, int64_t n_lo, int64_t n_hi, int64_t sample0,
                              int64_t nsamples, cudaStream_t stream, std::string *err) {
    SplitSegment seg;
    cudaError_t e = split_segment_begin(r, a, n_lo, n_hi, sample0, nsamples, stream, err, &seg);
    if (e != cudaSuccess || !err->empty()) return e;
    if (nsamples > 0) {
        const unsigned ev_flags = a.capture ? cudaEventRecordExternal : cudaEventRecordDefault;
        if (a.ev_start) cudaEventRecordWithFlags(a.ev_start, stream, ev_flags);
        for (int grp = 0; grp < r.ngroups; ++grp) {
            const SplitJobDesc d = split_segment_job(r, seg, grp);
            e = split_launch(&d, 1, stream);
            if (a.ev_stop && grp + 1 == r.ngroups) cudaEventRecordWithFlags(a.ev_stop, stream, ev_flags);
            if (a.launches) *a.launches += 2;
            if (e != cudaSuccess) return e;
            if ((e = split_segment_finalize(r, a, seg, grp, sample0, stream)) != cudaSuccess) return e;
        }
    }
    return split_segment_end(r, a, seg, stream);
}

cudaError_t split_check(SplitResident &r, cudaStream_t stream, std::string *err) {
    unsigned int h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, r.err, sizeof(h), cudaMemcpyDeviceToHost, stream);
    if (e != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
    if (h & 64u)
        *err = "split mode: a field term's phase range within one precession segment exceeds 4096 turns "
               "(max |basis value| x max |field integral|); run it in plain mode";
    else if (h != 0)
        *err = "split kernel: a bounded device wait timed out (code " + std::to_string(h) + ")";
    return cudaSuccess;
}

}  // namespace homs
