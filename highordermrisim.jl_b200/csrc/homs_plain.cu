// Plain fused kernels of libhoms: free precession and RF excitation in the
// phantom's own precision (FP64 or FP32) on CUDA cores, fused with a
// deterministic multi-coil reduction.  No per-spin ADC history is written to
// HBM: ADC states are staged in shared memory and contracted with the
// receive sensitivities on chip, one CTA partial per (CTA, sample, coil),
// then summed over CTAs in a fixed order.
//
// This translation unit is compiled with -fmad=false so that every product
// and sum rounds exactly as in HighOrderMRISim.jl's CPU path
// (src/simulation/Bloch/BlochHighOrderSimulatitonMethod.jl:43-134), which does
// not contract multiply-adds; the FP64 kernel therefore agrees with the FP64
// CPU restatement to ~1e-15.
#include <cfloat>

#include "homs_common.cuh"

namespace homs {

template <typename T>
struct Math;

template <>
struct Math<double> {
    static __device__ __forceinline__ double ex(double x) { return exp(x); }
    static __device__ __forceinline__ void sc(double x, double *s, double *c) { sincos(x, s, c); }
    static __device__ __forceinline__ double hyp(double a, double b) { return hypot(a, b); }
    static __device__ __forceinline__ double sq(double a) { return sqrt(a); }
    static __device__ __forceinline__ double eps() { return DBL_EPSILON; }
};

template <>
struct Math<float> {
    static __device__ __forceinline__ float ex(float x) { return expf(x); }
    static __device__ __forceinline__ void sc(float x, float *s, float *c) { sincosf(x, s, c); }
    static __device__ __forceinline__ float hyp(float a, float b) { return hypotf(a, b); }
    static __device__ __forceinline__ float sq(float a) { return sqrtf(a); }
    static __device__ __forceinline__ float eps() { return FLT_EPSILON; }
};

// Julia's complex product: (ar*br - ai*bi, ar*bi + ai*br).
template <typename T>
__device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b) {
    return cplx<T>{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}

// Sixteen unnormalised solid harmonics in the CPU expression order
// (BlochHighOrderSimulatitonMethod.jl:54-68).
template <typename T>
__device__ __forceinline__ void basis16(T x, T y, T z, T *b) {
    T x2 = x * x, y2 = y * y, z2 = z * z;
    T r2 = (x2 + y2) + z2;
    b[0] = T(1);
    b[1] = x;
    b[2] = y;
    b[3] = z;
    b[4] = x * y;
    b[5] = z * y;
    b[6] = T(3) * z2 - r2;
    b[7] = x * z;
    b[8] = x2 - y2;
    b[9] = (T(3) * y) * x2 - (y2 * y);
    b[10] = (x * z) * y;
    b[11] = (T(5) * z2 - r2) * y;
    b[12] = T(5) * (z2 * z) - (T(3) * z) * r2;
    b[13] = (T(5) * z2 - r2) * x;
    b[14] = x2 * z - y2 * z;
    b[15] = (x2 * x) - (T(3) * x) * y2;
}

constexpr int NODE_CHUNK = 32;

// Shared-memory node cache for one chunk of nodes [c0, c0 + NODE_CHUNK].
template <typename T>
struct NodeCache {
    T dt[NODE_CHUNK + 1];
    T g[3][NODE_CHUNK + 1];
    T h[16][NODE_CHUNK + 1];
    T df[NODE_CHUNK + 1];
    T psi[NODE_CHUNK + 1];
    cplx<T> b1[NODE_CHUNK + 1];
    T ab1[NODE_CHUNK + 1];  // |B1| of the node (RF segments)
    T dfg[NODE_CHUNK + 1];  // df / gamma of the node (RF segments)
    uint8_t adc[NODE_CHUNK + 1];
    uint8_t bnd[NODE_CHUNK + 1];
};

// Bz at a cached node (BlochHighOrderSimulatitonMethod.jl:70-75).
template <typename T>
__device__ __forceinline__ T field_cached(const NodeCache<T> &nc, int i, const T *b, T dwterm, uint32_t m) {
    T bz0 = (m & HOMS_HO0) ? nc.h[0][i] : T(0);
    T bz1;
    if (m & HOMS_HO1)
        bz1 = (b[1] * nc.h[1][i] + b[2] * nc.h[2][i]) + b[3] * nc.h[3][i];
    else
        bz1 = (b[1] * nc.g[0][i] + b[2] * nc.g[1][i]) + b[3] * nc.g[2][i];
    T bz2 = T(0), bz3 = T(0);
    if (m & HOMS_HO2)
        bz2 = (((b[4] * nc.h[4][i] + b[5] * nc.h[5][i]) + b[6] * nc.h[6][i]) + b[7] * nc.h[7][i]) +
              b[8] * nc.h[8][i];
    if (m & HOMS_HO3)
        bz3 = (((((b[9] * nc.h[9][i] + b[10] * nc.h[10][i]) + b[11] * nc.h[11][i]) + b[12] * nc.h[12][i]) +
                b[13] * nc.h[13][i]) +
               b[14] * nc.h[14][i]) +
              b[15] * nc.h[15][i];
    T bz = ((bz0 + bz1) + bz2) + bz3;
    if (m & HOMS_DW_PRECESSION) bz = bz + dwterm;
    return bz;
}

template <typename T, bool RF>
__device__ void load_nodes(NodeCache<T> &nc, const SeqDev<T> &q, int64_t c0, int64_t c_end, uint32_t m, T gamma) {
    // nodes c0 .. min(c0 + NODE_CHUNK, c_end) inclusive
    const int n = (int)imin64(NODE_CHUNK, c_end - c0) + 1;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        int64_t g = c0 + i;
        nc.dt[i] = (g < q.nnodes - 1) ? q.dt[g] : T(0);
        nc.adc[i] = q.adc[g];
        nc.bnd[i] = q.boundary[g];
        if (RF) {
            nc.g[0][i] = q.gx[g];
            nc.g[1][i] = q.gy[g];
            nc.g[2][i] = q.gz[g];
            const cplx<T> b1 = q.b1[g];
            nc.b1[i] = b1;
            nc.df[i] = q.df[g];
            nc.psi[i] = q.psi[g];
            // Spin-independent parts of the RF step, computed once per node
            // with the same operations as the per-spin code used.
            nc.ab1[i] = Math<T>::hyp(b1.re, b1.im);
            nc.dfg[i] = nc.df[i] / gamma;
        } else {
            if (!(m & HOMS_HO1)) {
                nc.g[0][i] = q.gx[g];
                nc.g[1][i] = q.gy[g];
                nc.g[2][i] = q.gz[g];
            }
#pragma unroll
            for (int k = 0; k < 16; ++k) nc.h[k][i] = q.h[k][g];
        }
    }
}

// Contract `na` staged ADC states X[a][s] (s < PLAIN_THREADS) with the
// sensitivities of this CTA's spins and write one partial row per sample:
// out[a * nc + c] = sum_s X[a][s] * csm[s][c], summed over spins in a fixed
// order (a per-lane sweep, then splits in index order).
template <typename T>
__device__ void reduce_stage(const cplx<T> *X, cplx<T> *P, int na, const cplx<T> *csm_rows, int csm_ld,
                             int nvalid, int32_t nc, cplx<T> *out) {
    const int t = threadIdx.x;
    for (int cg = 0; cg < nc; cg += 32) {
        const int left = min(32, nc - cg);
        int cw = 1;
        while (cw < left) cw <<= 1;
        const int cl = t % cw, split = t / cw;
        const int c = cg + cl;
        cplx<T> acc[PLAIN_STAGE];
#pragma unroll
        for (int a = 0; a < PLAIN_STAGE; ++a) acc[a] = cplx<T>{T(0), T(0)};
        if (cl < left) {
            for (int i = 0; i < cw; ++i) {
                const int s = split * cw + i;
                if (s >= nvalid) break;
                const cplx<T> w = csm_rows[(int64_t)s * csm_ld + c];
                // Complex multiply-accumulate as four fused multiply-adds: the
                // reference's coil sum is a BLAS product, which fuses them too.
#pragma unroll
                for (int a = 0; a < PLAIN_STAGE; ++a) {
                    if (a < na) {
                        const cplx<T> x = X[a * PLAIN_THREADS + s];
                        acc[a].re = fma(x.re, w.re, fma(-x.im, w.im, acc[a].re));
                        acc[a].im = fma(x.re, w.im, fma(x.im, w.re, acc[a].im));
                    }
                }
            }
        }
#pragma unroll
        for (int a = 0; a < PLAIN_STAGE; ++a)
            if (a < na) P[(split * PLAIN_STAGE + a) * cw + cl] = acc[a];
        __syncthreads();
        const int nsplit = PLAIN_THREADS / cw;
        if (t < na * cw) {
            const int a = t / cw, c2 = t % cw;
            cplx<T> s{T(0), T(0)};
            for (int j = 0; j < nsplit; ++j) {
                cplx<T> v = P[(j * PLAIN_STAGE + a) * cw + c2];
                s.re = s.re + v.re;
                s.im = s.im + v.im;
            }
            if (c2 < left) out[(int64_t)a * nc + cg + c2] = s;
        }
        __syncthreads();
    }
}

// Shared memory of a segment without ADC samples: the node cache alone (the
// kernel stages no samples and no sensitivities then).
template <typename T>
size_t segment_smem_bytes_no_adc() {
    return (sizeof(NodeCache<T>) + 127) & ~size_t(127);
}

template <typename T>
size_t segment_smem_bytes(int32_t nc) {
    size_t bytes = sizeof(NodeCache<T>) + 2 * sizeof(cplx<T>) * PLAIN_STAGE * PLAIN_THREADS;
    size_t csm_bytes = sizeof(cplx<T>) * (size_t)nc * PLAIN_THREADS;
    if (csm_bytes <= 128 * 1024) bytes += csm_bytes;
    return (bytes + 127) & ~size_t(127);
}

// Plain segment kernel.  One thread per spin; all threads of a CTA walk the
// same node range in lockstep, so ADC staging and the coil reduction are
// CTA-uniform.  RF=false: free precession (per-spin sequential trapezoid in
// the CPU order, BlochHighOrderSimulatitonMethod.jl:76-92).  RF=true:
// excitation (per-node hard-pulse spinor, :100-134; spinor of
// kernels/HighOrderGPU.jl:181-192).  The excitation variant asks for three
// CTAs per SM (80 registers: its launches without ADC samples use the node
// cache alone); the precession variant leaves the count to the compiler
// (0: none asked), which keeps it at 64 (FP32) and 128 (FP64) registers.
template <typename T, bool RF>
__global__ void __launch_bounds__(PLAIN_THREADS, RF ? 3 : 0)
    segment_kernel(PhantomDev<T> p, SeqDev<T> q, StateDev<T> st, SegmentArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    NodeCache<T> &nc = *reinterpret_cast<NodeCache<T> *>(smem_raw);
    cplx<T> *X = reinterpret_cast<cplx<T> *>(smem_raw + ((sizeof(NodeCache<T>) + 15) & ~size_t(15)));
    cplx<T> *P = X + PLAIN_STAGE * PLAIN_THREADS;
    cplx<T> *csm_s = P + PLAIN_STAGE * PLAIN_THREADS;

    const int64_t spin0 = (int64_t)blockIdx.x * PLAIN_THREADS;
    const int64_t s = spin0 + threadIdx.x;
    const bool active = s < p.ns;
    const int nvalid = (int)imin64(PLAIN_THREADS, p.ns - spin0);
    const int32_t ncoil = p.nc;
    // A segment without ADC samples stages nothing (and is launched with the
    // node cache alone).
    const bool stage_adc = a.nsamples > 0;
    const bool csm_in_smem = stage_adc && sizeof(cplx<T>) * (size_t)ncoil * PLAIN_THREADS <= 128 * 1024;

    // Stage this CTA's sensitivities (rows s, coil-fastest).
    const cplx<T> *csm_rows;
    int csm_ld = ncoil;
    if (csm_in_smem) {
        const int64_t total = (int64_t)nvalid * ncoil;
        for (int64_t i = threadIdx.x; i < total; i += PLAIN_THREADS) csm_s[i] = p.csm[spin0 * ncoil + i];
        csm_rows = csm_s;
    } else {
        csm_rows = p.csm + spin0 * ncoil;
    }

    const uint32_t m = a.method;
    const T gamma = a.gamma;
    // Constants converted from FP64 exactly as the reference's T(2π*γ).
    const double twopig_d = 2.0 * 3.141592653589793 * a.gamma_d;
    const T c_twopig = T(twopig_d);
    const T c_neg = T(-twopig_d);

    const int64_t si = active ? s : 0;
    const T px = p.x[si], py = p.y[si], pz = p.z[si];
    const T T1 = p.T1[si], T2 = p.T2[si], rho = p.rho[si];
    cplx<T> xy = active ? st.xy[si] : cplx<T>{T(0), T(0)};
    T mz = active ? st.z[si] : T(0);

    T b[16];
    T dwterm = T(0);
    T off = T(0);
    T acc = T(0);
    T tp = a.tp0;
    T prev = T(0);
    if (!RF) {
        basis16(px, py, pz, b);
        dwterm = p.dw[si] / c_twopig;
        acc = a.block_start ? T(0) : (active ? st.acc[si] : T(0));
    } else {
        off = (m & HOMS_DW_EXCITATION) ? p.dw[si] / c_twopig : T(0);
    }

    T dt_rel = T(-1), e1_rel = T(0), e2_rel = T(0);  // RF relaxation factors of the last dt
    int staged = 0;
    int64_t sample = 0;
    cplx<T> *out_base = a.partial + (int64_t)blockIdx.x * a.nsamples * ncoil;

    for (int64_t c0 = a.n_lo; c0 < a.n_hi; c0 += NODE_CHUNK) {
        __syncthreads();
        load_nodes<T, RF>(nc, q, c0, a.n_hi, m, gamma);
        __syncthreads();
        const int nint = (int)imin64(NODE_CHUNK, a.n_hi - c0);
        if (c0 == a.n_lo) {
            if (!RF) {
                prev = field_cached(nc, 0, b, dwterm, m);
            } else if (a.block_start) {
                T sn, cs;
                Math<T>::sc(-nc.psi[0], &sn, &cs);
                xy = cmul(xy, cplx<T>{cs, sn});
            }
        }
        for (int i = 0; i < nint; ++i) {
            const T dt = nc.dt[i];
            cplx<T> xs;
            bool have = false;
            if (!RF) {
                const T next = field_cached(nc, i + 1, b, dwterm, m);
                const T y = (next + prev) * dt;
                acc = acc + y;
                tp = tp + dt;
                prev = next;
                if (nc.adc[i + 1] || nc.bnd[i + 1]) {
                    const T phi = c_neg * (T(0.5) * acc);
                    const T e = Math<T>::ex(T(0) - tp / T2);
                    T sn, cs;
                    Math<T>::sc(phi, &sn, &cs);
                    xs = cmul(xy, cplx<T>{e * cs, e * sn});
                    have = true;
                }
            } else {
                const T dbz = off - nc.dfg[i];
                const T bz = ((nc.g[0][i] * px + nc.g[1][i] * py) + nc.g[2][i] * pz) + dbz;
                const cplx<T> b1 = nc.b1[i];
                const T ab1 = nc.ab1[i];
                T B = Math<T>::sq(ab1 * ab1 + bz * bz);
                if (B == T(0)) B = Math<T>::eps();
                const T phi = c_neg * (B * dt);
                T sh, ch;
                Math<T>::sc(phi / T(2), &sh, &ch);
                // Unit field direction (one reciprocal; within an ulp of three divisions).
                const T rB = T(1) / B;
                const T nz = bz * rB, nxr = b1.re * rB, nxi = b1.im * rB;
                const cplx<T> al{ch, -(nz * sh)};
                const cplx<T> be{nxi * sh, -(nxr * sh)};
                cplx<T> t1 = cmul(cplx<T>{T(2) * al.re, -(T(2) * al.im)}, be);
                t1.re = t1.re * mz;
                t1.im = t1.im * mz;
                const cplx<T> ca{al.re, -al.im};
                const cplx<T> t2 = cmul(cmul(ca, ca), xy);
                const cplx<T> t3 = cmul(cmul(be, be), cplx<T>{xy.re, -xy.im});
                const cplx<T> nxy{(t1.re + t2.re) - t3.re, (t1.im + t2.im) - t3.im};
                // |alpha|^2 - |beta|^2 as sums of squares (the reference's abs2;
                // within an ulp of hypot()^2).
                const T aa2 = al.re * al.re + al.im * al.im, bb2 = be.re * be.re + be.im * be.im;
                const cplx<T> pr = cmul(cmul(al, be), cplx<T>{xy.re, -xy.im});
                const T nz2 = (aa2 - bb2) * mz - T(2) * pr.re;
                // Relaxation factors depend on dt only: reuse them while dt repeats.
                if (!(dt == dt_rel)) {
                    e2_rel = Math<T>::ex(-dt / T2);
                    e1_rel = Math<T>::ex(-dt / T1);
                    dt_rel = dt;
                }
                xy = cplx<T>{nxy.re * e2_rel, nxy.im * e2_rel};
                mz = nz2 * e1_rel + rho * (T(1) - e1_rel);
                if (nc.adc[i + 1]) {
                    T sn, cs;
                    Math<T>::sc(nc.psi[i + 1], &sn, &cs);
                    xs = cmul(xy, cplx<T>{cs, sn});
                    have = true;
                }
            }
            if (stage_adc && nc.adc[i + 1]) {
                X[staged * PLAIN_THREADS + threadIdx.x] = active ? xs : cplx<T>{T(0), T(0)};
                staged++;
                if (staged == PLAIN_STAGE) {
                    __syncthreads();
                    reduce_stage(X, P, staged, csm_rows, csm_ld, nvalid, ncoil, out_base + sample * ncoil);
                    sample += staged;
                    staged = 0;
                }
            }
            if (nc.bnd[i + 1]) {
                if (!RF) {
                    // Block end: Mxy = last column, Mz relaxes over the block, phase restarts.
                    (void)have;
                    xy = xs;
                    const T e1 = Math<T>::ex(-tp / T1);
                    mz = mz * e1 + rho * (T(1) - e1);
                    acc = T(0);
                    tp = T(0);
                } else {
                    T sn, cs;
                    Math<T>::sc(nc.psi[i + 1], &sn, &cs);
                    xy = cmul(xy, cplx<T>{cs, sn});
                    if (c0 + i + 1 < a.n_hi) {
                        Math<T>::sc(-nc.psi[i + 1], &sn, &cs);
                        xy = cmul(xy, cplx<T>{cs, sn});
                    }
                }
            }
        }
    }
    if (staged > 0) {
        __syncthreads();
        reduce_stage(X, P, staged, csm_rows, csm_ld, nvalid, ncoil, out_base + sample * ncoil);
    }
    if (active) {
        st.xy[s] = xy;
        st.z[s] = mz;
        if (!RF) st.acc[s] = acc;
    }
}

// sig[(j) + c*ldsig] = sum over parts k of partial[(k*nsamples + j)*nc + c].
// A block takes 32 consecutive outputs; warp q of its 8 sums the parts
// k = q, q + 8, ... in increasing order (coalesced: 32 outputs of one part per
// load), then warp 0 adds the 8 sums in warp order.  The order depends only on
// nparts, so repeated runs are bit-identical.
constexpr int FIN_OUT = 32, FIN_SLICES = 8;
template <typename T>
__global__ void __launch_bounds__(FIN_OUT *FIN_SLICES)
    partial_finalize_kernel(const cplx<T> *partial, int64_t nparts, int64_t nsamples, int32_t nc, cplx<T> *sig,
                            int64_t ldsig) {
    __shared__ cplx<T> red[FIN_SLICES][FIN_OUT];
    const int64_t total = nsamples * nc;
    const int ol = threadIdx.x % FIN_OUT, q = threadIdx.x / FIN_OUT;
    for (int64_t o0 = (int64_t)blockIdx.x * FIN_OUT; o0 < total; o0 += (int64_t)gridDim.x * FIN_OUT) {
        const int64_t o = o0 + ol;
        cplx<T> acc{T(0), T(0)};
        if (o < total)
            for (int64_t k = q; k < nparts; k += FIN_SLICES) {
                const cplx<T> v = partial[k * total + o];
                acc.re = acc.re + v.re;
                acc.im = acc.im + v.im;
            }
        red[q][ol] = acc;
        __syncthreads();
        if (q == 0 && o < total) {
            cplx<T> s = red[0][ol];
            for (int qq = 1; qq < FIN_SLICES; ++qq) {
                s.re = s.re + red[qq][ol].re;
                s.im = s.im + red[qq][ol].im;
            }
            const int64_t jj = o / nc;
            const int32_t c = (int32_t)(o % nc);
            sig[jj + (int64_t)c * ldsig] = s;
        }
        __syncthreads();
    }
}

// Standalone coil reduction (states^T csm, no conjugation), split-K over spin
// ranges.  CTA (p, jt, ct) sums spins [ns p / P, ns (p + 1) / P) for samples
// 64 jt .. +63 and coils 32 ct .. +31 into its partial block: chunks of 16
// spins of both operands are staged in shared memory with coalesced loads
// along the spins (both arrays are column-major), then thread t accumulates
// sample t % 64 against coils 8 (t / 64) .. +7 in registers (a warp reads 32
// consecutive samples of one spin; the 8 sensitivities are broadcasts).
constexpr int CR_JB = 64, CR_CB = 32, CR_SK = 16, CR_THREADS = 256, CR_CTAS_PER_SM = 2;
constexpr int CR_XL = CR_SK * CR_JB / CR_THREADS, CR_CL = CR_SK * CR_CB / CR_THREADS;  // loads per thread and chunk
template <typename T>
__global__ void __launch_bounds__(CR_THREADS, CR_CTAS_PER_SM)
    coil_reduce_kernel(int64_t ns, int64_t nadc, int32_t nc, const cplx<T> *states, int64_t ldstates,
                       const cplx<T> *csm, int64_t ldcsm, int64_t parts, cplx<T> *partial) {
    __shared__ cplx<T> Xs[CR_SK][CR_JB + 1];
    __shared__ cplx<T> Cs[CR_SK][CR_CB + 1];
    const int64_t p = blockIdx.x;
    const int64_t j0 = (int64_t)blockIdx.y * CR_JB;
    const int c0 = (int)blockIdx.z * CR_CB;
    const int jn = (int)imin64(CR_JB, nadc - j0), cn = (int)imin64(CR_CB, nc - c0);
    const int64_t s_begin = ns * p / parts, s_end = ns * (p + 1) / parts;
    const int t = threadIdx.x;
    const int jl = t % CR_JB, cb = (t / CR_JB) * 8;
    // The next chunk's operands are fetched into registers while the current
    // chunk is contracted from shared memory.
    cplx<T> xr[CR_XL], cr[CR_CL];
    auto fetch = [&](int64_t s0) {
        const int sn = (int)imin64(CR_SK, s_end - s0);
#pragma unroll
        for (int r = 0; r < CR_XL; ++r) {
            const int i = t + r * CR_THREADS, sl = i % CR_SK, jj = i / CR_SK;
            xr[r] = (sl < sn && jj < jn) ? states[(s0 + sl) + (j0 + jj) * ldstates] : cplx<T>{T(0), T(0)};
        }
#pragma unroll
        for (int r = 0; r < CR_CL; ++r) {
            const int i = t + r * CR_THREADS, sl = i % CR_SK, c = i / CR_SK;
            cr[r] = (sl < sn && c < cn) ? csm[(s0 + sl) + (int64_t)(c0 + c) * ldcsm] : cplx<T>{T(0), T(0)};
        }
    };
    cplx<T> acc[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) acc[m] = cplx<T>{T(0), T(0)};
    if (s_begin < s_end) fetch(s_begin);
    for (int64_t s0 = s_begin; s0 < s_end; s0 += CR_SK) {
        const int sn = (int)imin64(CR_SK, s_end - s0);
        __syncthreads();
#pragma unroll
        for (int r = 0; r < CR_XL; ++r) {
            const int i = t + r * CR_THREADS;
            Xs[i % CR_SK][i / CR_SK] = xr[r];
        }
#pragma unroll
        for (int r = 0; r < CR_CL; ++r) {
            const int i = t + r * CR_THREADS;
            Cs[i % CR_SK][i / CR_SK] = cr[r];
        }
        __syncthreads();
        if (s0 + CR_SK < s_end) fetch(s0 + CR_SK);
        for (int sl = 0; sl < sn; ++sl) {
            const cplx<T> x = Xs[sl][jl];
#pragma unroll
            for (int m = 0; m < 8; ++m) {
                const cplx<T> w = Cs[sl][cb + m];
                acc[m].re = fma(x.re, w.re, fma(-x.im, w.im, acc[m].re));
                acc[m].im = fma(x.re, w.im, fma(x.im, w.re, acc[m].im));
            }
        }
    }
    if (jl < jn) {
        cplx<T> *out = partial + (p * nadc + j0 + jl) * nc + c0;
#pragma unroll
        for (int m = 0; m < 8; ++m)
            if (cb + m < cn) out[cb + m] = acc[m];
    }
}

template <typename T>
cudaError_t launch_segment(bool rf, const PhantomDev<T> &p, const SeqDev<T> &q, StateDev<T> &st,
                           const SegmentArgs<T> &a, int grid, cudaStream_t stream) {
    const size_t smem = a.nsamples > 0 ? segment_smem_bytes<T>(p.nc) : segment_smem_bytes_no_adc<T>();
    cudaError_t e;
    if (rf) {
        e = allow_max_dynamic_smem((const void *)segment_kernel<T, true>);
        if (e != cudaSuccess) return e;
        segment_kernel<T, true><<<grid, PLAIN_THREADS, smem, stream>>>(p, q, st, a);
    } else {
        e = allow_max_dynamic_smem((const void *)segment_kernel<T, false>);
        if (e != cudaSuccess) return e;
        segment_kernel<T, false><<<grid, PLAIN_THREADS, smem, stream>>>(p, q, st, a);
    }
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_partial_finalize(const cplx<T> *partial, int64_t nparts, int64_t nsamples, int32_t nc,
                                    cplx<T> *sig, int64_t ldsig, cudaStream_t stream) {
    const int64_t total = nsamples * nc;
    if (total == 0) return cudaSuccess;
    const int64_t blocks = std::min<int64_t>((total + FIN_OUT - 1) / FIN_OUT, 148 * 16);
    partial_finalize_kernel<T><<<(int)blocks, FIN_OUT * FIN_SLICES, 0, stream>>>(partial, nparts, nsamples, nc, sig,
                                                                                  ldsig);
    return cudaGetLastError();
}

// Parts of the split-K: one wave of CR_CTAS_PER_SM CTAs per SM over all
// (sample, coil) tiles, at least 256 spins per part (so at most
// ceil(ns / PLAIN_THREADS) parts).
int64_t coil_reduce_parts(int64_t ns, int64_t nadc, int32_t nc) {
    const int64_t tiles = ((nadc + CR_JB - 1) / CR_JB) * ((nc + CR_CB - 1) / CR_CB);
    const int64_t want = std::max<int64_t>(1, (148 * CR_CTAS_PER_SM) / tiles);
    return std::max<int64_t>(1, std::min<int64_t>(want, (ns + PLAIN_THREADS - 1) / PLAIN_THREADS));
}

template <typename T>
cudaError_t launch_coil_reduce(int64_t ns, int64_t nadc, int32_t nc, const cplx<T> *states, int64_t ldstates,
                               const cplx<T> *csm, int64_t ldcsm, cplx<T> *partial, cudaStream_t stream) {
    if (ns == 0 || nadc == 0 || nc == 0) return cudaSuccess;
    const int64_t parts = coil_reduce_parts(ns, nadc, nc);
    const int64_t jt = (nadc + CR_JB - 1) / CR_JB, ct = (nc + CR_CB - 1) / CR_CB;
    if (jt > 65535 || ct > 65535) return cudaErrorInvalidValue;
    dim3 grid((unsigned)parts, (unsigned)jt, (unsigned)ct);
    coil_reduce_kernel<T><<<grid, CR_THREADS, 0, stream>>>(ns, nadc, nc, states, ldstates, csm, ldcsm, parts,
                                                          partial);
    return cudaGetLastError();
}

template cudaError_t launch_segment<double>(bool, const PhantomDev<double> &, const SeqDev<double> &,
                                            StateDev<double> &, const SegmentArgs<double> &, int, cudaStream_t);
template cudaError_t launch_segment<float>(bool, const PhantomDev<float> &, const SeqDev<float> &,
                                           StateDev<float> &, const SegmentArgs<float> &, int, cudaStream_t);
template cudaError_t launch_partial_finalize<double>(const cplx<double> *, int64_t, int64_t, int32_t,
                                                     cplx<double> *, int64_t, cudaStream_t);
template cudaError_t launch_partial_finalize<float>(const cplx<float> *, int64_t, int64_t, int32_t, cplx<float> *,
                                                    int64_t, cudaStream_t);
template cudaError_t launch_coil_reduce<double>(int64_t, int64_t, int32_t, const cplx<double> *, int64_t,
                                                const cplx<double> *, int64_t, cplx<double> *, cudaStream_t);
template cudaError_t launch_coil_reduce<float>(int64_t, int64_t, int32_t, const cplx<float> *, int64_t,
                                               const cplx<float> *, int64_t, cplx<float> *, cudaStream_t);
template size_t segment_smem_bytes<double>(int32_t);
template size_t segment_smem_bytes<float>(int32_t);

}  // namespace homs
