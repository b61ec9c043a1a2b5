// Encoding export: the generalised k-space of a sampled sequence.
//
// grad2kspace (src/datatypes/HO_Sequence.jl:257-287) integrates every field
// column with KomaMRICore's cumtrapz over the intervals of the sequence, in
// parts cut at the RF pulses: part p restarts the integral and then adds
// sign_p times the value at the end of part p-1 (0 after an excitation, -1
// after a refocusing pulse, +1 otherwise or when the pulse is skipped), and
// multiplies by gamma.  The ADC-sampled copy interpolates that curve linearly
// at the ADC times over the knots t[n] + dt[n], 0 outside them
// (KomaMRIBase.linear_interpolate_samples with default = 0).
//
// On the device this is a segmented scan of the trapezoid terms
// y[n] = (g[n] + g[n+1]) * (dt[n] / 2), one column per grid row:
//   pass 1  per tile of 2048 intervals: segmented block scan with zero
//           carry-in; the tile's (has-part-start, sum since the last start)
//           and, for every part starting inside the tile, the sum of the
//           tile's elements before it (that part's predecessor's tail);
//   pass 2  per column, sequential over tiles and parts: carry into every
//           tile, the local sum of every part and the part offsets
//           sign_p * (end value of part p-1);
//   pass 3  per tile: the same block scan with the tile's carry-in, plus the
//           part offset, times gamma, written column-major;
//   query   per (ADC time, column): binary search over the knots, linear
//           interpolation.
// The traffic is one read of every column in passes 1 and 3 (the second read
// hits L2 at the sizes of a sequence) and one write of k: an HBM-bound scan.
#include <algorithm>
#include <cstdint>

#include "homs_kspace.cuh"

namespace homs {

namespace kspace {

constexpr int THREADS = 256;
constexpr int ITEMS = 8;
constexpr int TILE = THREADS * ITEMS;  // intervals per block
constexpr int NWARPS = THREADS / 32;

struct Seg {
    bool f;    // a part starts inside the range
    double v;  // sum since the last part start in the range (or over all of it)
};
__device__ __forceinline__ Seg combine(const Seg &a, const Seg &b) { return Seg{a.f || b.f, b.f ? b.v : a.v + b.v}; }

template <typename S>
__device__ __forceinline__ double trap(const S *g, const S *dt, int64_t n) {
    return ((double)g[n] + (double)g[n + 1]) * ((double)dt[n] * 0.5);
}

struct Shared {
    double y[TILE];
    uint32_t flag[TILE / 32];
    Seg warp_total[NWARPS];
    Seg warp_prefix[NWARPS + 1];
};

// Segmented inclusive scan of one tile (intervals t0 .. t0 + TILE - 1 of m)
// with `carry` entering the tile's first segment.  On return v[] holds this
// thread's ITEMS values (items tid*ITEMS + j), `bits` their part-start flags,
// and sh.warp_prefix[NWARPS] the tile's total (carry excluded when carry = 0).
template <typename S>
__device__ void tile_scan(const S *g, const S *dt, int64_t m, int64_t t0, const int64_t *starts, int nparts,
                          double carry, Shared &sh, double (&v)[ITEMS], uint32_t &bits) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < TILE / 32) sh.flag[tid] = 0u;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int i = j * THREADS + tid;
        const int64_t n = t0 + i;
        sh.y[i] = n < m ? trap(g, dt, n) : 0.0;
    }
    __syncthreads();
    for (int p = tid; p < nparts; p += THREADS) {
        const int64_t s = starts[p];
        if (s >= t0 && s < t0 + TILE && s < m) atomicOr(&sh.flag[(s - t0) >> 5], 1u << ((s - t0) & 31));
    }
    __syncthreads();
    const int base = tid * ITEMS;
    bits = (sh.flag[base >> 5] >> (base & 31)) & ((1u << ITEMS) - 1u);
    Seg agg{false, 0.0};
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const double y = sh.y[base + j];
        if ((bits >> j) & 1u) {
            agg.f = true;
            agg.v = y;
        } else {
            agg.v += y;
        }
        v[j] = agg.v;
    }
    // Warp inclusive scan of the thread aggregates.
    Seg inc = agg;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int uf = __shfl_up_sync(0xffffffffu, (int)inc.f, off);
        const double uv = __shfl_up_sync(0xffffffffu, inc.v, off);
        if (lane >= off) inc = combine(Seg{uf != 0, uv}, inc);
    }
    const int ef = __shfl_up_sync(0xffffffffu, (int)inc.f, 1);
    const double ev = __shfl_up_sync(0xffffffffu, inc.v, 1);
    const Seg wexcl = lane == 0 ? Seg{false, 0.0} : Seg{ef != 0, ev};
    if (lane == 31) sh.warp_total[warp] = inc;
    __syncthreads();
    if (tid == 0) {
        Seg pre{false, carry};
        for (int w = 0; w < NWARPS; ++w) {
            sh.warp_prefix[w] = pre;
            pre = combine(pre, sh.warp_total[w]);
        }
        sh.warp_prefix[NWARPS] = pre;
    }
    __syncthreads();
    const Seg excl = combine(sh.warp_prefix[warp], wexcl);
    // Items before this thread's first part start continue the segment
    // that runs into the thread.
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        if ((bits & ((2u << j) - 1u)) == 0u) v[j] += excl.v;
    }
}

// Pass 1: per (tile, column) aggregates and the tails of parts that end in
// the tile.
template <typename S>
__global__ void __launch_bounds__(THREADS) reduce_kernel(const S *dt, const void *const *cols, int64_t m,
                                                         const int64_t *starts, int nparts, int ntiles,
                                                         uint8_t *any, double *tail, double *head) {
    __shared__ Shared sh;
    const int tile = blockIdx.x, col = blockIdx.y;
    const S *g = static_cast<const S *>(cols[col]);
    const int64_t t0 = (int64_t)tile * TILE;
    double v[ITEMS];
    uint32_t bits;
    tile_scan<S>(g, dt, m, t0, starts, nparts, 0.0, sh, v, bits);
    const int base = threadIdx.x * ITEMS;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) sh.y[base + j] = v[j];
    __syncthreads();
    if (threadIdx.x == 0) {
        any[(size_t)col * ntiles + tile] = sh.warp_prefix[NWARPS].f ? 1 : 0;
        tail[(size_t)col * ntiles + tile] = sh.warp_prefix[NWARPS].v;
    }
    for (int p = threadIdx.x; p < nparts; p += THREADS) {
        const int64_t s = starts[p];
        if (p > 0 && s >= t0 && s < t0 + TILE && s < m) {
            const int i = (int)(s - t0);
            head[(size_t)col * nparts + p] = i > 0 ? sh.y[i - 1] : 0.0;
        }
    }
}

// Pass 2: carry into each tile, part sums and part offsets, per column.
__global__ void carry_kernel(int64_t m, int ntiles, const int64_t *starts, const int8_t *signs, int nparts,
                             const uint8_t *any, const double *tail, const double *head, double *carry_in,
                             double *part_sum, double *offset) {
    const int col = blockIdx.x;
    if (threadIdx.x != 0) return;
    const uint8_t *a = any + (size_t)col * ntiles;
    const double *tl = tail + (size_t)col * ntiles;
    const double *hd = head + (size_t)col * nparts;
    double *ci = carry_in + (size_t)col * ntiles;
    double *ps = part_sum + (size_t)col * nparts;
    double *off = offset + (size_t)col * nparts;
    double carry = 0.0;
    int p = 1;
    for (int i = 0; i < ntiles; ++i) {
        ci[i] = carry;
        bool first = true;
        while (p < nparts && starts[p] / TILE == i) {
            ps[p - 1] = (first ? carry : 0.0) + hd[p];
            first = false;
            ++p;
        }
        carry = a[i] ? tl[i] : carry + tl[i];
    }
    ps[nparts - 1] = carry;
    double prev = 0.0;
    for (int q = 0; q < nparts; ++q) {
        const double o = q == 0 ? 0.0 : (double)signs[q] * prev;
        off[q] = o;
        prev = ps[q] + o;
    }
    (void)m;
}

// Pass 3: k = gamma * (part-local prefix + part offset), column-major.
template <typename S>
__global__ void __launch_bounds__(THREADS) write_kernel(const S *dt, const void *const *cols, int64_t m,
                                                        const int64_t *starts, int nparts, int ntiles,
                                                        const double *carry_in, const double *offset, double gamma,
                                                        double *k) {
    __shared__ Shared sh;
    const int tile = blockIdx.x, col = blockIdx.y;
    const S *g = static_cast<const S *>(cols[col]);
    const int64_t t0 = (int64_t)tile * TILE;
    double v[ITEMS];
    uint32_t bits;
    tile_scan<S>(g, dt, m, t0, starts, nparts, carry_in[(size_t)col * ntiles + tile], sh, v, bits);
    // Part of this thread's first item: the last start at or before it.
    const int base = threadIdx.x * ITEMS;
    const int64_t n0 = t0 + base;
    int lo = 0, hi = nparts;  // first index with starts[idx] > n0
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (starts[mid] <= n0) lo = mid + 1;
        else hi = mid;
    }
    int p = lo - 1;
    const double *off = offset + (size_t)col * nparts;
    __syncthreads();  // every thread has read sh.y inside tile_scan
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        if (j > 0 && ((bits >> j) & 1u)) ++p;
        sh.y[base + j] = gamma * (v[j] + off[p]);
    }
    __syncthreads();
    double *kc = k + (size_t)col * m;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int i = j * THREADS + threadIdx.x;
        if (t0 + i < m) kc[t0 + i] = sh.y[i];
    }
}

// Query: k at the times q by linear interpolation over the knots
// t[n] + dt[n] (n < m), 0 outside [knot 0, knot m-1].
template <typename S>
__global__ void query_kernel(const S *t, const S *dt, int64_t m, const double *k, int32_t ncols, const double *q,
                             int64_t nq, double *kq) {
    const int64_t total = nq * ncols;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = idx % nq;
        const int64_t col = idx / nq;
        const double tau = q[j];
        auto knot = [&](int64_t n) { return (double)t[n] + (double)dt[n]; };
        double out = 0.0;
        if (tau >= knot(0) && tau <= knot(m - 1)) {
            int64_t lo = 0, hi = m;  // first n with knot(n) > tau
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                if (knot(mid) <= tau) lo = mid + 1;
                else hi = mid;
            }
            const int64_t n = lo - 1;
            const double *kc = k + (size_t)col * m;
            if (n == m - 1) {
                out = kc[n];
            } else {
                const double s0 = knot(n), s1 = knot(n + 1);
                const double w = (tau - s0) / (s1 - s0);
                out = kc[n] + w * (kc[n + 1] - kc[n]);
            }
        }
        kq[idx] = out;
    }
}

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

struct Work {
    uint8_t *any;
    double *tail, *head, *carry, *part_sum, *offset;
};

inline Work carve(void *w, int ntiles, int32_t ncols, int32_t nparts) {
    uint8_t *p = static_cast<uint8_t *>(w);
    Work out;
    out.any = p;
    p += align256((size_t)ntiles * ncols);
    out.tail = reinterpret_cast<double *>(p);
    p += align256(sizeof(double) * (size_t)ntiles * ncols);
    out.carry = reinterpret_cast<double *>(p);
    p += align256(sizeof(double) * (size_t)ntiles * ncols);
    out.head = reinterpret_cast<double *>(p);
    p += align256(sizeof(double) * (size_t)nparts * ncols);
    out.part_sum = reinterpret_cast<double *>(p);
    p += align256(sizeof(double) * (size_t)nparts * ncols);
    out.offset = reinterpret_cast<double *>(p);
    return out;
}

template <typename S>
cudaError_t launch_typed(const KspaceArgs &a, cudaStream_t stream) {
    const int64_t m = a.nnodes - 1;
    const int ntiles = (int)((m + TILE - 1) / TILE);
    Work w = carve(a.work, ntiles, a.ncols, a.nparts);
    const S *t = static_cast<const S *>(a.t);
    const S *dt = static_cast<const S *>(a.dt);
    const dim3 grid((unsigned)ntiles, (unsigned)a.ncols);
    reduce_kernel<S><<<grid, THREADS, 0, stream>>>(dt, a.cols, m, a.starts, a.nparts, ntiles, w.any, w.tail, w.head);
    carry_kernel<<<a.ncols, 32, 0, stream>>>(m, ntiles, a.starts, a.signs, a.nparts, w.any, w.tail, w.head, w.carry,
                                             w.part_sum, w.offset);
    write_kernel<S><<<grid, THREADS, 0, stream>>>(dt, a.cols, m, a.starts, a.nparts, ntiles, w.carry, w.offset,
                                                  a.gamma, a.k);
    if (a.nq > 0) {
        const int64_t total = a.nq * a.ncols;
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148 * 16));
        query_kernel<S><<<blocks, 256, 0, stream>>>(t, dt, m, a.k, a.ncols, a.q, a.nq, a.kq);
    }
    return cudaGetLastError();
}

}  // namespace kspace

size_t kspace_work_bytes(int64_t nnodes, int32_t ncols, int32_t nparts) {
    const int64_t m = std::max<int64_t>(nnodes - 1, 1);
    const size_t ntiles = (size_t)((m + kspace::TILE - 1) / kspace::TILE);
    using kspace::align256;
    return align256(ntiles * ncols) + 2 * align256(sizeof(double) * ntiles * ncols) +
           3 * align256(sizeof(double) * (size_t)nparts * ncols);
}

cudaError_t kspace_launch(const KspaceArgs &a, cudaStream_t stream) {
    if (a.nnodes < 2 || a.ncols < 1 || a.nparts < 1) return cudaErrorInvalidValue;
    return a.f64 ? kspace::launch_typed<double>(a, stream) : kspace::launch_typed<float>(a, stream);
}

}  // namespace homs
