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
//   pass 2  one warp per column: carry into every tile (segmented scan of
//           the tile aggregates), the local sum of every part and the part
//           offsets sign_p * (end value of part p-1) (an affine scan);
//   pass 3  per tile: the same block scan with the tile's carry-in, plus the
//           part offset, times gamma, written column-major;
//   query   per ADC time: binary search over the knots, then linear
//           interpolation of every column.
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

// Shared tile of trapezoid terms, one double of padding after every ITEMS
// (thread t's items t*ITEMS .. +ITEMS-1 then start 72 bytes apart: two-way
// bank use, the minimum for 8-byte words, where 64 bytes would be 16-way).
__device__ __forceinline__ int pad(int i) { return i + i / ITEMS; }

struct Shared {
    double y[TILE + TILE / ITEMS];
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
        sh.y[pad(i)] = n < m ? trap(g, dt, n) : 0.0;
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
        const double y = sh.y[pad(base + j)];
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
    for (int j = 0; j < ITEMS; ++j) sh.y[pad(base + j)] = v[j];
    __syncthreads();
    if (threadIdx.x == 0) {
        any[(size_t)col * ntiles + tile] = sh.warp_prefix[NWARPS].f ? 1 : 0;
        tail[(size_t)col * ntiles + tile] = sh.warp_prefix[NWARPS].v;
    }
    for (int p = threadIdx.x; p < nparts; p += THREADS) {
        const int64_t s = starts[p];
        if (p > 0 && s >= t0 && s < t0 + TILE && s < m) {
            const int i = (int)(s - t0);
            head[(size_t)col * nparts + p] = i > 0 ? sh.y[pad(i - 1)] : 0.0;
        }
    }
}

// Pass 2, one warp per column: the carry into every tile (a segmented scan
// of the tile aggregates, 32 tiles at a time), the local sum of every part
// (the carry into its first tile plus its head in that tile, or its head
// alone when an earlier part starts in the same tile), and the part offsets
// sign_p * (end value of part p-1), an affine scan prev_p = sign_p prev_{p-1}
// + S_p over the parts.
struct Affine {
    double a, b;  // x -> a x + b
};
__device__ __forceinline__ Affine then(const Affine &first, const Affine &second) {
    return Affine{second.a * first.a, second.a * first.b + second.b};
}

__global__ void __launch_bounds__(32) carry_kernel(int ntiles, const int64_t *starts, const int8_t *signs,
                                                   int nparts, const uint8_t *any, const double *tail,
                                                   const double *head, double *carry_in, double *part_sum,
                                                   double *offset) {
    const int col = blockIdx.x, lane = threadIdx.x;
    const uint8_t *a = any + (size_t)col * ntiles;
    const double *tl = tail + (size_t)col * ntiles;
    const double *hd = head + (size_t)col * nparts;
    double *ci = carry_in + (size_t)col * ntiles;
    double *ps = part_sum + (size_t)col * nparts;
    double *off = offset + (size_t)col * nparts;
    Seg run{false, 0.0};
    for (int base = 0; base < ntiles; base += 32) {
        const int i = base + lane;
        Seg x = i < ntiles ? Seg{a[i] != 0, tl[i]} : Seg{false, 0.0};
        Seg inc = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int uf = __shfl_up_sync(0xffffffffu, (int)inc.f, o);
            const double uv = __shfl_up_sync(0xffffffffu, inc.v, o);
            if (lane >= o) inc = combine(Seg{uf != 0, uv}, inc);
        }
        const int ef = __shfl_up_sync(0xffffffffu, (int)inc.f, 1);
        const double ev = __shfl_up_sync(0xffffffffu, inc.v, 1);
        const Seg excl = lane == 0 ? Seg{false, 0.0} : Seg{ef != 0, ev};
        if (i < ntiles) ci[i] = combine(run, excl).v;
        const int lf = __shfl_sync(0xffffffffu, (int)inc.f, 31);
        const double lv = __shfl_sync(0xffffffffu, inc.v, 31);
        run = combine(run, Seg{lf != 0, lv});
    }
    __syncwarp();
    for (int p = 1 + lane; p < nparts; p += 32) {
        const int64_t tile = starts[p] / TILE;
        const bool first = starts[p - 1] / TILE != tile;
        ps[p - 1] = (first ? ci[tile] : 0.0) + hd[p];
    }
    if (lane == 0) ps[nparts - 1] = run.v;
    __syncwarp();
    Affine acc{0.0, 0.0};  // prev_{-1} = 0 for every input
    for (int base = 0; base < nparts; base += 32) {
        const int p = base + lane;
        Affine f = p < nparts ? Affine{p == 0 ? 0.0 : (double)signs[p], ps[p]} : Affine{1.0, 0.0};
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double ua = __shfl_up_sync(0xffffffffu, f.a, o);
            const double ub = __shfl_up_sync(0xffffffffu, f.b, o);
            if (lane >= o) f = then(Affine{ua, ub}, f);
        }
        // prev_{p-1}: the composed map of the parts before p applied to 0.
        const double ea = __shfl_up_sync(0xffffffffu, f.a, 1);
        const double eb = __shfl_up_sync(0xffffffffu, f.b, 1);
        const Affine before = lane == 0 ? acc : then(acc, Affine{ea, eb});
        if (p < nparts) off[p] = p == 0 ? 0.0 : (double)signs[p] * before.b;
        const double la = __shfl_sync(0xffffffffu, f.a, 31);
        const double lb = __shfl_sync(0xffffffffu, f.b, 31);
        acc = then(acc, Affine{la, lb});
    }
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
        sh.y[pad(base + j)] = gamma * (v[j] + off[p]);
    }
    __syncthreads();
    double *kc = k + (size_t)col * m;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int i = j * THREADS + threadIdx.x;
        if (t0 + i < m) kc[t0 + i] = sh.y[pad(i)];
    }
}

// Query: k at the times q by linear interpolation over the knots
// t[n] + dt[n] (n < m), 0 outside [knot 0, knot m-1].  Each block first
// stages every stride-th knot in shared memory; a time's search runs there,
// then over one stride of global knots, and serves all columns.
constexpr int QTABLE = 1024;

template <typename S>
__global__ void __launch_bounds__(256) query_kernel(const S *t, const S *dt, int64_t m, const double *k,
                                                    int32_t ncols, const double *q, int64_t nq, double *kq) {
    __shared__ double table[QTABLE];
    auto knot = [&](int64_t n) { return (double)t[n] + (double)dt[n]; };
    const int64_t stride = (m + QTABLE - 1) / QTABLE;
    const int nrows = (int)((m + stride - 1) / stride);  // rows r: knot(r * stride), r * stride < m
    for (int r = threadIdx.x; r < nrows; r += blockDim.x) table[r] = knot((int64_t)r * stride);
    __syncthreads();
    const double last = knot(m - 1);
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nq; j += (int64_t)gridDim.x * blockDim.x) {
        const double tau = q[j];
        int64_t n = -1;
        double w = 0.0;
        if (tau >= table[0] && tau <= last) {
            int lo = 0, hi = nrows;  // first row whose knot exceeds tau (lo >= 1 here)
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (table[mid] <= tau) lo = mid + 1;
                else hi = mid;
            }
            // knot((lo-1) stride) <= tau < knot(lo stride) (or lo stride >= m):
            // the last knot <= tau lies in [(lo-1) stride, min(lo stride, m)).
            int64_t glo = (int64_t)(lo - 1) * stride + 1, ghi = std::min<int64_t>((int64_t)lo * stride, m);
            while (glo < ghi) {
                const int64_t mid = (glo + ghi) >> 1;
                if (knot(mid) <= tau) glo = mid + 1;
                else ghi = mid;
            }
            n = glo - 1;
            if (n < m - 1) {
                const double s0 = knot(n), s1 = knot(n + 1);
                w = (tau - s0) / (s1 - s0);
            }
        }
        for (int32_t col = 0; col < ncols; ++col) {
            const double *kc = k + (size_t)col * m;
            double out = 0.0;
            if (n == m - 1) out = kc[n];
            else if (n >= 0) out = kc[n] + w * (kc[n + 1] - kc[n]);
            kq[(size_t)col * nq + j] = out;
        }
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
    carry_kernel<<<a.ncols, 32, 0, stream>>>(ntiles, a.starts, a.signs, a.nparts, w.any, w.tail, w.head, w.carry,
                                             w.part_sum, w.offset);
    write_kernel<S><<<grid, THREADS, 0, stream>>>(dt, a.cols, m, a.starts, a.nparts, ntiles, w.carry, w.offset,
                                                  a.gamma, a.k);
    if (a.nq > 0) {
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((a.nq + 255) / 256, 148 * 4));
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
