// Phantom builders on the device.
//
// Brain phantom (src/phantom/hophantom_brain.jl:2-58): from a volume of
// tissue classes (column-major nx x ny x nz, as load_phantom_mat returns it)
// build the spin arrays of an HO_Phantom:
//   - voxel-centre grid of generate_grid (src/grid/Grid.jl:78-108) for
//     fov = matrix .* res, shifted by `offcenter`;
//   - T1, T2, T2s, rho per class from the 1.5 T or 7 T tables of
//     SpinProperty (src/phantom/SpinProperty.jl:1-118);
//   - dw = 2 pi * field map, or the fat shift -220 * 2 pi on the two fat
//     classes (b0_type = :fat);
//   - the receive sensitivities of the caller's map, or one unit coil;
// keeping the voxels whose density is not zero, in column-major voxel order
// (Julia's x[rho .!= 0]).  Every value is rounded as the reference rounds it
// (separately rounded products and sums: no contraction into FMAs).
//
// Birdcage map (src/phantom/csm/Birdcage.jl:21-42): 1/r * cis(phi) per coil
// on a ring of relative radius `relative_radius`, normalised per pixel by
// the root sum of squares over the coils.
//
// Compaction: blocks of 2048 voxels; pass 1 counts each block's kept voxels,
// a one-block scan turns the counts into offsets, pass 2 places each kept
// voxel by warp ballots, 256 consecutive voxels at a time, so the output
// keeps the voxel order and every access is coalesced.
#include <algorithm>
#include <cmath>
#include <cstdint>

#include "homs_phantom.cuh"

namespace homs {

namespace phantom {

constexpr int THREADS = 256;
constexpr int ITEMS = 8;
constexpr int VOX = THREADS * ITEMS;  // voxels per block
constexpr int NWARPS = THREADS / 32;
constexpr double TWO_PI = 6.283185307179586;  // Julia's 2π as a Float64

// Tissue classes of the brain phantom and their properties (T1, T2, T2s in
// ms as integers, scaled by 1e-3 like the reference; rho as given).
__device__ __forceinline__ int class_index(unsigned c) {
    switch (c) {
        case 23: return 0;    // CSF
        case 46: return 1;    // GM
        case 70: return 2;    // WM
        case 93: return 3;    // FAT1
        case 116: return 4;   // MUSCLE
        case 139: return 5;   // SKIN/MUSCLE
        case 162: return 6;   // SKULL
        case 185: return 7;   // VESSELS
        case 209: return 8;   // FAT2
        case 232: return 9;   // DURA
        case 255: return 10;  // MARROW
        default: return -1;
    }
}
__constant__ double RHO[11] = {1.0, 0.86, 0.77, 1.0, 1.0, 0.7, 0.0, 0.0, 0.77, 1.0, 0.77};
__constant__ int T1_MS[2][11] = {{2569, 833, 500, 350, 900, 569, 0, 0, 500, 2569, 500},
                                 {4400, 2100, 1200, 580, 1700, 1700, 0, 0, 1200, 4400, 1200}};
__constant__ int T2_MS[2][11] = {{329, 83, 70, 70, 47, 329, 0, 0, 70, 329, 70},
                                 {329, 50, 40, 46, 30, 30, 0, 0, 40, 329, 40}};
__constant__ int T2S_MS[2][11] = {{58, 69, 61, 58, 30, 58, 0, 0, 61, 58, 61},
                                  {58, 33, 27, 25, 23, 23, 0, 0, 27, 58, 27}};

__device__ __forceinline__ double rho_of(uint8_t c) {
    const int k = class_index(c);
    return k < 0 ? 0.0 : RHO[k];
}

// Warp-ballot compaction of 256 consecutive voxels: this thread's rank among
// the kept voxels of the slab, and the slab's count (shared by all threads).
__device__ __forceinline__ int slab_rank(bool keep, int *warp_off, int &slab_total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned ballot = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) warp_off[warp] = __popc(ballot);
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int w = 0; w < NWARPS; ++w) {
            const int c = warp_off[w];
            warp_off[w] = run;
            run += c;
        }
        warp_off[NWARPS] = run;
    }
    __syncthreads();
    const int rank = warp_off[warp] + __popc(ballot & ((1u << lane) - 1u));
    slab_total = warp_off[NWARPS];
    __syncthreads();  // warp_off is rewritten by the next slab
    return rank;
}

__global__ void __launch_bounds__(THREADS) count_kernel(const uint8_t *labels, int64_t nvox, int64_t *counts) {
    __shared__ int warp_off[NWARPS + 1];
    const int64_t base = (int64_t)blockIdx.x * VOX;
    int64_t total = 0;
    for (int j = 0; j < ITEMS; ++j) {
        const int64_t i = base + (int64_t)j * THREADS + threadIdx.x;
        const bool keep = i < nvox && rho_of(labels[i]) != 0.0;
        int slab;
        slab_rank(keep, warp_off, slab);
        total += slab;
    }
    if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

// Exclusive scan of the block counts in place; the total goes to counts[nblocks].
__global__ void __launch_bounds__(1024) scan_kernel(int64_t *counts, int64_t nblocks) {
    __shared__ int64_t part[1024];
    int64_t carry = 0;
    for (int64_t b0 = 0; b0 < nblocks; b0 += 1024) {
        const int64_t b = b0 + threadIdx.x;
        const int64_t v = b < nblocks ? counts[b] : 0;
        part[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            const int64_t add = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
            __syncthreads();
            part[threadIdx.x] += add;
            __syncthreads();
        }
        if (b < nblocks) counts[b] = carry + part[threadIdx.x] - v;
        carry += part[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) counts[nblocks] = carry;
}

__global__ void __launch_bounds__(THREADS) fill_kernel(BrainArgs a, const int64_t *offsets, BrainOut o) {
    __shared__ int warp_off[NWARPS + 1];
    const int64_t nvox = a.nx * a.ny * a.nz;
    const int64_t base = (int64_t)blockIdx.x * VOX;
    const int fs = a.fieldstrength;
    // generate_grid: spacing = (n * res) / n, centres (k - (n - 1) / 2) * spacing.
    const double sx = __ddiv_rn(__dmul_rn((double)a.nx, a.res[0]), (double)a.nx);
    const double sy = __ddiv_rn(__dmul_rn((double)a.ny, a.res[1]), (double)a.ny);
    const double sz = __ddiv_rn(__dmul_rn((double)a.nz, a.res[2]), (double)a.nz);
    const double hx = (double)(a.nx - 1) / 2.0, hy = (double)(a.ny - 1) / 2.0, hz = (double)(a.nz - 1) / 2.0;
    const double dw_fat = __dmul_rn(-220.0, TWO_PI);
    int64_t pos0 = offsets[blockIdx.x];
    for (int j = 0; j < ITEMS; ++j) {
        const int64_t i = base + (int64_t)j * THREADS + threadIdx.x;
        const uint8_t c = i < nvox ? a.labels[i] : 0;
        const int k = class_index(c);
        const bool keep = i < nvox && k >= 0 && RHO[k] != 0.0;
        int slab;
        const int rank = slab_rank(keep, warp_off, slab);
        if (keep) {
            const int64_t s = pos0 + rank;
            const int64_t ix = i % a.nx, iy = (i / a.nx) % a.ny, iz = i / (a.nx * a.ny);
            o.x[s] = __dadd_rn(__dmul_rn((double)ix - hx, sx), a.offcenter[0]);
            o.y[s] = __dadd_rn(__dmul_rn((double)iy - hy, sy), a.offcenter[1]);
            o.z[s] = __dadd_rn(__dmul_rn((double)iz - hz, sz), a.offcenter[2]);
            o.rho[s] = RHO[k];
            o.T1[s] = __dmul_rn((double)T1_MS[fs][k], 1e-3);
            o.T2[s] = __dmul_rn((double)T2_MS[fs][k], 1e-3);
            if (o.T2s) o.T2s[s] = __dmul_rn((double)T2S_MS[fs][k], 1e-3);
            o.dw[s] = a.fieldmap ? __dmul_rn(a.fieldmap[i], TWO_PI) : ((c == 93 || c == 209) ? dw_fat : -0.0);
            if (a.ncoils == 0 || !a.csm) {
                o.csm[2 * s] = 1.0;
                o.csm[2 * s + 1] = 0.0;
            } else {
                for (int32_t q = 0; q < a.ncoils; ++q) {
                    const double2 v = reinterpret_cast<const double2 *>(a.csm)[i + (int64_t)q * nvox];
                    reinterpret_cast<double2 *>(o.csm)[s + (int64_t)q * o.nspins] = v;
                }
            }
        }
        pos0 += slab;
    }
}

__global__ void birdcage_kernel(int64_t nx, int64_t ny, int32_t nc, double radius, double *out) {
    const int64_t npix = nx * ny;
    const double step = TWO_PI / (double)nc;
    const double hx = (double)nx / 2.0, hy = (double)ny / 2.0;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npix; p += (int64_t)gridDim.x * blockDim.x) {
        const double x = (double)(p % nx), y = (double)(p / nx);
        double ss = 0.0;
        for (int32_t c = 0; c < nc; ++c) {
            const double ang = __dmul_rn((double)c, step);
            const double y_co = __dsub_rn(__ddiv_rn(__dsub_rn(y, hy), hy), __dmul_rn(radius, sin(ang)));
            const double x_co = __dsub_rn(__ddiv_rn(__dsub_rn(x, hx), hx), __dmul_rn(radius, cos(ang)));
            const double rr = sqrt(__dadd_rn(__dmul_rn(x_co, x_co), __dmul_rn(y_co, y_co)));
            const double phi = __dsub_rn(atan2(x_co, -y_co), ang);
            double sn, cs;
            sincos(phi, &sn, &cs);
            const double inv = __ddiv_rn(1.0, rr);
            const double re = __dmul_rn(inv, cs), im = __dmul_rn(inv, sn);
            const double m = hypot(re, im);
            ss = __dadd_rn(ss, __dmul_rn(m, m));
            out[2 * (p + (int64_t)c * npix)] = re;
            out[2 * (p + (int64_t)c * npix) + 1] = im;
        }
        const double norm = sqrt(ss);
        for (int32_t c = 0; c < nc; ++c) {
            double *v = out + 2 * (p + (int64_t)c * npix);
            v[0] = __ddiv_rn(v[0], norm);
            v[1] = __ddiv_rn(v[1], norm);
        }
    }
}

}  // namespace phantom

size_t brain_work_bytes(int64_t nvox) {
    const int64_t nblocks = (nvox + phantom::VOX - 1) / phantom::VOX;
    return sizeof(int64_t) * (size_t)(nblocks + 1);
}

cudaError_t brain_count(const BrainArgs &a, void *work, int64_t *count, cudaStream_t stream) {
    const int64_t nvox = a.nx * a.ny * a.nz;
    const int64_t nblocks = (nvox + phantom::VOX - 1) / phantom::VOX;
    int64_t *counts = static_cast<int64_t *>(work);
    if (nblocks > 0) phantom::count_kernel<<<(unsigned)nblocks, phantom::THREADS, 0, stream>>>(a.labels, nvox, counts);
    phantom::scan_kernel<<<1, 1024, 0, stream>>>(counts, nblocks);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(count, counts + nblocks, sizeof(int64_t), cudaMemcpyDeviceToDevice, stream);
}

cudaError_t brain_fill(const BrainArgs &a, const void *work, const BrainOut &o, cudaStream_t stream) {
    const int64_t nvox = a.nx * a.ny * a.nz;
    const int64_t nblocks = (nvox + phantom::VOX - 1) / phantom::VOX;
    if (nblocks > 0)
        phantom::fill_kernel<<<(unsigned)nblocks, phantom::THREADS, 0, stream>>>(a, static_cast<const int64_t *>(work),
                                                                                o);
    return cudaGetLastError();
}

cudaError_t birdcage(int64_t nx, int64_t ny, int32_t ncoils, double relative_radius, double *out,
                     cudaStream_t stream) {
    const int64_t npix = nx * ny;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((npix + 255) / 256, 148 * 16));
    phantom::birdcage_kernel<<<blocks, 256, 0, stream>>>(nx, ny, ncoils, relative_radius, out);
    return cudaGetLastError();
}

}  // namespace homs
