// Phantom builders of libhoms (homs_brain_phantom_*, homs_csm_birdcage):
// interface between the host runtime and the kernels in homs_phantom.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace homs {

struct BrainArgs {
    int64_t nx, ny, nz;
    double res[3], offcenter[3];
    int fieldstrength;            // 0: 1.5 T, 1: 7 T
    int32_t ncoils;               // csm columns (0: one unit coil)
    const uint8_t *labels;        // device [nx*ny*nz], column-major
    const double *fieldmap;       // device [nx*ny*nz] Hz, or nullptr: the fat shift
    const double *csm;            // device complex [nx*ny*nz*ncoils], column-major, or nullptr
};

struct BrainOut {
    int64_t nspins;
    double *x, *y, *z, *rho, *T1, *T2, *T2s, *dw;  // device [nspins]
    double *csm;                                    // device complex [nspins*max(ncoils,1)], column-major
};

// Work area: one int64 per block of voxels, plus the scan's total.
size_t brain_work_bytes(int64_t nvox);

// Count the voxels whose density is not zero (*count is a device int64).
cudaError_t brain_count(const BrainArgs &a, void *work, int64_t *count, cudaStream_t stream);

// Write the voxels whose density is not zero, in column-major voxel order,
// after brain_count ran on the same arguments and work area.
cudaError_t brain_fill(const BrainArgs &a, const void *work, const BrainOut &o, cudaStream_t stream);

// Birdcage receive map of csm_Birdcage (nx x ny x ncoils complex, column-major).
cudaError_t birdcage(int64_t nx, int64_t ny, int32_t ncoils, double relative_radius, double *out,
                     cudaStream_t stream);

}  // namespace homs
