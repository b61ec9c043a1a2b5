// Encoding export of libhoms (homs_kspace): interface between the host
// runtime and the segmented trapezoid-scan kernels in homs_kspace.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace homs {

// k[n, c] = gamma * (part-local cumulative trapezoid of column c up to interval
// n + offset of the part), n = 0 .. nnodes-2, as grad2kspace
// (src/datatypes/HO_Sequence.jl:257-287); then k at the query times by linear
// interpolation over the knots t[n] + dt[n] (0 outside them).
struct KspaceArgs {
    int64_t nnodes = 0;          // intervals: nnodes - 1
    bool f64 = true;             // element type of t, dt and the columns
    const void *t = nullptr;     // device [nnodes]
    const void *dt = nullptr;    // device [nnodes - 1]
    int32_t ncols = 0;
    const void *const *cols = nullptr;  // device array of ncols device pointers [nnodes]
    int32_t nparts = 1;
    const int64_t *starts = nullptr;    // device [nparts], first interval of each part (starts[0] = 0)
    const int8_t *signs = nullptr;      // device [nparts], weight of the previous part's end value
    double gamma = 0.0;
    int64_t nq = 0;
    const double *q = nullptr;   // device [nq] query (ADC) times
    double *k = nullptr;         // device [(nnodes - 1) x ncols], column-major
    double *kq = nullptr;        // device [nq x ncols], column-major
    void *work = nullptr;        // device workspace of kspace_work_bytes()
};

size_t kspace_work_bytes(int64_t nnodes, int32_t ncols, int32_t nparts);

// Enqueue the scan (three kernels) and the interpolation on `stream`.
cudaError_t kspace_launch(const KspaceArgs &a, cudaStream_t stream);

}  // namespace homs
