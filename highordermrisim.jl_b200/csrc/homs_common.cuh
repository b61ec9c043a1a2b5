// Shared definitions for libhoms kernels and host runtime.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "../../include/homs.h"

namespace homs {

template <typename T>
struct cplx {
    T re, im;
};

__host__ __device__ __forceinline__ int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ int64_t imax64(int64_t a, int64_t b) { return a > b ? a : b; }

// Per-node arrays of a sampled sequence resident on the device, in type T.
template <typename T>
struct SeqDev {
    int64_t nnodes;
    const T *t, *dt, *gx, *gy, *gz, *df, *psi;
    const cplx<T> *b1;
    const uint8_t *adc;
    const uint8_t *boundary;  // 1 if the node ends a block (and starts the next)
    const T *h[16];
};

// Phantom arrays resident on the device, in type T.
template <typename T>
struct PhantomDev {
    int64_t ns;
    int32_t nc;
    const T *x, *y, *z, *rho, *T1, *T2, *dw;
    const cplx<T> *csm;  // column-major ns x nc
    int64_t ldcsm;
};

// Mutable per-spin state.
template <typename T>
struct StateDev {
    cplx<T> *xy;
    T *z;
    T *acc;  // running trapezoid sum of the current precession block
};

// One launch of the plain segment kernel: intervals [n_lo, n_hi) of a run of
// blocks of one kind (precession or excitation).
template <typename T>
struct SegmentArgs {
    int64_t n_lo, n_hi;
    int block_start;      // n_lo is the first node of a block
    T tp0;                // precession: elapsed block time at n_lo
    int64_t nsamples;     // ADC samples in (n_lo, n_hi]
    uint32_t method;
    T gamma;              // T(γ)
    double gamma_d;       // γ in FP64 (T(2π*γ) is formed from it)
    cplx<T> *partial;     // [grid][nsamples][nc]
};

constexpr int PLAIN_THREADS = 256;
constexpr int PLAIN_STAGE = 8;  // ADC samples staged per reduction

}  // namespace homs

// Internal launch entry points (host side, implemented in homs_plain.cu / homs_split.cu).
namespace homs {

template <typename T>
cudaError_t launch_segment(bool rf, const PhantomDev<T> &p, const SeqDev<T> &q, StateDev<T> &st,
                           const SegmentArgs<T> &a, int grid, cudaStream_t stream);

template <typename T>
cudaError_t launch_partial_finalize(const cplx<T> *partial, int64_t nparts, int64_t nsamples, int32_t nc,
                                    cplx<T> *sig, int64_t ldsig, cudaStream_t stream);

// Standalone coil reduction, split-K over spin ranges: coil_reduce_parts()
// partial (nadc x nc) blocks, at most ceil(ns / PLAIN_THREADS) of them, which
// launch_partial_finalize sums in part order.
int64_t coil_reduce_parts(int64_t ns, int64_t nadc, int32_t nc);

template <typename T>
cudaError_t launch_coil_reduce(int64_t ns, int64_t nadc, int32_t nc, const cplx<T> *states, int64_t ldstates,
                               const cplx<T> *csm, int64_t ldcsm, cplx<T> *partial, cudaStream_t stream);

template <typename T>
size_t segment_smem_bytes(int32_t nc);

// Allow `func` the device's largest opt-in dynamic shared memory.  The
// attribute belongs to the function, not to a launch: every caller sets the
// same value, so launches from concurrent host threads (each sizing its own
// shared memory below that limit) never see it lowered under them.
inline cudaError_t allow_max_dynamic_smem(const void *func) {
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    return e;
}

}  // namespace homs
