// Coil reduction for callers that cannot allocate device memory.
//
// Some callers of this library must not call cudaMalloc/cudaFree once they
// are running: a host that hands every device byte to its own pooled
// allocator (CUDA.jl's or PyTorch's caching allocator) and budgets it, or a
// latency-bound service loop in which an allocation would synchronise the
// device and stall every stream.  homs_coil_reduce_noalloc gives them the
// coil reduction of homs_coil_reduce with no allocation at all: the split-K
// partials live in one file-scope device array of fixed size, held by every
// GPU that loads this library until the process exits.
#include <mutex>

#include "homs_common.cuh"

namespace {

constexpr size_t kScratchBytes = size_t(16) << 20;  // 16 MiB of split-K partials per device
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_reduce_scratch[kScratchBytes];

std::mutex g_scratch_mu;
void *g_scratch_ptr[kMaxDevices];  // device address of g_reduce_scratch, per device

// Device address of the scratch array on the current device.  Host code only
// sees a host-side stand-in for the array's name, so the address is resolved
// with cudaGetSymbolAddress once per device, with that device current.  That
// first resolution may make the CUDA driver load this library's device code
// and back the array (an allocation of the driver's own, which can
// synchronise the device); later calls only read the cached address.  The
// cache is per device ordinal: after a cudaDeviceReset the address would be
// stale, so a device reset is not supported while the library is in use.
homs_status scratch_for_current_device(void **out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return HOMS_ECUDA;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_reduce_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return HOMS_ECUDA;
        }
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return HOMS_OK;
}

}  // namespace

extern "C" homs_status homs_coil_reduce_noalloc(void *stream, homs_dtype dtype, int64_t nspins, int64_t nadc,
                                                int32_t ncoils, const void *states, int64_t ldstates, const void *csm,
                                                int64_t ldcsm, void *sig, int64_t ldsig) {
    using homs::cplx;
    if (dtype != HOMS_F32 && dtype != HOMS_F64) return HOMS_EINVAL;
    if (nspins < 0 || nadc < 0 || ncoils < 1) return HOMS_EINVAL;
    if (nadc > 0 && (!sig || ldsig < nadc)) return HOMS_EINVAL;
    if (nspins > 0 && nadc > 0 && (!states || ldstates < nspins)) return HOMS_EINVAL;
    if (nspins > 0 && (!csm || ldcsm < nspins)) return HOMS_EINVAL;
    // Set-up first, even for an empty request, so that a call with nadc = 0
    // at initialisation resolves (and lets the driver back) the array.
    void *scratch = nullptr;
    homs_status s = scratch_for_current_device(&scratch);
    if (s != HOMS_OK) return s;
    if (nadc == 0) return HOMS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t es = dtype == HOMS_F64 ? 16 : 8;
    if (nspins == 0) {
        return cudaMemset2DAsync(sig, es * (size_t)ldsig, 0, es * (size_t)nadc, (size_t)ncoils, st) == cudaSuccess
                   ? HOMS_OK
                   : HOMS_ECUDA;
    }
    const int64_t tiles = (nspins + homs::PLAIN_THREADS - 1) / homs::PLAIN_THREADS;
    // Every partial entry read by the finalize step is written by the reduce
    // step of the same call, so nothing in the shared array has to start at zero.
    const double need = (double)es * (double)tiles * (double)nadc * (double)ncoils;
    if (need > (double)kScratchBytes) return HOMS_EINVAL;
    if ((nadc + homs::PLAIN_STAGE - 1) / homs::PLAIN_STAGE > 65535) return HOMS_EINVAL;  // grid.y of the reduce step
    // The reduce step writes coil_reduce_parts() <= tiles partial blocks, so they fit.
    const int64_t parts = homs::coil_reduce_parts(nspins, nadc, ncoils);
    cudaError_t e;
    if (dtype == HOMS_F64) {
        e = homs::launch_coil_reduce<double>(nspins, nadc, ncoils, (const cplx<double> *)states, ldstates,
                                             (const cplx<double> *)csm, ldcsm, (cplx<double> *)scratch, st);
        if (e == cudaSuccess)
            e = homs::launch_partial_finalize<double>((const cplx<double> *)scratch, parts, nadc, ncoils,
                                                      (cplx<double> *)sig, ldsig, st);
    } else {
        e = homs::launch_coil_reduce<float>(nspins, nadc, ncoils, (const cplx<float> *)states, ldstates,
                                            (const cplx<float> *)csm, ldcsm, (cplx<float> *)scratch, st);
        if (e == cudaSuccess)
            e = homs::launch_partial_finalize<float>((const cplx<float> *)scratch, parts, nadc, ncoils,
                                                     (cplx<float> *)sig, ldsig, st);
    }
    return e == cudaSuccess ? HOMS_OK : HOMS_ECUDA;
}
