// Split-precision path of libhoms (HOMS_SPLIT): interface between the host
// runtime and the tcgen05 kernels in homs_split.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace homs {

// Device operands that depend only on the phantom (built once per plan):
// per-spin FP64 basis rows and the receive sensitivities, scaled per coil by a
// power of two and split into FP16 hi/lo pairs, laid out in the canonical
// no-swizzle K-major UMMA layout, one operand per group of 32 coils.
struct SplitResident {
    void *basis = nullptr;     // [ns_pad][16] double
    void *b_operand = nullptr; // [groups][nchunks][4 ksteps][2N rows (hi, lo)][16 f16]
    void *spin_table = nullptr;  // per-segment spin parameters, [nchunks][608] double
    void *prefix = nullptr;    // per-segment phase table, [nadc_seg_pad][24] double
    void *tvec = nullptr;      // unused (the ADC ranks and column pointers come with SplitRunArgs)
    void *partial = nullptr;   // FP64 split-K partials, [tiles][slabs][128][N]
    void *coil_exp = nullptr;  // per coil: max |Re|,|Im| (u64 bits), then the scale exponent (int)
    void *amp = nullptr;       // per segment: bits of the largest |m0| (u64)
    void *err = nullptr;       // device error word
    size_t basis_bytes = 0, b_bytes = 0, spin_bytes = 0, prefix_bytes = 0, tvec_bytes = 0, partial_bytes = 0,
           coil_exp_bytes = 0;
    int64_t ns = 0, ns_pad = 0;
    int32_t nc = 0, n_mma = 0, ngroups = 1;
    // basis, b_operand and coil_exp belong to another SplitResident (a
    // device-resident phantom shared by many runs); the rest is this one's.
    bool phantom_view = false;
    SplitResident() = default;
    SplitResident(const SplitResident &) = delete;
    SplitResident &operator=(const SplitResident &) = delete;
    ~SplitResident();
    size_t device_bytes() const {
        return (phantom_view ? 0 : basis_bytes + b_bytes + coil_exp_bytes) + spin_bytes + prefix_bytes + tvec_bytes +
               partial_bytes;
    }
};

struct SplitRunArgs {
    size_t sizeof_T;
    int64_t ns, nt, nadc;
    int32_t nc;
    uint32_t method;
    double gamma;
    const int64_t *first, *last;
    const uint8_t *exc;
    int32_t nblocks;
    const uint8_t *adc_host;
    // device tables built once per sequence and method: the global ADC
    // sample index of every node (0-based, ownership as in the block plan)
    // and the 17 field-column pointers of the prefix table
    const int32_t *grank = nullptr;
    const void *const *src_dev = nullptr;
    bool capture = false;  // the stream is being captured into a CUDA graph
    // resident device arrays (type T = double or float per sizeof_T)
    const void *t, *dt, *gx, *gy, *gz, *b1, *df, *psi, *adc, *bnd, *h[16];
    const void *x, *y, *z, *rho, *T1, *T2, *dw, *csm_rows;
    void *xy, *mz, *acc, *sig;
    // instrumentation (optional): events bracketing the fused kernel launch and
    // a counter of kernels launched
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    int64_t *launches = nullptr;
};

// Build the phantom-dependent operands.  Sets *err (and returns cudaSuccess)
// for valid requests the split path does not serve.
cudaError_t split_prepare(SplitResident &r, int64_t ns, int32_t nc, const void *x, const void *y, const void *z,
                          const void *dw, const void *csm_rows, bool is_f64, cudaStream_t stream, std::string *err);

// Use the phantom operands of `src` (built by split_prepare, never written
// again) in runs of `r`; `src` keeps owning them and must outlive those runs.
// r's per-run buffers stay its own, so runs of different SplitResidents that
// share one `src` may overlap on the device.
cudaError_t split_attach(SplitResident &r, const SplitResident &src);

// Clear the device error word before a run.
cudaError_t split_reset_error(SplitResident &r, cudaStream_t stream);

// The 17 prefix-table column sources for a method mask: h_k when its order
// is on, the nominal gradient for k = 1..3 when the first order is off,
// NULL (zero) otherwise, and the constant-one marker for the dw column.
void split_column_sources(uint32_t method, const void *const h[16], const void *gx, const void *gy, const void *gz,
                          const void *out[17]);

// One precession segment (a run of consecutive precession blocks, nodes
// [n_lo, n_hi]) on the split tcgen05 kernel; its samples go to sig rows
// sample0 .. sample0+nsamples-1.  Updates the FP64 state.  Issues only
// kernels, memsets and (with a.capture, graph-external) event records, so it
// may run under stream capture once its buffers have their sizes.
cudaError_t split_run_segment(SplitResident &r, const SplitRunArgs &a, int64_t n_lo, int64_t n_hi, int64_t sample0,
                              int64_t nsamples, cudaStream_t stream, std::string *err);

// Launch the bounded-wait self-test: a wait that nothing completes runs out
// after `budget_cycles` and sets code 256 in *err (device word, cleared first).
cudaError_t wait_selftest(unsigned int *err, long long budget_cycles, cudaStream_t stream);

// Read the device error word (synchronises the stream).  Sets *err if a
// bounded wait timed out or the phase range check failed.
cudaError_t split_check(SplitResident &r, cudaStream_t stream, std::string *err);

}  // namespace homs
