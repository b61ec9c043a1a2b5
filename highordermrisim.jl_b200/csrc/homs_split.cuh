// Split-precision path of libhoms (HOMS_SPLIT): interface between the host
// runtime and the tcgen05 kernels in homs_split.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace homs {

// Device operands of the split path.  The phantom-dependent ones are built
// once (split_prepare) and may be shared read-only by many runs
// (split_attach); the per-segment ones belong to each SplitResident.
//
// Phantom operands (all exact integer digits of fixed-point values):
//   basis     per-spin FP64 basis rows (state update, phase operand)
//   phase_b   per 32-spin chunk: the phase MMAs' B operand, five balanced
//             int8 digits of every spin's 16 field-term coefficients
//             (basis terms 1..15 and dw/(2 pi)), laid out for the three
//             phase MMAs
//   coil_b    per coil group and chunk: three balanced int8 digits of the
//             scaled sensitivities (real embedding of the complex product)
//   colsum    per coil group and output column: sum of the sensitivity
//             integers (undoes the offset of the top magnetisation digit)
//   term_max  per field term: the largest |coefficient| over the spins (FP64)
//   coil_exp  per coil: max |Re|,|Im| (u64 bits), then the scale exponent
struct SplitResident {
    void *basis = nullptr;
    void *phase_b = nullptr;
    void *coil_b = nullptr;
    void *colsum = nullptr;
    void *term_max = nullptr;
    void *coil_exp = nullptr;
    // per-segment work
    void *params = nullptr;   // per chunk: turn of arg(m0), -log2(e)/T2, log2|m0|
    void *prefix = nullptr;   // FP64 trapezoid prefix table, [rows][24]
    void *phase_a = nullptr;  // per 128-sample tile: the phase MMAs' A operand
    void *rows = nullptr;     // per sample: base turn (h0 term + offsets), elapsed time
    void *accum = nullptr;    // int64 coil accumulators, [tiles][slots][N][128], zero between launches
    void *amp = nullptr;      // bits of the largest |m0| of the segment (u64)
    void *err = nullptr;      // device error word
    size_t basis_bytes = 0, phase_b_bytes = 0, coil_b_bytes = 0, colsum_bytes = 0, term_max_bytes = 0,
           coil_exp_bytes = 0, params_bytes = 0, prefix_bytes = 0, phase_a_bytes = 0, rows_bytes = 0,
           accum_bytes = 0;
    int64_t ns = 0, ns_pad = 0;
    int32_t nc = 0, n_mma = 0, ngroups = 1;
    // The phantom operands belong to another SplitResident (a device-resident
    // phantom shared by many runs); the rest is this one's.
    bool phantom_view = false;
    SplitResident() = default;
    SplitResident(const SplitResident &) = delete;
    SplitResident &operator=(const SplitResident &) = delete;
    ~SplitResident();
    size_t device_bytes() const {
        return (phantom_view ? 0
                             : basis_bytes + phase_b_bytes + coil_b_bytes + colsum_bytes + term_max_bytes +
                                   coil_exp_bytes) +
               params_bytes + prefix_bytes + phase_a_bytes + rows_bytes + accum_bytes;
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

// One precession segment in pieces, for runs that share launches: the
// prologue (split_segment_begin), per coil group grp one job
// (split_segment_job) run by split_launch (alone, or with other runs' jobs of
// the same n_mma in one persistent launch) and its finalize, then the state
// update (split_segment_end).  split_run_segment is exactly this sequence for
// one run.
struct SplitSegment {
    int64_t nsamples = 0, tiles = 0, nchunks = 0;
    int32_t slabs = 0, nacc = 0;
};
struct SplitJobDesc {
    const void *phase_a, *phase_b, *coil_b, *params, *rows;
    void *accum;
    unsigned int *err;
    int32_t n_chunks, tiles, slabs, n_mma;
};
constexpr int SPLIT_MAX_JOBS = 32;  // jobs per launch
cudaError_t split_segment_begin(SplitResident &r, const SplitRunArgs &a, int64_t n_lo, int64_t n_hi, int64_t sample0,
                                int64_t nsamples, cudaStream_t stream, std::string *err, SplitSegment *seg);
SplitJobDesc split_segment_job(const SplitResident &r, const SplitSegment &seg, int grp);
cudaError_t split_launch(const SplitJobDesc *jobs, int n_jobs, cudaStream_t stream);
cudaError_t split_segment_finalize(SplitResident &r, const SplitRunArgs &a, const SplitSegment &seg, int grp,
                                   int64_t sample0, cudaStream_t stream);
cudaError_t split_segment_end(SplitResident &r, const SplitRunArgs &a, const SplitSegment &seg, cudaStream_t stream);

// Launch the bounded-wait self-test: a wait that nothing completes runs out
// after `budget_cycles` and sets code 256 in *err (device word, cleared first).
cudaError_t wait_selftest(unsigned int *err, long long budget_cycles, cudaStream_t stream);

// Read the device error word (synchronises the stream).  Sets *err if a
// bounded wait timed out or a segment's phase range is out of bounds.
cudaError_t split_check(SplitResident &r, cudaStream_t stream, std::string *err);

// Device bytes of the split path's operands per spin (phantom operands of one
// simulation with `ncoils` coils), for admission estimates.
double split_bytes_per_spin(int32_t ncoils);

}  // namespace homs
