/*
 * homs.h -- C ABI of libhoms, the B200 (sm_100a) engine for HighOrderMRISim.jl's
 * BlochHighOrder simulation path.
 *
 * Plain C types only: pointers, sizes, enums.  A caller (Julia `ccall`, Python
 * `ctypes`, C/C++) passes phantom and sampled-sequence arrays that live either
 * in host memory or in device memory of the same primary CUDA context
 * (`homs_memory`), and receives the multi-coil signal and the final spin state.
 * Nothing keeps a caller pointer after a call returns.
 *
 * Array conventions follow the reference (Julia, column-major):
 *   - complex values are interleaved (re, im) pairs of the array's dtype;
 *   - csm is Ns x Nc, element (s, c) at index s + c*Ns;
 *   - the signal is Nadc x Nc, element (j, c) at index j + c*ldsig;
 *   - block ranges are 0-based inclusive node pairs (first, last); adjacent
 *     blocks share a node and its ADC belongs to the earlier block.
 *
 * Errors are returned as `homs_status`; nothing aborts, exits or traps.  The
 * message of the last failure on a context is available from
 * `homs_last_error`.  Explicit GPU requests never fall back to a CPU path.
 */
#ifndef HOMS_H
#define HOMS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HOMS_ABI_VERSION 1

typedef enum homs_status {
    HOMS_OK = 0,
    HOMS_EINVAL = 1,       /* invalid argument (the reference's ArgumentError/DimensionMismatch) */
    HOMS_ENOMEM = 2,       /* device or host allocation failed, or admission refused */
    HOMS_EUNSUPPORTED = 3, /* valid request this library cannot serve (e.g. no sm_100 device) */
    HOMS_ETIMEDOUT = 4,    /* a bounded device-side wait gave up; the context stays usable */
    HOMS_ECUDA = 5,        /* CUDA runtime error */
    HOMS_ECLOSED = 6,      /* object already closed */
    HOMS_EBUSY = 7         /* request not finished yet (polling) */
} homs_status;

typedef enum homs_dtype { HOMS_F32 = 0, HOMS_F64 = 1 } homs_dtype;

typedef enum homs_memory { HOMS_HOST = 0, HOMS_DEVICE = 1 } homs_memory;

/* Arithmetic of a run.
 *   HOMS_PLAIN  -- the reference's per-spin sequential trapezoid and fused coil
 *                  sum in the phantom's dtype (CUDA cores only);
 *   HOMS_SPLIT  -- exact integer arithmetic on the tcgen05 tensor cores: the
 *                  phase as a fixed-point turn fraction from int8 digit
 *                  products of the prefix-integrated field table and the
 *                  spins' basis values (the mod-2pi reduction is integer
 *                  wraparound), FP32 trigonometry and decay, and the coil
 *                  contraction as int8 digit products of 30-bit magnetisation
 *                  and 23-bit sensitivity integers, summed exactly (int32 per
 *                  work item, int64 across items); RF blocks and the state in
 *                  FP64.  Results are the same bit for bit on every run.
 *                  FP32 phantom and sequence arrays are widened on upload and
 *                  the signal and state are returned in FP32 (signal NRMSE
 *                  <= 1e-6 against an FP64 computation on the same inputs). */
typedef enum homs_mode { HOMS_PLAIN = 0, HOMS_SPLIT = 1 } homs_mode;

/* BlochHighOrder flags (src/simulation/BlochHighOrder.jl:21-43). */
#define HOMS_HO0 0x1u           /* zeroth order h0 */
#define HOMS_HO1 0x2u           /* first order h1..h3 (replaces nominal gradients) */
#define HOMS_HO2 0x4u           /* second order h4..h8 */
#define HOMS_HO3 0x8u           /* third order h9..h15 */
#define HOMS_DW_EXCITATION 0x10u
#define HOMS_DW_PRECESSION 0x20u

/* Phantom (src/datatypes/HO_Phantom.jl:47-71), structure of arrays. */
typedef struct homs_phantom {
    int64_t nspins;
    int32_t ncoils;
    homs_dtype dtype;
    homs_memory memory;
    const void *x, *y, *z;   /* m */
    const void *rho;
    const void *T1, *T2;     /* s */
    const void *dw;          /* rad/s */
    const void *csm;         /* complex, Ns x Nc column-major */
} homs_phantom;

/* Sampled sequence (src/datatypes/HO_DiscreteSequence.jl:31-80) plus the
 * block plan of KomaMRICore.get_sim_ranges (src/simulation/Simulate.jl:116-123). */
typedef struct homs_sequence {
    int64_t nnodes;
    homs_dtype dtype;
    homs_memory memory;
    const void *t;            /* nnodes, s */
    const void *dt;           /* nnodes-1, s */
    const void *gx, *gy, *gz; /* nnodes, T/m */
    const void *b1;           /* nnodes, complex, T */
    const void *df;           /* nnodes, Hz */
    const void *psi;          /* nnodes, rad */
    const uint8_t *adc;       /* nnodes, 0/1 */
    const void *h[16];        /* nnodes each; h0 T, h1..3 T/m, h4..8 T/m^2, h9..15 T/m^3 */
    int32_t nblocks;
    const int64_t *block_first;      /* host memory */
    const int64_t *block_last;       /* host memory */
    const uint8_t *block_excitation; /* host memory */
    double gamma;                    /* Hz/T (KomaMRIBase: 42.5774688e6) */
} homs_sequence;

typedef struct homs_run_options {
    uint32_t method; /* HOMS_HO* | HOMS_DW_* */
    homs_mode mode;
    int32_t reserved[6];
} homs_run_options;

/* Spin state (KomaMRICore Mag): xy complex, z real, Ns each, phantom dtype. */
typedef struct homs_state {
    void *xy;
    void *z;
    homs_memory memory;
} homs_state;

typedef struct homs_context homs_context;
typedef struct homs_plan homs_plan;
typedef struct homs_server homs_server;
typedef struct homs_resident homs_resident;

/* ---- library --------------------------------------------------------------- */

int homs_abi_version(void);
const char *homs_status_string(homs_status status);

/* ---- context: one device, one stream, serialised calls ----------------------- */

/* Bind a context to `device` and the caller's CUDA stream (cudaStream_t, NULL
 * for the per-thread default created by the library).  The reference binds work
 * to the current CUDA.jl device and stream (src/simulation/Simulate.jl:153-157).
 * HOST inputs and outputs of 1 MiB or more in pageable memory are staged
 * through two page-locked 8 MiB chunks that the context allocates on first use
 * (the host copy of one chunk overlaps the transfer of the other); page-locked
 * arrays are transferred as they are.  Either way a call returns once its host
 * inputs may be reused and its host outputs hold the results. */
homs_status homs_context_create(int device, void *stream, homs_context **out);
homs_status homs_context_destroy(homs_context *ctx);
const char *homs_last_error(const homs_context *ctx);
/* Wait for all work queued by this context. */
homs_status homs_synchronize(homs_context *ctx);

/* ---- block kernels: device pointers, caller's stream --------------------------
 * These replace the reference's per-block CUDA kernels one for one. */

/* Free precession over nodes [first,last] of a sampled sequence whose arrays are
 * DEVICE pointers in the phantom's dtype.  Updates state (device) in place and
 * writes the block's ADC samples to sig (device, Nadc_b x Nc, leading dimension
 * ldsig, complex of the phantom's dtype).
 * Replaces run_high_order_precession! (src/simulation/kernels/HighOrderGPU.jl:124-140)
 * with the fused kernel of src/simulation/kernels/FusedCoilGPU.jl:70-133. */
homs_status homs_precession_block(homs_context *ctx, const homs_phantom *phantom, const homs_sequence *seq,
                                  int64_t first, int64_t last, uint32_t method, homs_state *state, void *sig,
                                  int64_t ldsig);

/* RF excitation over nodes [first,last] (hard-pulse spinor per node, T2/T1 per
 * step, ADC-during-RF samples multiplied by cis(psi), psi framing at both ends).
 * Replaces run_high_order_excitation! (src/simulation/kernels/HighOrderGPU.jl:194-233). */
homs_status homs_excitation_block(homs_context *ctx, const homs_phantom *phantom, const homs_sequence *seq,
                                  int64_t first, int64_t last, uint32_t method, homs_state *state, void *sig,
                                  int64_t ldsig);

/* sig(Nadc x Nc) = transpose(states(Ns x Nadc)) * csm(Ns x Nc), no conjugation,
 * deterministic two-stage reduction; device pointers, complex of `dtype`.
 * Replaces reduce_high_order_signal! (src/simulation/kernels/CoilReductionGPU.jl:212-233)
 * and high_order_gemm! (src/simulation/kernels/HighOrderGPU.jl:162-178). */
homs_status homs_coil_reduce(homs_context *ctx, homs_dtype dtype, int64_t nspins, int64_t nadc, int32_t ncoils,
                             const void *states, int64_t ldstates, const void *csm, int64_t ldcsm, void *sig,
                             int64_t ldsig);

/* homs_coil_reduce without a context and without any device allocation; it has
 * no counterpart in the reference.  It is for callers that may not allocate
 * once running: a host whose own pooled allocator owns and budgets all device
 * memory (CUDA.jl's, PyTorch's), or a service loop where a cudaMalloc would
 * synchronise the device.  The split-K partials live in a fixed 16 MiB device
 * array inside this library (one per GPU, kept until the process exits), so
 * 16 * ceil(nspins/256) * nadc * ncoils bytes (8 * ... for f32) must fit in
 * 16 MiB and nadc may be at most 524280; larger requests return HOMS_EINVAL.
 * `stream` is a cudaStream_t on the current device (NULL = default stream);
 * the call only enqueues work.  Calls on the same device share that array, so
 * two calls whose work can overlap on the GPU (other streams, other host
 * threads) race: order them on one stream.  The first call on each device
 * (any call, also one with nadc = 0) resolves the array's address, which may
 * make the CUDA driver load this library's device code and back the array:
 * make that call at initialisation, before any stream capture; later calls
 * allocate nothing.  A device reset (cudaDeviceReset) is not supported while
 * the library is in use: the resolved address would be stale. */
homs_status homs_coil_reduce_noalloc(void *stream, homs_dtype dtype, int64_t nspins, int64_t nadc, int32_t ncoils,
                                     const void *states, int64_t ldstates, const void *csm, int64_t ldcsm, void *sig,
                                     int64_t ldsig);

/* ---- phantom builders -------------------------------------------------------------
 * The brain phantom of hophantom_brain (src/phantom/hophantom_brain.jl:2-58) built
 * on the device from a volume of tissue classes: the voxel-centre grid of
 * generate_grid (src/grid/Grid.jl:78-108) for fov = matrix .* res, plus
 * `offcenter`; T1, T2, T2s and rho per class from SpinProperty's 1.5 T or 7 T
 * tables (src/phantom/SpinProperty.jl:1-118); dw = 2 pi * field map, or the
 * fat shift -220 * 2 pi rad/s on the fat classes 93 and 209 (b0_type = :fat);
 * the caller's receive map, or one unit coil.  Only voxels with nonzero rho
 * are kept, in column-major voxel order (the reference's x[rho .!= 0]).
 * The volume is what load_phantom_mat returns: the reference reads and
 * resamples its .mat files in Julia, and those stay on the caller's side. */
typedef struct homs_brain_spec {
    int64_t nx, ny, nz;        /* target matrix */
    double res[3];             /* target resolution, m */
    double offcenter[3];       /* grid shift, m */
    int32_t fieldstrength;     /* 0: "1.5T", 1: "7T" */
    int32_t ncoils;            /* columns of csm; 0: one unit coil */
    homs_memory memory;        /* where labels, fieldmap and csm live */
    const uint8_t *labels;     /* nx*ny*nz tissue classes, column-major */
    const double *fieldmap;    /* nx*ny*nz off-resonance in Hz, or NULL for the fat shift */
    const double *csm;         /* nx*ny*nz*ncoils complex (re, im), column-major, or NULL */
} homs_brain_spec;

/* Output arrays of homs_brain_phantom_fill: nspins doubles each (T2s may be
 * NULL) and csm nspins x max(ncoils, 1) complex doubles, column-major. */
typedef struct homs_brain_out {
    int64_t nspins;            /* from homs_brain_phantom_count */
    homs_memory memory;
    double *x, *y, *z, *rho, *T1, *T2, *T2s, *dw, *csm;
} homs_brain_out;

/* Number of spins of the phantom (voxels with nonzero rho). */
homs_status homs_brain_phantom_count(homs_context *ctx, const homs_brain_spec *spec, int64_t *nspins);
/* Write the phantom's spin arrays; out->nspins must be the count above. */
homs_status homs_brain_phantom_fill(homs_context *ctx, const homs_brain_spec *spec, const homs_brain_out *out);
/* Birdcage receive map of csm_Birdcage (src/phantom/csm/Birdcage.jl:21-42):
 * nx x ny x ncoils complex doubles, column-major, in out_memory. */
homs_status homs_csm_birdcage(homs_context *ctx, int64_t nx, int64_t ny, int32_t ncoils, double relative_radius,
                              double *out, homs_memory out_memory);

/* ---- encoding export ------------------------------------------------------------
 * Generalised k-space of a sampled sequence: replaces get_kspace / grad2kspace
 * (src/datatypes/HO_Sequence.jl:236-287).  Columns 0..2 integrate the nominal
 * gradients gx, gy, gz (K_nominal) and columns 3..18 the field coefficients
 * h0..h15 (K_dfc).  Over the intervals n = 0 .. nnodes-2 of `seq`, each column
 * is KomaMRICore's cumtrapz of its node values, restarted at every RF break:
 * rf_start[i] (0-based interval index, strictly increasing, 1 <= rf_start[i] <
 * nnodes-1) begins part i+1, whose values then add rf_sign[i] times the value
 * at the end of part i (0 after an excitation, -1 after a refocusing pulse, +1
 * otherwise or when the pulse is skipped).  All values are multiplied by
 * seq->gamma (cycles/m^order).  k is (nnodes-1) x 19 FP64, column-major.
 * k_q (nq x 19, column-major) holds k at the times q_times by linear
 * interpolation over the knots t[n] + dt[n], 0 outside them (the ADC-sampled
 * K_nominal_adc / K_dfc_adc with q_times = the ADC times).  The knots must be
 * non-decreasing, as they are when dt is the difference of consecutive t;
 * otherwise k_q is unspecified (every access stays inside the arrays).
 * The RF breaks and their signs come from the caller: the reference derives
 * them from the unsampled sequence (KomaMRIBase.get_RF_types), which does not
 * cross this ABI.  seq's arrays may be host or device memory (seq->memory);
 * rf_start, rf_sign and q_times are host memory; k and k_q are in out_memory.
 * The block-plan fields of seq are not used.  Returns when k and k_q are ready. */
homs_status homs_kspace(homs_context *ctx, const homs_sequence *seq, int32_t nrf, const int64_t *rf_start,
                        const int8_t *rf_sign, int64_t nq, const double *q_times, double *k, double *k_q,
                        homs_memory out_memory);
/* Self-test of failure detection, with no counterpart in the reference: one
 * device thread waits, with a budget of `budget_cycles` (1e3 .. 4e9), on an
 * mbarrier that nothing arrives at, through the same bounded-wait code the
 * split kernel uses.  The wait runs out, the kernel records it in a device
 * error word and returns, and the call returns HOMS_ETIMEDOUT with the
 * context still usable (no trap, no fault, no hang). */
homs_status homs_selftest_wait_timeout(homs_context *ctx, int64_t budget_cycles);

/* Device time (CUDA events) of the kernels of the last homs_kspace call on ctx. */
homs_status homs_kspace_timing(homs_context *ctx, double *ms);

/* ---- whole simulation ---------------------------------------------------------- */

/* Run every block of `seq` on `phantom` (host or device arrays).
 * state: initial state in / final state out (NULL: start from Mxy=0, Mz=rho and
 * discard the final state).  sig: Nadc_total x Nc complex of the phantom's dtype
 * in `sig_memory`, leading dimension Nadc_total.
 * Replaces simulate_shard + run_sim_time_iter! (src/simulation/Simulate.jl:138-193,
 * src/simulation/SimulatorCore.jl:96-152).  The caller applies KomaMRI's ADC phase
 * compensation and builds `mat`/`state`/`raw` (src/simulation/Simulate.jl:195-214). */
homs_status homs_simulate(homs_context *ctx, const homs_phantom *phantom, const homs_sequence *seq,
                          const homs_run_options *opts, homs_state *state, void *sig, homs_memory sig_memory);

/* ---- device-resident phantoms ---------------------------------------------------
 * A phantom copied to the device once and reused by many simulations: its
 * arrays in the arithmetic's precision (FP64 for HOMS_SPLIT, the phantom's
 * dtype for HOMS_PLAIN) and, for HOMS_SPLIT, its spherical-harmonic basis table
 * and pre-split sensitivity operand.  The serving counterpart of the
 * reference's resident per-device simulation state
 * (src/simulation/PreparedSimulation.jl:144-212), kept per phantom so that
 * simulations of different sequences share it.  Immutable after creation:
 * simulations on any contexts of the same device may use it at once.  Keep it
 * alive until every simulation using it has returned (or, for the server, its
 * ticket has completed). */
homs_status homs_resident_create(homs_context *ctx, const homs_phantom *phantom, homs_mode mode,
                                 homs_resident **out);
homs_status homs_resident_device_bytes(const homs_resident *res, size_t *bytes);
homs_status homs_resident_destroy(homs_resident *res);
/* homs_simulate on a device-resident phantom: only the sequence, the state
 * and the signal move.  opts->mode must be the resident's mode (opts NULL: all
 * terms of the resident's mode).  state and sig are in the phantom's dtype as
 * given to homs_resident_create. */
homs_status homs_simulate_resident(homs_context *ctx, const homs_resident *res, const homs_sequence *seq,
                                   const homs_run_options *opts, homs_state *state, void *sig,
                                   homs_memory sig_memory);

/* Number of ADC samples the blocks of `seq` own (sum of ADC[first+1..last]). */
homs_status homs_count_adc(const homs_sequence *seq, int64_t *nadc);

/* ---- prepared plans: resident inputs, repeated runs --------------------------
 * prepare_simulation / simulate(plan) / close(plan)
 * (src/simulation/PreparedSimulation.jl:144-258).  Inputs are copied into the
 * plan's device memory at creation; each run restarts from Mxy=0, Mz=rho. */
homs_status homs_plan_create(homs_context *ctx, const homs_phantom *phantom, const homs_sequence *seq,
                             const homs_run_options *opts, homs_plan **out);
homs_status homs_plan_run(homs_plan *plan, void *sig, homs_memory sig_memory, homs_state *state_out);
/* Device bytes held by a plan (resident phantom, basis, operands, work). */
homs_status homs_plan_device_bytes(const homs_plan *plan, size_t *bytes);

/* Device timing of the plan's last run: summed CUDA-event time of the
 * dominant fused kernel (the split tcgen05 kernel in HOMS_SPLIT, the segment
 * kernel in HOMS_PLAIN), its launch count, and all kernels launched.  Plays
 * the role of the reference's per-run `sim_time_sec` (src/simulation/Simulate.jl:210)
 * at kernel granularity. */
typedef struct homs_timing {
    double fused_kernel_ms;
    int64_t fused_launches;
    int64_t kernel_launches;
} homs_timing;
homs_status homs_plan_timing(const homs_plan *plan, homs_timing *out);
/* How a plan's runs are issued.  The first run issues its kernels directly and
 * sizes every buffer; the second is captured into a CUDA graph, which later
 * runs replay (one launch of the whole block plan).  *state: 0 before the
 * capture, 1 while runs replay the graph, -1 if capture failed and runs are
 * issued directly (*why, if not NULL, then holds the reason; it stays valid
 * until the plan is destroyed).  Not in the reference, which relaunches its
 * kernels block by block (src/simulation/PreparedSimulation.jl:214-258). */
homs_status homs_plan_graph(const homs_plan *plan, int32_t *state, const char **why);
homs_status homs_plan_destroy(homs_plan *plan);

/* ---- serving: continuous batching of independent simulations --------------
 * The serving counterpart of the reference's persistent per-device worker
 * (src/simulation/PreparedSimulation.jl:2-287), which runs one simulation at a
 * time.  A server owns `slots` contexts (each with its own stream and cached
 * device workspace) and one worker thread per slot.  Requests are admitted in
 * submission order as soon as a slot is free and their estimated device
 * footprint fits in `max_device_bytes` together with the requests already in
 * flight; admitted requests run concurrently, so their kernels overlap on the
 * device.  Each request computes exactly what homs_simulate computes for it,
 * whatever else runs beside it.
 * Submission copies nothing: the phantom, sequence (including the block
 * arrays), state and signal buffers must stay valid and unchanged until the
 * request completes. */
typedef struct homs_server_options {
    int device;
    int32_t slots;            /* concurrent requests (0: 4) */
    int64_t max_device_bytes; /* admission budget for in-flight requests (0: 3/4 of free device memory) */
    int32_t reserved[4];
} homs_server_options;

/* Seconds since the server was created. */
typedef struct homs_request_times {
    double submitted, started, finished;
} homs_request_times;

homs_status homs_server_create(const homs_server_options *opts, homs_server **out);
/* Queue a simulation (the arguments of homs_simulate); *ticket identifies it. */
homs_status homs_server_submit(homs_server *srv, const homs_phantom *phantom, const homs_sequence *seq,
                               const homs_run_options *opts, homs_state *state, void *sig, homs_memory sig_memory,
                               int64_t *ticket);
/* Queue a simulation on a device-resident phantom of the server's device
 * (the arguments of homs_simulate_resident).  Its admission estimate leaves
 * out the phantom, which is already on the device. */
homs_status homs_server_submit_resident(homs_server *srv, const homs_resident *res, const homs_sequence *seq,
                                        const homs_run_options *opts, homs_state *state, void *sig,
                                        homs_memory sig_memory, int64_t *ticket);
/* HOMS_OK when the request has finished, HOMS_EBUSY while it is queued or
 * running, otherwise the status it failed with (message: homs_server_error). */
homs_status homs_server_poll(homs_server *srv, int64_t ticket);
/* Block until the request finishes or `timeout_seconds` pass (HOMS_ETIMEDOUT). */
homs_status homs_server_wait(homs_server *srv, int64_t ticket, double timeout_seconds);
homs_status homs_server_times(homs_server *srv, int64_t ticket, homs_request_times *out);
/* The request's admission estimate of its device footprint, in bytes (the
 * amount it holds of max_device_bytes while it is in flight). */
homs_status homs_server_estimate(homs_server *srv, int64_t ticket, int64_t *bytes);
const char *homs_server_error(homs_server *srv, int64_t ticket);
/* Forget a finished request. */
homs_status homs_server_release(homs_server *srv, int64_t ticket);
/* Finish every admitted and queued request, then free the server. */
homs_status homs_server_destroy(homs_server *srv);

#ifdef __cplusplus
}
#endif

#endif /* HOMS_H */
