// Internal interfaces between the libhoms translation units (not part of the
// C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/homs.h"
#include "homs_split.cuh"

namespace homs {

// Shape of a device-resident phantom, for the serving loop's admission
// estimate (homs_server.cu) without knowing its layout.
struct ResidentShape {
    int64_t nspins;
    int32_t ncoils;
    homs_dtype compute;  // precision its arrays are kept in
    homs_mode mode;
    int device;
};
bool resident_shape(const homs_resident *r, ResidentShape *out);

// A split-mode simulation prepared on a context for the server's rounds
// (homs_server.cu), which issue its work on a stream of their own:
//   server_run_prepare  uploads (or attaches) the phantom and the sequence,
//                       sets the initial state and builds the split tables on
//                       the context's stream; the context stays locked until
//                       server_run_free;
//   server_run_next     issues the run's work up to its next fused job on
//                       `stream` and returns it (*has_job false: the run is
//                       complete); the first call waits for the preparation;
//   server_run_after    the job's finalize (and the state update at the end
//                       of a segment);
//   server_run_done     marks the end of the run's work on `stream`;
//   server_run_finish   waits for it on the context's stream, reads the error
//                       word and copies the signal and state out.
// Failures go to the context's last error, as in homs_simulate.
struct ServerRun;
bool server_run_eligible(const homs_phantom *p, const homs_run_options *opts);
homs_status server_run_prepare(homs_context *ctx, const homs_phantom *phantom, const homs_resident *resident,
                               const homs_sequence *seq, const homs_run_options *opts, const homs_state *state,
                               ServerRun **out);
homs_status server_run_next(ServerRun *run, cudaStream_t stream, SplitJobDesc *job, bool *has_job);
homs_status server_run_after(ServerRun *run, cudaStream_t stream);
void server_run_done(ServerRun *run, cudaStream_t stream);
cudaStream_t server_run_stream(const ServerRun *run);  // the run's context's stream
homs_status server_run_finish(ServerRun *run, void *sig, homs_memory sig_memory, homs_state *state);
void server_run_free(ServerRun *run);

}  // namespace homs
