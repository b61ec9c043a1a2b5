// libhoms host runtime and C ABI (include/homs.h).
//
// A context owns one device and one stream; calls on a context are serialised
// by a mutex (the reference serialises runs of a prepared plan with plan.lock,
// src/simulation/PreparedSimulation.jl:224).  Inputs are copied into resident
// device buffers in the phantom's precision (FP64 in split mode); the block loop of
// src/simulation/SimulatorCore.jl:96-152 is planned on the host into launches
// of the fused segment kernels.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "homs_common.cuh"
#include "homs_internal.cuh"
#include "homs_kspace.cuh"
#include "homs_phantom.cuh"
#include "homs_split.cuh"

using namespace homs;

// ---------------------------------------------------------------------------
// Small utilities
// ---------------------------------------------------------------------------

namespace {

// Device buffer that grows on demand.  It owns its memory, or is a
// read-only view of another buffer (a device-resident phantom's arrays):
// ensure() never writes through a view, it replaces it with owned memory.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    bool owned = true;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), bytes(o.bytes), owned(o.owned) { o.p = nullptr; o.bytes = 0; o.owned = true; }
    DevBuf &operator=(DevBuf &&o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            bytes = o.bytes;
            owned = o.owned;
            o.p = nullptr;
            o.bytes = 0;
            o.owned = true;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    void release() {
        if (p && owned) cudaFree(p);
        p = nullptr;
        bytes = 0;
        owned = true;
    }
    void view(const DevBuf &src) {
        release();
        p = src.p;
        bytes = src.bytes;
        owned = false;
    }
    cudaError_t ensure(size_t n) {
        if (n <= bytes && p && owned) return cudaSuccess;
        release();
        if (n == 0) n = 16;
        cudaError_t e = cudaMalloc(&p, n);
        if (e == cudaSuccess) bytes = n;
        else p = nullptr;
        return e;
    }
    template <typename U>
    U *as() const { return reinterpret_cast<U *>(p); }
};

struct Failure {
    homs_status status;
    std::string msg;
};

#define HOMS_CUDA(expr)                                                                                   \
    do {                                                                                                  \
        cudaError_t e_ = (expr);                                                                          \
        if (e_ != cudaSuccess) {                                                                          \
            throw Failure{e_ == cudaErrorMemoryAllocation ? HOMS_ENOMEM : HOMS_ECUDA,                     \
                          std::string(#expr) + ": " + cudaGetErrorString(e_)};                            \
        }                                                                                                 \
    } while (0)

#define HOMS_REQUIRE(cond, msg)                         \
    do {                                                \
        if (!(cond)) throw Failure{HOMS_EINVAL, (msg)}; \
    } while (0)

size_t dsize(homs_dtype d) { return d == HOMS_F64 ? 8 : 4; }

// Element conversion kernel (device arrays of a different dtype).
template <typename D, typename S>
__global__ void convert_kernel(D *dst, const S *src, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = D(src[i]);
}

// csm column-major (s + c*ld) -> rows (s*nc + c), with type conversion.
template <typename D, typename S>
__global__ void transpose_csm_kernel(cplx<D> *dst, const S *src, int64_t ns, int32_t nc, int64_t ld) {
    const int64_t total = ns * nc;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = i / nc;
        const int32_t c = (int32_t)(i % nc);
        const S *v = src + 2 * (s + (int64_t)c * ld);
        dst[i] = cplx<D>{D(v[0]), D(v[1])};
    }
}

inline int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32)); }

}  // namespace

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------

struct homs_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string last_error;
    std::mutex mu;
    // reusable scratch
    DevBuf scratch_csm, scratch_partial, scratch_acc, scratch_bnd, scratch_sig, scratch_conv;
    // encoding export (homs_kspace): staged inputs, metadata, work and outputs,
    // and the events around its kernels
    DevBuf kspace_in, kspace_meta, kspace_work, kspace_out;
    // phantom builders: staged inputs, work area, staged outputs
    DevBuf build_in, build_work, build_out;
    DevBuf selftest_err;  // error word of homs_selftest_wait_timeout
    cudaEvent_t kspace_ev[2] = {nullptr, nullptr};
    bool kspace_timed = false;
    // Page-locked staging of pageable host inputs: two chunks and the events
    // that mark the copies reading them (created on first use).
    void *stage[2] = {nullptr, nullptr};
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};
    int stage_next = 0;  // the chunk the next staged copy fills
    // Device workspace of homs_simulate, kept between calls (per dtype) so that
    // repeated simulations reuse their buffers instead of reallocating them.
    std::unique_ptr<struct ResidentBase> cache[2];
};

namespace {

homs_status fail(homs_context *ctx, const Failure &f) {
    if (ctx) ctx->last_error = f.msg;
    return f.status;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

constexpr size_t STAGE_CHUNK = size_t(8) << 20;  // bytes per staging chunk
constexpr size_t STAGE_MIN = size_t(1) << 20;    // smaller pageable copies go to the driver as they are

bool stage_ready(homs_context *ctx) {
    if (ctx->stage[1]) return true;
    for (int b = 0; b < 2; ++b) {
        if (!ctx->stage[b] && cudaHostAlloc(&ctx->stage[b], STAGE_CHUNK, cudaHostAllocDefault) != cudaSuccess) {
            ctx->stage[b] = nullptr;
            break;
        }
        if (!ctx->stage_ev[b] && cudaEventCreateWithFlags(&ctx->stage_ev[b], cudaEventDisableTiming) != cudaSuccess) {
            ctx->stage_ev[b] = nullptr;
            break;
        }
    }
    cudaGetLastError();
    return ctx->stage[0] && ctx->stage[1] && ctx->stage_ev[0] && ctx->stage_ev[1];
}

// Ordinary pageable host memory: the only kind the staging below copies with
// the CPU.  Page-locked, managed and device memory (the last one a caller
// error under HOMS_HOST) go to cudaMemcpyAsync as they are.
bool pageable(const void *p) {
    cudaPointerAttributes at;
    const bool ok = cudaPointerGetAttributes(&at, p) == cudaSuccess;
    cudaGetLastError();
    return ok && at.type == cudaMemoryTypeUnregistered;
}

// Host -> device copy of `bytes` on the context's stream.  A page-locked
// source (allocated or registered through CUDA) goes to the copy engine as it
// is.  A pageable one is staged through the context's two page-locked
// chunks: this thread copies chunk k into one while the copy engine reads
// chunk k - 1 from the other, so contexts driven by different threads upload
// side by side.  Returns once the source may be reused, as a copy from
// pageable memory does.
void h2d(homs_context *ctx, void *dst, const void *src, size_t bytes) {
    if (bytes == 0) return;
    if (!pageable(src) || bytes < STAGE_MIN || !stage_ready(ctx)) {
        HOMS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
        return;
    }
    const char *s = static_cast<const char *>(src);
    char *d = static_cast<char *>(dst);
    for (size_t off = 0; off < bytes; off += STAGE_CHUNK) {
        const size_t n = std::min(STAGE_CHUNK, bytes - off);
        const int b = ctx->stage_next;
        ctx->stage_next ^= 1;
        HOMS_CUDA(cudaEventSynchronize(ctx->stage_ev[b]));  // the copy that last read this chunk is done
        std::memcpy(ctx->stage[b], s + off, n);
        HOMS_CUDA(cudaMemcpyAsync(d + off, ctx->stage[b], n, cudaMemcpyHostToDevice, ctx->stream));
        HOMS_CUDA(cudaEventRecord(ctx->stage_ev[b], ctx->stream));
    }
}

// Device -> host copy of `bytes` on the context's stream, the mirror of h2d: a
// page-locked destination is written by the copy engine as it is (the call
// returns at once); a pageable one receives the data through the two
// page-locked chunks (the copy engine fills one while this thread copies the
// other out) and holds it when the call returns.
void d2h(homs_context *ctx, void *dst, const void *src, size_t bytes) {
    if (bytes == 0) return;
    if (!pageable(dst) || bytes < STAGE_MIN || !stage_ready(ctx)) {
        HOMS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
        return;
    }
    const char *s = static_cast<const char *>(src);
    char *d = static_cast<char *>(dst);
    int prev = -1;
    size_t prev_off = 0, prev_n = 0;
    for (size_t off = 0; off < bytes; off += STAGE_CHUNK) {
        const size_t n = std::min(STAGE_CHUNK, bytes - off);
        const int b = ctx->stage_next;
        ctx->stage_next ^= 1;
        // The chunk's last reader was a transfer earlier on this stream, or this
        // thread's copy-out two chunks back, which has returned.
        HOMS_CUDA(cudaMemcpyAsync(ctx->stage[b], s + off, n, cudaMemcpyDeviceToHost, ctx->stream));
        HOMS_CUDA(cudaEventRecord(ctx->stage_ev[b], ctx->stream));
        if (prev >= 0) {
            HOMS_CUDA(cudaEventSynchronize(ctx->stage_ev[prev]));
            std::memcpy(d + prev_off, ctx->stage[prev], prev_n);
        }
        prev = b;
        prev_off = off;
        prev_n = n;
    }
    HOMS_CUDA(cudaEventSynchronize(ctx->stage_ev[prev]));
    std::memcpy(d + prev_off, ctx->stage[prev], prev_n);
}

// Copy `n` elements of dtype `src_dt` at `src` (host or device) into a device
// buffer of type T.
template <typename T>
void upload(homs_context *ctx, DevBuf &dst, const void *src, homs_dtype src_dt, homs_memory mem, int64_t n) {
    HOMS_CUDA(dst.ensure(sizeof(T) * (size_t)std::max<int64_t>(n, 1)));
    if (n == 0) return;
    HOMS_REQUIRE(src != nullptr, "a required input array is NULL");
    const bool same = (src_dt == HOMS_F64) == (sizeof(T) == 8);
    if (same) {
        if (mem == HOMS_HOST)
            h2d(ctx, dst.p, src, sizeof(T) * (size_t)n);
        else
            HOMS_CUDA(cudaMemcpyAsync(dst.p, src, sizeof(T) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream));
        return;
    }
    if (mem == HOMS_HOST) {
        // Staged as-is through the context's conversion buffer and converted on
        // the device; the next upload reuses the buffer only after this
        // conversion, in stream order.
        const size_t raw = dsize(src_dt) * (size_t)n;
        HOMS_CUDA(ctx->scratch_conv.ensure(raw));
        h2d(ctx, ctx->scratch_conv.p, src, raw);
        src = ctx->scratch_conv.p;
    }
    if (src_dt == HOMS_F64)
        convert_kernel<T, double><<<grid_for(n), 256, 0, ctx->stream>>>(reinterpret_cast<T *>(dst.p), static_cast<const double *>(src), n);
    else
        convert_kernel<T, float><<<grid_for(n), 256, 0, ctx->stream>>>(reinterpret_cast<T *>(dst.p), static_cast<const float *>(src), n);
    HOMS_CUDA(cudaGetLastError());
}

template <typename T>
void upload_csm_rows(homs_context *ctx, DevBuf &dst, const void *src, homs_dtype src_dt, homs_memory mem, int64_t ns,
                     int32_t nc, int64_t ld) {
    const int64_t total = ns * nc;
    HOMS_CUDA(dst.ensure(sizeof(cplx<T>) * (size_t)std::max<int64_t>(total, 1)));
    if (total == 0) return;
    HOMS_REQUIRE(src != nullptr, "csm is NULL");
    const void *dsrc = src;
    if (mem == HOMS_HOST) {
        // Staged through the context's scratch buffer (kept between calls).
        const size_t bytes = 2 * dsize(src_dt) * (size_t)(ld * (nc - 1) + ns);
        HOMS_CUDA(ctx->scratch_csm.ensure(bytes));
        h2d(ctx, ctx->scratch_csm.p, src, bytes);
        dsrc = ctx->scratch_csm.p;
    }
    if (src_dt == HOMS_F64)
        transpose_csm_kernel<T, double><<<grid_for(total), 256, 0, ctx->stream>>>(
            reinterpret_cast<cplx<T> *>(dst.p), static_cast<const double *>(dsrc), ns, nc, ld);
    else
        transpose_csm_kernel<T, float><<<grid_for(total), 256, 0, ctx->stream>>>(
            reinterpret_cast<cplx<T> *>(dst.p), static_cast<const float *>(dsrc), ns, nc, ld);
    HOMS_CUDA(cudaGetLastError());
}

void validate_phantom(const homs_phantom *p) {
    HOMS_REQUIRE(p != nullptr, "phantom is NULL");
    HOMS_REQUIRE(p->nspins >= 1, "The phantom must contain at least one spin.");
    HOMS_REQUIRE(p->ncoils >= 1, "The CSM must contain at least one coil.");
    HOMS_REQUIRE(p->dtype == HOMS_F32 || p->dtype == HOMS_F64, "phantom dtype must be f32 or f64");
    HOMS_REQUIRE(p->memory == HOMS_HOST || p->memory == HOMS_DEVICE, "invalid phantom memory kind");
    HOMS_REQUIRE(p->x && p->y && p->z && p->rho && p->T1 && p->T2 && p->dw && p->csm,
                 "every phantom array must be provided");
}

void validate_sequence(const homs_sequence *q) {
    HOMS_REQUIRE(q != nullptr, "sequence is NULL");
    HOMS_REQUIRE(q->nnodes >= 2, "The sequence must contain a simulation interval.");
    HOMS_REQUIRE(q->dtype == HOMS_F32 || q->dtype == HOMS_F64, "sequence dtype must be f32 or f64");
    HOMS_REQUIRE(q->t && q->dt && q->gx && q->gy && q->gz && q->b1 && q->df && q->psi && q->adc,
                 "every sequence array must be provided");
    for (int k = 0; k < 16; ++k) HOMS_REQUIRE(q->h[k] != nullptr, "every field coefficient array must be provided");
    HOMS_REQUIRE(q->nblocks >= 1 && q->block_first && q->block_last && q->block_excitation,
                 "The sequence must contain a simulation interval.");
    HOMS_REQUIRE(std::isfinite(q->gamma) && q->gamma > 0, "gamma must be finite and positive");
    int64_t expect = q->block_first[0];
    HOMS_REQUIRE(expect >= 0, "block ranges must be nonnegative");
    for (int32_t k = 0; k < q->nblocks; ++k) {
        HOMS_REQUIRE(q->block_first[k] == expect, "blocks must be contiguous and share boundary nodes");
        HOMS_REQUIRE(q->block_last[k] > q->block_first[k], "every block must contain at least one interval");
        HOMS_REQUIRE(q->block_last[k] < q->nnodes, "block range exceeds the sequence");
        expect = q->block_last[k];
    }
}

// Host copy of the ADC flags (the sequence may live on the device).
std::vector<uint8_t> host_adc(homs_context *ctx, const homs_sequence *q) {
    std::vector<uint8_t> adc((size_t)q->nnodes);
    if (q->memory == HOMS_HOST) {
        std::memcpy(adc.data(), q->adc, adc.size());
    } else {
        HOMS_CUDA(cudaMemcpyAsync(adc.data(), q->adc, adc.size(), cudaMemcpyDeviceToHost, ctx->stream));
        HOMS_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    return adc;
}

template <typename T>
std::vector<T> host_array(homs_context *ctx, const void *src, homs_dtype dt, homs_memory mem, int64_t n) {
    std::vector<T> out((size_t)n);
    if (n == 0) return out;
    std::vector<unsigned char> raw((size_t)n * dsize(dt));
    if (mem == HOMS_HOST) {
        std::memcpy(raw.data(), src, raw.size());
    } else {
        HOMS_CUDA(cudaMemcpyAsync(raw.data(), src, raw.size(), cudaMemcpyDeviceToHost, ctx->stream));
        HOMS_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    for (int64_t i = 0; i < n; ++i)
        out[i] = dt == HOMS_F64 ? T(reinterpret_cast<double *>(raw.data())[i]) : T(reinterpret_cast<float *>(raw.data())[i]);
    return out;
}

}  // namespace

// ---------------------------------------------------------------------------
// Resident simulation data (used by homs_simulate and prepared plans)
// ---------------------------------------------------------------------------

struct ResidentBase {
    virtual ~ResidentBase() = default;
    homs_dtype dtype = HOMS_F64;
    int64_t ns = 0, nt = 0, nadc = 0;
    int32_t nc = 0;
    virtual size_t device_bytes() const = 0;
    virtual void timing(homs_timing *out) const = 0;
};

template <typename T>
struct Resident : ResidentBase {
    DevBuf x, y, z, rho, T1, T2, dw, csm_rows;
    DevBuf t, dt, gx, gy, gz, b1, df, psi, adc, bnd, h[16];
    DevBuf xy, mz, acc, rho_init;
    DevBuf partial, sig;
    std::vector<int64_t> first, last;
    std::vector<uint8_t> exc, adc_host;
    std::vector<T> dt_host;
    double gamma = 0;
    SplitResident split;  // split-precision operands (built on demand)
    bool split_ready = false;
    // Split-path tables of the sequence: the global ADC sample index of every
    // node, and the 17 prefix-table column sources of `src_method`.
    DevBuf grank, src_table;
    bool grank_ready = false;
    uint32_t src_method = ~0u;
    // Instrumentation of the last run: events around every launch of the
    // dominant fused kernel, and a count of all kernels launched.
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
    size_t events_used = 0;
    int64_t launches = 0;

    std::pair<cudaEvent_t, cudaEvent_t> next_events() {
        if (events_used == events.size()) {
            cudaEvent_t a = nullptr, b = nullptr;
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            events.emplace_back(a, b);
        }
        return events[events_used++];
    }
    ~Resident() override {
        for (auto &e : events) {
            if (e.first) cudaEventDestroy(e.first);
            if (e.second) cudaEventDestroy(e.second);
        }
    }

    size_t device_bytes() const override {
        size_t b = x.bytes + y.bytes + z.bytes + rho.bytes + T1.bytes + T2.bytes + dw.bytes + csm_rows.bytes + t.bytes +
                   dt.bytes + gx.bytes + gy.bytes + gz.bytes + b1.bytes + df.bytes + psi.bytes + adc.bytes + bnd.bytes +
                   xy.bytes + mz.bytes + acc.bytes + rho_init.bytes + partial.bytes + sig.bytes + split.device_bytes();
        for (int k = 0; k < 16; ++k) b += h[k].bytes;
        return b;
    }

    void timing(homs_timing *out) const override {
        double ms = 0.0;
        for (size_t i = 0; i < events_used; ++i) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, events[i].first, events[i].second) == cudaSuccess) ms += t;
        }
        out->fused_kernel_ms = ms;
        out->fused_launches = (int64_t)events_used;
        out->kernel_launches = launches;
    }

    PhantomDev<T> phantom() const {
        return PhantomDev<T>{ns, nc, reinterpret_cast<T *>(x.p), reinterpret_cast<T *>(y.p), reinterpret_cast<T *>(z.p), reinterpret_cast<T *>(rho.p), reinterpret_cast<T *>(T1.p), reinterpret_cast<T *>(T2.p),
                             reinterpret_cast<T *>(dw.p), reinterpret_cast<cplx<T> *>(csm_rows.p), (int64_t)nc};
    }
    SeqDev<T> seq() const {
        SeqDev<T> q;
        q.nnodes = nt;
        q.t = reinterpret_cast<T *>(t.p);
        q.dt = reinterpret_cast<T *>(dt.p);
        q.gx = reinterpret_cast<T *>(gx.p);
        q.gy = reinterpret_cast<T *>(gy.p);
        q.gz = reinterpret_cast<T *>(gz.p);
        q.df = reinterpret_cast<T *>(df.p);
        q.psi = reinterpret_cast<T *>(psi.p);
        q.b1 = reinterpret_cast<cplx<T> *>(b1.p);
        q.adc = reinterpret_cast<uint8_t *>(adc.p);
        q.boundary = reinterpret_cast<uint8_t *>(bnd.p);
        for (int k = 0; k < 16; ++k) q.h[k] = reinterpret_cast<T *>(h[k].p);
        return q;
    }
};

namespace {

// Upload a phantom into `r` (fresh or reused: device buffers only grow).
// Host arrays may be released when this returns: copies from pageable memory
// are staged before cudaMemcpyAsync returns.
template <typename T>
void fill_phantom(homs_context *ctx, Resident<T> *r, const homs_phantom *p) {
    r->split_ready = false;
    r->dtype = sizeof(T) == 8 ? HOMS_F64 : HOMS_F32;
    r->ns = p->nspins;
    r->nc = p->ncoils;
    const int64_t ns = p->nspins;
    upload<T>(ctx, r->x, p->x, p->dtype, p->memory, ns);
    upload<T>(ctx, r->y, p->y, p->dtype, p->memory, ns);
    upload<T>(ctx, r->z, p->z, p->dtype, p->memory, ns);
    upload<T>(ctx, r->rho, p->rho, p->dtype, p->memory, ns);
    upload<T>(ctx, r->T1, p->T1, p->dtype, p->memory, ns);
    upload<T>(ctx, r->T2, p->T2, p->dtype, p->memory, ns);
    upload<T>(ctx, r->dw, p->dw, p->dtype, p->memory, ns);
    upload_csm_rows<T>(ctx, r->csm_rows, p->csm, p->dtype, p->memory, ns, p->ncoils, ns);
}

// Make `r`'s phantom a read-only view of `src`'s (a device-resident phantom
// that outlives the run), split operands included when `src` has them.
template <typename T>
void attach_phantom(Resident<T> *r, const Resident<T> &src) {
    r->dtype = src.dtype;
    r->ns = src.ns;
    r->nc = src.nc;
    r->x.view(src.x);
    r->y.view(src.y);
    r->z.view(src.z);
    r->rho.view(src.rho);
    r->T1.view(src.T1);
    r->T2.view(src.T2);
    r->dw.view(src.dw);
    r->csm_rows.view(src.csm_rows);
    r->split_ready = false;
    if (src.split_ready) {
        HOMS_CUDA(split_attach(r->split, src.split));
        r->split_ready = true;
    }
}

// Upload a sampled sequence and size the run's state and signal buffers for
// the phantom already in `r`.
template <typename T>
void fill_sequence(homs_context *ctx, Resident<T> *r, const homs_sequence *q) {
    r->nt = q->nnodes;
    r->gamma = q->gamma;
    r->grank_ready = false;
    r->src_method = ~0u;
    const int64_t ns = r->ns, nt = q->nnodes;
    upload<T>(ctx, r->t, q->t, q->dtype, q->memory, nt);
    upload<T>(ctx, r->dt, q->dt, q->dtype, q->memory, nt - 1);
    upload<T>(ctx, r->gx, q->gx, q->dtype, q->memory, nt);
    upload<T>(ctx, r->gy, q->gy, q->dtype, q->memory, nt);
    upload<T>(ctx, r->gz, q->gz, q->dtype, q->memory, nt);
    upload<T>(ctx, r->b1, q->b1, q->dtype, q->memory, 2 * nt);
    upload<T>(ctx, r->df, q->df, q->dtype, q->memory, nt);
    upload<T>(ctx, r->psi, q->psi, q->dtype, q->memory, nt);
    for (int k = 0; k < 16; ++k) upload<T>(ctx, r->h[k], q->h[k], q->dtype, q->memory, nt);
    r->adc_host = host_adc(ctx, q);
    HOMS_CUDA(r->adc.ensure((size_t)nt));
    HOMS_CUDA(cudaMemcpyAsync(r->adc.p, r->adc_host.data(), (size_t)nt, cudaMemcpyHostToDevice, ctx->stream));
    r->first.assign(q->block_first, q->block_first + q->nblocks);
    r->last.assign(q->block_last, q->block_last + q->nblocks);
    r->exc.assign(q->block_excitation, q->block_excitation + q->nblocks);
    std::vector<uint8_t> bnd((size_t)nt, 0);
    for (int64_t l : r->last) bnd[(size_t)l] = 1;
    HOMS_CUDA(r->bnd.ensure((size_t)nt));
    HOMS_CUDA(cudaMemcpyAsync(r->bnd.p, bnd.data(), (size_t)nt, cudaMemcpyHostToDevice, ctx->stream));
    r->dt_host = host_array<T>(ctx, q->dt, q->dtype, q->memory, nt - 1);
    int64_t nadc = 0;
    for (size_t k = 0; k < r->first.size(); ++k)
        for (int64_t n = r->first[k] + 1; n <= r->last[k]; ++n) nadc += r->adc_host[(size_t)n] ? 1 : 0;
    r->nadc = nadc;
    HOMS_CUDA(r->xy.ensure(sizeof(cplx<T>) * (size_t)ns));
    HOMS_CUDA(r->mz.ensure(sizeof(T) * (size_t)ns));
    HOMS_CUDA(r->acc.ensure(sizeof(T) * (size_t)ns));
    HOMS_CUDA(r->sig.ensure(sizeof(cplx<T>) * (size_t)std::max<int64_t>(nadc * r->nc, 1)));
}

template <typename T>
void fill_resident(homs_context *ctx, Resident<T> *r, const homs_phantom *p, const homs_sequence *q) {
    fill_phantom<T>(ctx, r, p);
    fill_sequence<T>(ctx, r, q);
}

template <typename T>
std::unique_ptr<Resident<T>> make_resident(homs_context *ctx, const homs_phantom *p, const homs_sequence *q) {
    auto r = std::make_unique<Resident<T>>();
    fill_resident<T>(ctx, r.get(), p, q);
    HOMS_CUDA(cudaStreamSynchronize(ctx->stream));
    return r;
}

// The context's cached workspace for dtype T, refilled with this phantom and sequence.
template <typename T>
Resident<T> *cached_resident(homs_context *ctx, const homs_phantom *p, const homs_sequence *q) {
    auto &slot = ctx->cache[sizeof(T) == 8 ? 1 : 0];
    if (!slot) slot = std::make_unique<Resident<T>>();
    Resident<T> *r = static_cast<Resident<T> *>(slot.get());
    fill_resident<T>(ctx, r, p, q);
    return r;
}

// Launch plan of the plain path: runs of same-kind blocks cut into launches
// of at most `max_samples` ADC samples.
struct Launch {
    int64_t run;
    bool rf;
    int64_t n_lo, n_hi;
    int block_start;
    double tp0;  // informational; the typed value is recomputed below
    int64_t sample0, nsamples;
};

template <typename T>
std::vector<std::pair<Launch, T>> plan_plain(const Resident<T> &r, int64_t max_samples) {
    std::vector<std::pair<Launch, T>> out;
    const auto &adc = r.adc_host;
    int64_t sample = 0;
    size_t k = 0;
    const size_t nb = r.first.size();
    while (k < nb) {
        const bool rf = r.exc[k] != 0;
        size_t k2 = k;
        while (k2 < nb && (r.exc[k2] != 0) == rf) ++k2;
        // run: blocks k .. k2-1, nodes first[k] .. last[k2-1]
        size_t blk = k;
        T tp = T(0);
        int64_t n = r.first[k];
        const int64_t n_end = r.last[k2 - 1];
        while (n < n_end) {
            Launch L{(int64_t)k, rf, n, n, n == r.first[blk] ? 1 : 0, 0.0, sample, 0};
            const T tp0 = tp;
            int64_t cnt = 0;
            int64_t m = n;
            while (m < n_end) {
                // interval m -> node m+1
                tp = tp + r.dt_host[(size_t)m];
                const bool a = adc[(size_t)(m + 1)] != 0;
                if (a) ++cnt;
                ++m;
                if (m == r.last[blk]) {
                    tp = T(0);
                    if (blk + 1 < k2) ++blk;
                }
                if (cnt >= max_samples) break;
            }
            L.n_hi = m;
            L.nsamples = cnt;
            sample += cnt;
            out.emplace_back(L, tp0);
            n = m;
        }
        k = k2;
    }
    return out;
}

template <typename T>
void run_plain(homs_context *ctx, Resident<T> &r, uint32_t method, bool capture) {
    const unsigned ev_flags = capture ? cudaEventRecordExternal : cudaEventRecordDefault;
    const int grid = (int)((r.ns + PLAIN_THREADS - 1) / PLAIN_THREADS);
    const size_t row_bytes = sizeof(cplx<T>) * (size_t)r.nc * (size_t)grid;
    const size_t budget = size_t(768) << 20;
    int64_t max_samples = std::max<int64_t>(PLAIN_STAGE, (int64_t)(budget / row_bytes));
    max_samples = std::min<int64_t>(max_samples, std::max<int64_t>(r.nadc, 1));
    auto plan = plan_plain<T>(r, max_samples);
    int64_t need = 0;
    for (auto &pl : plan) need = std::max(need, pl.first.nsamples);
    HOMS_CUDA(r.partial.ensure(row_bytes * (size_t)std::max<int64_t>(need, 1)));
    PhantomDev<T> p = r.phantom();
    SeqDev<T> q = r.seq();
    StateDev<T> st{reinterpret_cast<cplx<T> *>(r.xy.p), reinterpret_cast<T *>(r.mz.p), reinterpret_cast<T *>(r.acc.p)};
    for (auto &pl : plan) {
        const Launch &L = pl.first;
        SegmentArgs<T> a;
        a.n_lo = L.n_lo;
        a.n_hi = L.n_hi;
        a.block_start = L.block_start;
        a.tp0 = pl.second;
        a.nsamples = L.nsamples;
        a.method = method;
        a.gamma = T(r.gamma);
        a.gamma_d = r.gamma;
        a.partial = reinterpret_cast<cplx<T> *>(r.partial.p);
        auto ev = r.next_events();
        HOMS_CUDA(cudaEventRecordWithFlags(ev.first, ctx->stream, ev_flags));
        HOMS_CUDA(launch_segment<T>(L.rf, p, q, st, a, grid, ctx->stream));
        HOMS_CUDA(cudaEventRecordWithFlags(ev.second, ctx->stream, ev_flags));
        r.launches += 1;
        if (L.nsamples > 0) {
            HOMS_CUDA(launch_partial_finalize<T>(a.partial, grid, L.nsamples, r.nc,
                                                 reinterpret_cast<cplx<T> *>(r.sig.p) + L.sample0, r.nadc, ctx->stream));
            r.launches += 1;
        }
    }
}

template <typename T>
void init_state(homs_context *ctx, Resident<T> &r, const homs_state *state, homs_dtype pdt) {
    if (state && state->xy && state->z) {
        HOMS_REQUIRE(state->memory == HOMS_HOST || state->memory == HOMS_DEVICE, "invalid state memory kind");
        upload<T>(ctx, r.xy, state->xy, pdt, state->memory, 2 * r.ns);
        upload<T>(ctx, r.mz, state->z, pdt, state->memory, r.ns);
    } else {
        HOMS_CUDA(cudaMemsetAsync(r.xy.p, 0, sizeof(cplx<T>) * (size_t)r.ns, ctx->stream));
        HOMS_CUDA(cudaMemcpyAsync(r.mz.p, r.rho.p, sizeof(T) * (size_t)r.ns, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    HOMS_CUDA(cudaMemsetAsync(r.acc.p, 0, sizeof(T) * (size_t)r.ns, ctx->stream));
}

// Build the split path's phantom operands (basis table, pre-split
// sensitivities) unless `r` has them, its own or a resident phantom's.
template <typename T>
void ensure_split(homs_context *ctx, Resident<T> &r) {
    if (r.split_ready) return;
    std::string err;
    cudaError_t e = split_prepare(r.split, r.ns, r.nc, r.x.p, r.y.p, r.z.p, r.dw.p, r.csm_rows.p, sizeof(T) == 8,
                                  ctx->stream, &err);
    if (e != cudaSuccess) throw Failure{e == cudaErrorMemoryAllocation ? HOMS_ENOMEM : HOMS_ECUDA,
                                        std::string("split_prepare: ") + cudaGetErrorString(e)};
    if (!err.empty()) throw Failure{HOMS_EUNSUPPORTED, err};
    r.split_ready = true;
}

// Read the split kernel's device error word (synchronises the stream).
template <typename T>
void check_split(homs_context *ctx, Resident<T> &r) {
    std::string err;
    HOMS_CUDA(split_check(r.split, ctx->stream, &err));
    if (!err.empty())
        throw Failure{err.find("timed out") != std::string::npos ? HOMS_ETIMEDOUT : HOMS_EUNSUPPORTED, err};
}

// The split path's sequence tables: the global ADC sample index of every
// owned node (blocks share boundary nodes; a node belongs to the block that
// ends on it) and the prefix-table column sources of `method`.  Uploaded
// from the host only when the sequence or the method changed.
template <typename T>
void ensure_split_tables(homs_context *ctx, Resident<T> &r, uint32_t method) {
    if (!r.grank_ready) {
        std::vector<int32_t> g((size_t)r.nt, 0);
        int64_t c = 0;
        for (size_t k = 0; k < r.first.size(); ++k)
            for (int64_t n = r.first[k] + 1; n <= r.last[k]; ++n) {
                g[(size_t)n] = (int32_t)c;
                if (r.adc_host[(size_t)n]) ++c;
            }
        HOMS_REQUIRE(c <= INT32_MAX, "too many ADC samples for the split path");
        HOMS_CUDA(r.grank.ensure(sizeof(int32_t) * (size_t)r.nt));
        HOMS_CUDA(cudaMemcpyAsync(r.grank.p, g.data(), sizeof(int32_t) * (size_t)r.nt, cudaMemcpyHostToDevice,
                                  ctx->stream));
        r.grank_ready = true;
    }
    if (r.src_method != method) {
        const void *h[16];
        for (int k = 0; k < 16; ++k) h[k] = r.h[k].p;
        const void *src[17];
        split_column_sources(method, h, r.gx.p, r.gy.p, r.gz.p, src);
        HOMS_CUDA(r.src_table.ensure(sizeof(src)));
        HOMS_CUDA(cudaMemcpyAsync(r.src_table.p, src, sizeof(src), cudaMemcpyHostToDevice, ctx->stream));
        r.src_method = method;
    }
}

// One split-mode run of the block plan, issued in steps so that several
// runs can share the fused launches (the server's rounds):
//   next()  issues everything up to the run's next fused job -- the RF
//           launches before it and, at a segment's first coil group, the
//           segment's prologue -- and returns the job;
//   after() issues the job's finalize and, after the segment's last coil
//           group, the state update.
// A run on its own launches each job alone in between (run_resident).
template <typename T>
struct SplitRunner {
    homs_context *ctx = nullptr;
    Resident<T> *r = nullptr;
    SplitRunArgs sa{};
    std::vector<std::pair<Launch, T>> plan;
    size_t i = 0;  // next plan entry
    int grid = 0;
    size_t row_bytes = 0;
    // the segment in progress
    bool in_segment = false;
    size_t seg_next = 0;  // plan entry after the segment
    int64_t seg_sample0 = 0;
    int grp = 0;
    SplitSegment seg;

    void init(homs_context *c, Resident<T> &res, uint32_t method, bool capture) {
        ctx = c;
        r = &res;
        sa.sizeof_T = sizeof(T);
        sa.ns = res.ns;
        sa.nc = res.nc;
        sa.nt = res.nt;
        sa.nadc = res.nadc;
        sa.method = method;
        sa.gamma = res.gamma;
        sa.first = res.first.data();
        sa.last = res.last.data();
        sa.exc = res.exc.data();
        sa.nblocks = (int32_t)res.first.size();
        sa.adc_host = res.adc_host.data();
        sa.grank = reinterpret_cast<const int32_t *>(res.grank.p);
        sa.src_dev = reinterpret_cast<const void *const *>(res.src_table.p);
        sa.capture = capture;
        sa.t = res.t.p;
        sa.dt = res.dt.p;
        sa.gx = res.gx.p;
        sa.gy = res.gy.p;
        sa.gz = res.gz.p;
        sa.b1 = res.b1.p;
        sa.df = res.df.p;
        sa.psi = res.psi.p;
        sa.adc = res.adc.p;
        sa.bnd = res.bnd.p;
        for (int k = 0; k < 16; ++k) sa.h[k] = res.h[k].p;
        sa.x = res.x.p;
        sa.y = res.y.p;
        sa.z = res.z.p;
        sa.rho = res.rho.p;
        sa.T1 = res.T1.p;
        sa.T2 = res.T2.p;
        sa.dw = res.dw.p;
        sa.csm_rows = res.csm_rows.p;
        sa.xy = res.xy.p;
        sa.mz = res.mz.p;
        sa.acc = res.acc.p;
        sa.sig = res.sig.p;
        sa.launches = &res.launches;
        // RF runs use the plain FP64 excitation kernel; precession runs are
        // whole segments on the split kernel.
        grid = (int)((res.ns + PLAIN_THREADS - 1) / PLAIN_THREADS);
        row_bytes = sizeof(cplx<T>) * (size_t)res.nc * (size_t)grid;
        const int64_t max_samples = std::max<int64_t>(PLAIN_STAGE, (int64_t)((size_t(512) << 20) / row_bytes));
        plan = plan_plain<T>(res, max_samples);
        i = 0;
        in_segment = false;
    }

    void rf_launch(const Launch &L, T tp0, cudaStream_t stream) {
        HOMS_CUDA(r->partial.ensure(row_bytes * (size_t)std::max<int64_t>(L.nsamples, 1)));
        SegmentArgs<T> a;
        a.n_lo = L.n_lo;
        a.n_hi = L.n_hi;
        a.block_start = L.block_start;
        a.tp0 = tp0;
        a.nsamples = L.nsamples;
        a.method = sa.method;
        a.gamma = T(r->gamma);
        a.gamma_d = r->gamma;
        a.partial = reinterpret_cast<cplx<T> *>(r->partial.p);
        PhantomDev<T> p = r->phantom();
        SeqDev<T> q = r->seq();
        StateDev<T> st{reinterpret_cast<cplx<T> *>(r->xy.p), reinterpret_cast<T *>(r->mz.p),
                       reinterpret_cast<T *>(r->acc.p)};
        HOMS_CUDA(launch_segment<T>(true, p, q, st, a, grid, stream));
        r->launches += 1;
        if (L.nsamples > 0) {
            HOMS_CUDA(launch_partial_finalize<T>(a.partial, grid, L.nsamples, r->nc,
                                                 reinterpret_cast<cplx<T> *>(r->sig.p) + L.sample0, r->nadc, stream));
            r->launches += 1;
        }
    }

    bool next(cudaStream_t stream, SplitJobDesc *job) {
        if (in_segment) {
            *job = split_segment_job(r->split, seg, grp);
            return true;
        }
        while (i < plan.size()) {
            const Launch &L = plan[i].first;
            if (L.rf) {
                rf_launch(L, plan[i].second, stream);
                ++i;
                continue;
            }
            // merge consecutive precession launches of one run into a segment
            size_t j = i;
            int64_t ns_total = 0;
            while (j < plan.size() && !plan[j].first.rf && plan[j].first.run == L.run) {
                ns_total += plan[j].first.nsamples;
                ++j;
            }
            std::string err;
            const cudaError_t e =
                split_segment_begin(r->split, sa, L.n_lo, plan[j - 1].first.n_hi, L.sample0, ns_total, stream, &err,
                                    &seg);
            if (e != cudaSuccess) throw Failure{e == cudaErrorMemoryAllocation ? HOMS_ENOMEM : HOMS_ECUDA,
                                                std::string("split segment: ") + cudaGetErrorString(e)};
            if (!err.empty()) throw Failure{HOMS_EUNSUPPORTED, err};
            if (ns_total == 0) {
                HOMS_CUDA(split_segment_end(r->split, sa, seg, stream));
                i = j;
                continue;
            }
            in_segment = true;
            seg_next = j;
            seg_sample0 = L.sample0;
            grp = 0;
            *job = split_segment_job(r->split, seg, grp);
            return true;
        }
        return false;
    }

    void after(cudaStream_t stream) {
        HOMS_CUDA(split_segment_finalize(r->split, sa, seg, grp, seg_sample0, stream));
        if (++grp < r->split.ngroups) return;
        HOMS_CUDA(split_segment_end(r->split, sa, seg, stream));
        in_segment = false;
        i = seg_next;
    }

    bool first_group() const { return grp == 0; }
    bool last_group() const { return grp + 1 == r->split.ngroups; }
};

// Issue one run of the block plan on ctx's stream.  With `capture` the
// stream is being captured into a CUDA graph: every host-side table and
// buffer must already be in place (an earlier run of the same plan built
// them), and only kernels, memsets, device copies and graph-external event
// records are issued.  `check` reads the split kernel's error word
// afterwards (a synchronisation; not possible under capture).
template <typename T>
void run_resident(homs_context *ctx, Resident<T> &r, const homs_run_options *opts, bool capture = false,
                  bool check = true) {
    r.events_used = 0;
    r.launches = 0;
    const uint32_t method = opts ? opts->method : 0x3Fu;
    const homs_mode mode = opts ? opts->mode : HOMS_PLAIN;
    HOMS_REQUIRE((method & ~0x3Fu) == 0, "unknown method flag bits");
    if (mode == HOMS_PLAIN) {
        run_plain<T>(ctx, r, method, capture);
    } else if (mode == HOMS_SPLIT) {
        if (sizeof(T) != 8) throw Failure{HOMS_EUNSUPPORTED, "internal: split mode runs on FP64 resident arrays"};
        if (capture) {
            HOMS_REQUIRE(r.split_ready && r.grank_ready && r.src_method == method,
                         "internal: split tables missing under capture");
        } else {
            ensure_split<T>(ctx, r);
            ensure_split_tables<T>(ctx, r, method);
        }
        HOMS_CUDA(split_reset_error(r.split, ctx->stream));
        SplitRunner<T> run;
        run.init(ctx, r, method, capture);
        const unsigned ev_flags = capture ? cudaEventRecordExternal : cudaEventRecordDefault;
        std::pair<cudaEvent_t, cudaEvent_t> ev{nullptr, nullptr};
        SplitJobDesc job;
        while (run.next(ctx->stream, &job)) {
            // CUDA events around each segment's fused launches (all its coil groups)
            if (run.first_group()) {
                ev = r.next_events();
                cudaEventRecordWithFlags(ev.first, ctx->stream, ev_flags);
            }
            const cudaError_t e = split_launch(&job, 1, ctx->stream);
            if (run.last_group()) cudaEventRecordWithFlags(ev.second, ctx->stream, ev_flags);
            r.launches += 2;
            if (e != cudaSuccess) throw Failure{HOMS_ECUDA, std::string("split segment: ") + cudaGetErrorString(e)};
            run.after(ctx->stream);
        }
        if (check) check_split<T>(ctx, r);
    } else {
        throw Failure{HOMS_EINVAL, "unknown run mode"};
    }
}

// Copy `n` device elements of type T to `dst` (host or device) as `out_dt`.
// Narrowing FP64 -> FP32 runs on the device, through the conversion buffer
// when the destination is host memory.
template <typename T>
void download(homs_context *ctx, void *dst, homs_memory mem, const void *src, int64_t n, homs_dtype out_dt) {
    if (n == 0) return;
    if ((out_dt == HOMS_F64) == (sizeof(T) == 8)) {
        if (mem == HOMS_HOST)
            d2h(ctx, dst, src, sizeof(T) * (size_t)n);
        else
            HOMS_CUDA(cudaMemcpyAsync(dst, src, sizeof(T) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream));
        return;
    }
    HOMS_REQUIRE(sizeof(T) == 8 && out_dt == HOMS_F32, "internal: unsupported output conversion");
    float *narrow = static_cast<float *>(dst);
    if (mem == HOMS_HOST) {
        HOMS_CUDA(ctx->scratch_conv.ensure(sizeof(float) * (size_t)n));
        narrow = ctx->scratch_conv.as<float>();
    }
    convert_kernel<float, double><<<grid_for(n), 256, 0, ctx->stream>>>(narrow, static_cast<const double *>(src), n);
    HOMS_CUDA(cudaGetLastError());
    if (mem == HOMS_HOST) d2h(ctx, dst, narrow, sizeof(float) * (size_t)n);
}

// Signal and final state out, in the caller's dtype `out_dt`.
template <typename T>
void copy_out(homs_context *ctx, Resident<T> &r, void *sig, homs_memory sig_memory, homs_state *state,
              homs_dtype out_dt) {
    if (r.nadc * r.nc > 0) {
        HOMS_REQUIRE(sig != nullptr, "sig is NULL");
        download<T>(ctx, sig, sig_memory, r.sig.p, 2 * r.nadc * r.nc, out_dt);
    }
    if (state && state->xy && state->z) {
        download<T>(ctx, state->xy, state->memory, r.xy.p, 2 * r.ns, out_dt);
        download<T>(ctx, state->z, state->memory, r.mz.p, r.ns, out_dt);
    }
    HOMS_CUDA(cudaStreamSynchronize(ctx->stream));
}

// Split mode computes in FP64 whatever the caller's dtype: FP32 phantom and
// sequence arrays are widened on upload, and the signal and state are
// narrowed on the way out.
inline bool compute_f64(const homs_phantom *p, const homs_run_options *opts) {
    return p->dtype == HOMS_F64 || (opts && opts->mode == HOMS_SPLIT);
}

}  // namespace

// ---------------------------------------------------------------------------
// Plans
// ---------------------------------------------------------------------------

// A plan's runs are identical launch sequences on the same device buffers:
// the first run is issued directly (it builds every table and sizes every
// buffer), the second is captured into a CUDA graph, and later runs replay
// that graph.  If capture fails, the plan keeps issuing its runs directly.
struct homs_plan {
    homs_context *ctx = nullptr;
    homs_run_options opts{};
    std::unique_ptr<ResidentBase> res;
    homs_dtype out_dtype = HOMS_F64;  // the caller's dtype (the resident copy may be wider)
    cudaGraphExec_t exec = nullptr;
    int64_t runs = 0;
    bool graph_failed = false;
    std::string graph_error;
    ~homs_plan() {
        if (exec) cudaGraphExecDestroy(exec);
    }
};

// A phantom kept on one device for many simulations: its arrays in the
// arithmetic's precision and, for split mode, its basis table and pre-split
// sensitivity operand.  Immutable after creation, so runs on any number of
// contexts of that device may read it at once.
struct homs_resident {
    int device = 0;
    homs_mode mode = HOMS_PLAIN;
    homs_dtype in_dtype = HOMS_F64;  // the caller's dtype: results come back in it
    std::unique_ptr<ResidentBase> res;
};

namespace homs {
bool resident_shape(const homs_resident *r, ResidentShape *out) {
    if (!r || !r->res || !out) return false;
    out->nspins = r->res->ns;
    out->ncoils = r->res->nc;
    out->compute = r->res->dtype;
    out->mode = r->mode;
    out->device = r->device;
    return true;
}
}  // namespace homs

namespace {

// The context's cached workspace for dtype T, created empty if needed.
template <typename T>
Resident<T> *cache_slot(homs_context *ctx) {
    auto &slot = ctx->cache[sizeof(T) == 8 ? 1 : 0];
    if (!slot) slot = std::make_unique<Resident<T>>();
    return static_cast<Resident<T> *>(slot.get());
}

template <typename T>
void simulate_on_resident(homs_context *ctx, const homs_resident *res, const homs_sequence *seq,
                          const homs_run_options *opts, homs_state *state, void *sig, homs_memory sig_memory) {
    const auto &src = static_cast<const Resident<T> &>(*res->res);
    Resident<T> *r = cache_slot<T>(ctx);
    attach_phantom<T>(r, src);
    fill_sequence<T>(ctx, r, seq);
    init_state<T>(ctx, *r, state, res->in_dtype);
    run_resident<T>(ctx, *r, opts);
    copy_out<T>(ctx, *r, sig, sig_memory, state, res->in_dtype);
}

}  // namespace

namespace {

// One run of a prepared plan: directly, by capturing it into the plan's CUDA
// graph, or by replaying that graph (see homs_plan).
template <typename T>
void plan_run_typed(homs_plan *plan, void *sig, homs_memory sig_memory, homs_state *state_out) {
    homs_context *ctx = plan->ctx;
    auto &r = static_cast<Resident<T> &>(*plan->res);
    const homs_dtype rdt = sizeof(T) == 8 ? HOMS_F64 : HOMS_F32;
    bool issued = false;
    if (!plan->exec && plan->runs >= 1 && !plan->graph_failed) {
        cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            std::string why;
            try {
                init_state<T>(ctx, r, nullptr, rdt);
                run_resident<T>(ctx, r, &plan->opts, /*capture=*/true, /*check=*/false);
            } catch (const Failure &f) {
                why = f.msg;
            }
            cudaGraph_t graph = nullptr;
            e = cudaStreamEndCapture(ctx->stream, &graph);
            if (why.empty() && e == cudaSuccess && graph) {
                e = cudaGraphInstantiate(&plan->exec, graph, 0);
                if (e != cudaSuccess) {
                    plan->exec = nullptr;
                    why = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e);
                }
            } else if (why.empty()) {
                why = std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e);
            }
            if (graph) cudaGraphDestroy(graph);
            if (!why.empty()) {
                cudaGetLastError();
                plan->graph_failed = true;
                plan->graph_error = why;
            }
        } else {
            cudaGetLastError();
            plan->graph_failed = true;
            plan->graph_error = std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(e);
        }
    }
    if (plan->exec) {
        HOMS_CUDA(cudaGraphLaunch(plan->exec, ctx->stream));
        issued = true;
    }
    if (!issued) {
        init_state<T>(ctx, r, nullptr, rdt);
        run_resident<T>(ctx, r, &plan->opts, /*capture=*/false, /*check=*/false);
    }
    if (plan->opts.mode == HOMS_SPLIT) check_split<T>(ctx, r);
    copy_out<T>(ctx, r, sig, sig_memory, state_out, plan->out_dtype);
    ++plan->runs;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" {

int homs_abi_version(void) { return HOMS_ABI_VERSION; }

const char *homs_status_string(homs_status s) {
    switch (s) {
        case HOMS_OK: return "ok";
        case HOMS_EINVAL: return "invalid argument";
        case HOMS_ENOMEM: return "out of memory";
        case HOMS_EUNSUPPORTED: return "unsupported";
        case HOMS_ETIMEDOUT: return "timed out";
        case HOMS_ECUDA: return "CUDA error";
        case HOMS_ECLOSED: return "closed";
        case HOMS_EBUSY: return "busy";
    }
    return "unknown status";
}

homs_status homs_context_create(int device, void *stream, homs_context **out) {
    if (!out) return HOMS_EINVAL;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return HOMS_EUNSUPPORTED;
    }
    if (device < 0 || device >= count) return HOMS_EINVAL;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return HOMS_ECUDA;
    if (prop.major != 10) return HOMS_EUNSUPPORTED;  // sm_100a code only
    auto *ctx = new (std::nothrow) homs_context();
    if (!ctx) return HOMS_ENOMEM;
    ctx->device = device;
    DeviceGuard g(device);
    if (stream) {
        ctx->stream = static_cast<cudaStream_t>(stream);
    } else {
        if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete ctx;
            return HOMS_ECUDA;
        }
        ctx->own_stream = true;
    }
    *out = ctx;
    return HOMS_OK;
}

homs_status homs_context_destroy(homs_context *ctx) {
    if (!ctx) return HOMS_EINVAL;
    {
        DeviceGuard g(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        ctx->scratch_csm.release();
        ctx->scratch_partial.release();
        ctx->scratch_acc.release();
        ctx->scratch_bnd.release();
        ctx->scratch_sig.release();
        ctx->scratch_conv.release();
        ctx->kspace_in.release();
        ctx->kspace_meta.release();
        ctx->kspace_work.release();
        ctx->kspace_out.release();
        ctx->build_in.release();
        ctx->build_work.release();
        ctx->build_out.release();
        ctx->selftest_err.release();
        for (int b = 0; b < 2; ++b) {
            if (ctx->stage[b]) cudaFreeHost(ctx->stage[b]);
            if (ctx->stage_ev[b]) cudaEventDestroy(ctx->stage_ev[b]);
            ctx->stage[b] = nullptr;
            ctx->stage_ev[b] = nullptr;
        }
        for (cudaEvent_t &e : ctx->kspace_ev)
            if (e) cudaEventDestroy(e);
        ctx->cache[0].reset();
        ctx->cache[1].reset();
        if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    }
    delete ctx;
    return HOMS_OK;
}

const char *homs_last_error(const homs_context *ctx) { return ctx ? ctx->last_error.c_str() : "no context"; }

homs_status homs_synchronize(homs_context *ctx) {
    if (!ctx) return HOMS_EINVAL;
    DeviceGuard g(ctx->device);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return fail(ctx, Failure{HOMS_ECUDA, cudaGetErrorString(e)});
    return HOMS_OK;
}

homs_status homs_count_adc(const homs_sequence *seq, int64_t *nadc) {
    if (!seq || !nadc || !seq->adc || !seq->block_first || !seq->block_last) return HOMS_EINVAL;
    if (seq->memory != HOMS_HOST) return HOMS_EINVAL;
    int64_t c = 0;
    for (int32_t k = 0; k < seq->nblocks; ++k)
        for (int64_t n = seq->block_first[k] + 1; n <= seq->block_last[k] && n < seq->nnodes; ++n) c += seq->adc[n] ? 1 : 0;
    *nadc = c;
    return HOMS_OK;
}

homs_status homs_simulate(homs_context *ctx, const homs_phantom *phantom, const homs_sequence *seq,
                          const homs_run_options *opts, homs_state *state, void *sig, homs_memory sig_memory) {
    if (!ctx) return HOMS_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DeviceGuard g(ctx->device);
    try {
        validate_phantom(phantom);
        validate_sequence(seq);
        HOMS_REQUIRE(sig_memory == HOMS_HOST || sig_memory == HOMS_DEVICE, "invalid signal memory kind");
        if (compute_f64(phantom, opts)) {
            Resident<double> *r = cached_resident<double>(ctx, phantom, seq);
            init_state<double>(ctx, *r, state, phantom->dtype);
            run_resident<double>(ctx, *r, opts);
            copy_out<double>(ctx, *r, sig, sig_memory, state, phantom->dtype);
        } else {
            Resident<float> *r = cached_resident<float>(ctx, phantom, seq);
            init_state<float>(ctx, *r, state, phantom->dtype);
            run_resident<float>(ctx, *r, opts);
            copy_out<float>(ctx, *r, sig, sig_memory, state, phantom->dtype);
        }
        return HOMS_OK;
    } catch (const Failure &f) {
        cudaStreamSynchronize(ctx->stream);
        ctx->cache[0].reset();
        ctx->cache[1].reset();
        return fail(ctx, f);
    } catch (const std::bad_alloc &) {
        cudaStreamSynchronize(ctx->stream);
        ctx->cache[0].reset();
        ctx->cache[1].reset();
        return fail(ctx, Failure{HOMS_ENOMEM, "host allocation failed"});
    }
}

homs_status homs_plan_create(homs_context *ctx, const homs_phantom *phantom, const homs_sequence *seq,
                             const homs_run_options *opts, homs_plan **out) {
    if (!ctx || !out) return HOMS_EINVAL;
    *out = nullptr;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DeviceGuard g(ctx->device);
    try {
        validate_phantom(phantom);
        validate_sequence(seq);
        auto plan = std::make_unique<homs_plan>();
        plan->ctx = ctx;
        if (opts) plan->opts = *opts;
        else plan->opts.method = 0x3Fu;
        plan->out_dtype = phantom->dtype;
        if (compute_f64(phantom, &plan->opts)) plan->res = make_resident<double>(ctx, phantom, seq);
        else plan->res = make_resident<float>(ctx, phantom, seq);
        *out = plan.release();
        return HOMS_OK;
    } catch (const Failure &f) {
        cudaStreamSynchronize(ctx->stream);
        return fail(ctx, f);
    } catch (const std::bad_alloc &) {
        return fail(ctx, Failure{HOMS_ENOMEM, "host allocation failed"});
    }
}

homs_status homs_plan_run(homs_plan *plan, void *sig, homs_memory sig_memory, homs_state *state_out) {
    if (!plan || !plan->res) return plan ? HOMS_ECLOSED : HOMS_EINVAL;
    homs_context *ctx = plan->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DeviceGuard g(ctx->device);
    try {
        HOMS_REQUIRE(sig_memory == HOMS_HOST || sig_memory == HOMS_DEVICE, "invalid signal memory kind");
        if (plan->res->dtype == HOMS_F64) plan_run_typed<double>(plan, sig, sig_memory, state_out);
        else plan_run_typed<float>(plan, sig, sig_memory, state_out);
        return HOMS_OK;
    } catch (const Failure &f) {
        cudaStreamSynchronize(ctx->stream);
        return fail(ctx, f);
    }
}

homs_status homs_plan_device_bytes(const homs_plan *plan, size_t *bytes) {
    if (!plan || !bytes) return HOMS_EINVAL;
    if (!plan->res) return HOMS_ECLOSED;
    *bytes = plan->res->device_bytes();
    return HOMS_OK;
}

homs_status homs_plan_timing(const homs_plan *plan, homs_timing *out) {
    if (!plan || !out) return HOMS_EINVAL;
    if (!plan->res) return HOMS_ECLOSED;
    plan->res->timing(out);
    return HOMS_OK;
}

homs_status homs_plan_graph(const homs_plan *plan, int32_t *state, const char **why) {
    if (!plan || !state) return HOMS_EINVAL;
    if (!plan->res) return HOMS_ECLOSED;
    *state = plan->exec ? 1 : (plan->graph_failed ? -1 : 0);
    if (why) *why = plan->graph_error.c_str();
    return HOMS_OK;
}

homs_status homs_plan_destroy(homs_plan *plan) {
    if (!plan) return HOMS_EINVAL;
    if (plan->ctx) {
        std::lock_guard<std::mutex> lock(plan->ctx->mu);
        DeviceGuard g(plan->ctx->device);
        cudaStreamSynchronize(plan->ctx->stream);
        if (plan->exec) cudaGraphExecDestroy(plan->exec);
        plan->exec = nullptr;
        plan->res.reset();
    }
    delete plan;
    return HOMS_OK;
}

}  // extern "C"

// ---- block kernels on caller device arrays -----------------------------------

namespace {

template <typename T>
homs_status block_impl(homs_context *ctx, bool rf, const homs_phantom *p, const homs_sequence *q, int64_t first,
                       int64_t last, uint32_t method, homs_state *state, void *sig, int64_t ldsig) {
    validate_phantom(p);
    HOMS_REQUIRE(p->memory == HOMS_DEVICE, "block kernels take device arrays");
    HOMS_REQUIRE(q && q->memory == HOMS_DEVICE && q->dtype == p->dtype, "sequence must be device arrays of the phantom dtype");
    HOMS_REQUIRE(q->nnodes >= 2, "The sequence must contain a simulation interval.");
    HOMS_REQUIRE(first >= 0 && last > first && last < q->nnodes, "invalid block node range");
    HOMS_REQUIRE(state && state->xy && state->z && state->memory == HOMS_DEVICE, "state must be device arrays");
    HOMS_REQUIRE((method & ~0x3Fu) == 0, "unknown method flag bits");
    const int64_t ns = p->nspins, nt = q->nnodes;
    const int32_t nc = p->ncoils;
    // ADC count of the block.
    std::vector<uint8_t> adc((size_t)(last - first));
    HOMS_CUDA(cudaMemcpyAsync(adc.data(), q->adc + first + 1, adc.size(), cudaMemcpyDeviceToHost, ctx->stream));
    HOMS_CUDA(cudaStreamSynchronize(ctx->stream));
    int64_t nadc = 0;
    for (auto v : adc) nadc += v ? 1 : 0;
    HOMS_REQUIRE(nadc == 0 || (sig != nullptr && ldsig >= nadc), "sig is NULL or its leading dimension is too small");
    // Boundary flags: only `last` ends a block.
    HOMS_CUDA(ctx->scratch_bnd.ensure((size_t)nt));
    HOMS_CUDA(cudaMemsetAsync(ctx->scratch_bnd.p, 0, (size_t)nt, ctx->stream));
    const uint8_t one = 1;
    HOMS_CUDA(cudaMemcpyAsync(reinterpret_cast<uint8_t *>(ctx->scratch_bnd.p) + last, &one, 1, cudaMemcpyHostToDevice, ctx->stream));
    upload_csm_rows<T>(ctx, ctx->scratch_csm, p->csm, p->dtype, HOMS_DEVICE, ns, nc, ns);
    HOMS_CUDA(ctx->scratch_acc.ensure(sizeof(T) * (size_t)ns));
    const int grid = (int)((ns + PLAIN_THREADS - 1) / PLAIN_THREADS);
    HOMS_CUDA(ctx->scratch_partial.ensure(sizeof(cplx<T>) * (size_t)grid * (size_t)std::max<int64_t>(nadc, 1) * nc));
    HOMS_CUDA(ctx->scratch_sig.ensure(sizeof(cplx<T>) * (size_t)std::max<int64_t>(nadc, 1) * nc));
    PhantomDev<T> pd{ns, nc, (const T *)p->x, (const T *)p->y, (const T *)p->z, (const T *)p->rho, (const T *)p->T1,
                     (const T *)p->T2, (const T *)p->dw, reinterpret_cast<cplx<T> *>(ctx->scratch_csm.p), nc};
    SeqDev<T> qd;
    qd.nnodes = nt;
    qd.t = (const T *)q->t;
    qd.dt = (const T *)q->dt;
    qd.gx = (const T *)q->gx;
    qd.gy = (const T *)q->gy;
    qd.gz = (const T *)q->gz;
    qd.df = (const T *)q->df;
    qd.psi = (const T *)q->psi;
    qd.b1 = (const cplx<T> *)q->b1;
    qd.adc = q->adc;
    qd.boundary = reinterpret_cast<uint8_t *>(ctx->scratch_bnd.p);
    for (int k = 0; k < 16; ++k) qd.h[k] = (const T *)q->h[k];
    StateDev<T> st{(cplx<T> *)state->xy, (T *)state->z, reinterpret_cast<T *>(ctx->scratch_acc.p)};
    SegmentArgs<T> a;
    a.n_lo = first;
    a.n_hi = last;
    a.block_start = 1;
    a.tp0 = T(0);
    a.nsamples = nadc;
    a.method = method;
    a.gamma = T(q->gamma);
    a.gamma_d = q->gamma;
    a.partial = reinterpret_cast<cplx<T> *>(ctx->scratch_partial.p);
    HOMS_CUDA(launch_segment<T>(rf, pd, qd, st, a, grid, ctx->stream));
    if (nadc > 0) {
        HOMS_CUDA(launch_partial_finalize<T>(a.partial, grid, nadc, nc, reinterpret_cast<cplx<T> *>(ctx->scratch_sig.p), nadc, ctx->stream));
        HOMS_CUDA(cudaMemcpy2DAsync(sig, sizeof(cplx<T>) * (size_t)ldsig, ctx->scratch_sig.p, sizeof(cplx<T>) * (size_t)nadc,
                                    sizeof(cplx<T>) * (size_t)nadc, (size_t)nc, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    return HOMS_OK;
}

}  // namespace

extern "C" {

homs_status homs_precession_block(homs_context *ctx, const homs_phantom *phantom, const homs_sequence *seq,
                                  int64_t first, int64_t last, uint32_t method, homs_state *state, void *sig,
                                  int64_t ldsig) {
    if (!ctx) return HOMS_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DeviceGuard g(ctx->device);
    try {
        if (!phantom) throw Failure{HOMS_EINVAL, "phantom is NULL"};
        return phantom->dtype == HOMS_F64
                   ? block_impl<double>(ctx, false, phantom, seq, first, last, method, state, sig, ldsig)
                   : block_impl<float>(ctx, false, phantom, seq, first, last, method, state, sig, ldsig);
    } catch (const Failure &f) {
        return fail(ctx, f);
    }
}

homs_status homs_excitation_block(homs_context *ctx, const homs_phantom *phantom, const homs_sequence *seq,
                                  int64_t first, int64_t last, uint32_t method, homs_state *state, void *sig,
                                  int64_t ldsig) {
    if (!ctx) return HOMS_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DeviceGuard g(ctx->device);
    try {
        if (!phantom) throw Failure{HOMS_EINVAL, "phantom is NULL"};
        return phantom->dtype == HOMS_F64
                   ? block_impl<double>(ctx, true, phantom, seq, first, last, method, state, sig, ldsig)
                   : block_impl<float>(ctx, true, phantom, seq, first, last, method, state, sig, ldsig);
    } catch (const Failure &f) {
        return fail(ctx, f);
    }
}

homs_status homs_coil_reduce(homs_context *ctx, homs_dtype dtype, int64_t nspins, int64_t nadc, int32_t ncoils,
                             const void *states, int64_t ldstates, const void *csm, int64_t ldcsm, void *sig,
                             int64_t ldsig) {
    if (!ctx) return HOMS_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DeviceGuard g(ctx->device);
    try {
        HOMS_REQUIRE(dtype == HOMS_F32 || dtype == HOMS_F64, "dtype must be f32 or f64");
        HOMS_REQUIRE(nspins >= 0 && nadc >= 0 && ncoils >= 1, "States, CSM, and signal dimensions do not match.");
        HOMS_REQUIRE(nadc == 0 || (sig && ldsig >= nadc), "sig is NULL or its leading dimension is too small");
        HOMS_REQUIRE(nspins == 0 || nadc == 0 || (states && ldstates >= nspins), "states is NULL or ldstates < nspins");
        HOMS_REQUIRE(nspins == 0 || (csm && ldcsm >= nspins), "csm is NULL or ldcsm < nspins");
        if (nadc == 0) return HOMS_OK;
        const size_t es = dtype == HOMS_F64 ? 16 : 8;
        if (nspins == 0) {
            HOMS_CUDA(cudaMemset2DAsync(sig, es * (size_t)ldsig, 0, es * (size_t)nadc, (size_t)ncoils, ctx->stream));
            return HOMS_OK;
        }
        HOMS_REQUIRE((nadc + PLAIN_STAGE - 1) / PLAIN_STAGE <= 65535,
                     "nadc above 524280 samples per call (the reduction's grid)");
        const int64_t parts = coil_reduce_parts(nspins, nadc, ncoils);
        HOMS_CUDA(ctx->scratch_partial.ensure(es * (size_t)parts * (size_t)nadc * (size_t)ncoils));
        if (dtype == HOMS_F64) {
            HOMS_CUDA(launch_coil_reduce<double>(nspins, nadc, ncoils, (const cplx<double> *)states, ldstates,
                                                 (const cplx<double> *)csm, ldcsm, reinterpret_cast<cplx<double> *>(ctx->scratch_partial.p),
                                                 ctx->stream));
            HOMS_CUDA(launch_partial_finalize<double>(reinterpret_cast<cplx<double> *>(ctx->scratch_partial.p), parts, nadc, ncoils,
                                                      (cplx<double> *)sig, ldsig, ctx->stream));
        } else {
            HOMS_CUDA(launch_coil_reduce<float>(nspins, nadc, ncoils, (const cplx<float> *)states, ldstates,
                                                (const cplx<float> *)csm, ldcsm, reinterpret_cast<cplx<float> *>(ctx->scratch_partial.p),
                                                ctx->stream));
            HOMS_CUDA(launch_partial_finalize<float>(reinterpret_cast<cplx<float> *>(ctx->scratch_partial.p), parts, nadc, ncoils,
                                                     (cplx<float> *)sig, ldsig, ctx->stream));
        }
        return HOMS_OK;
    } catch (const Failure &f) {
        return fail(ctx, f);
    }
}

homs_status homs_resident_create(homs_context *ctx, const homs_phantom *phantom, homs_mode mode,
                                 homs_resident **out) {
    if (!ctx || !out) return HOMS_EINVAL;
    *out = nullptr;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DeviceGuard g(ctx->device);
    try {
        validate_phantom(phantom);
        HOMS_REQUIRE(mode == HOMS_PLAIN || mode == HOMS_SPLIT, "unknown run mode");
        auto h = std::make_unique<homs_resident>();
        h->device = ctx->device;
        h->mode = mode;
        h->in_dtype = phantom->dtype;
        homs_run_options o{};
        o.mode = mode;
        if (compute_f64(phantom, &o)) {
            auto r = std::make_unique<Resident<double>>();
            fill_phantom<double>(ctx, r.get(), phantom);
            if (mode == HOMS_SPLIT) ensure_split<double>(ctx, *r);
            h->res = std::move(r);
        } else {
            auto r = std::make_unique<Resident<float>>();
            fill_phantom<float>(ctx, r.get(), phantom);
            h->res = std::move(r);
        }
        HOMS_CUDA(cudaStreamSynchronize(ctx->stream));
        *out = h.release();
        return HOMS_OK;
    } catch (const Failure &f) {
        cudaStreamSynchronize(ctx->stream);
        return fail(ctx, f);
    } catch (const std::bad_alloc &) {
        return fail(ctx, Failure{HOMS_ENOMEM, "host allocation failed"});
    }
}

homs_status homs_resident_device_bytes(const homs_resident *res, size_t *bytes) {
    if (!res || !res->res || !bytes) return HOMS_EINVAL;
    *bytes = res->res->device_bytes();
    return HOMS_OK;
}

homs_status homs_resident_destroy(homs_resident *res) {
    if (!res) return HOMS_EINVAL;
    {
        DeviceGuard g(res->device);
        res->res.reset();
    }
    delete res;
    return HOMS_OK;
}

homs_status homs_simulate_resident(homs_context *ctx, const homs_resident *res, const homs_sequence *seq,
                                   const homs_run_options *opts, homs_state *state, void *sig,
                                   homs_memory sig_memory) {
    if (!ctx || !res || !res->res) return HOMS_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DeviceGuard g(ctx->device);
    try {
        HOMS_REQUIRE(res->device == ctx->device, "the resident phantom lives on another device than the context");
        validate_sequence(seq);
        HOMS_REQUIRE(sig_memory == HOMS_HOST || sig_memory == HOMS_DEVICE, "invalid signal memory kind");
        homs_run_options o{};
        o.method = 0x3Fu;
        o.mode = res->mode;
        if (opts) o = *opts;
        HOMS_REQUIRE(o.mode == res->mode, "the run mode must be the one the resident phantom was prepared for");
        if (res->res->dtype == HOMS_F64) simulate_on_resident<double>(ctx, res, seq, &o, state, sig, sig_memory);
        else simulate_on_resident<float>(ctx, res, seq, &o, state, sig, sig_memory);
        return HOMS_OK;
    } catch (const Failure &f) {
        cudaStreamSynchronize(ctx->stream);
        ctx->cache[0].reset();
        ctx->cache[1].reset();
        return fail(ctx, f);
    } catch (const std::bad_alloc &) {
        cudaStreamSynchronize(ctx->stream);
        ctx->cache[0].reset();
        ctx->cache[1].reset();
        return fail(ctx, Failure{HOMS_ENOMEM, "host allocation failed"});
    }
}

}  // extern "C"

namespace {

// Device view of a brain spec: host inputs are staged into ctx->build_in.
BrainArgs brain_args(homs_context *ctx, const homs_brain_spec *spec) {
    HOMS_REQUIRE(spec != nullptr, "spec is NULL");
    HOMS_REQUIRE(spec->nx >= 1 && spec->ny >= 1 && spec->nz >= 1, "Target matrix dimensions must be positive.");
    for (int k = 0; k < 3; ++k) {
        HOMS_REQUIRE(std::isfinite(spec->res[k]) && spec->res[k] > 0, "Target voxel sizes must be finite and positive.");
        HOMS_REQUIRE(std::isfinite(spec->offcenter[k]), "The off-centre shift must be finite.");
    }
    HOMS_REQUIRE(spec->fieldstrength == 0 || spec->fieldstrength == 1, "Field strength available: 1.5T, 7T");
    HOMS_REQUIRE(spec->ncoils >= 0 && (spec->ncoils == 0 || spec->csm), "csm is NULL for ncoils > 0");
    HOMS_REQUIRE(spec->labels != nullptr, "labels is NULL");
    HOMS_REQUIRE(spec->memory == HOMS_HOST || spec->memory == HOMS_DEVICE, "invalid memory kind");
    const int64_t nvox = spec->nx * spec->ny * spec->nz;
    HOMS_REQUIRE(nvox / spec->nx / spec->ny == spec->nz, "target matrix too large");
    BrainArgs a;
    a.nx = spec->nx;
    a.ny = spec->ny;
    a.nz = spec->nz;
    for (int k = 0; k < 3; ++k) {
        a.res[k] = spec->res[k];
        a.offcenter[k] = spec->offcenter[k];
    }
    a.fieldstrength = spec->fieldstrength;
    a.ncoils = spec->ncoils;
    a.labels = spec->labels;
    a.fieldmap = spec->fieldmap;
    a.csm = spec->ncoils > 0 ? spec->csm : nullptr;
    if (spec->memory == HOMS_HOST) {
        // Every staged array starts on a 256-byte boundary (the kernel reads
        // the sensitivities as 16-byte pairs).
        const size_t lab = ((size_t)nvox + 255) & ~size_t(255);
        const size_t fm = spec->fieldmap ? ((sizeof(double) * (size_t)nvox + 255) & ~size_t(255)) : 0;
        const size_t cs = a.csm ? 2 * sizeof(double) * (size_t)nvox * (size_t)spec->ncoils : 0;
        HOMS_CUDA(ctx->build_in.ensure(lab + fm + cs));
        uint8_t *b = ctx->build_in.as<uint8_t>();
        h2d(ctx, b, spec->labels, (size_t)nvox);
        a.labels = b;
        if (fm) {
            h2d(ctx, b + lab, spec->fieldmap, sizeof(double) * (size_t)nvox);
            a.fieldmap = reinterpret_cast<const double *>(b + lab);
        }
        if (cs) {
            h2d(ctx, b + lab + fm, a.csm, cs);
            a.csm = reinterpret_cast<const double *>(b + lab + fm);
        }
    }
    HOMS_REQUIRE(!a.csm || (reinterpret_cast<uintptr_t>(a.csm) & 15) == 0, "csm must be 16-byte aligned");
    HOMS_CUDA(ctx->build_work.ensure(brain_work_bytes(nvox) + sizeof(int64_t)));
    return a;
}

int64_t brain_count_sync(homs_context *ctx, const BrainArgs &a) {
    int64_t *dcount = reinterpret_cast<int64_t *>(ctx->build_work.as<uint8_t>() + brain_work_bytes(a.nx * a.ny * a.nz));
    HOMS_CUDA(brain_count(a, ctx->build_work.p, dcount, ctx->stream));
    int64_t n = 0;
    HOMS_CUDA(cudaMemcpyAsync(&n, dcount, sizeof(n), cudaMemcpyDeviceToHost, ctx->stream));
    HOMS_CUDA(cudaStreamSynchronize(ctx->stream));
    return n;
}

}  // namespace

extern "C" {

homs_status homs_brain_phantom_count(homs_context *ctx, const homs_brain_spec *spec, int64_t *nspins) {
    if (!ctx || !nspins) return HOMS_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DeviceGuard g(ctx->device);
    try {
        const BrainArgs a = brain_args(ctx, spec);
        *nspins = brain_count_sync(ctx, a);
        return HOMS_OK;
    } catch (const Failure &f) {
        cudaStreamSynchronize(ctx->stream);
        return fail(ctx, f);
    }
}

homs_status homs_brain_phantom_fill(homs_context *ctx, const homs_brain_spec *spec, const homs_brain_out *out) {
    if (!ctx || !out) return HOMS_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DeviceGuard g(ctx->device);
    try {
        const BrainArgs a = brain_args(ctx, spec);
        HOMS_REQUIRE(out->memory == HOMS_HOST || out->memory == HOMS_DEVICE, "invalid output memory kind");
        HOMS_REQUIRE(out->x && out->y && out->z && out->rho && out->T1 && out->T2 && out->dw && out->csm,
                     "every output array but T2s must be provided");
        const int64_t n = brain_count_sync(ctx, a);
        HOMS_REQUIRE(out->nspins == n, "out->nspins must be the spin count of the phantom");
        const int64_t nc = std::max<int32_t>(spec->ncoils, 1);
        BrainOut o;
        o.nspins = n;
        double *host[9] = {out->x, out->y, out->z, out->rho, out->T1, out->T2, out->T2s, out->dw, out->csm};
        const size_t len[9] = {1, 1, 1, 1, 1, 1, 1, 1, 2 * (size_t)nc};
        double *dev[9];
        if (out->memory == HOMS_DEVICE) {
            for (int k = 0; k < 9; ++k) dev[k] = host[k];
            HOMS_REQUIRE((reinterpret_cast<uintptr_t>(out->csm) & 15) == 0, "out->csm must be 16-byte aligned");
        } else {
            auto padded = [&](int k) {
                return (sizeof(double) * len[k] * (size_t)std::max<int64_t>(n, 1) + 255) & ~size_t(255);
            };
            size_t total = 0;
            for (int k = 0; k < 9; ++k) total += padded(k);
            HOMS_CUDA(ctx->build_out.ensure(total));
            uint8_t *p = ctx->build_out.as<uint8_t>();
            for (int k = 0; k < 9; ++k) {
                dev[k] = host[k] ? reinterpret_cast<double *>(p) : nullptr;
                p += padded(k);
            }
        }
        o.x = dev[0];
        o.y = dev[1];
        o.z = dev[2];
        o.rho = dev[3];
        o.T1 = dev[4];
        o.T2 = dev[5];
        o.T2s = dev[6];
        o.dw = dev[7];
        o.csm = dev[8];
        if (n > 0) HOMS_CUDA(brain_fill(a, ctx->build_work.p, o, ctx->stream));
        if (out->memory == HOMS_HOST && n > 0)
            for (int k = 0; k < 9; ++k)
                if (host[k])
                    d2h(ctx, host[k], dev[k], sizeof(double) * len[k] * (size_t)n);
        HOMS_CUDA(cudaStreamSynchronize(ctx->stream));
        return HOMS_OK;
    } catch (const Failure &f) {
        cudaStreamSynchronize(ctx->stream);
        return fail(ctx, f);
    }
}

homs_status homs_csm_birdcage(homs_context *ctx, int64_t nx, int64_t ny, int32_t ncoils, double relative_radius,
                              double *out, homs_memory out_memory) {
    if (!ctx) return HOMS_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DeviceGuard g(ctx->device);
    try {
        HOMS_REQUIRE(nx >= 1 && ny >= 1 && ncoils >= 1, "nX, nY and nCoil must be positive");
        HOMS_REQUIRE(std::isfinite(relative_radius), "relative_radius must be finite");
        HOMS_REQUIRE(out != nullptr, "out is NULL");
        HOMS_REQUIRE(out_memory == HOMS_HOST || out_memory == HOMS_DEVICE, "invalid output memory kind");
        const size_t bytes = 2 * sizeof(double) * (size_t)nx * (size_t)ny * (size_t)ncoils;
        double *dst = out;
        if (out_memory == HOMS_HOST) {
            HOMS_CUDA(ctx->build_out.ensure(bytes));
            dst = ctx->build_out.as<double>();
        }
        HOMS_CUDA(birdcage(nx, ny, ncoils, relative_radius, dst, ctx->stream));
        if (out_memory == HOMS_HOST) d2h(ctx, out, dst, bytes);
        HOMS_CUDA(cudaStreamSynchronize(ctx->stream));
        return HOMS_OK;
    } catch (const Failure &f) {
        cudaStreamSynchronize(ctx->stream);
        return fail(ctx, f);
    }
}

homs_status homs_kspace(homs_context *ctx, const homs_sequence *seq, int32_t nrf, const int64_t *rf_start,
                        const int8_t *rf_sign, int64_t nq, const double *q_times, double *k, double *k_q,
                        homs_memory out_memory) {
    if (!ctx) return HOMS_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DeviceGuard g(ctx->device);
    ctx->kspace_timed = false;
    try {
        HOMS_REQUIRE(seq != nullptr, "sequence is NULL");
        HOMS_REQUIRE(seq->nnodes >= 2, "Cannot integrate an empty sequence.");
        HOMS_REQUIRE(seq->dtype == HOMS_F32 || seq->dtype == HOMS_F64, "sequence dtype must be f32 or f64");
        HOMS_REQUIRE(seq->memory == HOMS_HOST || seq->memory == HOMS_DEVICE, "invalid sequence memory kind");
        HOMS_REQUIRE(seq->t && seq->dt && seq->gx && seq->gy && seq->gz, "t, dt, gx, gy and gz must be provided");
        for (int c = 0; c < 16; ++c) HOMS_REQUIRE(seq->h[c] != nullptr, "every field coefficient array must be provided");
        HOMS_REQUIRE(std::isfinite(seq->gamma) && seq->gamma > 0, "gamma must be finite and positive");
        HOMS_REQUIRE(out_memory == HOMS_HOST || out_memory == HOMS_DEVICE, "invalid output memory kind");
        HOMS_REQUIRE(k != nullptr, "k is NULL");
        HOMS_REQUIRE(nrf >= 0 && (nrf == 0 || (rf_start && rf_sign)), "RF break arrays are NULL");
        HOMS_REQUIRE(nq >= 0 && (nq == 0 || (q_times && k_q)), "query times or k_q is NULL");
        const int64_t nn = seq->nnodes, m = nn - 1;
        for (int32_t i = 0; i < nrf; ++i) {
            HOMS_REQUIRE(rf_start[i] >= 1 && rf_start[i] < m, "RF breaks must lie inside the sequence's intervals");
            HOMS_REQUIRE(i == 0 || rf_start[i] > rf_start[i - 1], "RF breaks must be strictly increasing");
            HOMS_REQUIRE(rf_sign[i] >= -1 && rf_sign[i] <= 1, "RF signs must be -1, 0 or 1");
        }
        for (int64_t j = 0; j < nq; ++j) HOMS_REQUIRE(std::isfinite(q_times[j]), "query times must be finite");
        constexpr int32_t NCOLS = 19;  // gx, gy, gz, h0 .. h15
        const int32_t nparts = nrf + 1;
        const size_t es = dsize(seq->dtype);
        // Device inputs: the caller's arrays, or a staged copy of host arrays.
        const void *dev_t = seq->t, *dev_dt = seq->dt;
        const void *cols[NCOLS] = {seq->gx, seq->gy, seq->gz};
        for (int c = 0; c < 16; ++c) cols[3 + c] = seq->h[c];
        if (seq->memory == HOMS_HOST) {
            const size_t col_bytes = (es * (size_t)nn + 255) & ~size_t(255);
            HOMS_CUDA(ctx->kspace_in.ensure(col_bytes * (NCOLS + 2)));
            uint8_t *base = ctx->kspace_in.as<uint8_t>();
            h2d(ctx, base, seq->t, es * (size_t)nn);
            h2d(ctx, base + col_bytes, seq->dt, es * (size_t)m);
            dev_t = base;
            dev_dt = base + col_bytes;
            for (int c = 0; c < NCOLS; ++c) {
                uint8_t *dst = base + (size_t)(2 + c) * col_bytes;
                h2d(ctx, dst, cols[c], es * (size_t)nn);
                cols[c] = dst;
            }
        }
        // Metadata: column pointers, part starts, query times, part signs.
        std::vector<uint8_t> meta;
        const size_t off_starts = sizeof(void *) * NCOLS;
        const size_t off_q = off_starts + sizeof(int64_t) * (size_t)nparts;
        const size_t off_signs = off_q + sizeof(double) * (size_t)nq;
        meta.resize(off_signs + (size_t)nparts);
        std::memcpy(meta.data(), cols, sizeof(void *) * NCOLS);
        int64_t *st = reinterpret_cast<int64_t *>(meta.data() + off_starts);
        int8_t *sg = reinterpret_cast<int8_t *>(meta.data() + off_signs);
        st[0] = 0;
        sg[0] = 0;
        for (int32_t i = 0; i < nrf; ++i) {
            st[i + 1] = rf_start[i];
            sg[i + 1] = rf_sign[i];
        }
        if (nq > 0) std::memcpy(meta.data() + off_q, q_times, sizeof(double) * (size_t)nq);
        HOMS_CUDA(ctx->kspace_meta.ensure(meta.size()));
        uint8_t *dmeta = ctx->kspace_meta.as<uint8_t>();
        HOMS_CUDA(cudaMemcpyAsync(dmeta, meta.data(), meta.size(), cudaMemcpyHostToDevice, ctx->stream));
        // Outputs: the caller's device arrays or a staging buffer.
        double *dk = k, *dkq = k_q;
        const size_t k_bytes = sizeof(double) * (size_t)m * NCOLS, kq_bytes = sizeof(double) * (size_t)nq * NCOLS;
        if (out_memory == HOMS_HOST) {
            const size_t k_pad = (k_bytes + 255) & ~size_t(255);
            HOMS_CUDA(ctx->kspace_out.ensure(k_pad + kq_bytes));
            dk = ctx->kspace_out.as<double>();
            dkq = reinterpret_cast<double *>(ctx->kspace_out.as<uint8_t>() + k_pad);
        }
        HOMS_CUDA(ctx->kspace_work.ensure(kspace_work_bytes(nn, NCOLS, nparts)));
        KspaceArgs a;
        a.nnodes = nn;
        a.f64 = seq->dtype == HOMS_F64;
        a.t = dev_t;
        a.dt = dev_dt;
        a.ncols = NCOLS;
        a.cols = reinterpret_cast<const void *const *>(dmeta);
        a.nparts = nparts;
        a.starts = reinterpret_cast<const int64_t *>(dmeta + off_starts);
        a.signs = reinterpret_cast<const int8_t *>(dmeta + off_signs);
        a.gamma = seq->gamma;
        a.nq = nq;
        a.q = reinterpret_cast<const double *>(dmeta + off_q);
        a.k = dk;
        a.kq = dkq;
        a.work = ctx->kspace_work.p;
        for (cudaEvent_t &e : ctx->kspace_ev)
            if (!e) HOMS_CUDA(cudaEventCreate(&e));
        HOMS_CUDA(cudaEventRecord(ctx->kspace_ev[0], ctx->stream));
        HOMS_CUDA(kspace_launch(a, ctx->stream));
        HOMS_CUDA(cudaEventRecord(ctx->kspace_ev[1], ctx->stream));
        if (out_memory == HOMS_HOST) {
            d2h(ctx, k, dk, k_bytes);
            if (nq > 0) d2h(ctx, k_q, dkq, kq_bytes);
        }
        HOMS_CUDA(cudaStreamSynchronize(ctx->stream));
        ctx->kspace_timed = true;
        return HOMS_OK;
    } catch (const Failure &f) {
        cudaStreamSynchronize(ctx->stream);
        return fail(ctx, f);
    }
}

homs_status homs_selftest_wait_timeout(homs_context *ctx, int64_t budget_cycles) {
    if (!ctx) return HOMS_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DeviceGuard g(ctx->device);
    try {
        HOMS_REQUIRE(budget_cycles >= 1000 && budget_cycles <= 4000000000LL,
                     "budget_cycles must lie in [1e3, 4e9]");
        HOMS_CUDA(ctx->selftest_err.ensure(sizeof(unsigned int)));
        HOMS_CUDA(wait_selftest(ctx->selftest_err.as<unsigned int>(), (long long)budget_cycles, ctx->stream));
        unsigned int h = 0;
        HOMS_CUDA(cudaMemcpyAsync(&h, ctx->selftest_err.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        HOMS_CUDA(cudaStreamSynchronize(ctx->stream));
        if (h & 256u) throw Failure{HOMS_ETIMEDOUT, "self-test: the bounded device wait timed out (code 256)"};
        return HOMS_OK;
    } catch (const Failure &f) {
        cudaStreamSynchronize(ctx->stream);
        return fail(ctx, f);
    }
}

homs_status homs_kspace_timing(homs_context *ctx, double *ms) {
    if (!ctx || !ms) return HOMS_EINVAL;
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (!ctx->kspace_timed) return fail(ctx, Failure{HOMS_EINVAL, "no completed homs_kspace call on this context"});
    float t = 0.f;
    cudaError_t e = cudaEventElapsedTime(&t, ctx->kspace_ev[0], ctx->kspace_ev[1]);
    if (e != cudaSuccess) return fail(ctx, Failure{HOMS_ECUDA, cudaGetErrorString(e)});
    *ms = (double)t;
    return HOMS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Split-mode runs driven by the server's rounds (homs_server.cu)
// ---------------------------------------------------------------------------

namespace homs {

struct ServerRun {
    homs_context *ctx = nullptr;
    std::unique_lock<std::mutex> lock;  // the context is the run's until server_run_free
    Resident<double> *r = nullptr;
    SplitRunner<double> runner;
    homs_dtype out_dt = HOMS_F64;
    cudaEvent_t ready = nullptr, done = nullptr;
    bool waited = false, failed = false, done_recorded = false;
};

bool server_run_eligible(const homs_phantom *p, const homs_run_options *opts) {
    (void)p;
    return opts && opts->mode == HOMS_SPLIT;
}

homs_status server_run_prepare(homs_context *ctx, const homs_phantom *phantom, const homs_resident *resident,
                               const homs_sequence *seq, const homs_run_options *opts, const homs_state *state,
                               ServerRun **out) {
    if (!ctx || !out || !opts) return HOMS_EINVAL;
    *out = nullptr;
    auto run = std::make_unique<ServerRun>();
    run->ctx = ctx;
    run->lock = std::unique_lock<std::mutex>(ctx->mu);
    DeviceGuard g(ctx->device);
    try {
        validate_sequence(seq);
        HOMS_REQUIRE(opts->mode == HOMS_SPLIT, "internal: server rounds run split mode");
        HOMS_REQUIRE((opts->method & ~0x3Fu) == 0, "unknown method flag bits");
        Resident<double> *r = nullptr;
        if (resident) {
            HOMS_REQUIRE(resident->res && resident->device == ctx->device,
                         "the resident phantom lives on another device than the context");
            HOMS_REQUIRE(resident->mode == HOMS_SPLIT,
                         "the run mode must be the one the resident phantom was prepared for");
            HOMS_REQUIRE(resident->res->dtype == HOMS_F64, "internal: split-mode residents are FP64");
            const auto &src = static_cast<const Resident<double> &>(*resident->res);
            r = cache_slot<double>(ctx);
            attach_phantom<double>(r, src);
            fill_sequence<double>(ctx, r, seq);
            run->out_dt = resident->in_dtype;
        } else {
            validate_phantom(phantom);
            r = cached_resident<double>(ctx, phantom, seq);
            run->out_dt = phantom->dtype;
        }
        init_state<double>(ctx, *r, state, run->out_dt);
        ensure_split<double>(ctx, *r);
        ensure_split_tables<double>(ctx, *r, opts->method);
        HOMS_CUDA(split_reset_error(r->split, ctx->stream));
        r->events_used = 0;
        r->launches = 0;
        run->r = r;
        run->runner.init(ctx, *r, opts->method, false);
        HOMS_CUDA(cudaEventCreateWithFlags(&run->ready, cudaEventDisableTiming));
        HOMS_CUDA(cudaEventCreateWithFlags(&run->done, cudaEventDisableTiming));
        HOMS_CUDA(cudaEventRecord(run->ready, ctx->stream));
    } catch (const Failure &f) {
        cudaStreamSynchronize(ctx->stream);
        ctx->cache[0].reset();
        ctx->cache[1].reset();
        const homs_status s = fail(ctx, f);
        server_run_free(run.release());
        return s;
    } catch (const std::bad_alloc &) {
        cudaStreamSynchronize(ctx->stream);
        ctx->cache[0].reset();
        ctx->cache[1].reset();
        const homs_status s = fail(ctx, Failure{HOMS_ENOMEM, "host allocation failed"});
        server_run_free(run.release());
        return s;
    }
    *out = run.release();
    return HOMS_OK;
}

homs_status server_run_next(ServerRun *run, cudaStream_t stream, SplitJobDesc *job, bool *has_job) {
    *has_job = false;
    DeviceGuard g(run->ctx->device);
    try {
        if (!run->waited) {
            HOMS_CUDA(cudaStreamWaitEvent(stream, run->ready, 0));
            run->waited = true;
        }
        *has_job = run->runner.next(stream, job);
        return HOMS_OK;
    } catch (const Failure &f) {
        run->failed = true;
        return fail(run->ctx, f);
    }
}

homs_status server_run_after(ServerRun *run, cudaStream_t stream) {
    DeviceGuard g(run->ctx->device);
    try {
        run->runner.after(stream);
        return HOMS_OK;
    } catch (const Failure &f) {
        run->failed = true;
        return fail(run->ctx, f);
    }
}

cudaStream_t server_run_stream(const ServerRun *run) { return run->ctx->stream; }

void server_run_done(ServerRun *run, cudaStream_t stream) {
    DeviceGuard g(run->ctx->device);
    if (run->done && cudaEventRecord(run->done, stream) == cudaSuccess) run->done_recorded = true;
}

homs_status server_run_finish(ServerRun *run, void *sig, homs_memory sig_memory, homs_state *state) {
    homs_context *ctx = run->ctx;
    DeviceGuard g(ctx->device);
    try {
        HOMS_REQUIRE(run->done_recorded, "internal: the run's work was not issued");
        HOMS_CUDA(cudaStreamWaitEvent(ctx->stream, run->done, 0));
        HOMS_REQUIRE(sig_memory == HOMS_HOST || sig_memory == HOMS_DEVICE, "invalid signal memory kind");
        check_split<double>(ctx, *run->r);
        copy_out<double>(ctx, *run->r, sig, sig_memory, state, run->out_dt);
        return HOMS_OK;
    } catch (const Failure &f) {
        run->failed = true;
        return fail(ctx, f);
    }
}

void server_run_free(ServerRun *run) {
    if (!run) return;
    homs_context *ctx = run->ctx;
    {
        DeviceGuard g(ctx->device);
        // No work of the run may still use the context's buffers.
        if (run->done_recorded) cudaEventSynchronize(run->done);
        cudaStreamSynchronize(ctx->stream);
        if (run->failed) {
            ctx->cache[0].reset();
            ctx->cache[1].reset();
        }
        if (run->ready) cudaEventDestroy(run->ready);
        if (run->done) cudaEventDestroy(run->done);
    }
    delete run;  // releases the context
}

}  // namespace homs
