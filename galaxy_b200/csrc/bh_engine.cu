// SPDX-License-Identifier: Apache-2.0
//
// Host runtime of the B200 Barnes-Hut engine and the C ABI of galaxy_bh.h.
//
// A Batch lays one or more simulations out in a shared "position space":
// simulation s owns positions [off_s, off_s + n_s), off_s a multiple of 32,
// so a warp never straddles two simulations.  Radix tiles (4096 keys) never
// straddle simulations either.  Per-rebuild scratch (keys, sorted bodies,
// cells, control block) is one device arena carved at batch creation and
// sized for the worst case, so no step ever allocates.  The plain API
// (tree_create / rebuild / force) is a batch of one.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "bh_internal.cuh"

using namespace gbh;

// ------------------------------------------------------------------ errors --

static thread_local std::string g_last_error;

static int set_error(int status, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return status;
}

static int cuda_fail(cudaError_t e, const char* what) {
    cudaGetLastError();
    return set_error(e == cudaErrorMemoryAllocation ? BH_OOM : BH_CUDA_ERROR, "%s: %s (%s)", what,
                     cudaGetErrorName(e), cudaGetErrorString(e));
}

#define CK(expr, what)                                  \
    do {                                                \
        cudaError_t _e = (expr);                        \
        if (_e != cudaSuccess) return cuda_fail(_e, what); \
    } while (0)

int gbh::set_error_message(int status, const char* message) {
    return set_error(status, "%s", message);
}

extern "C" size_t galaxy_bh_last_error(char* buf, size_t len) {
    if (buf && len) {
        size_t n = std::min(len - 1, g_last_error.size());
        memcpy(buf, g_last_error.data(), n);
        buf[n] = 0;
    }
    return g_last_error.size();
}

extern "C" uint32_t galaxy_bh_abi_version(void) { return GALAXY_BH_ABI_VERSION; }

// ------------------------------------------------------------------ device --

struct bh_device {
    int ordinal = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[8] = {};
    cudaDeviceProp prop{};
    int refs = 0;         // live states, trees and batches on this device
    bool closed = false;  // galaxy_bh_device_close was called
    // Stream-ordered pool of the per-state buffers and the batch / tree
    // arenas.  It keeps released memory for reuse (trimmed only when an
    // allocation runs short): cudaFree synchronizes the whole device and
    // unmaps pages, which cost a serving loop seconds per burst of finished
    // requests and would stall it on its stager's work.
    cudaMemPool_t pool = nullptr;
};

static void device_free(bh_device* dev) {
    cudaSetDevice(dev->ordinal);
    cudaStreamSynchronize(dev->stream);
    if (dev->pool) cudaMemPoolDestroy(dev->pool);
    for (auto& ev : dev->ev) cudaEventDestroy(ev);
    cudaStreamDestroy(dev->stream);
    delete dev;
}

static void device_ref(bh_device* dev) { ++dev->refs; }

// Drops one handle's reference; frees a closed device with no handles left.
static void device_unref(bh_device* dev) {
    if (!dev) return;
    if (--dev->refs == 0 && dev->closed) device_free(dev);
}

static int enter(bh_device* dev) {
    if (!dev) return set_error(BH_INVALID_ARG, "null device handle");
    if (dev->closed) return set_error(BH_INVALID_ARG, "device handle is closed");
    CK(cudaSetDevice(dev->ordinal), "cudaSetDevice");
    return BH_OK;
}

extern "C" int galaxy_bh_device_open(int ordinal, bh_device** out) {
    if (!out) return set_error(BH_INVALID_ARG, "null output pointer");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return set_error(BH_NO_DEVICE, "No CUDA device is available (%s)",
                         e == cudaSuccess ? "0 devices" : cudaGetErrorName(e));
    }
    if (ordinal < 0 || ordinal >= count)
        return set_error(BH_NO_DEVICE, "CUDA device ordinal %d out of range (0..%d)", ordinal,
                         count - 1);
    bh_device* d = new bh_device();
    d->ordinal = ordinal;
    cudaMemPoolProps pool_props{};
    pool_props.allocType = cudaMemAllocationTypePinned;
    pool_props.location.type = cudaMemLocationTypeDevice;
    pool_props.location.id = ordinal;
    const uint64_t keep = ~0ull;
    if ((e = cudaSetDevice(ordinal)) != cudaSuccess ||
        (e = cudaGetDeviceProperties(&d->prop, ordinal)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaMemPoolCreate(&d->pool, &pool_props)) != cudaSuccess ||
        (e = cudaMemPoolSetAttribute(d->pool, cudaMemPoolAttrReleaseThreshold,
                                     (void*)&keep)) != cudaSuccess) {
        if (d->pool) cudaMemPoolDestroy(d->pool);
        if (d->stream) cudaStreamDestroy(d->stream);
        delete d;
        return cuda_fail(e, "device open");
    }
    for (auto& ev : d->ev) cudaEventCreate(&ev);
    *out = d;
    return BH_OK;
}

extern "C" int galaxy_bh_device_close(bh_device* dev) {
    if (!dev || dev->closed) return BH_OK;
    dev->closed = true;
    if (dev->refs == 0) device_free(dev);
    return BH_OK;
}

extern "C" int galaxy_bh_device_info(bh_device* dev, char* buf, size_t len) {
    int rc = enter(dev);
    if (rc) return rc;
    int rt = 0, drv = 0;
    cudaRuntimeGetVersion(&rt);
    cudaDriverGetVersion(&drv);
    char tmp[768];
    snprintf(tmp, sizeof tmp,
             "{\"index\": %d, \"name\": \"%s\", \"backend\": \"CUDA\", \"device_type\": "
             "\"DiscreteGpu\", \"compute_capability\": \"%d.%d\", \"sm_count\": %d, "
             "\"memory_bytes\": %zu, \"cuda_runtime\": %d, \"cuda_driver\": %d, "
             "\"software\": false}",
             dev->ordinal, dev->prop.name, dev->prop.major, dev->prop.minor,
             dev->prop.multiProcessorCount, (size_t)dev->prop.totalGlobalMem, rt, drv);
    if (buf && len) {
        strncpy(buf, tmp, len - 1);
        buf[len - 1] = 0;
    }
    return BH_OK;
}

extern "C" int galaxy_bh_device_stream(bh_device* dev, void** stream) {
    if (!dev || !stream) return set_error(BH_INVALID_ARG, "null argument");
    *stream = (void*)dev->stream;
    return BH_OK;
}

// ------------------------------------------------------------ config -------

static int validate_config(const bh_config* c) {
    if (!c) return set_error(BH_INVALID_ARG, "null config");
    // nbody/src/lib.rs:48-66
    if (!std::isfinite(c->theta) || c->theta < 0.0)
        return set_error(BH_INVALID_ARG, "theta must be finite and >= 0");
    if (!std::isfinite(c->softening) || c->softening < 0.0)
        return set_error(BH_INVALID_ARG, "softening_kpc must be finite and >= 0");
    if (!std::isfinite(c->g) || c->g <= 0.0)
        return set_error(BH_INVALID_ARG, "g must be positive and finite");
    if (c->bucket == 0 || c->bucket > 1024)
        return set_error(BH_INVALID_ARG, "bucket must be in 1..=1024");
    if (c->max_depth == 0 || c->max_depth > 128)
        return set_error(BH_INVALID_ARG, "max_depth must be in 1..=128");
    // nbody_parallel.rs:848-850: physics must stay finite as f32
    const float t = (float)c->theta, s = (float)c->softening, g = (float)c->g;
    if (!std::isfinite(t) || !std::isfinite(s) || !std::isfinite(g) || g <= 0.f)
        return set_error(BH_INVALID_ARG, "force settings are not representable as finite f32");
    return BH_OK;
}

static uint32_t eff_depth(const bh_config& c) { return std::min<uint32_t>(c.max_depth, kMortonDepth); }

// Upper bound on cells: leaves are disjoint (<= n); internal cells exist at
// depths 0..max_depth-1, and those at depth d are at most 4^d (one per
// quadtree square) and hold disjoint ranges of > bucket bodies (at most
// n/(bucket+1)).  At bucket 1 this is ~3.8n cells for n = 2^22 (a
// depth-blind n/(bucket+1) per depth would be 9n); trees of real
// distributions hold ~1.7n.
static uint64_t cell_bound(uint32_t n, const bh_config& c) {
    const uint64_t per_depth = n / ((uint64_t)c.bucket + 1);
    uint64_t internal = 0, squares = 1;
    for (uint32_t d = 0; d < eff_depth(c); ++d, squares *= 4)
        internal += std::min(squares, per_depth);
    return (uint64_t)n + internal + 1;
}

static void fill_physics(SimDesc& sd, const bh_config& c) {
    sd.bucket = c.bucket;
    sd.max_depth = eff_depth(c);
    sd.flags = c.flags;
    sd.theta = c.theta;
    sd.theta_f = (float)c.theta;
    sd.inv_theta_f = c.theta > 0.0 ? (float)(1.0 / c.theta) : INFINITY;
    sd.eps_f = (float)c.softening;
    sd.g_f = (float)c.g;
}

// ------------------------------------------------------------------- state --

struct bh_state {
    bh_device* dev = nullptr;
    uint32_t n = 0;
    GpuEvolveState* d_state = nullptr;
    float4* d_accel = nullptr;
    float* d_potential = nullptr;
    // a one-simulation layout for stand-alone kick / drift launches
    SimDesc* d_sim = nullptr;
    uint32_t* d_chunk_sim = nullptr;
    uint32_t* d_minmax = nullptr;
    double* d_cons = nullptr;  // conservation partials + result
    uint32_t* d_check = nullptr;         // first invalid record index of the last check
    GpuEvolveState* d_stage = nullptr;   // upload staging (first galaxy_bh_write_state)
    uint32_t nchunks = 0;
    SimDesc h_sim{};
};

static int enqueue_check(bh_state* st, const void* records, int kind, uint32_t n);
static int fetch_check(bh_state* st, uint32_t* first_bad);

extern "C" int galaxy_bh_state_create(bh_device* dev, const GpuEvolveState* host, uint32_t n,
                                      bh_state** out, bh_stage_timing* timing) {
    int rc = enter(dev);
    if (rc) return rc;
    if (!out || !host) return set_error(BH_INVALID_ARG, "null argument");
    *out = nullptr;
    // nbody_gpu.rs:787-789
    if (n < 2 || n > (1u << 30))
        return set_error(BH_INVALID_ARG, "GPU evolving state requires 2..=%u resident bodies",
                         1u << 30);
    bh_state* st = new bh_state();
    st->dev = dev;
    device_ref(dev);
    st->n = n;
    st->nchunks = (n + kChunk - 1) / kChunk;
    cudaEventRecord(dev->ev[0], dev->stream);
    cudaError_t e;
    std::vector<uint32_t> chunk(st->nchunks, 0u);
    auto pool_alloc = [&](auto** ptr, size_t bytes) {
        cudaError_t r = cudaMallocFromPoolAsync((void**)ptr, bytes, dev->pool, dev->stream);
        if (r == cudaErrorMemoryAllocation) {
            // give back what the pool keeps unused, then retry
            cudaGetLastError();
            cudaStreamSynchronize(dev->stream);
            cudaMemPoolTrimTo(dev->pool, 0);
            r = cudaMallocFromPoolAsync((void**)ptr, bytes, dev->pool, dev->stream);
        }
        return r;
    };
    if ((e = pool_alloc(&st->d_state, sizeof(GpuEvolveState) * (size_t)n)) ||
        (e = pool_alloc(&st->d_accel, sizeof(float4) * (size_t)n)) ||
        (e = pool_alloc(&st->d_sim, sizeof(SimDesc))) ||
        (e = pool_alloc(&st->d_chunk_sim, sizeof(uint32_t) * st->nchunks)) ||
        (e = pool_alloc(&st->d_minmax, 16)) || (e = pool_alloc(&st->d_check, 16))) {
        galaxy_bh_state_destroy(st);
        return cuda_fail(e, "evolving state allocation");
    }
    st->h_sim.state = st->d_state;
    st->h_sim.accel = st->d_accel;
    st->h_sim.off = 0;
    st->h_sim.n = n;
    if ((e = cudaMemcpyAsync(st->d_state, host, sizeof(GpuEvolveState) * (size_t)n,
                             cudaMemcpyHostToDevice, dev->stream)) ||
        (e = cudaMemsetAsync(st->d_accel, 0, sizeof(float4) * (size_t)n, dev->stream)) ||
        (e = cudaMemcpyAsync(st->d_chunk_sim, chunk.data(), 4 * chunk.size(),
                             cudaMemcpyHostToDevice, dev->stream)) ||
        (e = cudaMemcpyAsync(st->d_sim, &st->h_sim, sizeof(SimDesc), cudaMemcpyHostToDevice,
                             dev->stream))) {
        galaxy_bh_state_destroy(st);
        return cuda_fail(e, "evolving state upload");
    }
    cudaEventRecord(dev->ev[1], dev->stream);
    // nbody_gpu.rs:802-810: every record finite with a positive mass, tested
    // on the uploaded copy; the smallest failing index is reported and no
    // state is created
    uint32_t bad = kNone;
    if ((rc = enqueue_check(st, st->d_state, 0, n)) || (rc = fetch_check(st, &bad))) {
        galaxy_bh_state_destroy(st);
        return rc;
    }
    if (bad != kNone) {
        galaxy_bh_state_destroy(st);
        return set_error(BH_NONFINITE, "body %u contains invalid evolving state", bad);
    }
    if (timing) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, dev->ev[0], dev->ev[1]);
        *timing = bh_stage_timing{ms * 1e-3, 0.0, 0.0};
    }
    *out = st;
    return BH_OK;
}

extern "C" int galaxy_bh_state_destroy(bh_state* st) {
    if (!st) return BH_OK;
    if (st->dev) {
        cudaSetDevice(st->dev->ordinal);
        cudaStreamSynchronize(st->dev->stream);
        // back to the device's pool, in stream order (no device-wide sync)
        for (void* p : {(void*)st->d_state, (void*)st->d_accel, (void*)st->d_sim,
                        (void*)st->d_chunk_sim, (void*)st->d_minmax, (void*)st->d_check})
            if (p) cudaFreeAsync(p, st->dev->stream);
    }
    if (st->d_potential) cudaFree(st->d_potential);
    if (st->d_cons) cudaFree(st->d_cons);
    if (st->d_stage) cudaFree(st->d_stage);
    bh_device* dev = st->dev;
    delete st;
    device_unref(dev);
    return BH_OK;
}

// Hands a state made on one device handle to another handle of the same
// GPU (the serving loop's stager uploads and solves on its own handle and
// stream): the state's pending work finishes first; its buffers stay where
// they are and are later released on the new handle's stream.
int gbh::state_move(bh_state* st, bh_device* to) {
    if (!st || !to) return set_error(BH_INVALID_ARG, "null argument");
    if (st->dev == to) return BH_OK;
    if (st->dev->ordinal != to->ordinal)
        return set_error(BH_INVALID_ARG, "state and device handle are on different GPUs");
    CK(cudaSetDevice(st->dev->ordinal), "cudaSetDevice");
    CK(cudaStreamSynchronize(st->dev->stream), "state move");
    bh_device* old = st->dev;
    device_ref(to);
    st->dev = to;
    device_unref(old);
    return BH_OK;
}

extern "C" int galaxy_bh_state_count(bh_state* st, uint32_t* n) {
    if (!st || !n) return set_error(BH_INVALID_ARG, "null argument");
    *n = st->n;
    return BH_OK;
}

extern "C" int galaxy_bh_state_bytes(bh_state* st, uint64_t* bytes) {
    if (!st || !bytes) return set_error(BH_INVALID_ARG, "null argument");
    *bytes = (uint64_t)st->n * (sizeof(GpuEvolveState) + sizeof(float4));
    return BH_OK;
}

static int checked_dt(double dt, float* out) {
    if (!std::isfinite(dt) || dt <= 0.0)
        return set_error(BH_INVALID_ARG, "dt_myr must be positive and finite");
    float f = (float)dt;
    if (!std::isfinite(f) || f <= 0.f)
        return set_error(BH_INVALID_ARG, "dt_myr cannot be represented as finite f32");
    *out = f;
    return BH_OK;
}

static int stage_time(bh_device* dev, bh_stage_timing* t) {
    CK(cudaEventRecord(dev->ev[1], dev->stream), "event record");
    CK(cudaStreamSynchronize(dev->stream), "stream synchronize");
    if (t) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, dev->ev[0], dev->ev[1]);
        *t = bh_stage_timing{0.0, ms * 1e-3, 0.0};
    }
    return BH_OK;
}

static int integrate_state(bh_device* dev, bh_state* st, double dt, int mode,
                           bh_stage_timing* timing) {
    int rc = enter(dev);
    if (rc) return rc;
    if (!st || st->dev != dev) return set_error(BH_INVALID_ARG, "state does not belong to device");
    float f = 0.f;
    if ((rc = checked_dt(dt, &f))) return rc;
    st->h_sim.dt = f;
    CK(cudaMemcpyAsync(st->d_sim, &st->h_sim, sizeof(SimDesc), cudaMemcpyHostToDevice,
                       dev->stream),
       "settings upload");
    CK(cudaMemsetAsync(st->d_minmax, 0, 16, dev->stream), "memset");
    CK(cudaEventRecord(dev->ev[0], dev->stream), "event record");
    BatchBuffers b{};
    b.sims = st->d_sim;
    b.chunk_sim = st->d_chunk_sim;
    b.nchunks = st->nchunks;
    b.minmax = st->d_minmax;
    CK(launch_integrate(b, mode, dev->stream), "integrate launch");
    return stage_time(dev, timing);
}

extern "C" int galaxy_bh_kick_drift(bh_device* dev, bh_state* st, double dt,
                                    bh_stage_timing* timing) {
    return integrate_state(dev, st, dt, 1, timing);
}

extern "C" int galaxy_bh_final_kick(bh_device* dev, bh_state* st, double dt,
                                    bh_stage_timing* timing) {
    return integrate_state(dev, st, dt, 2, timing);
}

extern "C" int galaxy_bh_final_kick_drift(bh_device* dev, bh_state* st, double dt,
                                          bh_stage_timing* timing) {
    return integrate_state(dev, st, dt, 3, timing);
}

// Enqueues the record check of n records at `records` (kind 0: evolving
// states, 1: accelerations) and the copy of its result word to *first_bad.
static int enqueue_check(bh_state* st, const void* records, int kind, uint32_t n) {
    bh_device* dev = st->dev;
    CK(cudaMemsetAsync(st->d_check, 0xff, 4, dev->stream), "memset");
    CK(launch_check_records(records, kind, n, st->d_check, dev->stream), "record check");
    return BH_OK;
}

static int fetch_check(bh_state* st, uint32_t* first_bad) {
    CK(cudaMemcpyAsync(first_bad, st->d_check, 4, cudaMemcpyDeviceToHost, st->dev->stream),
       "record check readback");
    CK(cudaStreamSynchronize(st->dev->stream), "record check readback");
    return BH_OK;
}

extern "C" int galaxy_bh_read_state(bh_device* dev, bh_state* st, GpuEvolveState* out,
                                    uint32_t n, bh_stage_timing* timing) {
    int rc = enter(dev);
    if (rc) return rc;
    if (!st || !out) return set_error(BH_INVALID_ARG, "null argument");
    if (n != st->n) return set_error(BH_INVALID_ARG, "readback count %u != resident bodies %u", n, st->n);
    // nbody_gpu.rs:1043-1053 checks the host copy; the same test runs on the
    // device records (bitwise the same values) while they are copied out
    if ((rc = enqueue_check(st, st->d_state, 0, n))) return rc;
    CK(cudaEventRecord(dev->ev[0], dev->stream), "event record");
    CK(cudaMemcpyAsync(out, st->d_state, sizeof(GpuEvolveState) * (size_t)n,
                       cudaMemcpyDeviceToHost, dev->stream),
       "state readback");
    CK(cudaEventRecord(dev->ev[1], dev->stream), "event record");
    uint32_t bad = kNone;
    if ((rc = fetch_check(st, &bad))) return rc;
    if (timing) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, dev->ev[0], dev->ev[1]);
        *timing = bh_stage_timing{0.0, 0.0, ms * 1e-3};
    }
    if (bad != kNone)
        return set_error(BH_NONFINITE, "GPU produced invalid evolving body state at %u", bad);
    return BH_OK;
}

extern "C" int galaxy_bh_read_accel(bh_device* dev, bh_state* st, GpuAccel* out, uint32_t n,
                                    bh_stage_timing* timing) {
    int rc = enter(dev);
    if (rc) return rc;
    if (!st || !out) return set_error(BH_INVALID_ARG, "null argument");
    if (n != st->n) return set_error(BH_INVALID_ARG, "readback count %u != resident bodies %u", n, st->n);
    // nbody_gpu.rs:1097-1101, evaluated on the device records
    if ((rc = enqueue_check(st, st->d_accel, 1, n))) return rc;
    CK(cudaEventRecord(dev->ev[0], dev->stream), "event record");
    CK(cudaMemcpyAsync(out, st->d_accel, sizeof(float4) * (size_t)n, cudaMemcpyDeviceToHost,
                       dev->stream),
       "acceleration readback");
    CK(cudaEventRecord(dev->ev[1], dev->stream), "event record");
    uint32_t bad = kNone;
    if ((rc = fetch_check(st, &bad))) return rc;
    if (timing) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, dev->ev[0], dev->ev[1]);
        *timing = bh_stage_timing{0.0, 0.0, ms * 1e-3};
    }
    if (bad != kNone)
        return set_error(BH_NONFINITE, "GPU produced invalid evolving acceleration at %u", bad);
    return BH_OK;
}

extern "C" int galaxy_bh_write_state(bh_device* dev, bh_state* st, const GpuEvolveState* host,
                                     uint32_t n) {
    int rc = enter(dev);
    if (rc) return rc;
    if (!st || !host) return set_error(BH_INVALID_ARG, "null argument");
    if (n != st->n) return set_error(BH_INVALID_ARG, "write count %u != resident bodies %u", n, st->n);
    // Upload into a staging buffer, check the records there and only then
    // replace the resident state: an invalid upload leaves it untouched.
    if (!st->d_stage)
        CK(cudaMalloc(&st->d_stage, sizeof(GpuEvolveState) * (size_t)n), "staging allocation");
    CK(cudaMemcpyAsync(st->d_stage, host, sizeof(GpuEvolveState) * (size_t)n,
                       cudaMemcpyHostToDevice, dev->stream),
       "state upload");
    if ((rc = enqueue_check(st, st->d_stage, 0, n))) return rc;
    uint32_t bad = kNone;
    if ((rc = fetch_check(st, &bad))) return rc;
    if (bad != kNone) return set_error(BH_NONFINITE, "body %u contains invalid evolving state", bad);
    CK(cudaMemcpyAsync(st->d_state, st->d_stage, sizeof(GpuEvolveState) * (size_t)n,
                       cudaMemcpyDeviceToDevice, dev->stream),
       "state upload");
    return BH_OK;
}

static int ensure_potential(bh_state* st) {
    if (!st->d_potential) {
        CK(cudaMalloc(&st->d_potential, sizeof(float) * (size_t)st->n), "potential allocation");
        CK(cudaMemsetAsync(st->d_potential, 0, sizeof(float) * (size_t)st->n, st->dev->stream),
           "memset");
    }
    return BH_OK;
}

extern "C" int galaxy_bh_direct_probes(bh_device* dev, bh_state* st, const bh_config* cfg,
                                       const uint32_t* probes, uint32_t nprobes, double* out) {
    int rc = enter(dev);
    if (rc) return rc;
    if (!st || !cfg || !probes || !out) return set_error(BH_INVALID_ARG, "null argument");
    if ((rc = validate_config(cfg))) return rc;
    if (nprobes == 0) return BH_OK;
    for (uint32_t k = 0; k < nprobes; ++k)
        if (probes[k] >= st->n) return set_error(BH_INVALID_ARG, "body index is out of range");
    uint32_t* d_p = nullptr;
    double* d_o = nullptr;
    cudaError_t e = cudaMalloc(&d_p, 4ull * nprobes);
    if (!e) e = cudaMalloc(&d_o, 16ull * nprobes);
    if (!e) e = cudaMemcpyAsync(d_p, probes, 4ull * nprobes, cudaMemcpyHostToDevice, dev->stream);
    if (!e)
        e = launch_direct_probes(st->d_state, st->n, d_p, nprobes, cfg->softening, cfg->g, d_o,
                                 dev->stream);
    if (!e) e = cudaMemcpyAsync(out, d_o, 16ull * nprobes, cudaMemcpyDeviceToHost, dev->stream);
    if (!e) e = cudaStreamSynchronize(dev->stream);
    cudaFree(d_p);
    cudaFree(d_o);
    if (e) return cuda_fail(e, "direct probes");
    return BH_OK;
}

extern "C" int galaxy_bh_conservation(bh_device* dev, bh_state* st, double out[10]) {
    int rc = enter(dev);
    if (rc) return rc;
    if (!st || !out) return set_error(BH_INVALID_ARG, "null argument");
    const uint32_t nb = conservation_blocks(st->n);
    if (!st->d_cons) CK(cudaMalloc(&st->d_cons, sizeof(double) * (9 * (size_t)nb + 16)), "alloc");
    CK(launch_conservation(st->d_state, st->d_potential, st->n, st->d_cons, nb,
                           st->d_cons + 9 * (size_t)nb, dev->stream),
       "conservation launch");
    double r[9];
    CK(cudaMemcpyAsync(r, st->d_cons + 9 * (size_t)nb, sizeof r, cudaMemcpyDeviceToHost,
                       dev->stream),
       "readback");
    CK(cudaStreamSynchronize(dev->stream), "conservation");
    out[0] = r[0];
    out[1] = r[1] / r[0];
    out[2] = r[2] / r[0];
    out[3] = r[3];
    out[4] = r[4];
    out[5] = r[5];
    out[6] = r[6];
    out[7] = r[7];
    out[8] = r[8];
    out[9] = r[6] + r[7];
    return BH_OK;
}

// ------------------------------------------------------------------- batch --

struct Batch {
    bh_device* dev = nullptr;
    std::vector<bh_state*> states;
    std::vector<bh_config> cfgs;
    std::vector<SimDesc> h_sims;
    std::vector<uint32_t> h_chunk_sim;
    std::vector<Tile> h_tiles;
    uint32_t npos = 0, nchunks = 0, ntiles = 0, nscan_tiles = 0;
    uint64_t cell_capacity = 0;
    void* arena = nullptr;
    size_t arena_bytes = 0;
    void* control = nullptr;
    size_t control_bytes = 0;
    BatchBuffers bb{};
    SimDesc* d_sims = nullptr;
    // graphs: [0] first step, [1] middle step, [2] final kick
    cudaGraphExec_t graphs[3] = {nullptr, nullptr, nullptr};
    uint32_t graph_flags = 0xffffffffu;
    bool stats_valid = false;
    // theta and G the cell records (G*m, MAC bounds) were last computed with
    // (single-simulation trees; batches keep their creation configs)
    double built_theta = NAN, built_g = NAN;

    size_t arena_capacity = 0;  // bytes held

    ~Batch() {
        for (auto& g : graphs)
            if (g) cudaGraphExecDestroy(g);
        // back to the device handle's pool in stream order: no device-wide
        // synchronisation (a cudaFree would wait for every stream of the GPU,
        // e.g. a serving loop's rounds while its stager releases a tree)
        if (arena) cudaFreeAsync(arena, dev->stream);
    }
};

struct Layout {
    uint32_t npos = 0, nchunks = 0, ntiles = 0, nscan_tiles = 0;
    uint64_t cells = 0;
    std::vector<uint32_t> off;
};

static Layout plan_layout(const uint32_t* counts, const bh_config* cfgs, uint32_t count) {
    Layout L;
    uint64_t pos = 0;
    L.off.resize(count);
    for (uint32_t s = 0; s < count; ++s) {
        L.off[s] = (uint32_t)pos;
        pos += (counts[s] + kChunk - 1) / kChunk * kChunk;
        L.ntiles += (counts[s] + kTile - 1) / kTile;
        L.cells += cell_bound(counts[s], cfgs[s]);
    }
    L.npos = (uint32_t)pos;
    L.nchunks = L.npos / kChunk;
    L.nscan_tiles = (L.npos + 1 + kScanTile - 1) / kScanTile;
    return L;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Byte sizes of the arena regions, in carve order.
struct ArenaPlan {
    size_t control, sims, simout, chunk, tiles, keys, vals, sbody, base, cell_u, groups,
        cell_d, cell_child, cell_parent, cell_counter, err, stats;
    size_t total() const {
        return control + sims + simout + chunk + tiles + 2 * keys + 2 * vals + sbody + base +
               cell_u + groups + cell_d + cell_child + cell_parent + cell_counter +
               err + stats;
    }
};

static ArenaPlan plan_arena(const Layout& L, uint32_t nsims) {
    ArenaPlan a;
    a.control = align256(4ull * nsims * 4 + 4ull * nsims * kRadixPasses * kRadixDigits + 4ull * 16 +
                         4ull * kRadixPasses * L.ntiles * kRadixDigits) +
                align256(8ull * L.nscan_tiles);
    a.sims = align256(sizeof(SimDesc) * nsims);
    a.simout = align256(sizeof(SimOut) * nsims);
    a.chunk = align256(4ull * L.nchunks);
    a.tiles = align256(sizeof(Tile) * L.ntiles);
    a.keys = align256(4ull * L.npos);
    a.vals = align256(4ull * L.npos);
    a.sbody = align256(16ull * L.npos);
    a.base = align256(4ull * (L.npos + 1));
    a.cell_u = align256(sizeof(uint4) * L.cells);
    a.groups = align256(4ull * sizeof(CellRec) * (L.cells + nsims));
    a.cell_d = align256(32ull * L.cells);
    a.cell_child = align256(16ull * L.cells);
    a.cell_parent = align256(4ull * L.cells);
    a.cell_counter = align256(4ull * L.cells);
    a.err = 256;
    a.stats = 256;
    return a;
}

extern "C" int galaxy_bh_batch_footprint(const uint32_t* counts, const bh_config* cfgs,
                                         uint32_t count, uint64_t* bytes) {
    if (!counts || !cfgs || !bytes || !count) return set_error(BH_INVALID_ARG, "null argument");
    Layout L = plan_layout(counts, cfgs, count);
    uint64_t persistent = 0;
    for (uint32_t s = 0; s < count; ++s)
        persistent += (uint64_t)counts[s] * (sizeof(GpuEvolveState) + sizeof(float4) + 4) +
                      ((counts[s] + 31) / 32) * 4 + 1024;
    *bytes = plan_arena(L, count).total() + persistent;
    return BH_OK;
}

// Builds a batch of `count` states.  A `donor` batch of the same device
// handle (or null) gives up its arena when that is large enough, and is
// freed either way: re-forming a batch, or pointing a tree at another state,
// then allocates nothing (the donor's work precedes the new batch's on the
// handle's stream).
static int batch_build(bh_device* dev, bh_state* const* states, const bh_config* cfgs,
                       uint32_t count, Batch** out, Batch* donor_batch = nullptr) {
    std::unique_ptr<Batch> donor(donor_batch);
    *out = nullptr;
    if (!count) return set_error(BH_INVALID_ARG, "batch needs at least one state");
    std::vector<uint32_t> counts(count);
    for (uint32_t s = 0; s < count; ++s) {
        if (!states[s] || states[s]->dev != dev)
            return set_error(BH_INVALID_ARG, "state %u does not belong to this device", s);
        int rc = validate_config(&cfgs[s]);
        if (rc) return rc;
        counts[s] = states[s]->n;
    }
    Layout L = plan_layout(counts.data(), cfgs, count);
    if (L.cells >= (1ull << 31) || (uint64_t)L.npos + 1 >= (1ull << 31))
        return set_error(BH_CAPACITY_OVERFLOW, "batch exceeds 2^31 positions or cells");
    ArenaPlan A = plan_arena(L, count);
    Batch* b = new Batch();
    b->dev = dev;
    b->states.assign(states, states + count);
    b->cfgs.assign(cfgs, cfgs + count);
    b->npos = L.npos;
    b->nchunks = L.nchunks;
    b->ntiles = L.ntiles;
    b->nscan_tiles = L.nscan_tiles;
    b->cell_capacity = L.cells;
    b->arena_bytes = A.total();
    cudaError_t e = cudaSuccess;
    if (donor && donor->arena && donor->arena_capacity >= b->arena_bytes) {
        b->arena = donor->arena;
        b->arena_capacity = donor->arena_capacity;
        donor->arena = nullptr;
    }
    donor.reset();  // a donor arena too small goes back to the pool first
    // the arena comes from the device handle's stream-ordered pool, which
    // keeps released arenas and state buffers for reuse
    if (!b->arena) {
        e = cudaMallocFromPoolAsync(&b->arena, b->arena_bytes, dev->pool, dev->stream);
        if (e == cudaErrorMemoryAllocation) {
            // give back what the pool keeps, then retry
            cudaGetLastError();
            cudaStreamSynchronize(dev->stream);
            cudaMemPoolTrimTo(dev->pool, 0);
            e = cudaMallocFromPoolAsync(&b->arena, b->arena_bytes, dev->pool, dev->stream);
        }
        b->arena_capacity = b->arena_bytes;
    }
    if (e != cudaSuccess) {
        b->arena = nullptr;
        delete b;
        return cuda_fail(e, "batch arena allocation");
    }
    char* p = (char*)b->arena;
    auto take = [&](size_t bytes) {
        char* q = p;
        p += bytes;
        return (void*)q;
    };
    BatchBuffers& bb = b->bb;
    b->control = p;
    b->control_bytes = A.control;
    char* cp = (char*)take(A.control);
    bb.minmax = (uint32_t*)cp;
    cp += 4ull * count * 4;
    bb.hist = (uint32_t*)cp;
    cp += 4ull * count * kRadixPasses * kRadixDigits;
    bb.counters = (uint32_t*)cp;
    cp += 4ull * 16;
    bb.sort_flags = (uint32_t*)cp;
    cp += 4ull * kRadixPasses * L.ntiles * kRadixDigits;
    bb.scan_flags = (unsigned long long*)((char*)b->control +
                                          align256((size_t)(cp - (char*)b->control)));
    b->d_sims = (SimDesc*)take(A.sims);
    bb.sims = b->d_sims;
    bb.simout = (SimOut*)take(A.simout);
    bb.chunk_sim = (const uint32_t*)take(A.chunk);
    bb.tiles = (const Tile*)take(A.tiles);
    bb.keys_a = (uint32_t*)take(A.keys);
    bb.keys_b = (uint32_t*)take(A.keys);
    bb.vals_a = (uint32_t*)take(A.vals);
    bb.vals_b = (uint32_t*)take(A.vals);
    bb.sbody = (float4*)take(A.sbody);
    bb.base = (uint32_t*)take(A.base);
    bb.cell_u = (uint4*)take(A.cell_u);
    bb.groups = (CellRec*)take(A.groups);
    bb.cell_d = (double4*)take(A.cell_d);
    bb.cell_child = (uint4*)take(A.cell_child);
    bb.cell_parent = (uint32_t*)take(A.cell_parent);
    bb.cell_counter = (uint32_t*)take(A.cell_counter);
    bb.err = (uint32_t*)take(A.err);
    bb.force_stats = (unsigned long long*)take(A.stats);
    bb.nsims = count;
    bb.npos = L.npos;
    bb.nchunks = L.nchunks;
    bb.ntiles = L.ntiles;
    bb.nscan_tiles = L.nscan_tiles;
    bb.cell_capacity = (uint32_t)L.cells;
    bb.radix_bits = 8;
    bb.trav_warps = 4;

    b->h_sims.resize(count);
    b->h_chunk_sim.assign(L.nchunks, kNone);
    uint32_t tile = 0;
    for (uint32_t s = 0; s < count; ++s) {
        SimDesc& sd = b->h_sims[s];
        memset(&sd, 0, sizeof sd);
        sd.state = states[s]->d_state;
        sd.accel = states[s]->d_accel;
        sd.potential = states[s]->d_potential;
        sd.off = L.off[s];
        sd.n = counts[s];
        sd.first_tile = tile;
        sd.dt = 0.f;
        fill_physics(sd, cfgs[s]);
        for (uint32_t c = 0; c < (counts[s] + kChunk - 1) / kChunk; ++c)
            b->h_chunk_sim[L.off[s] / kChunk + c] = s;
        for (uint32_t t0 = 0; t0 < counts[s]; t0 += kTile) {
            Tile tl{};
            tl.sim = s;
            tl.start = L.off[s] + t0;
            tl.count = std::min<uint32_t>(kTile, counts[s] - t0);
            b->h_tiles.push_back(tl);
            ++tile;
        }
    }
    cudaStream_t st = dev->stream;
    if ((e = cudaMemcpyAsync(b->d_sims, b->h_sims.data(), sizeof(SimDesc) * count,
                             cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync((void*)bb.chunk_sim, b->h_chunk_sim.data(), 4ull * L.nchunks,
                             cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync((void*)bb.tiles, b->h_tiles.data(), sizeof(Tile) * L.ntiles,
                             cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemsetAsync(bb.err, 0, 256, st)) ||
        (e = cudaMemsetAsync(bb.force_stats, 0, 256, st)) ||
        (e = cudaMemsetAsync(bb.simout, 0, sizeof(SimOut) * count, st)) ||
        (e = cudaStreamSynchronize(st))) {
        delete b;
        return cuda_fail(e, "batch upload");
    }
    *out = b;
    return BH_OK;
}

static int upload_sims(Batch* b) {
    CK(cudaMemcpyAsync(b->d_sims, b->h_sims.data(), sizeof(SimDesc) * b->h_sims.size(),
                       cudaMemcpyHostToDevice, b->dev->stream),
       "settings upload");
    return BH_OK;
}

// Reads (and clears) the device error word; maps bits to a status.
static int check_device_errors(Batch* b) {
    uint32_t err = 0;
    CK(cudaMemcpyAsync(&err, b->bb.err, 4, cudaMemcpyDeviceToHost, b->dev->stream), "readback");
    CK(cudaStreamSynchronize(b->dev->stream), "stream synchronize");
    if (!err) return BH_OK;
    cudaMemsetAsync(b->bb.err, 0, 4, b->dev->stream);
    cudaStreamSynchronize(b->dev->stream);
    if (err & kErrLookbackTimeout)
        return set_error(BH_TIMEOUT, "device look-back wait timed out (error bits 0x%x)", err);
    if (err & kErrCapacity)
        return set_error(BH_CAPACITY_OVERFLOW, "GPU tree reported cell-capacity overflow");
    return set_error(BH_CUDA_ERROR, "device traversal reported error bits 0x%x", err);
}

enum Stage { kStBounds, kStMorton, kStRadix, kStTopology, kStAggregate };

// memset(control) + bounds/integrate + Morton + radix + topology + aggregates.
// With ev != null, records events between stages (ev[0..5]).
static int enqueue_rebuild(Batch* b, int integrate_mode, cudaEvent_t* ev) {
    cudaStream_t s = b->dev->stream;
    if (ev) CK(cudaEventRecord(ev[0], s), "event");
    CK(cudaMemsetAsync(b->control, 0, b->control_bytes, s), "control memset");
    CK(launch_integrate(b->bb, integrate_mode, s), "integrate launch");
    if (ev) CK(cudaEventRecord(ev[1], s), "event");
    CK(launch_morton(b->bb, s), "morton launch");
    if (ev) CK(cudaEventRecord(ev[2], s), "event");
    CK(launch_radix(b->bb, s), "radix launch");
    if (ev) CK(cudaEventRecord(ev[3], s), "event");
    CK(launch_count_scan(b->bb, s), "count/scan launch");
    CK(launch_cells(b->bb, s), "cells launch");
    if (ev) CK(cudaEventRecord(ev[4], s), "event");
    CK(launch_aggregate(b->bb, s), "aggregate launch");
    if (ev) CK(cudaEventRecord(ev[5], s), "event");
    return BH_OK;
}

static bool any_flag(Batch* b, uint32_t flag) {
    for (auto& c : b->cfgs)
        if (c.flags & flag) return true;
    return false;
}

static bool any_without_flag(Batch* b, uint32_t flag) {
    for (auto& c : b->cfgs)
        if (!(c.flags & flag)) return true;
    return false;
}

static int enqueue_force(Batch* b, bool stats) {
    cudaStream_t s = b->dev->stream;
    if (stats) CK(cudaMemsetAsync(b->bb.force_stats, 0, 40, s), "memset");
    CK(launch_traverse(b->bb, any_flag(b, BH_FLAG_COMPENSATED),
                       any_without_flag(b, BH_FLAG_COMPENSATED), any_flag(b, BH_FLAG_POTENTIAL),
                       stats, s),
       "traverse launch");
    return BH_OK;
}

// Installs per-simulation configs.  A rebuild under a config needing more
// cells than the arena holds must be preceded by tree_fit.
static int apply_configs(Batch* b, const bh_config* cfgs, bool for_rebuild) {
    for (size_t s = 0; s < b->states.size(); ++s) {
        int rc = validate_config(&cfgs[s]);
        if (rc) return rc;
        if (for_rebuild && cell_bound(b->states[s]->n, cfgs[s]) > b->cell_capacity)
            return set_error(BH_CAPACITY_OVERFLOW,
                             "config needs more tree cells than this tree holds");
        if (cfgs[s].flags & BH_FLAG_POTENTIAL) {
            if ((rc = ensure_potential(b->states[s]))) return rc;
        }
        b->cfgs[s] = cfgs[s];
        b->h_sims[s].potential = b->states[s]->d_potential;
        fill_physics(b->h_sims[s], cfgs[s]);
    }
    return upload_sims(b);
}

static int run_graphs(Batch* b, uint32_t nsteps) {
    cudaStream_t s = b->dev->stream;
    const uint32_t flags = (any_flag(b, BH_FLAG_COMPENSATED) ? 1u : 0u) |
                           (any_flag(b, BH_FLAG_POTENTIAL) ? 2u : 0u) |
                           (any_without_flag(b, BH_FLAG_COMPENSATED) ? 4u : 0u);
    if (b->graph_flags != flags) {
        for (auto& g : b->graphs)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
        for (int k = 0; k < 3; ++k) {
            cudaGraph_t graph;
            CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
            int rc = BH_OK;
            if (k < 2) {
                rc = enqueue_rebuild(b, k == 0 ? 1 : 3, nullptr);
                if (!rc) rc = enqueue_force(b, false);
            } else {
                cudaError_t e = launch_integrate(b->bb, 2, s);
                if (e) rc = cuda_fail(e, "integrate launch");
            }
            cudaError_t e = cudaStreamEndCapture(s, &graph);
            if (rc) return rc;
            CK(e, "end capture");
            e = cudaGraphInstantiate(&b->graphs[k], graph, 0);
            cudaGraphDestroy(graph);
            CK(e, "graph instantiate");
        }
        b->graph_flags = flags;
    }
    for (uint32_t k = 0; k < nsteps; ++k)
        CK(cudaGraphLaunch(b->graphs[k == 0 ? 0 : 1], s), "graph launch");
    CK(cudaGraphLaunch(b->graphs[2], s), "graph launch");
    b->stats_valid = false;
    return check_device_errors(b);
}

// -------------------------------------------------------------------- tree --

struct bh_tree {
    bh_device* dev = nullptr;
    bh_state* st = nullptr;
    Batch* batch = nullptr;
    bool built = false;
};

extern "C" int galaxy_bh_tree_create(bh_device* dev, bh_state* st, const bh_config* cfg,
                                     bh_tree** out) {
    int rc = enter(dev);
    if (rc) return rc;
    if (!out || !st) return set_error(BH_INVALID_ARG, "null argument");
    *out = nullptr;
    if ((rc = validate_config(cfg))) return rc;
    if (st->dev != dev) return set_error(BH_INVALID_ARG, "state does not belong to device");
    Batch* b = nullptr;
    if ((rc = batch_build(dev, &st, cfg, 1, &b))) return rc;
    bh_tree* t = new bh_tree();
    t->dev = dev;
    device_ref(dev);
    t->st = st;
    t->batch = b;
    *out = t;
    return BH_OK;
}

extern "C" int galaxy_bh_tree_destroy(bh_tree* tree) {
    if (!tree) return BH_OK;
    cudaSetDevice(tree->dev->ordinal);
    cudaStreamSynchronize(tree->dev->stream);
    delete tree->batch;
    bh_device* dev = tree->dev;
    delete tree;
    device_unref(dev);
    return BH_OK;
}

// Points *tree at state st under cfg (creating the tree when null), keeping
// its arena when that is large enough: a serving loop's stager solves each
// newcomer's boundary on one tree instead of allocating one per request.
int gbh::tree_retarget(bh_device* dev, bh_tree** tree, bh_state* st, const bh_config* cfg) {
    if (!tree) return set_error(BH_INVALID_ARG, "null argument");
    if (!*tree) return galaxy_bh_tree_create(dev, st, cfg, tree);
    int rc = enter(dev);
    if (rc) return rc;
    bh_tree* t = *tree;
    if (!st) return set_error(BH_INVALID_ARG, "null argument");
    if (t->dev != dev || st->dev != dev)
        return set_error(BH_INVALID_ARG, "tree or state belongs to another device handle");
    if ((rc = validate_config(cfg))) return rc;
    Batch* b = nullptr;
    Batch* donor = t->batch;
    t->batch = nullptr;
    t->built = false;
    if ((rc = batch_build(dev, &st, cfg, 1, &b, donor))) {
        galaxy_bh_tree_destroy(t);
        *tree = nullptr;
        return rc;
    }
    t->batch = b;
    t->st = st;
    return BH_OK;
}

static int tree_check(bh_device* dev, bh_state* st, bh_tree* tree) {
    int rc = enter(dev);
    if (rc) return rc;
    if (!tree || !st) return set_error(BH_INVALID_ARG, "null argument");
    if (tree->st != st || tree->dev != dev)
        return set_error(BH_INVALID_ARG, "tree count does not match evolving state");
    return BH_OK;
}

// Re-carves the tree's arena when cfg needs more cells than it holds.
static int tree_fit(bh_tree* tree, const bh_config* cfg) {
    int rc = validate_config(cfg);
    if (rc) return rc;
    if (cell_bound(tree->st->n, *cfg) <= tree->batch->cell_capacity) return BH_OK;
    Batch* nb = nullptr;
    if ((rc = batch_build(tree->dev, &tree->st, cfg, 1, &nb))) return rc;
    nb->bb.radix_bits = tree->batch->bb.radix_bits;  // keep the tree's tuning
    nb->bb.trav_warps = tree->batch->bb.trav_warps;
    delete tree->batch;
    tree->batch = nb;
    tree->built = false;
    return BH_OK;
}

extern "C" int galaxy_bh_tree_rebuild(bh_device* dev, bh_state* st, bh_tree* tree,
                                      const bh_config* cfg, bh_build_timing* timing) {
    int rc = tree_check(dev, st, tree);
    if (rc) return rc;
    if ((rc = tree_fit(tree, cfg))) return rc;
    if ((rc = apply_configs(tree->batch, cfg, true))) return rc;
    if ((rc = enqueue_rebuild(tree->batch, 0, dev->ev))) return rc;
    CK(cudaStreamSynchronize(dev->stream), "rebuild");
    if ((rc = check_device_errors(tree->batch))) return rc;
    if (timing) {
        float ms[5];
        for (int k = 0; k < 5; ++k) cudaEventElapsedTime(&ms[k], dev->ev[k], dev->ev[k + 1]);
        timing->bounds_seconds = ms[0] * 1e-3;
        timing->morton_seconds = ms[1] * 1e-3;
        timing->radix_seconds = ms[2] * 1e-3;
        timing->positions_seconds = 0.0;  // fused into the last radix pass
        timing->topology_seconds = ms[3] * 1e-3;
        timing->aggregate_seconds = ms[4] * 1e-3;
    }
    tree->built = true;
    tree->batch->built_theta = cfg->theta;
    tree->batch->built_g = cfg->g;
    return BH_OK;
}

extern "C" int galaxy_bh_force(bh_device* dev, bh_state* st, bh_tree* tree, const bh_config* cfg,
                               bh_stage_timing* timing) {
    int rc = tree_check(dev, st, tree);
    if (rc) return rc;
    if (!tree->built) return set_error(BH_INVALID_ARG, "force requires a rebuilt tree");
    if ((rc = apply_configs(tree->batch, cfg, false))) return rc;
    Batch* b = tree->batch;
    if (cfg->theta != b->built_theta || cfg->g != b->built_g) {
        CK(launch_refresh_mac(b->bb, 0, dev->stream), "refresh launch");
        b->built_theta = cfg->theta;
        b->built_g = cfg->g;
    }
    CK(cudaEventRecord(dev->ev[0], dev->stream), "event");
    const bool stats = !(cfg->flags & BH_FLAG_NO_STATS);
    if ((rc = enqueue_force(tree->batch, stats))) return rc;
    if ((rc = stage_time(dev, timing))) return rc;
    tree->batch->stats_valid = stats;
    return check_device_errors(tree->batch);
}

extern "C" int galaxy_bh_force_stats(bh_device* dev, bh_tree* tree, bh_force_stats* out) {
    int rc = enter(dev);
    if (rc) return rc;
    if (!tree || !out) return set_error(BH_INVALID_ARG, "null argument");
    if (!tree->batch->stats_valid)
        return set_error(BH_INVALID_ARG, "no force statistics since the last galaxy_bh_force");
    unsigned long long v[5];
    CK(cudaMemcpyAsync(v, tree->batch->bb.force_stats, sizeof v, cudaMemcpyDeviceToHost,
                       dev->stream),
       "readback");
    CK(cudaStreamSynchronize(dev->stream), "readback");
    out->visited_nodes = v[0];
    out->approximated_cells = v[1];
    out->direct_terms = v[2];
    out->exact_mac_fallbacks = v[3];
    out->warp_iterations = v[4];
    return BH_OK;
}

extern "C" int galaxy_bh_force_f64(bh_device* dev, bh_state* st, bh_tree* tree,
                                   const bh_config* cfg, double* accel, double* abs_sum,
                                   bh_force_stats* stats) {
    int rc = tree_check(dev, st, tree);
    if (rc) return rc;
    if (!cfg || !accel) return set_error(BH_INVALID_ARG, "null argument");
    if ((rc = validate_config(cfg))) return rc;
    if (!tree->built) return set_error(BH_INVALID_ARG, "force requires a rebuilt tree");
    const size_t n = st->n;
    const size_t bytes = 16 * n + (abs_sum ? 8 * n : 0) + 32;
    char* d = nullptr;
    CK(cudaMalloc(&d, bytes), "f64 traversal allocation");
    double* d_acc = reinterpret_cast<double*>(d);
    double* d_abs = abs_sum ? reinterpret_cast<double*>(d + 16 * n) : nullptr;
    unsigned long long* d_stats = reinterpret_cast<unsigned long long*>(d + bytes - 32);
    unsigned long long h_stats[3] = {0, 0, 0};
    cudaError_t e = cudaMemsetAsync(d_stats, 0, 32, dev->stream);
    if (!e)
        e = launch_traverse_f64(tree->batch->bb, 0, st->n, cfg->theta, cfg->softening, cfg->g,
                                d_acc, d_abs, d_stats, dev->stream);
    if (!e) e = cudaMemcpyAsync(accel, d_acc, 16 * n, cudaMemcpyDeviceToHost, dev->stream);
    if (!e && abs_sum)
        e = cudaMemcpyAsync(abs_sum, d_abs, 8 * n, cudaMemcpyDeviceToHost, dev->stream);
    if (!e) e = cudaMemcpyAsync(h_stats, d_stats, 24, cudaMemcpyDeviceToHost, dev->stream);
    if (!e) e = cudaStreamSynchronize(dev->stream);
    cudaFree(d);
    if (e) return cuda_fail(e, "f64 traversal");
    if (stats) {
        *stats = bh_force_stats{};
        stats->visited_nodes = h_stats[0];
        stats->approximated_cells = h_stats[1];
        stats->direct_terms = h_stats[2];
    }
    return BH_OK;
}

extern "C" int galaxy_bh_wait_probe(bh_device* dev, uint64_t spin_cycles) {
    int rc = enter(dev);
    if (rc) return rc;
    if (spin_cycles > (uint64_t)4000000000ull)
        return set_error(BH_INVALID_ARG, "spin_cycles above 4e9 (about two seconds)");
    // flags of the never-published first tile, the error word, the results
    constexpr size_t kWords = 2 * kRadixDigits + 1;
    uint32_t* d = nullptr;
    CK(cudaMalloc(&d, kWords * 4), "probe allocation");
    cudaError_t e = cudaMemsetAsync(d, 0, kWords * 4, dev->stream);
    if (e == cudaSuccess)
        e = launch_wait_probe(d, d + kRadixDigits, (long long)spin_cycles, d + kRadixDigits + 1,
                              dev->stream);
    uint32_t err = 0;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&err, d + kRadixDigits, 4, cudaMemcpyDeviceToHost, dev->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(dev->stream);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "wait probe");
    if (err & kErrLookbackTimeout)
        return set_error(BH_TIMEOUT, "device wait (look-back) timed out (error bits 0x%x)", err);
    return set_error(BH_CUDA_ERROR, "wait probe: the bounded wait did not report its timeout");
}

extern "C" int galaxy_bh_read_tree_evidence(bh_device* dev, bh_tree* tree, TreeMeta* meta,
                                            GpuEntry* entries, GpuBody* bodies, uint32_t n,
                                            GpuCell* cells, uint32_t cell_capacity,
                                            uint32_t* cell_count) {
    int rc = enter(dev);
    if (rc) return rc;
    if (!tree) return set_error(BH_INVALID_ARG, "null tree");
    if (!tree->built) return set_error(BH_INVALID_ARG, "tree has not been rebuilt");
    Batch* b = tree->batch;
    const uint32_t sn = tree->st->n;
    if ((entries || bodies) && n != sn)
        return set_error(BH_INVALID_ARG, "evidence count %u != resident bodies %u", n, sn);
    cudaStream_t s = dev->stream;
    uint32_t cb_ce[2];
    CK(cudaMemcpyAsync(&cb_ce[0], b->bb.base + b->h_sims[0].off, 4, cudaMemcpyDeviceToHost, s), "readback");
    CK(cudaMemcpyAsync(&cb_ce[1], b->bb.base + b->h_sims[0].off + sn, 4, cudaMemcpyDeviceToHost, s), "readback");
    SimOut so;
    CK(cudaMemcpyAsync(&so, b->bb.simout, sizeof so, cudaMemcpyDeviceToHost, s), "readback");
    CK(cudaStreamSynchronize(s), "readback");
    const uint32_t ncell = cb_ce[1] - cb_ce[0];
    if (cell_count) *cell_count = ncell;
    if (meta) {
        meta->data[0] = ncell;
        meta->data[1] = sn;
        meta->data[2] = b->h_sims[0].max_depth;
        meta->data[3] = 0;
        meta->bounds[0] = (float)so.cx;
        meta->bounds[1] = (float)so.cy;
        meta->bounds[2] = (float)so.half;
        meta->bounds[3] = 0.f;
    }
    if (cells && cell_capacity < ncell)
        return set_error(BH_CAPACITY_OVERFLOW, "cell buffer holds %u records, tree has %u",
                         cell_capacity, ncell);
    GpuEntry* d_e = nullptr;
    GpuBody* d_b = nullptr;
    GpuCell* d_c = nullptr;
    cudaError_t e = cudaSuccess;
    if (entries) e = cudaMalloc(&d_e, sizeof(GpuEntry) * (size_t)sn);
    if (!e && bodies) e = cudaMalloc(&d_b, sizeof(GpuBody) * (size_t)sn);
    if (!e && cells && ncell) e = cudaMalloc(&d_c, sizeof(GpuCell) * (size_t)ncell);
    if (!e) e = launch_export(b->bb, 0, d_e, d_b, d_c, s);
    if (!e && entries) e = cudaMemcpyAsync(entries, d_e, sizeof(GpuEntry) * (size_t)sn, cudaMemcpyDeviceToHost, s);
    if (!e && bodies) e = cudaMemcpyAsync(bodies, d_b, sizeof(GpuBody) * (size_t)sn, cudaMemcpyDeviceToHost, s);
    if (!e && cells && ncell) e = cudaMemcpyAsync(cells, d_c, sizeof(GpuCell) * (size_t)ncell, cudaMemcpyDeviceToHost, s);
    if (!e) e = cudaStreamSynchronize(s);
    cudaFree(d_e);
    cudaFree(d_b);
    cudaFree(d_c);
    if (e) return cuda_fail(e, "tree evidence");
    return BH_OK;
}

extern "C" int galaxy_bh_tree_footprint(uint32_t n, const bh_config* cfg, uint64_t* bytes) {
    if (!cfg || !bytes) return set_error(BH_INVALID_ARG, "null argument");
    int rc = validate_config(cfg);
    if (rc) return rc;
    const uint32_t counts[1] = {n};
    Layout L = plan_layout(counts, cfg, 1);
    *bytes = plan_arena(L, 1).total();
    return BH_OK;
}

extern "C" int galaxy_bh_tree_buffer_bytes(bh_tree* tree, uint64_t* bytes) {
    if (!tree || !bytes) return set_error(BH_INVALID_ARG, "null argument");
    *bytes = tree->batch->arena_bytes;
    return BH_OK;
}

extern "C" int galaxy_bh_step(bh_device* dev, bh_state* st, bh_tree* tree, const bh_config* cfg,
                              double dt, uint32_t nsteps) {
    int rc = tree_check(dev, st, tree);
    if (rc) return rc;
    if (!tree->built) return set_error(BH_INVALID_ARG, "step requires rebuild + force first");
    float f = 0.f;
    if ((rc = checked_dt(dt, &f))) return rc;
    if (nsteps == 0) return BH_OK;
    tree->batch->h_sims[0].dt = f;
    if ((rc = apply_configs(tree->batch, cfg, true))) return rc;
    tree->batch->built_theta = cfg->theta;
    tree->batch->built_g = cfg->g;
    return run_graphs(tree->batch, nsteps);
}

// ----------------------------------------------------------- packed (2B1) --

static int packed_checks(const BhSettings* settings, const GpuBody* bodies, uint32_t n,
                         const GpuEntry* entries, const GpuCell* cells, uint32_t cell_count) {
    if (!settings || !bodies || !entries || !cells)
        return set_error(BH_INVALID_ARG, "null argument");
    if (n == 0 || cell_count == 0)
        return set_error(BH_INVALID_ARG, "Barnes-Hut bodies/cells requires a non-empty buffer");
    if (settings->info[0] != n) return set_error(BH_INVALID_ARG, "flat tree/body cardinality mismatch");
    if (settings->info[2] >= cell_count) return set_error(BH_INVALID_ARG, "flat tree has invalid root");
    return BH_OK;
}

static int run_packed(bh_device* dev, const BhSettings* settings, const GpuBody* bodies,
                      uint32_t n, const GpuEntry* entries, const GpuCell* cells,
                      uint32_t cell_count, float4* d_out, bh_stage_timing* timing) {
    cudaStream_t s = dev->stream;
    BhSettings* d_s = nullptr;
    GpuBody* d_b = nullptr;
    GpuEntry* d_e = nullptr;
    GpuCell* d_c = nullptr;
    uint32_t* d_err = nullptr;
    cudaError_t e = cudaSuccess;
    uint32_t err = 0;
    float t_up = 0.f, t_k = 0.f;
    if ((e = cudaMalloc(&d_s, sizeof(BhSettings))) ||
        (e = cudaMalloc(&d_b, sizeof(GpuBody) * (size_t)n)) ||
        (e = cudaMalloc(&d_e, sizeof(GpuEntry) * (size_t)n)) ||
        (e = cudaMalloc(&d_c, sizeof(GpuCell) * (size_t)cell_count)) ||
        (e = cudaMalloc(&d_err, 8)))
        goto done;
    cudaEventRecord(dev->ev[0], s);
    if ((e = cudaMemcpyAsync(d_s, settings, sizeof(BhSettings), cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(d_b, bodies, sizeof(GpuBody) * (size_t)n, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(d_e, entries, sizeof(GpuEntry) * (size_t)n, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(d_c, cells, sizeof(GpuCell) * (size_t)cell_count, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemsetAsync(d_err, 0, 8, s)))
        goto done;
    cudaEventRecord(dev->ev[1], s);
    if ((e = launch_traverse_packed(d_s, d_b, d_e, d_c, n, cell_count, d_out, d_err, s))) goto done;
    cudaEventRecord(dev->ev[2], s);
    if ((e = cudaMemcpyAsync(&err, d_err, 4, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaStreamSynchronize(s)))
        goto done;
    cudaEventElapsedTime(&t_up, dev->ev[0], dev->ev[1]);
    cudaEventElapsedTime(&t_k, dev->ev[1], dev->ev[2]);
    if (timing) *timing = bh_stage_timing{t_up * 1e-3, t_k * 1e-3, 0.0};
done:
    cudaFree(d_s);
    cudaFree(d_b);
    cudaFree(d_e);
    cudaFree(d_c);
    cudaFree(d_err);
    if (e) return cuda_fail(e, "packed traversal");
    if (err & kErrPackedStack)
        return set_error(BH_CAPACITY_OVERFLOW, "packed traversal stack exceeded 64 entries");
    if (err) return set_error(BH_INVALID_ARG, "packed tree holds an out-of-range index");
    return BH_OK;
}

extern "C" int galaxy_bh_traverse_packed(bh_device* dev, const BhSettings* settings,
                                         const GpuBody* bodies, uint32_t n,
                                         const GpuEntry* entries, const GpuCell* cells,
                                         uint32_t cell_count, GpuAccel* out,
                                         bh_stage_timing* timing) {
    int rc = enter(dev);
    if (rc) return rc;
    if (!out) return set_error(BH_INVALID_ARG, "null argument");
    if ((rc = packed_checks(settings, bodies, n, entries, cells, cell_count))) return rc;
    float4* d_out = nullptr;
    CK(cudaMalloc(&d_out, sizeof(float4) * (size_t)n), "output allocation");
    cudaMemsetAsync(d_out, 0, sizeof(float4) * (size_t)n, dev->stream);
    rc = run_packed(dev, settings, bodies, n, entries, cells, cell_count, d_out, timing);
    cudaEvent_t* ev = dev->ev;
    if (!rc) {
        cudaEventRecord(ev[3], dev->stream);
        cudaError_t e = cudaMemcpyAsync(out, d_out, sizeof(float4) * (size_t)n,
                                        cudaMemcpyDeviceToHost, dev->stream);
        if (!e) e = cudaStreamSynchronize(dev->stream);
        if (e) rc = cuda_fail(e, "acceleration readback");
        if (!rc && timing) {
            float ms = 0.f;
            cudaEventRecord(ev[4], dev->stream);
            cudaEventSynchronize(ev[4]);
            cudaEventElapsedTime(&ms, ev[3], ev[4]);
            timing->readback_seconds = ms * 1e-3;
        }
    }
    cudaFree(d_out);
    if (rc) return rc;
    for (uint32_t i = 0; i < n; ++i)
        if (!std::isfinite(out[i].value[0]) || !std::isfinite(out[i].value[1]))
            return set_error(BH_NONFINITE, "GPU produced non-finite acceleration for body %u", i);
    return BH_OK;
}

extern "C" int galaxy_bh_force_into(bh_device* dev, bh_state* st, const BhSettings* settings,
                                    const GpuBody* bodies, const GpuEntry* entries,
                                    const GpuCell* cells, uint32_t cell_count,
                                    bh_stage_timing* timing) {
    int rc = enter(dev);
    if (rc) return rc;
    if (!st) return set_error(BH_INVALID_ARG, "null state");
    if ((rc = packed_checks(settings, bodies, st->n, entries, cells, cell_count)))
        return set_error(rc, "Barnes-Hut force/tree count does not match evolving state");
    return run_packed(dev, settings, bodies, st->n, entries, cells, cell_count, st->d_accel, timing);
}

// ------------------------------------------------------------ batch API ----

struct bh_batch {
    bh_device* dev = nullptr;
    Batch* batch = nullptr;
    bool solved = false;
};

extern "C" int galaxy_bh_batch_create(bh_device* dev, bh_state* const* states,
                                      const bh_config* cfgs, uint32_t count, bh_batch** out) {
    int rc = enter(dev);
    if (rc) return rc;
    if (!states || !cfgs || !out) return set_error(BH_INVALID_ARG, "null argument");
    *out = nullptr;
    for (uint32_t s = 0; s < count; ++s)
        if (cfgs[s].flags & BH_FLAG_POTENTIAL) {
            if (!states[s]) return set_error(BH_INVALID_ARG, "null state %u", s);
            if ((rc = ensure_potential(states[s]))) return rc;
        }
    Batch* b = nullptr;
    if ((rc = batch_build(dev, states, cfgs, count, &b))) return rc;
    bh_batch* h = new bh_batch();
    h->dev = dev;
    device_ref(dev);
    h->batch = b;
    *out = h;
    return BH_OK;
}

extern "C" int galaxy_bh_batch_destroy(bh_batch* batch) {
    if (!batch) return BH_OK;
    cudaSetDevice(batch->dev->ordinal);
    cudaStreamSynchronize(batch->dev->stream);
    delete batch->batch;
    bh_device* dev = batch->dev;
    delete batch;
    device_unref(dev);
    return BH_OK;
}

// Re-forms *batch over `count` states (creating it when null, destroying it
// when count is 0), keeping its arena when that is large enough: a serving
// loop's joins and leaves then allocate nothing once the arena has grown to
// the largest active set.
int gbh::batch_reform(bh_device* dev, bh_batch** batch, bh_state* const* states,
                      const bh_config* cfgs, uint32_t count) {
    if (!batch) return set_error(BH_INVALID_ARG, "null argument");
    if (count == 0) {
        galaxy_bh_batch_destroy(*batch);
        *batch = nullptr;
        return BH_OK;
    }
    if (!*batch) return galaxy_bh_batch_create(dev, states, cfgs, count, batch);
    int rc = enter(dev);
    if (rc) return rc;
    bh_batch* h = *batch;
    if (h->dev != dev) return set_error(BH_INVALID_ARG, "batch belongs to another device handle");
    if (!states || !cfgs) return set_error(BH_INVALID_ARG, "null argument");
    for (uint32_t s = 0; s < count; ++s)
        if (cfgs[s].flags & BH_FLAG_POTENTIAL) {
            if (!states[s]) return set_error(BH_INVALID_ARG, "null state %u", s);
            if ((rc = ensure_potential(states[s]))) return rc;
        }
    Batch* b = nullptr;
    Batch* donor = h->batch;
    h->batch = nullptr;
    h->solved = false;
    if ((rc = batch_build(dev, states, cfgs, count, &b, donor))) {
        galaxy_bh_batch_destroy(h);
        *batch = nullptr;
        return rc;
    }
    h->batch = b;
    return BH_OK;
}

extern "C" int galaxy_bh_batch_solve(bh_device* dev, bh_batch* batch) {
    int rc = enter(dev);
    if (rc) return rc;
    if (!batch || batch->dev != dev) return set_error(BH_INVALID_ARG, "batch does not belong to device");
    Batch* b = batch->batch;
    if ((rc = upload_sims(b))) return rc;
    if ((rc = enqueue_rebuild(b, 0, nullptr))) return rc;
    if ((rc = enqueue_force(b, false))) return rc;
    batch->solved = true;
    return check_device_errors(b);
}

extern "C" int galaxy_bh_batch_step(bh_device* dev, bh_batch* batch, const double* dts,
                                    uint32_t nsteps) {
    int rc = enter(dev);
    if (rc) return rc;
    if (!batch || !dts || batch->dev != dev) return set_error(BH_INVALID_ARG, "null argument");
    // Each member's acceleration buffer must already hold its boundary
    // acceleration (from galaxy_bh_batch_solve, galaxy_bh_force, or earlier
    // steps of any batch or tree): a batch re-formed after members left can
    // step at once.
    Batch* b = batch->batch;
    for (size_t s = 0; s < b->h_sims.size(); ++s) {
        float f = 0.f;
        if ((rc = checked_dt(dts[s], &f))) return rc;
        b->h_sims[s].dt = f;
    }
    if (nsteps == 0) return BH_OK;
    if ((rc = upload_sims(b))) return rc;
    return run_graphs(b, nsteps);
}

// Installs launch-shape knobs; the next step re-captures its graphs.
static int apply_tuning(Batch* b, const bh_tuning* t) {
    if (!t) return set_error(BH_INVALID_ARG, "null argument");
    if (t->radix_bits != 4 && t->radix_bits != 8)
        return set_error(BH_INVALID_ARG, "radix_bits must be 4 or 8, got %u", t->radix_bits);
    if (t->traverse_warps != 2 && t->traverse_warps != 4 && t->traverse_warps != 8)
        return set_error(BH_INVALID_ARG, "traverse_warps must be 2, 4 or 8, got %u",
                         t->traverse_warps);
    if (t->radix_bits != b->bb.radix_bits || t->traverse_warps != b->bb.trav_warps) {
        b->bb.radix_bits = t->radix_bits;
        b->bb.trav_warps = t->traverse_warps;
        b->graph_flags = 0xffffffffu;  // graphs hold the old launch shapes
    }
    return BH_OK;
}

extern "C" int galaxy_bh_batch_tune(bh_batch* batch, const bh_tuning* tuning) {
    if (!batch) return set_error(BH_INVALID_ARG, "null batch");
    return apply_tuning(batch->batch, tuning);
}

extern "C" int galaxy_bh_tree_tune(bh_tree* tree, const bh_tuning* tuning) {
    if (!tree) return set_error(BH_INVALID_ARG, "null tree");
    return apply_tuning(tree->batch, tuning);
}

extern "C" int galaxy_bh_batch_bytes(bh_batch* batch, uint64_t* bytes) {
    if (!batch || !bytes) return set_error(BH_INVALID_ARG, "null argument");
    *bytes = batch->batch->arena_bytes;
    return BH_OK;
}
