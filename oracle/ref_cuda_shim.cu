// SPDX-License-Identifier: Apache-2.0
//
// Host launcher for the reference's own CUDA kernels (test infrastructure).
// The reference file runtime/cuda/barnes_hut_flat.cu is compiled unmodified
// from where it lies (REF_CU is its path, passed by oracle/Makefile); this
// translation unit only adds C entry points that upload packed records, launch
// the kernels the way runtime/src/nbody_gpu.rs:640-780 and :940-1009 dispatch
// them (ceil(N/128) groups of 128), and copy the result back.  The engine never
// links this; the GPU tests use it as a second, independent checker.
#include REF_CU

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <vector>

namespace {
struct Timer {
    cudaEvent_t a, b;
    Timer() { cudaEventCreate(&a); cudaEventCreate(&b); }
    ~Timer() { cudaEventDestroy(a); cudaEventDestroy(b); }
};

// Median device time of `repeats` single launches, each bracketed by its own
// events; with flush, a 256 MiB memset before each launch evicts L2 (126 MB)
// so the launch reads its inputs from DRAM.
template <typename F>
cudaError_t time_single(F launch, int repeats, bool flush, float* ms_out) {
    void* scratch = nullptr;
    cudaError_t err = cudaSuccess;
    const size_t kFlush = 256ull << 20;
    if (flush && (err = cudaMalloc(&scratch, kFlush))) return err;
    std::vector<float> ms;
    Timer t;
    for (int r = 0; r < std::max(repeats, 1); ++r) {
        if (flush) cudaMemsetAsync(scratch, r & 0xff, kFlush);
        cudaEventRecord(t.a);
        launch();
        cudaEventRecord(t.b);
        if ((err = cudaEventSynchronize(t.b))) break;
        float v = 0.f;
        cudaEventElapsedTime(&v, t.a, t.b);
        ms.push_back(v);
    }
    if (scratch) cudaFree(scratch);
    if (!err) err = cudaGetLastError();
    if (!err && !ms.empty()) {
        std::sort(ms.begin(), ms.end());
        *ms_out = ms[ms.size() / 2];
    }
    return err;
}
}  // namespace

extern "C" int ref_bh_traverse(const void* settings, const void* bodies, uint32_t n,
                               const void* entries, const void* cells, uint32_t n_cells,
                               void* accel_out, float* kernel_ms, int repeats) {
    BhSettings* d_s = nullptr;
    BhBody* d_b = nullptr;
    BhEntry* d_e = nullptr;
    BhCell* d_c = nullptr;
    float4* d_a = nullptr;
    cudaError_t err = cudaSuccess;
    if ((err = cudaMalloc(&d_s, sizeof(BhSettings))) ||
        (err = cudaMalloc(&d_b, sizeof(BhBody) * (size_t)n)) ||
        (err = cudaMalloc(&d_e, sizeof(BhEntry) * (size_t)n)) ||
        (err = cudaMalloc(&d_c, sizeof(BhCell) * (size_t)n_cells)) ||
        (err = cudaMalloc(&d_a, sizeof(float4) * (size_t)n)))
        goto done;
    cudaMemcpy(d_s, settings, sizeof(BhSettings), cudaMemcpyHostToDevice);
    cudaMemcpy(d_b, bodies, sizeof(BhBody) * (size_t)n, cudaMemcpyHostToDevice);
    cudaMemcpy(d_e, entries, sizeof(BhEntry) * (size_t)n, cudaMemcpyHostToDevice);
    cudaMemcpy(d_c, cells, sizeof(BhCell) * (size_t)n_cells, cudaMemcpyHostToDevice);
    {
        Timer t;
        if (repeats < 1) repeats = 1;
        bh_traverse<<<(n + 127) / 128, 128>>>(d_s, d_b, d_e, d_c, d_a);
        cudaEventRecord(t.a);
        for (int r = 0; r < repeats; ++r) bh_traverse<<<(n + 127) / 128, 128>>>(d_s, d_b, d_e, d_c, d_a);
        cudaEventRecord(t.b);
        if ((err = cudaEventSynchronize(t.b))) goto done;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t.a, t.b);
        if (kernel_ms) *kernel_ms = ms / (float)repeats;
    }
    if ((err = cudaGetLastError())) goto done;
    err = cudaMemcpy(accel_out, d_a, sizeof(float4) * (size_t)n, cudaMemcpyDeviceToHost);
done:
    cudaFree(d_s); cudaFree(d_b); cudaFree(d_e); cudaFree(d_c); cudaFree(d_a);
    return (int)err;
}

// bh_traverse over an uploaded packed tree: median single-launch device
// time with L2 warm (ms_warm) and flushed before each launch (ms_cold).
extern "C" int ref_bh_traverse_single(const void* settings, const void* bodies, uint32_t n,
                                      const void* entries, const void* cells, uint32_t n_cells,
                                      float* ms_warm, float* ms_cold, int repeats) {
    BhSettings* d_s = nullptr;
    BhBody* d_b = nullptr;
    BhEntry* d_e = nullptr;
    BhCell* d_c = nullptr;
    float4* d_a = nullptr;
    cudaError_t err = cudaSuccess;
    auto launch = [&] { bh_traverse<<<(n + 127) / 128, 128>>>(d_s, d_b, d_e, d_c, d_a); };
    if ((err = cudaMalloc(&d_s, sizeof(BhSettings))) ||
        (err = cudaMalloc(&d_b, sizeof(BhBody) * (size_t)n)) ||
        (err = cudaMalloc(&d_e, sizeof(BhEntry) * (size_t)n)) ||
        (err = cudaMalloc(&d_c, sizeof(BhCell) * (size_t)n_cells)) ||
        (err = cudaMalloc(&d_a, sizeof(float4) * (size_t)n)))
        goto done;
    cudaMemcpy(d_s, settings, sizeof(BhSettings), cudaMemcpyHostToDevice);
    cudaMemcpy(d_b, bodies, sizeof(BhBody) * (size_t)n, cudaMemcpyHostToDevice);
    cudaMemcpy(d_e, entries, sizeof(BhEntry) * (size_t)n, cudaMemcpyHostToDevice);
    cudaMemcpy(d_c, cells, sizeof(BhCell) * (size_t)n_cells, cudaMemcpyHostToDevice);
    launch();
    if ((err = time_single(launch, repeats, false, ms_warm))) goto done;
    err = time_single(launch, repeats, true, ms_cold);
done:
    cudaFree(d_s); cudaFree(d_b); cudaFree(d_e); cudaFree(d_c); cudaFree(d_a);
    return (int)err;
}

static int run_integrate(int final_kick, void* states, const void* accel, uint32_t n, float dt,
                         float* kernel_ms, int repeats) {
    EvolveSettings s = {};
    s.info[0] = n;
    s.motion[0] = dt;
    EvolveSettings* d_s = nullptr;
    EvolveState* d_st = nullptr;
    float4* d_a = nullptr;
    cudaError_t err = cudaSuccess;
    if ((err = cudaMalloc(&d_s, sizeof s)) ||
        (err = cudaMalloc(&d_st, sizeof(EvolveState) * (size_t)n)) ||
        (err = cudaMalloc(&d_a, sizeof(float4) * (size_t)n)))
        goto done;
    cudaMemcpy(d_s, &s, sizeof s, cudaMemcpyHostToDevice);
    cudaMemcpy(d_st, states, sizeof(EvolveState) * (size_t)n, cudaMemcpyHostToDevice);
    cudaMemcpy(d_a, accel, sizeof(float4) * (size_t)n, cudaMemcpyHostToDevice);
    if (final_kick)
        bh_final_kick<<<(n + 127) / 128, 128>>>(d_s, d_st, d_a);
    else
        bh_kick_drift<<<(n + 127) / 128, 128>>>(d_s, d_st, d_a);
    if ((err = cudaGetLastError())) goto done;
    err = cudaMemcpy(states, d_st, sizeof(EvolveState) * (size_t)n, cudaMemcpyDeviceToHost);
    if (!err && kernel_ms) {
        // further launches on the device copy, timed (the state keeps moving)
        Timer t;
        if (repeats < 1) repeats = 1;
        cudaEventRecord(t.a);
        for (int r = 0; r < repeats; ++r) {
            if (final_kick)
                bh_final_kick<<<(n + 127) / 128, 128>>>(d_s, d_st, d_a);
            else
                bh_kick_drift<<<(n + 127) / 128, 128>>>(d_s, d_st, d_a);
        }
        cudaEventRecord(t.b);
        if ((err = cudaEventSynchronize(t.b))) goto done;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t.a, t.b);
        *kernel_ms = ms / (float)repeats;
        err = cudaGetLastError();
    }
done:
    cudaFree(d_s); cudaFree(d_st); cudaFree(d_a);
    return (int)err;
}

extern "C" int ref_bh_kick_drift(void* states, const void* accel, uint32_t n, float dt) {
    return run_integrate(0, states, accel, n, dt, nullptr, 0);
}

extern "C" int ref_bh_final_kick(void* states, const void* accel, uint32_t n, float dt) {
    return run_integrate(1, states, accel, n, dt, nullptr, 0);
}

// One launch whose result goes to `states`, then `repeats` timed launches on
// the device copy; *kernel_ms = mean device time of those.
extern "C" int ref_bh_integrate_timed(int final_kick, void* states, const void* accel, uint32_t n,
                                      float dt, float* kernel_ms, int repeats) {
    return run_integrate(final_kick, states, accel, n, dt, kernel_ms, repeats);
}

// bh_kick_drift / bh_final_kick over uploaded (states, accel): median
// single-launch device time with L2 warm and flushed before each launch.
extern "C" int ref_bh_integrate_single(int final_kick, const void* states, const void* accel,
                                       uint32_t n, float dt, float* ms_warm, float* ms_cold,
                                       int repeats) {
    EvolveSettings s = {};
    s.info[0] = n;
    s.motion[0] = dt;
    EvolveSettings* d_s = nullptr;
    EvolveState* d_st = nullptr;
    float4* d_a = nullptr;
    cudaError_t err = cudaSuccess;
    auto launch = [&] {
        if (final_kick)
            bh_final_kick<<<(n + 127) / 128, 128>>>(d_s, d_st, d_a);
        else
            bh_kick_drift<<<(n + 127) / 128, 128>>>(d_s, d_st, d_a);
    };
    if ((err = cudaMalloc(&d_s, sizeof s)) ||
        (err = cudaMalloc(&d_st, sizeof(EvolveState) * (size_t)n)) ||
        (err = cudaMalloc(&d_a, sizeof(float4) * (size_t)n)))
        goto done;
    cudaMemcpy(d_s, &s, sizeof s, cudaMemcpyHostToDevice);
    cudaMemcpy(d_st, states, sizeof(EvolveState) * (size_t)n, cudaMemcpyHostToDevice);
    cudaMemcpy(d_a, accel, sizeof(float4) * (size_t)n, cudaMemcpyHostToDevice);
    launch();
    if ((err = time_single(launch, repeats, false, ms_warm))) goto done;
    err = time_single(launch, repeats, true, ms_cold);
done:
    cudaFree(d_s); cudaFree(d_st); cudaFree(d_a);
    return (int)err;
}
