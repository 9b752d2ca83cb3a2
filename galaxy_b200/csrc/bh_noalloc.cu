// SPDX-License-Identifier: Apache-2.0
//
// FP64 conservation sums that allocate nothing.
//
// galaxy_bh_conservation allocates its per-block partial-sum buffer with
// cudaMalloc on first use.  Some callers cannot allocate device memory when
// they want these sums: a serving loop that reserved its whole memory budget
// up front and must not grow it between steps, a host runtime whose own
// allocator owns all device memory (a cudaMalloc from a plug-in would fail or
// fragment its pool), or a caller that works only with device buffers it was
// handed.  galaxy_bh_conservation_noalloc serves them: the caller passes the
// device input (state records, optional potentials) and the device output,
// and the partial sums live in a file-scope __device__ array below, which
// every GPU that loads this library holds until the process exits.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "bh_internal.cuh"

namespace {

constexpr uint32_t kThreads = 256;
constexpr uint32_t kItems = 16;
constexpr uint32_t kSliceBodies = kThreads * kItems;  // bodies per block
constexpr uint32_t kMaxBlocks = 1024;
constexpr uint32_t kTerms = 9;
constexpr uint32_t kMaxBodies = kMaxBlocks * kSliceBodies;  // 4,194,304
constexpr int kMaxDevices = 64;

}  // namespace

// Scratch: one row of kTerms partial sums per block, 73,728 bytes.  Each call
// overwrites the rows of the blocks it launches before it reads them, so no
// row needs clearing; rows beyond the call's block count are never read.
static __device__ __align__(256) double g_conservation_scratch[kMaxBlocks * kTerms];

// Block b sums bodies [b*kSliceBodies, min(n, (b+1)*kSliceBodies)) in a fixed
// order and writes its kTerms partial sums to row b.
__global__ void __launch_bounds__(kThreads) k_conservation_slices(const GpuEvolveState* __restrict__ state,
                                                                  const float* __restrict__ potential,
                                                                  uint32_t n, double* partials) {
    __shared__ double sh[kTerms][kThreads];
    double t[kTerms] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const uint32_t base = blockIdx.x * kSliceBodies;
#pragma unroll 4
    for (uint32_t k = 0; k < kItems; ++k) {
        const uint32_t i = base + k * kThreads + threadIdx.x;
        if (i >= n) break;
        const GpuEvolveState s = state[i];
        const double m = s.position_mass[2], x = s.position_mass[0], y = s.position_mass[1];
        const double vx = s.velocity[0], vy = s.velocity[1];
        t[0] += m;
        t[1] += m * x;
        t[2] += m * y;
        t[3] += m * vx;
        t[4] += m * vy;
        t[5] += m * (x * vy - y * vx);
        t[6] += 0.5 * m * (vx * vx + vy * vy);
        if (potential) t[7] += 0.5 * m * (double)potential[i];
        t[8] += m * hypot(vx, vy);
    }
#pragma unroll
    for (int k = 0; k < (int)kTerms; ++k) sh[k][threadIdx.x] = t[k];
    __syncthreads();
    for (int stride = kThreads / 2; stride > 0; stride >>= 1) {
        if ((int)threadIdx.x < stride)
#pragma unroll
            for (int k = 0; k < (int)kTerms; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + stride];
        __syncthreads();
    }
    if (threadIdx.x < kTerms) partials[blockIdx.x * kTerms + threadIdx.x] = sh[threadIdx.x][0];
}

// Adds the rows of this call's blocks in block order into out[0..kTerms).
__global__ void k_conservation_rows(const double* partials, uint32_t nblocks, double* out) {
    if (threadIdx.x >= kTerms) return;
    double acc = 0.0;
    for (uint32_t b = 0; b < nblocks; ++b) acc += partials[b * kTerms + threadIdx.x];
    out[threadIdx.x] = acc;
}

static std::mutex g_setup_mutex;
static double* g_scratch_address[kMaxDevices] = {};

// Device address of g_conservation_scratch on the current device, looked up
// once per device with that device current.  The address belongs to the
// device's context: a cudaDeviceReset in this process ends that context and
// the cached address with it, so the entry point must not be called on a
// device after a reset (the header says so).
static int scratch_address(double** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        char msg[256];
        snprintf(msg, sizeof msg, "cudaGetDevice failed: %s", cudaGetErrorName(e));
        return gbh::set_error_message(BH_NO_DEVICE, msg);
    }
    if (dev < 0 || dev >= kMaxDevices)
        return gbh::set_error_message(BH_NO_DEVICE, "device ordinal beyond 63");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_address[dev]) {
        double* p = nullptr;
        e = cudaGetSymbolAddress((void**)&p, g_conservation_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            char msg[256];
            snprintf(msg, sizeof msg, "cudaGetSymbolAddress of the conservation scratch failed: %s",
                     cudaGetErrorName(e));
            return gbh::set_error_message(BH_CUDA_ERROR, msg);
        }
        g_scratch_address[dev] = p;
    }
    *out = g_scratch_address[dev];
    return BH_OK;
}

extern "C" int galaxy_bh_conservation_noalloc(const GpuEvolveState* state, const float* potential,
                                              uint32_t n, double* sums, void* stream) {
    if (!state || !sums)
        return gbh::set_error_message(BH_INVALID_ARG, "null state or sums pointer");
    if (n == 0) return gbh::set_error_message(BH_INVALID_ARG, "n must be at least 1");
    if (n > kMaxBodies) {
        char msg[256];
        snprintf(msg, sizeof msg,
                 "n = %u exceeds the no-allocation limit of %u bodies (%u blocks of scratch)", n,
                 kMaxBodies, kMaxBlocks);
        return gbh::set_error_message(BH_INVALID_ARG, msg);
    }
    double* scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;
    const uint32_t blocks = (n + kSliceBodies - 1) / kSliceBodies;
    cudaStream_t s = (cudaStream_t)stream;
    if (s) {
        // the scratch address is the current device's: the stream must run there
        int cur = -1, sdev = -1;
        cudaError_t e = cudaGetDevice(&cur);
        if (e == cudaSuccess) e = cudaStreamGetDevice(s, &sdev);
        if (e != cudaSuccess) {
            cudaGetLastError();
            char msg[256];
            snprintf(msg, sizeof msg, "stream device query failed: %s", cudaGetErrorName(e));
            return gbh::set_error_message(BH_INVALID_ARG, msg);
        }
        if (sdev != cur) {
            char msg[256];
            snprintf(msg, sizeof msg,
                     "stream belongs to device %d but device %d is current; make the "
                     "stream's device current before the call", sdev, cur);
            return gbh::set_error_message(BH_INVALID_ARG, msg);
        }
    }
    k_conservation_slices<<<blocks, kThreads, 0, s>>>(state, potential, n, scratch);
    k_conservation_rows<<<1, 32, 0, s>>>(scratch, blocks, sums);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        char msg[256];
        snprintf(msg, sizeof msg, "conservation launch failed: %s", cudaGetErrorName(e));
        return gbh::set_error_message(BH_CUDA_ERROR, msg);
    }
    return BH_OK;
}
