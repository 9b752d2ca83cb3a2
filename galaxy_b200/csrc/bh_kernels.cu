// SPDX-License-Identifier: Apache-2.0
//
// sm_100a kernels of the Barnes-Hut evolution step.  Every kernel covers all
// simulations of a batch in one launch (the plain path is a batch of one):
//
//   k_integrate   kick/drift/final-kick (runtime/src/nbody_evolve.wgsl) fused
//                 with the per-simulation f32 min/max bounds reduction
//   k_morton      f64 root bounds + 16-bit/axis quantization + Morton code
//                 (nbody/src/lib.rs:137-154, nbody/src/flat.rs:67-94), fused
//                 with the four 8-bit digit histograms of the radix sort
//   k_radix_pass  one stable LSD pass (onesweep: decoupled look-back, warp
//                 match ranking, shared-memory staged scatter); the last pass
//                 also gathers the bodies into Morton order
//   k_count_scan  cells per position + exclusive scan (cell numbering in the
//                 reference's recursive preorder, nbody/src/flat.rs:127-177)
//   k_cells       ranges, children, skip pointers of every cell
//   k_aggregate   bottom-up f64 mass / centre of mass, identical arithmetic
//                 and order to nbody/src/flat.rs:179-215
//   k_traverse    lane-parallel theta-MAC walk over node groups with per-warp
//                 interaction lists (nbody/src/flat.rs:270-346 decisions per
//                 body), f32 forces, exact f64 MAC in the guard band
//
// The f64 expressions that must reproduce the reference bit for bit use the
// explicit round-to-nearest intrinsics (__dadd_rn, __dmul_rn, ...), which
// nvcc never contracts into FMAs.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "bh_internal.cuh"

namespace gbh {

namespace {

constexpr unsigned kFull = 0xffffffffu;

#ifndef GBH_PDL
#define GBH_PDL 1
#endif

// Launches a kernel of the step with programmatic stream serialization, so
// its launch overlaps the previous kernel's tail (see wait_for_predecessor).
template <typename... KArgs, typename... Args>
static cudaError_t launch_step(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                               cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = GBH_PDL;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ void set_err(uint32_t* err, uint32_t bits) { atomicOr(err, bits); }

// Programmatic dependent launch: a kernel of the step may be launched while
// its predecessor drains; it waits here, before touching any memory, until
// the predecessor has completed and its writes are visible (a no-op for a
// launch without the attribute).
__device__ __forceinline__ void wait_for_predecessor() {
#if GBH_PDL
    asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}

// Order-preserving float <-> uint mapping (for integer atomics on floats).
__device__ __forceinline__ uint32_t enc_f32(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float dec_f32(uint32_t e) {
    uint32_t u = (e & 0x80000000u) ? (e & 0x7fffffffu) : ~e;
    return __uint_as_float(u);
}

struct RootBounds {
    double cx, cy, half;
};

// nbody/src/lib.rs:137-154 over the f32 min/max promoted to f64.
__device__ __forceinline__ RootBounds root_bounds_from(const uint32_t* mm) {
    double min_x = (double)dec_f32(~mm[0]);
    double min_y = (double)dec_f32(~mm[1]);
    double max_x = (double)dec_f32(mm[2]);
    double max_y = (double)dec_f32(mm[3]);
    double span = fmax(fmax(__dsub_rn(max_x, min_x), __dsub_rn(max_y, min_y)), 1e-12);
    RootBounds r;
    r.cx = __dmul_rn(__dadd_rn(min_x, max_x), 0.5);
    r.cy = __dmul_rn(__dadd_rn(min_y, max_y), 0.5);
    r.half = __dadd_rn(__dmul_rn(span, 0.500000000001), 1e-12);
    return r;
}

// nbody/src/flat.rs:82-87
__device__ __forceinline__ uint32_t quantize_axis(double value, double center, double half) {
    double low = __dsub_rn(center, half);
    double width = __dmul_rn(half, 2.0);
    double scaled = floor(__dmul_rn(__ddiv_rn(__dsub_rn(value, low), width), 65536.0));
    scaled = fmin(fmax(scaled, 0.0), 65535.0);
    return (uint32_t)scaled;
}

// nbody/src/flat.rs:67-80
__device__ __forceinline__ uint32_t spread16(uint32_t v) {
    v &= 0x0000ffffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}
__device__ __forceinline__ uint32_t morton2(uint32_t x, uint32_t y) {
    return spread16(x) | (spread16(y) << 1);
}

// Number of leading quadtree levels (2 bits each) two codes share; 16 when equal.
__device__ __forceinline__ uint32_t shared_levels(uint32_t a, uint32_t b) {
    return a == b ? 16u : ((uint32_t)__clz(a ^ b) >> 1);
}

// 2^-d as an exact double.
__device__ __forceinline__ double pow2_neg(uint32_t d) {
    return __longlong_as_double((long long)(1023 - (int)d) << 52);
}

// First index in [lo, hi) whose code is >= x, given codes[j] < x for j < lo.
// Exponential probe from lo, then binary search: O(log distance).
__device__ __forceinline__ uint32_t gallop_lower_bound(const uint32_t* codes, uint32_t lo,
                                                       uint32_t hi, uint32_t x) {
    uint32_t step = 1;
    uint32_t probe = lo;
    while (probe < hi && codes[probe] < x) {
        lo = probe + 1;
        probe = lo + step;
        step <<= 1;
    }
    uint32_t r = probe < hi ? probe : hi;
    while (lo < r) {
        uint32_t m = lo + ((r - lo) >> 1);
        if (codes[m] < x)
            lo = m + 1;
        else
            r = m;
    }
    return lo;
}

// First index in [lo, hi) whose code is >= x (codes ascending there; hi if
// none), for NT targets at once, by 8-way partition: each round loads seven
// evenly spaced codes per unfinished target — all of them one round trip —
// and keeps the eighth of the range that holds the bound; the last <= 8
// positions are counted with independent loads.  A range of D positions
// takes log8(D) + 1 round trips instead of the ~2 log2(D) dependent loads of
// a binary search, which is what the few cells spanning most of the
// positions (near the root) wait for.
template <int NT>
__device__ __forceinline__ void kary_lower_bound(const uint32_t* codes, uint32_t lo, uint32_t hi,
                                                 const uint32_t (&x)[NT], uint32_t (&out)[NT]) {
    uint32_t l[NT], h[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) {
        l[t] = lo;
        h[t] = hi;
    }
    while (true) {
        bool more = false;
#pragma unroll
        for (int t = 0; t < NT; ++t) more = more || h[t] - l[t] > 8u;
        if (!more) break;
        uint32_t c[NT][7];
#pragma unroll
        for (int t = 0; t < NT; ++t) {
            const uint32_t step = (h[t] - l[t]) / 8u;
#pragma unroll
            for (int j = 0; j < 7; ++j)
                c[t][j] = step ? __ldg(codes + l[t] + step * (uint32_t)(j + 1)) : 0u;
        }
#pragma unroll
        for (int t = 0; t < NT; ++t) {
            const uint32_t step = (h[t] - l[t]) / 8u;
            if (!step) continue;
            uint32_t below = 0;  // probes below x: the probes are ascending
#pragma unroll
            for (int j = 0; j < 7; ++j) below += c[t][j] < x[t] ? 1u : 0u;
            const uint32_t nl = below ? l[t] + step * below + 1u : l[t];
            const uint32_t nh = below < 7u ? l[t] + step * (below + 1u) : h[t];
            l[t] = nl;
            h[t] = nh;
        }
    }
#pragma unroll
    for (int t = 0; t < NT; ++t) {
        uint32_t below = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j)
            below += (l[t] + (uint32_t)j < h[t] && __ldg(codes + l[t] + j) < x[t]) ? 1u : 0u;
        out[t] = l[t] + below;
    }
}

// Exclusive scan over a 256-thread block; *total gets the block sum.
__device__ __forceinline__ uint32_t block_exclusive_scan_256(uint32_t v, uint32_t* total,
                                                             uint32_t* smem8) {
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) smem8[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < 8 ? smem8[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            uint32_t y = __shfl_up_sync(kFull, w, o);
            if (lane >= (uint32_t)o) w += y;
        }
        if (lane < 8) smem8[lane] = w;
    }
    __syncthreads();
    uint32_t wp = warp ? smem8[warp - 1] : 0u;
    *total = smem8[7];
    __syncthreads();
    return wp + x - v;
}

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) {
    return *(const volatile uint32_t*)p;
}
__device__ __forceinline__ unsigned long long ld_volatile64(const unsigned long long* p) {
    return *(const volatile unsigned long long*)p;
}

// Bounded wait budget for look-back spins (~1 s at 2 GHz).
constexpr long long kSpinCycles = 2000000000ll;

}  // namespace

// ============================================================ integrate ====

// runtime/src/nbody_evolve.wgsl:19-46 with explicit f32 roundings (no FMA):
// half_velocity = v + (0.5*dt)*a ; x = x + dt*half_velocity.  Mode 3 runs the
// final kick of one step and the kick-drift of the next with the same two
// roundings as two separate launches.  Modes 0, 1, 3 also reduce the
// per-simulation f32 bounds of the (new) positions.
#ifndef GBH_INTEGRATE_UNROLL
#define GBH_INTEGRATE_UNROLL 4
#endif
// chunks whose loads a warp keeps in flight (modes with the bounds reduction)
constexpr int kIntegrateUnrollBounds = GBH_INTEGRATE_UNROLL;

template <int MODE>
__global__ void __launch_bounds__(256) k_integrate(const SimDesc* __restrict__ sims,
                                                   const uint32_t* __restrict__ chunk_sim,
                                                   uint32_t nchunks, uint32_t* minmax) {
    wait_for_predecessor();
    constexpr bool kBounds = MODE != 2;
    // without the bounds reduction (no atomics) one warp per chunk streams
    // best; with it, fewer blocks each keeping several chunks' loads in flight
    constexpr int kIntegrateUnroll = kBounds ? kIntegrateUnrollBounds : 1;
    __shared__ uint32_t s_sim[8];
    __shared__ float s_val[8][4];
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    // grid-stride over chunks, kIntegrateUnroll strides per round: at any
    // moment the warps of the grid stream one contiguous region
    const uint32_t nwarps = gridDim.x * 8;
    const uint32_t gw = blockIdx.x * 8 + warp;
    uint32_t cur = kNone;
    // fields of simulation `cur`, reloaded only when the simulation changes
    GpuEvolveState* st = nullptr;
    const float4* acc = nullptr;
    uint32_t off = 0, n = 0;
    float dt = 0.f;
    float mnx = INFINITY, mny = INFINITY, mxx = -INFINITY, mxy = -INFINITY;

    auto warp_reduce = [&]() {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mnx = fminf(mnx, __shfl_xor_sync(kFull, mnx, o));
            mny = fminf(mny, __shfl_xor_sync(kFull, mny, o));
            mxx = fmaxf(mxx, __shfl_xor_sync(kFull, mxx, o));
            mxy = fmaxf(mxy, __shfl_xor_sync(kFull, mxy, o));
        }
    };
    // warp-uniform: publishes the bounds of the previous simulation
    auto enter_sim = [&](uint32_t s) {
        if (s == cur) return;
        if (kBounds && cur != kNone) {
            warp_reduce();
            if (lane == 0) {
                atomicMax(&minmax[4 * cur + 0], ~enc_f32(mnx));
                atomicMax(&minmax[4 * cur + 1], ~enc_f32(mny));
                atomicMax(&minmax[4 * cur + 2], enc_f32(mxx));
                atomicMax(&minmax[4 * cur + 3], enc_f32(mxy));
            }
            mnx = mny = INFINITY;
            mxx = mxy = -INFINITY;
        }
        cur = s;
        const SimDesc& sd = sims[s];
        st = sd.state;
        acc = sd.accel;
        off = sd.off;
        n = sd.n;
        dt = sd.dt;
    };
    // the kick / drift of one record, with its bounds
    auto update = [&](float4& pm, float4& v, const float4& a) {
        const float hdt = __fmul_rn(0.5f, dt);
        if (MODE == 2 || MODE == 3) {
            v.x = __fadd_rn(v.x, __fmul_rn(hdt, a.x));
            v.y = __fadd_rn(v.y, __fmul_rn(hdt, a.y));
        }
        if (MODE == 1 || MODE == 3) {
            v.x = __fadd_rn(v.x, __fmul_rn(hdt, a.x));
            v.y = __fadd_rn(v.y, __fmul_rn(hdt, a.y));
            pm.x = __fadd_rn(pm.x, __fmul_rn(dt, v.x));
            pm.y = __fadd_rn(pm.y, __fmul_rn(dt, v.y));
        }
    };
    auto bound = [&](const float4& pm) {
        if (kBounds) {
            mnx = fminf(mnx, pm.x);
            mny = fminf(mny, pm.y);
            mxx = fmaxf(mxx, pm.x);
            mxy = fmaxf(mxy, pm.y);
        }
    };
    auto one_chunk = [&](uint32_t chunk, uint32_t s) {
        if (s == kNone) return;
        enter_sim(s);
        const uint32_t i = chunk * kChunk + lane - off;
        if (i >= n) return;
        float4* rec = reinterpret_cast<float4*>(st + i);
        float4 pm = rec[0];
        if (MODE != 0) {
            float4 v = rec[1];
            update(pm, v, acc[i]);
            if (MODE != 2) rec[0] = pm;
            rec[1] = v;
        }
        bound(pm);
    };

    constexpr uint32_t kPast = kNone - 1u;  // a slot past the last chunk
    for (uint32_t round = gw; round < nchunks; round += kIntegrateUnroll * nwarps) {
        uint32_t sv[kIntegrateUnroll], cv[kIntegrateUnroll];
#pragma unroll
        for (int j = 0; j < kIntegrateUnroll; ++j) {
            cv[j] = round + (uint32_t)j * nwarps;
            sv[j] = cv[j] < nchunks ? chunk_sim[cv[j]] : kPast;
        }
        bool same = sv[0] != kNone;
#pragma unroll
        for (int j = 1; j < kIntegrateUnroll; ++j) same = same && (sv[j] == sv[0] || sv[j] == kPast);
        if (!same) {
#pragma unroll 1
            for (int j = 0; j < kIntegrateUnroll; ++j)
                if (sv[j] != kPast) one_chunk(cv[j], sv[j]);
            continue;
        }
        // one simulation: every load of the run first, then the updates
        enter_sim(sv[0]);
        float4 pm[kIntegrateUnroll], v[kIntegrateUnroll], a[kIntegrateUnroll];
        bool ok[kIntegrateUnroll];
#pragma unroll
        for (int j = 0; j < kIntegrateUnroll; ++j) {
            const uint32_t i = cv[j] * kChunk + lane - off;
            ok[j] = sv[j] != kPast && i < n;
            if (ok[j]) {
                const float4* rec = reinterpret_cast<const float4*>(st + i);
                pm[j] = rec[0];
                if (MODE != 0) {
                    v[j] = rec[1];
                    a[j] = acc[i];
                }
            }
        }
#pragma unroll
        for (int j = 0; j < kIntegrateUnroll; ++j) {
            if (!ok[j]) continue;
            const uint32_t i = cv[j] * kChunk + lane - off;
            if (MODE != 0) {
                update(pm[j], v[j], a[j]);
                float4* rec = reinterpret_cast<float4*>(st + i);
                if (MODE != 2) rec[0] = pm[j];
                rec[1] = v[j];
            }
            bound(pm[j]);
        }
    }
    if (!kBounds) return;
    warp_reduce();
    if (lane == 0) {
        s_sim[warp] = cur;
        s_val[warp][0] = mnx;
        s_val[warp][1] = mny;
        s_val[warp][2] = mxx;
        s_val[warp][3] = mxy;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = kNone;
        float a0 = 0, a1 = 0, a2 = 0, a3 = 0;
        for (int w = 0; w <= 8; ++w) {
            const uint32_t sw = w < 8 ? s_sim[w] : kNone;
            if (w == 8 || sw != run) {
                if (run != kNone) {
                    atomicMax(&minmax[4 * run + 0], ~enc_f32(a0));
                    atomicMax(&minmax[4 * run + 1], ~enc_f32(a1));
                    atomicMax(&minmax[4 * run + 2], enc_f32(a2));
                    atomicMax(&minmax[4 * run + 3], enc_f32(a3));
                }
                if (w == 8) break;
                run = sw;
                a0 = s_val[w][0];
                a1 = s_val[w][1];
                a2 = s_val[w][2];
                a3 = s_val[w][3];
            } else {
                a0 = fminf(a0, s_val[w][0]);
                a1 = fminf(a1, s_val[w][1]);
                a2 = fmaxf(a2, s_val[w][2]);
                a3 = fmaxf(a3, s_val[w][3]);
            }
        }
    }
}

// ============================================================== morton ====

constexpr uint32_t kHistStride = kRadixPasses * kRadixDigits;  // histogram words per sim

// One block per radix tile: Morton codes of the tile's bodies (resident
// order) plus the tile's contribution to the digit histograms of every pass
// of a BITS-wide LSD sort (hist[sim][pass * 2^BITS + digit]).
// Threads per Morton block (one radix tile of kTile keys): 512 hide more of
// the quantization's f64 latency than 256 (and than 1024).
constexpr int kMortonThreads = 512;
constexpr int kMortonItems = (int)kTile / kMortonThreads;
static_assert(kMortonItems * kMortonThreads == (int)kTile, "a Morton block covers one tile");

template <int BITS>
__global__ void __launch_bounds__(kMortonThreads) k_morton(const SimDesc* __restrict__ sims,
                                                         const Tile* __restrict__ tiles,
                                                         const uint32_t* __restrict__ minmax,
                                                         uint32_t* __restrict__ keys,
                                                         uint32_t* hist, SimOut* simout) {
    wait_for_predecessor();
    constexpr int kPasses = 32 / BITS;
    constexpr uint32_t kDig = 1u << BITS;
    __shared__ uint32_t sh[kPasses * kDig];
    for (int k = threadIdx.x; k < kPasses * (int)kDig; k += kMortonThreads) sh[k] = 0;
    __syncthreads();
    const Tile t = tiles[blockIdx.x];
    const SimDesc& sd = sims[t.sim];
    const RootBounds rb = root_bounds_from(minmax + 4 * t.sim);
    if (threadIdx.x == 0 && t.start == sd.off) {
        simout[t.sim].cx = rb.cx;
        simout[t.sim].cy = rb.cy;
        simout[t.sim].half = rb.half;
    }
#pragma unroll
    for (int k = 0; k < kMortonItems; ++k) {
        const uint32_t idx = k * kMortonThreads + threadIdx.x;
        if (idx < t.count) {
            const uint32_t p = t.start + idx;
            const float2 xy = *reinterpret_cast<const float2*>(sd.state + (p - sd.off));
            const uint32_t code = morton2(quantize_axis((double)xy.x, rb.cx, rb.half),
                                          quantize_axis((double)xy.y, rb.cy, rb.half));
            keys[p] = code;
#pragma unroll
            for (int pass = 0; pass < kPasses; ++pass)
                atomicAdd(&sh[pass * kDig + ((code >> (BITS * pass)) & (kDig - 1u))], 1u);
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < kPasses * (int)kDig; k += kMortonThreads) {
        const uint32_t c = sh[k];
        if (c) atomicAdd(&hist[(size_t)t.sim * kHistStride + k], c);
    }
}

// ============================================================== radix =====

#ifndef GBH_LOOK_WINDOW
#define GBH_LOOK_WINDOW 8
#endif
constexpr int kLookWindow = GBH_LOOK_WINDOW;  // predecessor flags loaded per look-back round trip
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagInc = 2u << 30;
constexpr uint32_t kFlagMask = (1u << 30) - 1u;

// Decoupled look-back of tile t for one digit (flags[tile * stride] holds
// that tile's state | count): the sum of the predecessors' counts back to the
// nearest inclusive prefix, reading kLookWindow flags per round trip and
// re-polling from the first tile that has not published yet.  The
// simulation's first tile publishes an inclusive prefix at once, so the
// window never needs tiles before it.  The wait is bounded: once `limit`
// clock cycles have passed since it began and a round finds an unpublished
// predecessor, it sets kErrLookbackTimeout and returns the partial sum, which
// is at most the true prefix (the caller's writes stay in range).
__device__ __forceinline__ uint32_t lookback_digit(const uint32_t* flags, uint32_t stride,
                                                   uint32_t t, uint32_t first_tile,
                                                   uint32_t* err, long long limit) {
    uint32_t excl = 0;
    uint32_t tp = t - 1;
    const long long t0 = clock64();
    while (true) {
        uint32_t f[kLookWindow];
#pragma unroll
        for (int j = 0; j < kLookWindow; ++j)
            f[j] = tp >= first_tile + j ? ld_volatile(flags + (size_t)(tp - j) * stride) : 0u;
        bool done = false;
        int used = 0;
#pragma unroll
        for (int j = 0; j < kLookWindow; ++j) {
            if (done || used < j) continue;
            const uint32_t st = f[j] & ~kFlagMask;
            if (st == 0u) continue;
            excl += f[j] & kFlagMask;
            used = j + 1;
            done = st == kFlagInc;
        }
        if (done) break;
        tp -= used;
        if (used < kLookWindow && clock64() - t0 > limit) {
            set_err(err, kErrLookbackTimeout);
            break;
        }
    }
    return excl;
}

// Failure-detection probe: the sort's look-back wait run as tile 1 of a
// simulation whose first tile never publishes (flags all zero), one thread
// per digit, so every thread must give up after `limit` cycles and report
// the timeout.
__global__ void k_wait_probe(const uint32_t* flags, uint32_t* err, long long limit,
                             uint32_t* out) {
    const uint32_t d = threadIdx.x;
    out[d] = lookback_digit(flags + d, kRadixDigits, 1u, 0u, err, limit);
}

// One stable BITS-wide LSD pass (BITS = 8: 4 passes, 4: 8 passes) over every
// simulation's keys.  Tiles never cross simulations; within a simulation,
// tile order is key order and the decoupled look-back adds the digit counts
// of the preceding tiles.  Items are ranked warp by warp in key order (the
// lanes sharing a digit found with one ballot per digit bit), so equal
// digits keep their input order: the permutation equals a stable sort by
// code, as Rust's sort_by_key (nbody/src/flat.rs:233-234).
// MINB tiles share an SM: 2 (up to 128 registers) for sorts of one wave,
// 3 (80 registers) for sorts of many waves of tiles (large batches).
template <int BITS, int PASS, bool LAST, int MINB>
__global__ void __launch_bounds__(kSortThreads, MINB) k_radix_pass(
    const SimDesc* __restrict__ sims, const Tile* __restrict__ tiles, uint32_t* tile_counter,
    const uint32_t* __restrict__ hist, uint32_t* flags, const uint32_t* __restrict__ keys_in,
    const uint32_t* __restrict__ vals_in, uint32_t* __restrict__ keys_out,
    uint32_t* __restrict__ vals_out, float4* __restrict__ sbody, uint32_t* err) {
    wait_for_predecessor();
    constexpr uint32_t kDig = 1u << BITS;
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_whist[8][kDig];
    __shared__ uint32_t s_tprefix[kDig];
    __shared__ uint32_t s_out[kDig];
    __shared__ uint32_t s_keys[kTile];
    __shared__ uint32_t s_vals[kTile];
    __shared__ uint32_t s_scan[8];

    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    for (int k = threadIdx.x; k < 8 * (int)kDig; k += kSortThreads) (&s_whist[0][0])[k] = 0;
    __syncthreads();
    const uint32_t t = s_tile;
    const Tile tl = tiles[t];
    const SimDesc& sd = sims[tl.sim];
    const uint32_t shift = (uint32_t)BITS * PASS;
    const uint32_t lt_mask = (1u << lane) - 1u;

    uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t idx = warp * (kSortItems * 32u) + r * 32u + lane;
        const bool valid = idx < tl.count;
        const uint32_t p = tl.start + idx;
        key[r] = valid ? keys_in[p] : 0u;
        val[r] = valid ? (PASS == 0 ? p - sd.off : vals_in[p]) : 0u;
    }
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t idx = warp * (kSortItems * 32u) + r * 32u + lane;
        const bool valid = idx < tl.count;
        const uint32_t d = (key[r] >> shift) & (kDig - 1u);
        // valid lanes holding the same digit: one ballot per digit bit
        uint32_t peers = __ballot_sync(kFull, valid);
#pragma unroll
        for (int bit = 0; bit < BITS; ++bit) {
            const uint32_t m = __ballot_sync(kFull, (d >> bit) & 1u);
            peers &= ((d >> bit) & 1u) ? m : ~m;
        }
        const uint32_t leader = __ffs(peers) - 1u;
        uint32_t b = 0;
        if (valid && lane == leader) {
            b = s_whist[warp][d];
            s_whist[warp][d] = b + __popc(peers);
        }
        b = __shfl_sync(kFull, b, leader);
        rank[r] = b + __popc(peers & lt_mask);
        __syncwarp();
    }
    __syncthreads();

    // Thread d < 2^BITS owns digit d: warp offsets, tile count, look-back,
    // bases (the other threads feed zeros to the block scans).
    const uint32_t d = threadIdx.x;
    const bool owner = d < kDig;
    uint32_t run = 0;
    if (owner) {
#pragma unroll
        for (int w = 0; w < 8; ++w) {
            const uint32_t c = s_whist[w][d];
            s_whist[w][d] = run;
            run += c;
        }
    }
    const bool first = (t == sd.first_tile);
    uint32_t* my_flag = flags + (size_t)t * kDig + d;
    if (owner) atomicExch(my_flag, (first ? kFlagInc : kFlagAgg) | run);
    uint32_t excl = 0;
    if (owner && !first) {
        excl = lookback_digit(flags + d, kDig, t, sd.first_tile, err, kSpinCycles);
        atomicExch(my_flag, kFlagInc | (excl + run));
    }
    uint32_t tot;
    const uint32_t h = owner ? hist[(size_t)tl.sim * kHistStride + PASS * kDig + d] : 0u;
    const uint32_t gex = block_exclusive_scan_256(h, &tot, s_scan);
    const uint32_t tex = block_exclusive_scan_256(run, &tot, s_scan);
    if (owner) {
        s_tprefix[d] = tex;
        s_out[d] = sd.off + gex + excl - tex;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t idx = warp * (kSortItems * 32u) + r * 32u + lane;
        if (idx < tl.count) {
            const uint32_t dg = (key[r] >> shift) & (kDig - 1u);
            const uint32_t slot = s_tprefix[dg] + s_whist[warp][dg] + rank[r];
            s_keys[slot] = key[r];
            s_vals[slot] = val[r];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const uint32_t slot = k * kSortThreads + threadIdx.x;
        if (slot < tl.count) {
            const uint32_t kk = s_keys[slot];
            const uint32_t vv = s_vals[slot];
            const uint32_t dest = s_out[(kk >> shift) & (kDig - 1u)] + slot;
            keys_out[dest] = kk;
            vals_out[dest] = vv;
            if (LAST) {
                const float4 pm = *reinterpret_cast<const float4*>(sd.state + vv);
                sbody[dest] = make_float4(pm.x, pm.y, pm.z, __uint_as_float(vv));
            }
        }
    }
}

// ========================================================== count + scan ==

// Cells whose range starts at sorted position i (a "chain": depths
// d_min..D).  Cell (d, i) exists iff i starts a depth-d group and its parent
// group holds more than `bucket` bodies; it is internal iff it holds more
// than `bucket` bodies and d < max_depth (nbody/src/flat.rs:145).
__device__ __forceinline__ uint32_t chain_count(const uint32_t* __restrict__ sc, uint32_t i,
                                                uint32_t n, uint32_t bucket, uint32_t maxd,
                                                uint32_t* dmin_out) {
    const uint32_t ci = sc[i];
    const uint32_t dmin = i == 0 ? 0u : shared_levels(sc[i - 1], ci) + 1u;
    *dmin_out = dmin;
    if (dmin > maxd) return 0;
    if (i > 0 && bucket > 1) {
        // parent group (depth dmin-1) holds i-1 and i; needs > bucket bodies:
        // some window [j, j+bucket] containing both lies inside it.
        const uint32_t pd = dmin - 1u;
        const uint32_t jlo = i >= bucket ? i - bucket : 0u;
        bool ok = false;
        for (uint32_t j = jlo; j < i && j + bucket < n; ++j) {
            if (shared_levels(sc[j], sc[j + bucket]) >= pd) {
                ok = true;
                break;
            }
        }
        if (!ok) return 0;
    }
    const int lw = (i + bucket < n) ? (int)shared_levels(ci, sc[i + bucket]) : -1;
    const int deepest = max((int)dmin, min((int)maxd, lw + 1));
    return (uint32_t)(deepest - (int)dmin + 1);
}

constexpr unsigned long long kScanAgg = 1ull << 62;
constexpr unsigned long long kScanInc = 2ull << 62;
constexpr unsigned long long kScanMask = (1ull << 62) - 1ull;

__global__ void __launch_bounds__(kScanThreads) k_count_scan(
    const SimDesc* __restrict__ sims, const uint32_t* __restrict__ chunk_sim, uint32_t npos,
    const uint32_t* __restrict__ codes, uint32_t* __restrict__ base, uint32_t* tile_counter,
    unsigned long long* flags, uint32_t* err) {
    wait_for_predecessor();
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_scan[8];
    __shared__ unsigned long long s_excl;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint32_t t = s_tile;
    const uint32_t p0 = t * kScanTile + threadIdx.x * kScanItems;
    uint32_t cnt[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t p = p0 + k;
        uint32_t c = 0;
        if (p < npos) {
            const uint32_t s = chunk_sim[p >> 5];
            if (s != kNone) {
                const SimDesc& sd = sims[s];
                const uint32_t i = p - sd.off;
                if (i < sd.n) {
                    uint32_t dmin;
                    c = chain_count(codes + sd.off, i, sd.n, sd.bucket, sd.max_depth, &dmin);
                }
            }
        }
        cnt[k] = c;
        sum += c;
    }
    uint32_t tile_total;
    const uint32_t texcl = block_exclusive_scan_256(sum, &tile_total, s_scan);
    if (threadIdx.x < 32u) {
        // decoupled look-back by one warp: lane j reads tile tp - j, so a
        // round covers 32 predecessors; a round counts once every tile up to
        // the nearest inclusive prefix has published (tiles before 0 read as
        // inclusive 0), otherwise it polls again (bounded)
        const uint32_t lane = threadIdx.x;
        unsigned long long excl = 0;
        if (t == 0) {
            if (lane == 0) atomicExch(&flags[0], kScanInc | (unsigned long long)tile_total);
        } else {
            if (lane == 0) atomicExch(&flags[t], kScanAgg | (unsigned long long)tile_total);
            long long tp = (long long)t - 1;
            const long long c0 = clock64();
            while (true) {
                const long long idx = tp - (long long)lane;
                const unsigned long long f = idx >= 0 ? ld_volatile64(&flags[idx]) : kScanInc;
                const unsigned long long st = f & ~kScanMask;
                const uint32_t inc = __ballot_sync(kFull, st == kScanInc);
                const uint32_t pub = __ballot_sync(kFull, st != 0ull);
                const uint32_t upto = inc ? (inc & (0u - inc)) * 2u - 1u : 0xffffffffu;
                if ((pub & upto) == upto) {
                    unsigned long long v = ((upto >> lane) & 1u) ? (f & kScanMask) : 0ull;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
                    excl += v;
                    if (inc) break;
                    tp -= 32;
                } else if (__any_sync(kFull, clock64() - c0 > kSpinCycles)) {
                    if (lane == 0) set_err(err, kErrLookbackTimeout);
                    break;  // the whole warp: the vote is uniform
                }
            }
            if (lane == 0) atomicExch(&flags[t], kScanInc | (excl + tile_total));
        }
        if (lane == 0) s_excl = excl;
    }
    __syncthreads();
    uint32_t run = (uint32_t)s_excl + texcl;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t p = p0 + k;
        if (p <= npos) base[p] = run;
        run += cnt[k];
    }
}

// =============================================================== cells ====

// One thread per cell.  A block covers 256 positions, whose cells are the
// contiguous preorder range [base[P0], base[P0 + 256]); the codes and chain
// bases of the next kCellsWin positions sit in shared memory, so the range
// searches of almost every cell (all but the few that span more than the
// window) never touch global memory.
// Positions per k_aggregate block: cells whose range crosses a multiple of it
// are finished by cross-block climbs (the only users of the cell counters).
#ifndef GBH_AGG_POSITIONS
#define GBH_AGG_POSITIONS 256
#endif
constexpr uint32_t kAggBlockPositions = GBH_AGG_POSITIONS;
#ifndef GBH_CELLS_THREADS
#define GBH_CELLS_THREADS 256
#endif
constexpr uint32_t kCellsThreads = GBH_CELLS_THREADS;  // positions (and threads) per block
// 512 positions: wider windows load more than their searches save (1024 and
// 2048 measured slower at 2^20 and 2^24)
#ifndef GBH_CELLS_WIN
#define GBH_CELLS_WIN 512
#endif
constexpr uint32_t kCellsWin = GBH_CELLS_WIN;
constexpr uint32_t kMaxChain = kMortonDepth + 1;  // cells per position: depths 0..16

#ifndef GBH_CELLS_KARY
#define GBH_CELLS_KARY 1
#endif

struct CellsWindow {
    const uint32_t* s_code;  // codes of positions [w0, w0 + kCellsWin)
    const uint32_t* s_base;  // base of positions [w0, w0 + kCellsWin]
    const uint32_t* codes;
    const uint32_t* base;
    uint32_t w0;

    __device__ __forceinline__ uint32_t base_at(uint32_t gp) const {
        const uint32_t j = gp - w0;
        return j <= kCellsWin ? s_base[j] : base[gp];
    }
    // First position in [lo, hi) whose code is >= x, given codes < x before lo
    // (w0 <= lo).
    __device__ __forceinline__ uint32_t lower_bound(uint32_t lo, uint32_t hi, uint32_t x) const {
        const uint32_t wend = min(hi, w0 + kCellsWin);
        if (lo < wend) {
            if (s_code[wend - 1u - w0] >= x)
                return w0 + gallop_lower_bound(s_code, lo - w0, wend - w0, x);
            lo = wend;
        }
#if GBH_CELLS_KARY
        if (lo >= hi) return hi;
        const uint32_t xs[1] = {x};
        uint32_t r[1];
        kary_lower_bound<1>(codes, lo, hi, xs, r);
        return r[0];
#else
        return lo < hi ? gallop_lower_bound(codes, lo, hi, x) : hi;
#endif
    }
    // The three quadrant bounds of a cell's range [lo, hi): out[q] = first
    // position whose code is >= x[q] (x ascending), the window first, the
    // searches past it together.
    __device__ __forceinline__ void lower_bound3(uint32_t lo, uint32_t hi, const uint32_t (&x)[3],
                                                 uint32_t (&out)[3]) const {
#if GBH_CELLS_KARY
        const uint32_t wend = min(hi, w0 + kCellsWin);
        bool far = false;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            if (lo < wend && s_code[wend - 1u - w0] >= x[q]) {
                out[q] = w0 + gallop_lower_bound(s_code, lo - w0, wend - w0, x[q]);
            } else {
                out[q] = kNone;
                far = true;
            }
        }
        if (far) {
            const uint32_t flo = max(lo, wend);
            uint32_t r[3];
            if (flo < hi) {
                kary_lower_bound<3>(codes, flo, hi, x, r);
            } else {
                r[0] = r[1] = r[2] = hi;
            }
#pragma unroll
            for (int q = 0; q < 3; ++q)
                if (out[q] == kNone) out[q] = r[q];
        }
#else
        uint32_t l = lo;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            l = lower_bound(l, hi, x[q]);
            out[q] = l;
        }
#endif
    }
};

// six blocks per SM (40 registers): the k-ary searches spill a little in
// the few threads that run them instead of halving every block's occupancy
#ifndef GBH_CELLS_MIN_BLOCKS
#define GBH_CELLS_MIN_BLOCKS 6
#endif
__global__ void __launch_bounds__(kCellsThreads, GBH_CELLS_MIN_BLOCKS) k_cells(const SimDesc* __restrict__ sims,
                                                         const uint32_t* __restrict__ chunk_sim,
                                                         uint32_t npos, uint32_t capacity,
                                                         const uint32_t* __restrict__ codes,
                                                         const uint32_t* __restrict__ base,
                                                         uint4* cell_u,
                                                         uint4* cell_child, uint32_t* cell_parent,
                                                         uint32_t* cell_counter, CellRec* groups,
                                                         uint32_t* err) {
    wait_for_predecessor();
    __shared__ uint32_t s_code[kCellsWin];
    __shared__ uint32_t s_base[kCellsWin + 1];
    __shared__ uint8_t s_owner[kCellsThreads * kMaxChain];  // cell -> position in block
    __shared__ uint16_t s_end[kCellsThreads * kMaxChain];   // cell -> min(end - P0, 0xffff)
    const uint32_t t = threadIdx.x;
    const uint32_t P0 = blockIdx.x * kCellsThreads;
    for (uint32_t j = t; j <= kCellsWin; j += kCellsThreads) {
        const uint32_t gp = P0 + j;
        if (j < kCellsWin) s_code[j] = gp < npos ? codes[gp] : 0xffffffffu;
        s_base[j] = gp <= npos ? base[gp] : 0u;
    }
    __syncthreads();
    const uint32_t P1 = min(P0 + kCellsThreads, npos);
    const uint32_t kb = s_base[0], ke = s_base[P1 - P0];
    if (ke > capacity || ke - kb > kCellsThreads * kMaxChain) {
        if (t == 0) set_err(err, kErrCapacity);
        return;
    }
    if (P0 + t < P1) {
        const uint32_t c0 = s_base[t] - kb, c = s_base[t + 1] - s_base[t];
        for (uint32_t j = 0; j < c; ++j) s_owner[c0 + j] = (uint8_t)t;
    }
    __syncthreads();
    const CellsWindow w{s_code, s_base, codes, base, P0};
    const uint4 absent = make_uint4(0u, 0u, 0u, kNone);  // u.z == 0: no child in this slot
    // Position, depth and deepest chain depth of cell k of this block.
    auto locate = [&](uint32_t k, uint32_t* p, uint32_t* d, uint32_t* deepest) {
        const uint32_t tl = s_owner[k - kb];
        *p = P0 + tl;
        const SimDesc& sd = sims[chunk_sim[*p >> 5]];
        const uint32_t ci = s_code[tl];
        const uint32_t dmin = *p == sd.off
                                  ? 0u
                                  : shared_levels(tl ? s_code[tl - 1u] : codes[*p - 1u], ci) + 1u;
        const uint32_t k0 = s_base[tl];
        *deepest = dmin + (s_base[tl + 1] - k0) - 1u;
        *d = dmin + (k - k0);
    };
    // Pass 1: every cell's range end (one search each).
    for (uint32_t k = kb + t; k < ke; k += kCellsThreads) {
        uint32_t p, d, deepest;
        locate(k, &p, &d, &deepest);
        const uint32_t s = chunk_sim[p >> 5];
        const SimDesc& sd = sims[s];
        const uint32_t hi = sd.off + sd.n;
        const uint32_t ci = s_code[p - P0];
        // end of the depth-d group holding p
        uint32_t end = hi;
        if (d > 0) {
            const uint32_t sh = 32u - 2u * d;
            const unsigned long long next = ((unsigned long long)(ci >> sh) + 1ull) << sh;
            if (next <= 0xffffffffull) end = w.lower_bound(p + 1u, hi, (uint32_t)next);
        } else {
            cell_parent[k] = kNone;
            // the simulation's root group holds the root in slot 0 only
            CellRec* rg = groups + 4ull * (capacity + s);
            rg[1].u = absent;
            rg[2].u = absent;
            rg[3].u = absent;
        }
        cell_u[k] = make_uint4(end, w.base_at(end), p, d);
        // counters serve only cells that span aggregate blocks (cross-block climbs)
        if ((p / kAggBlockPositions) != ((end - 1u) / kAggBlockPositions)) cell_counter[k] = 0;
        s_end[k - kb] = (uint16_t)min(end - P0, 0xffffu);
    }
    __syncthreads();
    // Pass 2: children.  Children of (p, d) are the depth-(d+1) groups of its
    // range in position order (= quadrant order): (p, d+1) first, then the
    // chain head at each child's end.  While those ends lie in this block
    // they come from pass 1; otherwise the quadrant bounds are searched.
    for (uint32_t k = kb + t; k < ke; k += kCellsThreads) {
        uint32_t p, d, deepest;
        locate(k, &p, &d, &deepest);
        uint4 ch = make_uint4(kNone, kNone, kNone, kNone);
        uint32_t* chp = &ch.x;
        if (d < deepest) {
            const uint32_t end = cell_u[k].x;
            const uint32_t sh = 30u - 2u * d;
            uint32_t q = p, child = k + 1u;
            bool searched = false;
            while (true) {
                chp[(s_code[q - P0] >> sh) & 3u] = child;
                const uint32_t e = s_end[child - kb];
                if (P0 + e >= end) break;        // the last child
                if (e >= P1 - P0) {              // next child starts past this block
                    searched = true;
                    break;
                }
                q = P0 + e;
                child = s_base[e];               // chain head of position q
            }
            if (searched) {
                const uint32_t pre = d == 0 ? 0u : (s_code[p - P0] >> (32u - 2u * d));
                const uint32_t xs[3] = {((pre << 2) | 1u) << sh, ((pre << 2) | 2u) << sh,
                                        ((pre << 2) | 3u) << sh};
                uint32_t qb[3];
                w.lower_bound3(p, end, xs, qb);
                uint32_t bounds[5];
                bounds[0] = p;
                bounds[1] = qb[0];
                bounds[2] = qb[1];
                bounds[3] = qb[2];
                bounds[4] = end;
#pragma unroll
                for (uint32_t qd = 0; qd < 4; ++qd)
                    chp[qd] = bounds[qd] < bounds[qd + 1]
                                  ? (bounds[qd] == p ? k + 1u : w.base_at(bounds[qd]))
                                  : kNone;
            }
#pragma unroll
            for (uint32_t qd = 0; qd < 4; ++qd) {
                const uint32_t child = chp[qd];
                if (child == kNone) {
                    groups[4ull * k + qd].u = absent;
                } else if (child < capacity) {
                    cell_parent[child] = k;
                } else {
                    set_err(err, kErrCapacity);
                }
            }
        }
        cell_child[k] = ch;
    }
}

// =========================================================== aggregate ====

// Guard band of the f32 opening test.  The exact test (flat.rs:317-323) opens
// a cell unless width/dist < theta, i.e. approximates iff dist^2 > crit^2 with
// crit = width/theta.  The traversal computes d2 in f32 from the f32 centre of
// mass; with u = 2^-24 and C = |com_x| + |com_y| its error is at most
// 2u*C*d + 4u*d^2, and d <= (d^2 + crit^2)/(2 crit) turns that into a bound
// linear in d^2: |d2_f32 - d^2| <= d^2 * r + u*C*crit, r = u*C/crit + 4u.
// So d2_f32 > hi proves "approximate" and d2_f32 < lo proves "open" (with a
// 4x margin and 1e-4 relative slack); in between the traversal decides in f64.
__device__ __forceinline__ void mac_band(double width, double theta, float com_x, float com_y,
                                         float* lo, float* hi) {
    if (!(theta > 0.0)) {  // theta = 0: every cell opens
        *lo = INFINITY;
        *hi = INFINITY;
        return;
    }
    const double crit = width / theta;
    const double crit2 = crit * crit;
    if (!(crit2 < 1e38)) {  // beyond any f32 distance: always open
        *lo = INFINITY;
        *hi = INFINITY;
        return;
    }
    const double u = 5.9604644775390625e-8;
    const double C = fabs((double)com_x) + fabs((double)com_y);
    const double r = u * C / crit + 4.0 * u;
    const double slack = 4.0 * r + 1e-4;
    *hi = __double2float_ru(crit2 * (1.0 + slack) + 4.0 * u * C * crit);
    *lo = __double2float_rd(crit2 * (1.0 - slack) - 4.0 * u * C * crit);
}

// hi with the depth in its low 5 bits, rounded away from zero to make room:
// a larger positive bound (or a more negative -1) only widens the band, and
// +inf becomes a NaN, for which "d2 > hi" stays false.
__device__ __forceinline__ float pack_depth(float hi, uint32_t depth) {
    return __uint_as_float(((__float_as_uint(hi) + 32u) & ~31u) | depth);
}

// Writes the MAC fields of record k: internal cells get (hi|depth, lo); a
// leaf (count >= 1 bodies) is always summed directly: one body -> hi = -1 (it
// passes as a point mass at its own position, which is its f32 centre of
// mass exactly) and u.x = 1; several bodies -> hi = +inf (no point-mass
// term) and u.x = count, summed body by body.
// Where a cell sits for the traversal: slot `quadrant` of its parent's node
// group, or slot 0 of its simulation's root group (index capacity + sim).
struct SlotRef {
    uint32_t parent;      // kNone for a root
    uint32_t quadrant;
    uint32_t root_group;  // capacity + sim
};

__device__ __forceinline__ CellRec* slot_of(CellRec* groups, const SlotRef& r) {
    return groups + (r.parent == kNone ? 4ull * r.root_group : 4ull * r.parent + r.quadrant);
}

// Writes the MAC fields of cell k into its slot of the parent's node group
// (the traversal's record of the cell): internal cells get (hi|depth, lo); a leaf
// (count >= 1 bodies) is always summed directly: one body -> hi = -1 (it
// passes as a point mass at its own position, which is its f32 centre of
// mass exactly); several bodies -> hi = +inf (no point-mass term), summed
// body by body.  The slot's u = (lo | body count, start, body count, k or
// kNone for a leaf).
__device__ __forceinline__ void store_mac_fields(CellRec* groups, uint32_t k,
                                                 float fx, float fy, float gm, uint32_t depth,
                                                 uint32_t start, uint32_t count, bool leaf,
                                                 const SlotRef& slot, double root_half,
                                                 double theta) {
    float lo = 0.f, hi;
    uint32_t ux;
    if (leaf) {
        hi = count == 1u ? -1.0f : INFINITY;
        ux = count;
    } else {
        const double width = __dmul_rn(__dmul_rn(root_half, pow2_neg(depth)), 2.0);
        mac_band(width, theta, fx, fy, &lo, &hi);
        ux = __float_as_uint(lo);
    }
    const float4 f = make_float4(fx, fy, gm, pack_depth(hi, depth));
    CellRec* sl = slot_of(groups, slot);
    sl->f = f;
    sl->u = make_uint4(ux, start, count, leaf ? kNone : k);
}

// Writes a cell's f64 aggregates (centre of mass = weighted sums / mass, as
// flat.rs:193-212) and its traversal records.
__device__ __forceinline__ void store_cell_values(uint32_t k, double mass, double wx, double wy,
                                                  uint32_t depth, uint32_t start, uint32_t count,
                                                  bool leaf, const SlotRef& slot,
                                                  double root_half, double theta, float g,
                                                  double4* cell_d, CellRec* groups) {
    const double com_x = __ddiv_rn(wx, mass);
    const double com_y = __ddiv_rn(wy, mass);
    const float hx = (float)com_x, hy = (float)com_y;
    // the f32 residuals com - (float)com ride in the record's spare word: the
    // compensated traversal adds them back to its differences
    const float lo_x = (float)(com_x - (double)hx), lo_y = (float)(com_y - (double)hy);
    const unsigned long long lo_bits =
        ((unsigned long long)__float_as_uint(lo_y) << 32) | __float_as_uint(lo_x);
    cell_d[k] = make_double4(com_x, com_y, mass, __longlong_as_double((long long)lo_bits));
    store_mac_fields(groups, k, hx, hy, __fmul_rn(g, (float)mass),
                     depth, start, count, leaf, slot, root_half, theta);
}

// Slot of cell k given its parent: the quadrant is the 2-bit digit of the
// cell's codes at the parent's depth.
__device__ __forceinline__ SlotRef slot_ref(uint32_t parent, uint32_t depth, uint32_t start_code,
                                            uint32_t root_group) {
    SlotRef r;
    r.parent = parent;
    r.quadrant = depth ? (start_code >> (32u - 2u * depth)) & 3u : 0u;
    r.root_group = root_group;
    return r;
}

// Acquire-release fetch-add at GPU scope: the writes before it (this
// thread's cell values) are visible to whichever thread reads the counter's
// final value, and this thread sees the writes released before the
// increments it reads.
__device__ __forceinline__ uint32_t atomic_add_acq_rel(uint32_t* p, uint32_t v) {
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;"
                 : "=r"(old)
                 : "l"(p), "r"(v)
                 : "memory");
    return old;
}

struct AggArgs {
    const SimDesc* sims;
    const SimOut* simout;
    const uint32_t* chunk_sim;
    const float4* sbody;
    const uint32_t* codes;
    uint32_t capacity;
    const uint4* cell_u;
    const uint4* cell_child;
    const uint32_t* cell_parent;
    uint32_t* cell_counter;
    double4* cell_d;
    CellRec* groups;
};

// Aggregates of cell k (u = its links (end, skip, start, depth)): a leaf
// sums its bodies in Morton order, an internal cell its children in quadrant
// order 0..3 (nbody/src/flat.rs:179-215).
__device__ __forceinline__ void aggregate_cell(const AggArgs& a, uint32_t k, uint4 u, bool leaf) {
    const uint32_t start = u.z, depth = u.w, end = u.x;
    const uint32_t s = a.chunk_sim[start >> 5];
    const SimDesc& sd = a.sims[s];
    double mass = 0.0, wx = 0.0, wy = 0.0;
    if (leaf) {
        for (uint32_t q = start; q < end; ++q) {
            const float4 b = a.sbody[q];
            const double m = (double)b.z;
            mass = __dadd_rn(mass, m);
            wx = __dadd_rn(wx, __dmul_rn(m, (double)b.x));
            wy = __dadd_rn(wy, __dmul_rn(m, (double)b.y));
        }
    } else {
        const uint4 ch = a.cell_child[k];
        const uint32_t chv[4] = {ch.x, ch.y, ch.z, ch.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (chv[q] == kNone) continue;
            const double2 cxy = __ldcg(reinterpret_cast<const double2*>(a.cell_d + chv[q]));
            const double cm = __ldcg(reinterpret_cast<const double*>(a.cell_d + chv[q]) + 2);
            mass = __dadd_rn(mass, cm);
            wx = __dadd_rn(wx, __dmul_rn(cm, cxy.x));
            wy = __dadd_rn(wy, __dmul_rn(cm, cxy.y));
        }
    }
    store_cell_values(k, mass, wx, wy, depth, start, end - start, leaf,
                      slot_ref(a.cell_parent[k], depth, a.codes[start], a.capacity + s),
                      a.simout[s].half, sd.theta, sd.g_f, a.cell_d, a.groups);
}

// Cell k is done and its parent spans several blocks: count k in at the
// parent; the thread that completes a parent's last child computes the
// parent and carries on upwards.
__device__ void climb(const AggArgs& a, uint32_t k) {
    while (true) {
        const uint32_t par = a.cell_parent[k];
        if (par == kNone) return;
        const uint4 ch = a.cell_child[par];
        const uint32_t nchild =
            (ch.x != kNone) + (ch.y != kNone) + (ch.z != kNone) + (ch.w != kNone);
        if (atomic_add_acq_rel(a.cell_counter + par, 1u) + 1u != nchild) return;
        aggregate_cell(a, par, a.cell_u[par], false);
        k = par;
    }
}

// Bottom-up f64 aggregates.  A block covers the cells of 256 positions
// [P0, P1), the preorder range [kb, ke).  A cell whose positions lie inside
// [P0, P1) is local: the block computes every leaf first, then its local
// internal cells depth by depth, deepest first, with a block barrier between
// depths, so no local cell needs an atomic.  The other cells span several
// blocks (ancestors of block boundaries, about 1% of the internal cells);
// each is computed by the thread that completes its last child, found with
// one acquire-release counter per cell.  Same arithmetic and order as the
// reference, so the f64 mass and centre of mass equal its values bit for bit.
// 64 threads per 256 positions: a depth holds few cells, and small blocks
// let many blocks hide each other's per-depth latency.
constexpr uint32_t kAggPositions = kAggBlockPositions;
#ifndef GBH_AGG_THREADS
#define GBH_AGG_THREADS 64
#endif
constexpr uint32_t kAggThreads = GBH_AGG_THREADS;

__global__ void __launch_bounds__(kAggThreads) k_aggregate(const AggArgs a, uint32_t npos,
                                                           const uint32_t* __restrict__ base,
                                                           uint32_t* err) {
    wait_for_predecessor();
    // local internal cells by depth (offsets from kb), internal depths
    // 0..15: those of one depth hold disjoint ranges of at least two
    // positions, so at most half the block's positions per depth
    __shared__ uint16_t s_level[kMortonDepth][kAggPositions / 2];
    __shared__ uint32_t s_count[kMortonDepth];
    __shared__ uint32_t s_code[kAggPositions + 2];  // codes of positions P0-1 .. P0+256
    const uint32_t t = threadIdx.x;
    const uint32_t P0 = blockIdx.x * kAggPositions;
    const uint32_t P1 = min(P0 + kAggPositions, npos);
    if (t < kMortonDepth) s_count[t] = 0;
    for (uint32_t j = t; j < kAggPositions + 2; j += kAggThreads) {
        const uint32_t gp = P0 + j - 1u;
        s_code[j] = (j > 0 || P0 > 0) && gp < npos ? a.codes[gp] : 0u;
    }
    __syncthreads();
    const uint32_t kb = base[P0], ke = base[P1];
    // whether the depth-dd group holding position p lies inside [P0, P1):
    // its neighbours outside the block (within the simulation) differ in
    // the first dd levels
    auto inside = [&](uint32_t p, uint32_t dd, const SimDesc& sd) {
        const uint32_t c = s_code[p - P0 + 1u];
        const bool left = sd.off >= P0 || shared_levels(s_code[0], c) < dd;
        const bool right = sd.off + sd.n <= P1 || shared_levels(c, s_code[P1 - P0 + 1u]) < dd;
        return left && right;
    };
    // the next cell's links are loaded while this one is summed
    uint4 u_next = kb + t < ke ? a.cell_u[kb + t] : make_uint4(0u, 0u, 0u, 0u);
    for (uint32_t k = kb + t; k < ke; k += kAggThreads) {
        const uint4 u = u_next;  // (end, skip, start, depth)
        if (k + kAggThreads < ke) u_next = a.cell_u[k + kAggThreads];
        const SimDesc& sd = a.sims[a.chunk_sim[u.z >> 5]];
        if (u.y == k + 1u) {
            aggregate_cell(a, k, u, true);
            if (u.w > 0 && !inside(u.z, u.w - 1u, sd)) climb(a, k);
        } else if (inside(u.z, u.w, sd)) {
            const uint32_t slot = u.w < kMortonDepth ? atomicAdd(&s_count[u.w], 1u) : kNone;
            if (slot < kAggPositions / 2)
                s_level[u.w][slot] = (uint16_t)(k - kb);
            else
                set_err(err, kErrCapacity);
        }
    }
    __syncthreads();
    for (int d = (int)kMortonDepth - 1; d >= 0; --d) {
        const uint32_t cnt = min(s_count[d], kAggPositions / 2);
        if (cnt == 0) continue;
        for (uint32_t j = t; j < cnt; j += kAggThreads) {
            const uint32_t k = kb + s_level[d][j];
            const uint4 u = a.cell_u[k];
            aggregate_cell(a, k, u, false);
            if (d > 0 && !inside(u.z, (uint32_t)d - 1u, a.sims[a.chunk_sim[u.z >> 5]])) climb(a, k);
        }
        __syncthreads();
    }
}

// Recomputes G*m and the MAC band of every cell of one simulation from the
// f64 aggregates, for a force pass whose theta or G differs from the rebuild's.
__global__ void k_refresh_mac(const SimDesc* __restrict__ sims, const SimOut* __restrict__ simout,
                              uint32_t sim, const uint32_t* __restrict__ base,
                              const uint32_t* __restrict__ codes, uint32_t capacity,
                              const uint32_t* __restrict__ cell_parent,
                              const double4* __restrict__ cell_d,
                              const uint4* __restrict__ cell_u, CellRec* groups) {
    const SimDesc& sd = sims[sim];
    const uint32_t cb = base[sd.off], ce = base[sd.off + sd.n];
    const uint32_t k = cb + blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ce) return;
    const uint4 u = cell_u[k];
    const double4 v = cell_d[k];
    const bool leaf = u.y == k + 1u;
    const uint32_t start = u.z;
    store_mac_fields(groups, k, (float)v.x, (float)v.y, __fmul_rn(sd.g_f, (float)v.z), u.w, start,
                     u.x - start, leaf,
                     slot_ref(cell_parent[k], u.w, codes[start], capacity + sim),
                     simout[sim].half, sd.theta);
}

// ============================================================ traverse ====

// Paired f32 arithmetic (sm_100 FADD2 / FFMA2 / FMUL2) for the compensated
// form: both axes of a term in one instruction, each axis rounded exactly as
// its scalar operation; a - b is fma(b, -1, a) (exact negation, one
// rounding).  The plain form keeps scalar operations (paired ones measured
// slower there: 0.667 against 0.592 ms at N = 2^20).
template <bool PAIRED>
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    if (PAIRED) return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
    return make_float2(a.x - b.x, a.y - b.y);
}

template <bool COMP>
struct Acc {
    float2 v = make_float2(0.f, 0.f);  // the sum (x, y)
    float2 c = make_float2(0.f, 0.f);  // compensated form: the two-sum error terms
    // adds the term d * scale: the plain form with one fused multiply-add per
    // axis, the compensated form with the rounded product and Knuth's two-sum
    // (s + e == v + t exactly)
    __device__ __forceinline__ void add_scaled(float2 d, float scale) {
        if (COMP) {
            const float2 t = __fmul2_rn(d, make_float2(scale, scale));
            const float2 s = __fadd2_rn(v, t);
            const float2 bb = sub2<true>(s, v);
            c = __fadd2_rn(c, __fadd2_rn(sub2<true>(v, sub2<true>(s, bb)), sub2<true>(t, bb)));
            v = s;
        } else {
            v.x += d.x * scale;
            v.y += d.y * scale;
        }
    }
    __device__ __forceinline__ float fx() const { return COMP ? v.x + c.x : v.x; }
    __device__ __forceinline__ float fy() const { return COMP ? v.y + c.y : v.y; }
};

// Lane-parallel traversal with interaction lists.  A warp owns 32
// consecutive Morton positions (its lanes).  Every lane keeps exactly its
// own opening decisions of nbody/src/flat.rs:270-346, but the walk itself is
// spread over the lanes: the warp pops up to 8 (node group, lane mask)
// entries from a per-warp stack in shared memory, and lane 4i+q examines
// slot q of popped entry i for all lanes of its mask at once, against the
// bounding box of the warp's bodies:
//   * the box's nearest point has d2 > hi: every lane of the mask
//     approximates the cell (a lane whose own body the cell holds opens it);
//   * the box's farthest corner has d2 < lo: every lane of the mask opens it;
//   * otherwise the cell is mixed and the warp decides it lane by lane, as
//     a single lane would (f64 test inside the guard band).
// d2 is fma(dx, dx, dy*dy) in f32 with round-to-nearest, monotone in |dx|
// and |dy|, and each lane's |dx|, |dy| lie between the box's nearest and
// farthest distances, so a box decision is every lane's own decision.
// Approximated cells and one-body leaves go to a per-warp interaction list
// (centre of mass, G*m, mask of the lanes that take the term), which all
// lanes sum with one branch-free masked term per entry; mixed cells add
// their term directly and leaves of several bodies are summed body by body,
// self excluded.  Only the order of a lane's terms differs from the
// reference's depth-first order.

// Exact f64 opening test of flat.rs:317-323 for a lane inside the guard
// band; true = approximate.
__device__ __noinline__ bool exact_mac(const double4* __restrict__ cell_d, uint32_t c, float tx,
                                       float ty, double root_half, uint32_t depth,
                                       double theta) {
    const double2 com = *reinterpret_cast<const double2*>(cell_d + c);
    const double ddx = __dsub_rn(com.x, (double)tx);
    const double ddy = __dsub_rn(com.y, (double)ty);
    const double dist = hypot(ddx, ddy);
    const double width = __dmul_rn(__dmul_rn(root_half, pow2_neg(depth)), 2.0);
    return dist > 0.0 && __ddiv_rn(width, dist) < theta;
}

// Squared distance as the traversal computes it everywhere (monotone in |dx|
// and |dy|; its rounding is covered by the guard band of mac_band).
__device__ __forceinline__ float dist2(float dx, float dy) {
    return __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
}

// Lane mask of bits [a, b), 0 <= a <= b <= 32.
__device__ __forceinline__ uint32_t bit_range(uint32_t a, uint32_t b) {
    const uint32_t w = b - a;
    return w >= 32u ? 0xffffffffu : (((1u << w) - 1u) << a);
}

#ifndef GBH_TRAVERSE_WARPS
#define GBH_TRAVERSE_WARPS 8
#endif
#ifndef GBH_TRAVERSE_MIN_BLOCKS
#define GBH_TRAVERSE_MIN_BLOCKS 4  // 64 registers: 32 warps per SM
#endif
constexpr uint32_t kTravWarps = GBH_TRAVERSE_WARPS;
// Stack bound.  Each step pops the top <= 8 entries and pushes the opened
// children groups (<= 32) in the order of their parents' stack positions, so
// the stack stays sorted by depth with the deepest entries on top.  When
// entries of depth d are pushed, every earlier entry of depth d has already
// been popped (it sat above the depth d-1 parent), so at most 32 entries of
// one depth are held at once.  Groups belong to the 16 internal depths 0..15
// (Morton codes resolve 16 levels) or are a root group: 17 depths.
constexpr uint32_t kTravStack = 17u * 32u;
// Interaction list: flushed once it holds >= 32 entries; a step adds <= 32.
constexpr uint32_t kTravList = 64u;
static_assert(kTravList >= 64u, "the mixed cells of a step park in list[32, 64)");

template <bool COMP, bool POT, bool STATS, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, GBH_TRAVERSE_MIN_BLOCKS * kTravWarps / WARPS)
    k_traverse(
    const SimDesc* __restrict__ sims, const SimOut* __restrict__ simout,
    const uint32_t* __restrict__ chunk_sim, uint32_t nchunks, const float4* __restrict__ sbody,
    const CellRec* __restrict__ groups, const double4* __restrict__ cell_d, uint32_t capacity,
    unsigned long long* stats, uint32_t* err) {
    wait_for_predecessor();
    __shared__ uint2 s_stack[WARPS][kTravStack];  // (node group, lane mask)
    __shared__ float4 s_list[WARPS][kTravList];   // (com_x, com_y, G*m, lane mask bits)
    __shared__ uint4 s_mix[WARPS][32];  // mixed cells by rank: (lo bits, cell, deciding
                                        // lanes, opened); their f in list[32 + rank]
    // compensated form: the f32 residual of each list entry's centre of mass
    // (0 for bodies), added back to the difference (com_hi - x) + com_lo, so a
    // term's distance carries the f64 centre of mass to one f32 rounding of
    // the distance itself rather than of the centre's coordinates
    __shared__ float2 s_lo[WARPS][COMP ? kTravList : 1];
    const uint32_t lane = lane_id();
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t chunk = blockIdx.x * WARPS + warp;
    if (chunk >= nchunks) return;
    const uint32_t s = chunk_sim[chunk];
    if (s == kNone) return;
    const SimDesc& sd = sims[s];
    // each instance sums only the simulations that asked for its summation
    // form, so a simulation's forces do not depend on its batch mates
    if (((sd.flags & BH_FLAG_COMPENSATED) != 0u) != COMP) return;
    const uint32_t p0 = chunk * kChunk;
    const uint32_t p = p0 + lane;
    const bool valid = p < sd.off + sd.n;
    const float4 me = valid ? sbody[p] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float tx = me.x, ty = me.y;
    const float eps2 = sd.eps_f * sd.eps_f;
    const float g = sd.g_f;
    const uint32_t valid_mask = __ballot_sync(kFull, valid);
    const uint32_t lanes_below = (1u << lane) - 1u;
    float bx0 = valid ? tx : INFINITY, bx1 = valid ? tx : -INFINITY;
    float by0 = valid ? ty : INFINITY, by1 = valid ? ty : -INFINITY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        bx0 = fminf(bx0, __shfl_xor_sync(kFull, bx0, o));
        bx1 = fmaxf(bx1, __shfl_xor_sync(kFull, bx1, o));
        by0 = fminf(by0, __shfl_xor_sync(kFull, by0, o));
        by1 = fmaxf(by1, __shfl_xor_sync(kFull, by1, o));
    }
    uint2* stack = s_stack[warp];
    float4* list = s_list[warp];
    Acc<COMP> acc;
    float phi = 0.f;
    uint32_t n_visit = 0, n_approx = 0, n_direct = 0, n_exact = 0, n_iter = 0;

    const float2 txy = make_float2(tx, ty);
    // one point-mass term at difference d, scale 0 for lanes that do not take it
    auto term = [&](float2 d, float d2, float gm, bool take) {
        const float inv_r = rsqrtf(d2 + eps2);
        const float scale = take ? gm * inv_r * inv_r * inv_r : 0.f;
        acc.add_scaled(d, scale);
        if (POT) phi -= take ? gm * inv_r : 0.f;
    };
    const uint32_t lane_bit = 1u << lane;
    // A lane outside an entry's mask may sit at distance 0 from it (its own
    // body, with zero softening): its scale is selected to 0 after the
    // product, so the inf of that product never reaches the sums.
    auto flush = [&](uint32_t count) {
#pragma unroll 4
        for (uint32_t i = 0; i < count; ++i) {
            const float4 e = list[i];
            float2 d = sub2<COMP>(make_float2(e.x, e.y), txy);
            if constexpr (COMP) d = __fadd2_rn(d, s_lo[warp][i]);
            const float inv_r = rsqrtf(__fmaf_rn(d.x, d.x, __fmaf_rn(d.y, d.y, eps2)));
            const bool take = (__float_as_uint(e.w) & lane_bit) != 0u;
            const float scale = e.z * inv_r * inv_r * inv_r;
            if constexpr (!COMP && !POT) {
                // plain sums: lanes outside the mask skip the (predicated) adds
                if (take) acc.add_scaled(d, scale);
            } else {
                acc.add_scaled(d, take ? scale : 0.f);
                if (POT) phi -= take ? e.z * inv_r : 0.f;
            }
        }
    };

    if (lane == 0) stack[0] = make_uint2(capacity + s, valid_mask);
    __syncwarp();
    uint32_t len = 1, nlist = 0;
    while (len > 0) {
        const uint32_t ng = min(len, 8u);
        const uint32_t gi = lane >> 2;
        const bool have = gi < ng;
        uint2 e = make_uint2(0u, 0u);
        if (have) e = stack[len - ng + gi];
        __syncwarp();
        len -= ng;
        float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
        uint4 u = make_uint4(0u, 0u, 0u, 0u);  // lo | count, start, count, cell (kNone: leaf)
        if (have) {
            const CellRec* r = groups + 4ull * e.x + (lane & 3u);
            f = __ldg(&r->f);
            u = __ldg(&r->u);
        }
        const uint32_t A = e.y;
        const bool present = u.z != 0u;
        const bool leaf = u.w == kNone;
        float2 clo = make_float2(0.f, 0.f);  // compensated: residual of the centre of mass
        if (COMP && have && present && !leaf) {
            const unsigned long long b = __double_as_longlong(
                __ldg(reinterpret_cast<const double*>(cell_d + u.w) + 3));
            clo = make_float2(__uint_as_float((uint32_t)b), __uint_as_float((uint32_t)(b >> 32)));
        }
        // lanes whose own body the cell holds: positions [start, start + count)
        const uint32_t ha = max(u.y, p0), hb = min(u.y + u.z, p0 + 32u);
        const uint32_t H = (present && ha < hb) ? bit_range(ha - p0, hb - p0) : 0u;
        const uint32_t R = A & ~H;
        // classification, branch-free (a select per outcome): a one-body
        // leaf is a list term for R; an internal cell is a list term for R
        // when the box's nearest point is beyond hi, opened by R when its
        // farthest corner is inside lo, otherwise mixed; holding lanes open it
        const float nx = fmaxf(fmaxf(bx0 - f.x, f.x - bx1), 0.f);
        const float ny = fmaxf(fmaxf(by0 - f.y, f.y - by1), 0.f);
        const float fx = fmaxf(fabsf(f.x - bx0), fabsf(f.x - bx1));
        const float fy = fmaxf(fabsf(f.y - by0), fabsf(f.y - by1));
        const bool internal = present && !leaf;
        const bool far = dist2(nx, ny) > f.w;
        const bool near = dist2(fx, fy) < __uint_as_float(u.x);
        const bool multi = present && leaf && u.z != 1u;
        const uint32_t ap = ((present && leaf && u.z == 1u) || (internal && far)) ? R : 0u;
        uint32_t op = internal ? ((A & H) | ((!far && near) ? R : 0u)) : 0u;
        const bool mixed = internal && R != 0u && !far && !near;
        if (STATS && present) {
            n_visit += __popc(A);
            if (leaf)
                n_direct += __popc(ap);
            else
                n_approx += __popc(ap);
        }
        if (STATS) ++n_iter;

        // mixed cells: every lane of the mask that does not hold the cell
        // decides for itself, one cell after the other; holding lanes open
        // it (op).  The record's f waits in the free upper half of the
        // interaction list (at most 31 entries are pending between steps),
        // the rest and the masks in s_mix.
        const uint32_t bm = __ballot_sync(kFull, mixed);
        const uint32_t mrank = __popc(bm & lanes_below);
        if (mixed) {
            list[32u + mrank] = f;
            if (COMP) s_lo[warp][32u + mrank] = clo;
            s_mix[warp][mrank] = make_uint4(u.x, u.w, R, 0u);
        }
        __syncwarp();
        const uint32_t nm = __popc(bm);
        for (uint32_t i = 0; i < nm; ++i) {
            const float4 cf = list[32u + i];
            const uint4 cu = s_mix[warp][i];
            const bool active = (cu.z & lane_bit) != 0u;
            const float2 d = sub2<COMP>(make_float2(cf.x, cf.y), txy);
            const float d2 = dist2(d.x, d.y);
            bool approx = active && d2 > cf.w;
            bool open = active && d2 < __uint_as_float(cu.x);
            const bool undecided = active && !approx && !open;
            if (__any_sync(kFull, undecided)) {
                if (undecided) {
                    approx = exact_mac(cell_d, cu.y, tx, ty, simout[s].half,
                                       __float_as_uint(cf.w) & 31u, sd.theta);
                    open = !approx;
                    if (STATS) ++n_exact;
                }
            }
            // branch-free: lanes that do not approximate add a zero term
            if constexpr (COMP) {
                const float2 dc = __fadd2_rn(d, s_lo[warp][32u + i]);
                term(dc, dist2(dc.x, dc.y), cf.z, approx);
            } else {
                term(d, d2, cf.z, approx);
            }
            if (STATS) n_approx += approx;
            const uint32_t O = __ballot_sync(kFull, open);
            if (lane == 0) s_mix[warp][i].w = O;
            if (STATS) ++n_iter;
        }
        __syncwarp();
        if (mixed) op |= s_mix[warp][mrank].w;

        // leaves of several bodies: each body summed directly, self excluded
        uint32_t bl = __ballot_sync(kFull, multi);
        while (bl) {
            const uint32_t src = __ffs(bl) - 1u;
            bl &= bl - 1u;
            const uint32_t start = __shfl_sync(kFull, u.y, src);
            const uint32_t count = __shfl_sync(kFull, u.z, src);
            const uint32_t M = __shfl_sync(kFull, A, src);
            const bool active = (M >> lane) & 1u;
            for (uint32_t j = start; j < start + count; ++j) {
                const float4 o = sbody[j];
                const bool take = active && j != p;
                const float2 d = sub2<COMP>(make_float2(o.x, o.y), txy);
                term(d, dist2(d.x, d.y), __fmul_rn(g, o.z), take);
                if (STATS) n_direct += take;
            }
        }

        // append the uniform terms, push the opened groups in lane order
        const uint32_t la = __ballot_sync(kFull, ap != 0u);
        if (ap) {
            const uint32_t slot = nlist + __popc(la & lanes_below);
            list[slot] = make_float4(f.x, f.y, f.z, __uint_as_float(ap));
            if (COMP) s_lo[warp][slot] = clo;
        }
        nlist += __popc(la);
        const uint32_t lp = __ballot_sync(kFull, op != 0u);
        if (len + __popc(lp) > kTravStack) {  // unreachable by the bound above
            if (lane == 0) set_err(err, kErrTraversal);
            break;
        }
        if (op) stack[len + __popc(lp & lanes_below)] = make_uint2(u.w, op);
        len += __popc(lp);
        __syncwarp();
        if (nlist >= 32u) {
            flush(nlist);
            nlist = 0;
            __syncwarp();
        }
    }
    flush(nlist);
    if (valid) {
        const uint32_t idx = __float_as_uint(me.w);
        sd.accel[idx] = make_float4(acc.fx(), acc.fy(), 0.f, 0.f);
        if (POT && sd.potential) sd.potential[idx] = phi;
    }
    if (STATS) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            n_visit += __shfl_xor_sync(kFull, n_visit, o);
            n_approx += __shfl_xor_sync(kFull, n_approx, o);
            n_direct += __shfl_xor_sync(kFull, n_direct, o);
            n_exact += __shfl_xor_sync(kFull, n_exact, o);
        }
        if (lane == 0) {
            atomicAdd(&stats[0], (unsigned long long)n_visit);
            atomicAdd(&stats[1], (unsigned long long)n_approx);
            atomicAdd(&stats[2], (unsigned long long)n_direct);
            atomicAdd(&stats[3], (unsigned long long)n_exact);
            atomicAdd(&stats[4], (unsigned long long)n_iter);
        }
    }
}

// ======================================================== packed (2B1) ====

// runtime/src/nbody.wgsl:43-123 (and barnes_hut_flat.cu:65-146) over an
// arbitrary packed tree with explicit children: the same per-body decisions
// (f32 MAC with sqrt), self-exclusion and terms, computed for a warp of 32
// consecutive Morton positions at once.
constexpr int kPackedStack = 64;

__device__ __forceinline__ void packed_point_mass(float tx, float ty, float px, float py,
                                                  float mass, float soft, float g, float* ax,
                                                  float* ay) {
    const float dx = px - tx;
    const float dy = py - ty;
    const float r2 = dx * dx + dy * dy + soft * soft;
    const float inv_r = rsqrtf(r2);
    const float scale = g * mass * inv_r * inv_r * inv_r;
    *ax += dx * scale;
    *ay += dy * scale;
}

// Whether every position's entry names a body whose recorded Morton
// position is that position (bodies[entries[p].body].meta[0] == p), i.e. the
// entries are a permutation of the bodies and meta its inverse, as
// pack_flat_tree writes them.  *bad gets 1 otherwise.  The lane-parallel
// walk relies on it: a lane's own body is the one at its position.
__global__ void k_check_packed(const GpuBody* __restrict__ bodies,
                               const GpuEntry* __restrict__ entries, uint32_t n, uint32_t* bad) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const uint32_t o = entries[p].data[1];
    if (o >= n || bodies[o].meta[0] != p) atomicOr(bad, 1u);
}

// The walk one cell at a time: every lane of the warp tests the same cell
// and keeps the reference's depth-first order of its own terms (children
// pushed 3..0).  Used when the entries and bodies disagree or a tree is
// deeper than the lane-parallel walk's stack bound.  s_cell / s_mask hold
// kPackedStack entries each.
__device__ void packed_walk_cellwise(const BhSettings& st, const GpuBody* __restrict__ bodies,
                                     const GpuEntry* __restrict__ entries,
                                     const GpuCell* __restrict__ cells, uint32_t n,
                                     uint32_t ncells, uint32_t ti, float tx, float ty,
                                     uint32_t tpos, bool lane_ok, uint32_t* s_cell,
                                     uint32_t* s_mask, uint32_t* err, float* out_ax,
                                     float* out_ay) {
    const float theta = st.physics[0], soft = st.physics[1], g = st.physics[2];
    const uint32_t lane = lane_id();
    float ax = 0.f, ay = 0.f;
    int len = 1;
    const uint32_t vmask = __ballot_sync(kFull, lane_ok);
    if (lane == 0) {
        s_cell[0] = st.info[2];
        s_mask[0] = vmask;
    }
    __syncwarp();
    while (len > 0) {
        --len;
        const uint32_t ci = s_cell[len];
        const uint32_t M = s_mask[len];
        __syncwarp();
        if (ci >= ncells) {
            set_err(err, kErrPackedIndex);
            break;
        }
        const GpuCell cell = cells[ci];
        const bool active = (M >> lane) & 1u;
        const bool leaf = cell.children[0] == GALAXY_BH_NO_CHILD &&
                          cell.children[1] == GALAXY_BH_NO_CHILD &&
                          cell.children[2] == GALAXY_BH_NO_CHILD &&
                          cell.children[3] == GALAXY_BH_NO_CHILD;
        if (leaf) {
            for (uint32_t q = cell.range_depth[0]; q < cell.range_depth[1]; ++q) {
                if (q >= n) {
                    set_err(err, kErrPackedIndex);
                    break;
                }
                const uint32_t o = entries[q].data[1];
                if (active && o != ti && o < n) {
                    const GpuBody ob = bodies[o];
                    packed_point_mass(tx, ty, ob.position_mass[0], ob.position_mass[1],
                                      ob.position_mass[2], soft, g, &ax, &ay);
                }
            }
            continue;
        }
        bool open = false;
        if (active) {
            const float dx = cell.com[0] - tx;
            const float dy = cell.com[1] - ty;
            const float distance2 = dx * dx + dy * dy;
            const bool contains = tpos >= cell.range_depth[0] && tpos < cell.range_depth[1];
            open = true;
            if (!contains && distance2 > 0.0f) {
                const float distance = sqrtf(distance2);
                if ((2.0f * cell.center_half_mass[2]) / distance < theta) {
                    packed_point_mass(tx, ty, cell.com[0], cell.com[1], cell.center_half_mass[3],
                                      soft, g, &ax, &ay);
                    open = false;
                }
            }
        }
        const uint32_t O = __ballot_sync(kFull, open);
        if (O) {
            int nch = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) nch += cell.children[q] != GALAXY_BH_NO_CHILD;
            if (len + nch > kPackedStack) {
                set_err(err, kErrPackedStack);
                break;
            }
            if (lane == 0) {
                for (int q = 3; q >= 0; --q) {
                    if (cell.children[q] != GALAXY_BH_NO_CHILD) {
                        s_cell[len] = cell.children[q];
                        s_mask[len] = O;
                        ++len;
                    }
                }
            }
            len = __shfl_sync(kFull, len, 0);
            __syncwarp();
        }
    }
    *out_ax = ax;
    *out_ay = ay;
}

// Lane-parallel walk over the packed tree, the structure of k_traverse: a
// warp pops up to 8 opened cells from its shared-memory stack and lane 4i+q
// examines child q of popped cell i for all lanes of its mask at once,
// against the bounding box of the warp's bodies.  The reference decides in
// f32: a lane approximates a cell unless the cell holds its own body, if
// its squared distance d2 to the centre of mass is positive and
// (2 half) / sqrt(d2) < theta.  d2 = fma(dx, dx, dy*dy), sqrt and the
// division are monotone in |dx|, |dy| (round to nearest), so the test at
// the box's nearest point (all lanes approximate) or farthest corner (all
// open) is every lane's own test; other cells are decided lane by lane
// with the same expression.  Approximated cells and one-body leaves go to
// the interaction list, several-body leaves are summed body by body; a
// lane's own body is the one at its position (the entries are checked to be
// a permutation whose inverse the bodies record), so self-exclusion is
// the lane bit of that position.  Each lane sums exactly the reference's
// terms; only their order differs.
constexpr uint32_t kPkWarps = 4;
constexpr uint32_t kPkRoot = 0xfffffffeu;  // stack entry standing for the root cell itself
// (cell, lane mask) entries: the stack stays sorted by depth and one step
// pushes at most 32 opened cells, so 32 per level of a tree of depth 16
// (pack_flat_tree's trees); a deeper tree that overflows it is walked again
// cell by cell
constexpr uint32_t kPkStack = 17u * 32u;
static_assert(2u * kPkStack >= 2u * kPackedStack, "the cell-by-cell walk borrows the stack");

__global__ void __launch_bounds__(kPkWarps * 32) k_traverse_packed(
    const BhSettings* __restrict__ settings, const GpuBody* __restrict__ bodies,
    const GpuEntry* __restrict__ entries, const GpuCell* __restrict__ cells, uint32_t n,
    uint32_t ncells, float4* __restrict__ accel, uint32_t* err,
    const uint32_t* __restrict__ inconsistent) {
    __shared__ uint2 s_stack[kPkWarps][kPkStack];
    __shared__ float4 s_list[kPkWarps][kTravList];  // (x, y, G*m, lane mask bits)
    __shared__ uint32_t s_mix[kPkWarps][32][2];      // mixed cells by rank: deciding, opened
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    const uint32_t p0 = (blockIdx.x * kPkWarps + warp) * 32u;
    if (p0 >= n) return;
    const BhSettings st = *settings;
    const float theta = st.physics[0], soft = st.physics[1], g = st.physics[2];
    const uint32_t p = p0 + lane;
    const bool valid = p < n;
    uint32_t* s_cell = reinterpret_cast<uint32_t*>(s_stack[warp]);
    float ax = 0.f, ay = 0.f;
    if (*inconsistent) {
        // the reference's own indexing: lane p walks for body p, at the
        // Morton position that body records
        const GpuBody b = valid ? bodies[p] : GpuBody{};
        packed_walk_cellwise(st, bodies, entries, cells, n, ncells, p, b.position_mass[0],
                             b.position_mass[1], b.meta[0], valid, s_cell,
                             s_cell + kPackedStack, err, &ax, &ay);
        if (valid) accel[p] = make_float4(ax, ay, 0.f, 0.f);
        return;
    }
    // consistent input: the body at position p is ti, and it records p
    const uint32_t ti = valid ? entries[p].data[1] : 0u;
    const GpuBody tb = valid ? bodies[ti] : GpuBody{};
    const float tx = tb.position_mass[0], ty = tb.position_mass[1];
    const float eps2 = soft * soft;
    const uint32_t valid_mask = __ballot_sync(kFull, valid);
    const uint32_t lanes_below = (1u << lane) - 1u;
    const uint32_t lane_bit = 1u << lane;
    float bx0 = valid ? tx : INFINITY, bx1 = valid ? tx : -INFINITY;
    float by0 = valid ? ty : INFINITY, by1 = valid ? ty : -INFINITY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        bx0 = fminf(bx0, __shfl_xor_sync(kFull, bx0, o));
        bx1 = fmaxf(bx1, __shfl_xor_sync(kFull, bx1, o));
        by0 = fminf(by0, __shfl_xor_sync(kFull, by0, o));
        by1 = fmaxf(by1, __shfl_xor_sync(kFull, by1, o));
    }
    uint2* stack = s_stack[warp];
    float4* list = s_list[warp];
    // one point-mass term (the reference's add_point_mass) for lanes that take it
    auto term = [&](float dx, float dy, float gm, bool take) {
        const float inv_r = rsqrtf(__fmaf_rn(dx, dx, __fmaf_rn(dy, dy, eps2)));
        const float scale = gm * inv_r * inv_r * inv_r;
        if (take) {
            ax += dx * scale;
            ay += dy * scale;
        }
    };
    auto flush = [&](uint32_t count) {
#pragma unroll 4
        for (uint32_t i = 0; i < count; ++i) {
            const float4 e = list[i];
            term(e.x - tx, e.y - ty, e.z, (__float_as_uint(e.w) & lane_bit) != 0u);
        }
    };
    // the reference's opening test: true = approximate
    auto approximates = [&](float two_half, float d2) {
        return d2 > 0.0f && two_half / sqrtf(d2) < theta;
    };

    if (lane == 0) stack[0] = make_uint2(kPkRoot, valid_mask);
    __syncwarp();
    uint32_t len = 1, nlist = 0;
    bool overflow = false;
    while (len > 0) {
        const uint32_t ng = min(len, 8u);
        const uint32_t gi = lane >> 2, q = lane & 3u;
        const bool have = gi < ng;
        uint2 e = make_uint2(0u, 0u);
        if (have) e = stack[len - ng + gi];
        __syncwarp();
        len -= ng;
        uint32_t c = GALAXY_BH_NO_CHILD;
        if (have) c = e.x == kPkRoot ? (q == 0u ? st.info[2] : GALAXY_BH_NO_CHILD)
                                     : __ldg(&cells[e.x].children[q]);
        bool present = c != GALAXY_BH_NO_CHILD;
        if (present && c >= ncells) {
            set_err(err, kErrPackedIndex);
            present = false;
        }
        float4 chm = make_float4(0.f, 0.f, 0.f, 0.f);  // centre, half, mass
        float2 com = make_float2(0.f, 0.f);
        uint4 rd = make_uint4(0u, 0u, 0u, 0u);          // start, end, depth, valid
        uint4 chn = make_uint4(GALAXY_BH_NO_CHILD, GALAXY_BH_NO_CHILD, GALAXY_BH_NO_CHILD,
                               GALAXY_BH_NO_CHILD);
        if (present) {
            const GpuCell* cr = cells + c;
            chm = __ldg(reinterpret_cast<const float4*>(cr->center_half_mass));
            com = __ldg(reinterpret_cast<const float2*>(cr->com));
            rd = __ldg(reinterpret_cast<const uint4*>(cr->range_depth));
            chn = __ldg(reinterpret_cast<const uint4*>(cr->children));
        }
        const uint32_t A = e.y;
        const bool leaf = chn.x == GALAXY_BH_NO_CHILD && chn.y == GALAXY_BH_NO_CHILD &&
                          chn.z == GALAXY_BH_NO_CHILD && chn.w == GALAXY_BH_NO_CHILD;
        // lanes whose own body the cell holds: positions [start, end)
        const uint32_t ha = max(rd.x, p0), hb = min(rd.y, p0 + 32u);
        const uint32_t H = (present && ha < hb) ? bit_range(ha - p0, hb - p0) : 0u;
        const uint32_t R = A & ~H;
        const bool internal = present && !leaf;
        const bool one = present && leaf && rd.y == rd.x + 1u;
        const bool multi = present && leaf && rd.y > rd.x + 1u;
        // a one-body leaf is a term at its body (the reference sums leaves
        // from the bodies themselves)
        float ex = com.x, ey = com.y, em = chm.w;
        if (one) {
            if (rd.x < n) {
                const float4 b = __ldg(reinterpret_cast<const float4*>(
                    bodies[__ldg(&entries[rd.x].data[1])].position_mass));
                ex = b.x;
                ey = b.y;
                em = b.z;
            } else {
                set_err(err, kErrPackedIndex);
            }
        }
        const float two_half = 2.0f * chm.z;
        const float nx = fmaxf(fmaxf(bx0 - com.x, com.x - bx1), 0.f);
        const float ny = fmaxf(fmaxf(by0 - com.y, com.y - by1), 0.f);
        const float fx = fmaxf(fabsf(com.x - bx0), fabsf(com.x - bx1));
        const float fy = fmaxf(fabsf(com.y - by0), fabsf(com.y - by1));
        const bool far = internal && approximates(two_half, dist2(nx, ny));
        const bool near = internal && !approximates(two_half, dist2(fx, fy));
        const uint32_t ap = (one || far) ? R : 0u;
        uint32_t op = internal ? ((A & H) | (near ? R : 0u)) : 0u;
        const bool mixed = internal && R != 0u && !far && !near;

        // mixed cells: every lane of the mask that does not hold the cell
        // decides for itself, one cell after the other, from a copy of the
        // cell parked in the free upper half of the interaction list
        const uint32_t bm = __ballot_sync(kFull, mixed);
        const uint32_t mrank = __popc(bm & lanes_below);
        if (mixed) {
            list[32u + mrank] = make_float4(com.x, com.y, g * chm.w, two_half);
            s_mix[warp][mrank][0] = R;
        }
        __syncwarp();
        const uint32_t nm = __popc(bm);
        for (uint32_t i = 0; i < nm; ++i) {
            const float4 cf = list[32u + i];
            const bool active = (s_mix[warp][i][0] & lane_bit) != 0u;
            const float dx = cf.x - tx, dy = cf.y - ty;
            const bool approx = active && approximates(cf.w, dist2(dx, dy));
            term(dx, dy, cf.z, approx);
            const uint32_t O = __ballot_sync(kFull, active && !approx);
            if (lane == 0) s_mix[warp][i][1] = O;
        }
        __syncwarp();
        if (mixed) op |= s_mix[warp][mrank][1];

        // leaves of several bodies: each body summed directly, self excluded
        uint32_t bl = __ballot_sync(kFull, multi);
        while (bl) {
            const uint32_t src = __ffs(bl) - 1u;
            bl &= bl - 1u;
            const uint32_t start = __shfl_sync(kFull, rd.x, src);
            const uint32_t end = __shfl_sync(kFull, rd.y, src);
            const uint32_t M = __shfl_sync(kFull, A, src);
            const bool active = (M >> lane) & 1u;
            if (end > n) set_err(err, kErrPackedIndex);
            for (uint32_t j = start; j < min(end, n); ++j) {
                const float4 b = __ldg(reinterpret_cast<const float4*>(
                    bodies[__ldg(&entries[j].data[1])].position_mass));
                term(b.x - tx, b.y - ty, g * b.z, active && j != p);
            }
        }

        // append the list terms, push the opened cells in lane order
        const uint32_t la = __ballot_sync(kFull, ap != 0u);
        if (ap) list[nlist + __popc(la & lanes_below)] = make_float4(ex, ey, g * em,
                                                                      __uint_as_float(ap));
        nlist += __popc(la);
        const uint32_t lp = __ballot_sync(kFull, op != 0u);
        if (len + __popc(lp) > kPkStack) {  // deeper than the bound: walk again cell by cell
            overflow = true;
            break;
        }
        if (op) stack[len + __popc(lp & lanes_below)] = make_uint2(c, op);
        len += __popc(lp);
        __syncwarp();
        if (nlist >= 32u) {
            flush(nlist);
            nlist = 0;
            __syncwarp();
        }
    }
    if (overflow) {
        __syncwarp();
        packed_walk_cellwise(st, bodies, entries, cells, n, ncells, ti, tx, ty, p, valid, s_cell,
                             s_cell + kPackedStack, err, &ax, &ay);
    } else {
        flush(nlist);
    }
    if (valid) accel[ti] = make_float4(ax, ay, 0.f, 0.f);
}

// ============================================================ export =====

// Frozen 64-byte cells (pack_flat_tree, nbody_gpu.rs:211-229) of one
// simulation in the reference preorder, plus sorted entries and bodies with
// their Morton positions.  Cell centres are rebuilt from the code prefix
// with the same f64 steps as child_bounds (nbody/src/flat.rs:96-103).
__global__ void k_export_cells(const SimDesc* __restrict__ sims, const SimOut* __restrict__ simout,
                               uint32_t sim, const uint32_t* __restrict__ codes,
                               const uint32_t* __restrict__ base,
                               const uint4* __restrict__ cell_u,
                               const uint4* __restrict__ cell_child,
                               const double4* __restrict__ cell_d, GpuCell* out) {
    const SimDesc& sd = sims[sim];
    const uint32_t cb = base[sd.off], ce = base[sd.off + sd.n];
    const uint32_t k = cb + blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ce) return;
    const SimOut so = simout[sim];
    const uint4 u = cell_u[k];
    const uint32_t start = u.z - sd.off;
    const uint32_t code = codes[u.z];
    double cx = so.cx, cy = so.cy, half = so.half;
    for (uint32_t level = 0; level < u.w; ++level) {
        const uint32_t q = (code >> (30u - 2u * level)) & 3u;
        const double h = __dmul_rn(half, 0.5);
        cx = __dadd_rn(cx, (q & 1u) ? h : -h);
        cy = __dadd_rn(cy, (q & 2u) ? h : -h);
        half = h;
    }
    const double4 v = cell_d[k];
    const uint4 ch = cell_child[k];
    GpuCell c;
    c.center_half_mass[0] = (float)cx;
    c.center_half_mass[1] = (float)cy;
    c.center_half_mass[2] = (float)half;
    c.center_half_mass[3] = (float)v.z;
    c.com[0] = (float)v.x;
    c.com[1] = (float)v.y;
    c.com[2] = 0.f;
    c.com[3] = 0.f;
    c.range_depth[0] = start;
    c.range_depth[1] = u.x - sd.off;
    c.range_depth[2] = u.w;
    c.range_depth[3] = 0u;
    c.children[0] = ch.x == kNone ? kNone : ch.x - cb;
    c.children[1] = ch.y == kNone ? kNone : ch.y - cb;
    c.children[2] = ch.z == kNone ? kNone : ch.z - cb;
    c.children[3] = ch.w == kNone ? kNone : ch.w - cb;
    out[k - cb] = c;
}

__global__ void k_export_entries(const SimDesc* __restrict__ sims, uint32_t sim,
                                 const uint32_t* __restrict__ codes,
                                 const float4* __restrict__ sbody, GpuEntry* entries,
                                 GpuBody* bodies) {
    const SimDesc& sd = sims[sim];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sd.n) return;
    const float4 b = sbody[sd.off + i];
    const uint32_t idx = __float_as_uint(b.w);
    if (entries) {
        GpuEntry e;
        e.data[0] = codes[sd.off + i];
        e.data[1] = idx;
        e.data[2] = 0u;
        e.data[3] = 0u;
        entries[i] = e;
    }
    if (bodies) {
        GpuBody gb;
        gb.position_mass[0] = b.x;
        gb.position_mass[1] = b.y;
        gb.position_mass[2] = b.z;
        gb.position_mass[3] = 0.f;
        gb.meta[0] = i;
        gb.meta[1] = gb.meta[2] = gb.meta[3] = 0u;
        bodies[idx] = gb;
    }
}

// ===================================================== direct probes =====

constexpr int kProbeThreads = 256;
constexpr int kProbesPerBlock = 8;

// FP64 direct sums for probe bodies (direct_acceleration_for,
// nbody/src/lib.rs:315-329, over the f32 state promoted to f64): every term
// is nbody/src/lib.rs:247-255 with explicit round-to-nearest f64 operations;
// each thread sums a strided slice of the sources and the block adds the
// slices in a fixed order.
__global__ void __launch_bounds__(kProbeThreads) k_direct_probes(
    const GpuEvolveState* __restrict__ state, uint32_t n, const uint32_t* __restrict__ probes,
    uint32_t nprobes, double eps, double g, double* __restrict__ out) {
    __shared__ double sh[kProbesPerBlock][2][kProbeThreads];
    double tx[kProbesPerBlock], ty[kProbesPerBlock], ax[kProbesPerBlock], ay[kProbesPerBlock];
    uint32_t ti[kProbesPerBlock];
#pragma unroll
    for (int k = 0; k < kProbesPerBlock; ++k) {
        const uint32_t q = blockIdx.x * kProbesPerBlock + k;
        ti[k] = q < nprobes ? probes[q] : kNone;
        const bool ok = ti[k] < n;
        tx[k] = ok ? (double)state[ti[k]].position_mass[0] : 0.0;
        ty[k] = ok ? (double)state[ti[k]].position_mass[1] : 0.0;
        ax[k] = ay[k] = 0.0;
    }
    const double eps2 = __dmul_rn(eps, eps);
    for (uint32_t j = threadIdx.x; j < n; j += kProbeThreads) {
        const float4 pm = *reinterpret_cast<const float4*>(state + j);
        const double x = pm.x, y = pm.y, m = pm.z;
        const double gm = __dmul_rn(g, m);
#pragma unroll
        for (int k = 0; k < kProbesPerBlock; ++k) {
            if (j == ti[k]) continue;
            const double dx = __dsub_rn(x, tx[k]);
            const double dy = __dsub_rn(y, ty[k]);
            const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), eps2);
            const double inv_r = __ddiv_rn(1.0, __dsqrt_rn(r2));
            const double scale = __dmul_rn(__dmul_rn(__dmul_rn(gm, inv_r), inv_r), inv_r);
            ax[k] = __dadd_rn(ax[k], __dmul_rn(dx, scale));
            ay[k] = __dadd_rn(ay[k], __dmul_rn(dy, scale));
        }
    }
#pragma unroll
    for (int k = 0; k < kProbesPerBlock; ++k) {
        sh[k][0][threadIdx.x] = ax[k];
        sh[k][1][threadIdx.x] = ay[k];
    }
    __syncthreads();
    for (int stride = kProbeThreads / 2; stride > 0; stride >>= 1) {
        if ((int)threadIdx.x < stride)
#pragma unroll
            for (int k = 0; k < kProbesPerBlock; ++k) {
                sh[k][0][threadIdx.x] += sh[k][0][threadIdx.x + stride];
                sh[k][1][threadIdx.x] += sh[k][1][threadIdx.x + stride];
            }
        __syncthreads();
    }
    if (threadIdx.x < kProbesPerBlock) {
        const uint32_t q = blockIdx.x * kProbesPerBlock + threadIdx.x;
        if (q < nprobes) {
            out[2 * q] = sh[threadIdx.x][0][0];
            out[2 * q + 1] = sh[threadIdx.x][1][0];
        }
    }
}

cudaError_t launch_direct_probes(const GpuEvolveState* state, uint32_t n, const uint32_t* probes,
                                 uint32_t nprobes, double eps, double g, double* out,
                                 cudaStream_t s) {
    const uint32_t blocks = (nprobes + kProbesPerBlock - 1) / kProbesPerBlock;
    k_direct_probes<<<blocks, kProbeThreads, 0, s>>>(state, n, probes, nprobes, eps, g, out);
    return cudaGetLastError();
}

// ================================================= f64 flat traversal =====

// The reference CPU flat traversal (flat_acceleration_for,
// nbody/src/flat.rs:270-346) in f64 over this engine's tree, one thread per
// body in Morton order.  The cells are numbered in the reference's preorder,
// so its depth-first stack walk (children pushed 3..0, popped 0 first) is
// the walk k -> k + 1 when a cell opens and k -> skip when a leaf is summed
// or a cell approximated: each body meets the same cells in the same order,
// with the same f64 centres of mass and masses (bit-identical aggregates),
// the same MAC (hypot distance, width / distance < theta, a cell holding the
// body always opens) and the per-term arithmetic of nbody/src/lib.rs:247-255
// as explicit round-to-nearest operations, so the sum repeats the
// reference's additions one for one.  abs_sum (optional) gets the sum of
// the terms' magnitudes |G m d / r^3| per body; stats the reference's force
// counters (visited, approximated, direct).
constexpr int kF64Threads = 128;

__global__ void __launch_bounds__(kF64Threads) k_traverse_f64(
    const SimDesc* __restrict__ sims, const SimOut* __restrict__ simout, uint32_t sim,
    const float4* __restrict__ sbody, const uint4* __restrict__ cell_u,
    const double4* __restrict__ cell_d, const uint32_t* __restrict__ base, double theta,
    double eps, double g, double2* __restrict__ out, double* __restrict__ abs_sum,
    unsigned long long* __restrict__ stats) {
    const SimDesc& sd = sims[sim];
    const uint32_t i = blockIdx.x * kF64Threads + threadIdx.x;
    unsigned long long nv = 0, na = 0, nd = 0;
    if (i < sd.n) {
        const uint32_t p = sd.off + i;
        const float4 me = sbody[p];
        const double tx = me.x, ty = me.y;
        const double eps2 = __dmul_rn(eps, eps);
        const double root_half = simout[sim].half;
        double ax = 0.0, ay = 0.0, s = 0.0;
        auto add = [&](double x, double y, double mass) {
            const double dx = __dsub_rn(x, tx);
            const double dy = __dsub_rn(y, ty);
            const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), eps2);
            const double inv_r = __ddiv_rn(1.0, __dsqrt_rn(r2));
            const double scale =
                __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(g, mass), inv_r), inv_r), inv_r);
            const double fx = __dmul_rn(dx, scale), fy = __dmul_rn(dy, scale);
            ax = __dadd_rn(ax, fx);
            ay = __dadd_rn(ay, fy);
            if (abs_sum) s += hypot(fx, fy);
        };
        const uint32_t root = base[sd.off];
        const uint32_t stop = cell_u[root].y;  // the root's skip: past the last cell
        uint32_t k = root;
        while (k < stop) {
            const uint4 u = cell_u[k];  // (end, skip, start, depth)
            ++nv;
            if (u.y == k + 1u) {  // a leaf: its bodies directly, self excluded
                for (uint32_t q = u.z; q < u.x; ++q) {
                    if (q == p) continue;
                    const float4 o = sbody[q];
                    add((double)o.x, (double)o.y, (double)o.z);
                    ++nd;
                }
                k = u.y;
                continue;
            }
            const double4 c = cell_d[k];
            const double dist = hypot(__dsub_rn(c.x, tx), __dsub_rn(c.y, ty));
            const double width = __dmul_rn(__dmul_rn(root_half, pow2_neg(u.w)), 2.0);
            const bool contains = p >= u.z && p < u.x;
            if (!contains && dist > 0.0 && __ddiv_rn(width, dist) < theta) {
                add(c.x, c.y, c.z);
                ++na;
                k = u.y;
            } else {
                k = k + 1u;  // open: the first child follows its parent
            }
        }
        const uint32_t idx = __float_as_uint(me.w);
        out[idx] = make_double2(ax, ay);
        if (abs_sum) abs_sum[idx] = s;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        nv += __shfl_xor_sync(kFull, nv, o);
        na += __shfl_xor_sync(kFull, na, o);
        nd += __shfl_xor_sync(kFull, nd, o);
    }
    if (stats && lane_id() == 0 && nv) {
        atomicAdd(&stats[0], nv);
        atomicAdd(&stats[1], na);
        atomicAdd(&stats[2], nd);
    }
}

cudaError_t launch_traverse_f64(const BatchBuffers& b, uint32_t sim, uint32_t n, double theta,
                                double eps, double g, double* out, double* abs_sum,
                                unsigned long long* stats, cudaStream_t s) {
    const uint32_t blocks = (n + kF64Threads - 1) / kF64Threads;
    if (blocks == 0) return cudaSuccess;
    k_traverse_f64<<<blocks, kF64Threads, 0, s>>>(b.sims, b.simout, sim, b.sbody, b.cell_u,
                                                  b.cell_d, b.base, theta, eps, g,
                                                  reinterpret_cast<double2*>(out), abs_sum, stats);
    return cudaGetLastError();
}

// ======================================================= conservation =====

constexpr int kConsThreads = 256;
constexpr int kConsTerms = 9;

// Per-block f64 partial sums in a fixed order, then one block adds the
// partials in block order: the result does not depend on scheduling.
__global__ void __launch_bounds__(kConsThreads) k_conservation_partial(
    const GpuEvolveState* __restrict__ state, const float* __restrict__ potential, uint32_t n,
    double* partials) {
    __shared__ double sh[kConsTerms][kConsThreads];
    double t[kConsTerms] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t i = blockIdx.x * kConsThreads + threadIdx.x; i < n;
         i += gridDim.x * kConsThreads) {
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
    for (int k = 0; k < kConsTerms; ++k) sh[k][threadIdx.x] = t[k];
    __syncthreads();
    for (int stride = kConsThreads / 2; stride > 0; stride >>= 1) {
        if ((int)threadIdx.x < stride)
#pragma unroll
            for (int k = 0; k < kConsTerms; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + stride];
        __syncthreads();
    }
    if (threadIdx.x < kConsTerms) partials[blockIdx.x * kConsTerms + threadIdx.x] = sh[threadIdx.x][0];
}

__global__ void k_conservation_final(const double* partials, uint32_t nblocks, double* out) {
    if (threadIdx.x >= kConsTerms) return;
    double acc = 0.0;
    for (uint32_t b = 0; b < nblocks; ++b) acc += partials[b * kConsTerms + threadIdx.x];
    out[threadIdx.x] = acc;
}

// ============================================================ launchers ===

static int sm_count();

// One resident wave of integrate blocks (each warp then streams a contiguous
// run of chunks), fewer when there are fewer chunks than warps.
template <int MODE>
static uint32_t integrate_blocks(uint32_t nchunks) {
    static int per_sm[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    int& r = per_sm[dev & 63];
    if (!r) {
        int v = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_integrate<MODE>, 256, 0);
        r = v > 0 ? v : 1;
    }
#ifdef GBH_INTEGRATE_BLOCKS_PER_SM
    const uint32_t cap = (uint32_t)(sm_count() * GBH_INTEGRATE_BLOCKS_PER_SM);
#else
    // the final kick (no bounds atomics): one warp per chunk
    const uint32_t cap = MODE == 2 ? 0xffffffffu : (uint32_t)(sm_count() * r);
#endif
    const uint32_t blocks = (nchunks + 7) / 8;
    return blocks < cap ? (blocks ? blocks : 1u) : cap;
}

cudaError_t launch_integrate(const BatchBuffers& b, int mode, cudaStream_t s) {
    switch (mode) {
        case 0: return launch_step(k_integrate<0>, integrate_blocks<0>(b.nchunks), 256, 0, s, b.sims, b.chunk_sim, b.nchunks, b.minmax);
        case 1: return launch_step(k_integrate<1>, integrate_blocks<1>(b.nchunks), 256, 0, s, b.sims, b.chunk_sim, b.nchunks, b.minmax);
        case 2: return launch_step(k_integrate<2>, integrate_blocks<2>(b.nchunks), 256, 0, s, b.sims, b.chunk_sim, b.nchunks, b.minmax);
        default: return launch_step(k_integrate<3>, integrate_blocks<3>(b.nchunks), 256, 0, s, b.sims, b.chunk_sim, b.nchunks, b.minmax);
    }
    return cudaGetLastError();
}

cudaError_t launch_morton(const BatchBuffers& b, cudaStream_t s) {
    if (b.radix_bits == 4)
        return launch_step(k_morton<4>, b.ntiles, kMortonThreads, 0, s, b.sims, b.tiles, b.minmax,
                           b.keys_a, b.hist, b.simout);
    return launch_step(k_morton<8>, b.ntiles, kMortonThreads, 0, s, b.sims, b.tiles, b.minmax,
                       b.keys_a, b.hist, b.simout);
}

// Passes alternate a -> b -> a ...; an even pass count leaves the sorted keys
// in keys_a / vals_a, and the last pass also gathers the sorted bodies.
// Streaming multiprocessors of the current device (cached per device).
static int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cached[dev]) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cached[dev] = n > 0 ? n : 148;
    }
    return cached[dev];
}

template <int BITS, int PASS>
static cudaError_t radix_passes(const BatchBuffers& b, cudaStream_t s) {
    constexpr int kPasses = 32 / BITS;
    const size_t fstride = (size_t)b.ntiles << BITS;
    const bool even = (PASS % 2) == 0;
    const uint32_t* kin = even ? b.keys_a : b.keys_b;
    const uint32_t* vin = even ? b.vals_a : b.vals_b;
    uint32_t* kout = even ? b.keys_b : b.keys_a;
    uint32_t* vout = even ? b.vals_b : b.vals_a;
    // more than two waves of tiles at two per SM: three per SM instead
    const bool many = b.ntiles > 2u * 2u * (uint32_t)sm_count();
    const cudaError_t e =
        many ? launch_step(k_radix_pass<BITS, PASS, PASS == kPasses - 1, 3>, b.ntiles,
                           kSortThreads, 0, s, b.sims, b.tiles, b.counters + PASS, b.hist,
                           b.sort_flags + PASS * fstride, kin, PASS == 0 ? nullptr : vin, kout,
                           vout, b.sbody, b.err)
             : launch_step(k_radix_pass<BITS, PASS, PASS == kPasses - 1, 2>, b.ntiles,
                           kSortThreads, 0, s, b.sims, b.tiles, b.counters + PASS, b.hist,
                           b.sort_flags + PASS * fstride, kin, PASS == 0 ? nullptr : vin, kout,
                           vout, b.sbody, b.err);
    if (e != cudaSuccess) return e;
    if constexpr (PASS + 1 < kPasses) return radix_passes<BITS, PASS + 1>(b, s);
    return cudaSuccess;
}

cudaError_t launch_radix(const BatchBuffers& b, cudaStream_t s) {
    return b.radix_bits == 4 ? radix_passes<4, 0>(b, s) : radix_passes<8, 0>(b, s);
}

cudaError_t launch_count_scan(const BatchBuffers& b, cudaStream_t s) {
    return launch_step(k_count_scan, b.nscan_tiles, kScanThreads, 0, s, b.sims, b.chunk_sim,
                       b.npos, b.keys_a, b.base, b.counters + 8, b.scan_flags, b.err);
}

cudaError_t launch_cells(const BatchBuffers& b, cudaStream_t s) {
    return launch_step(k_cells, (b.npos + kCellsThreads - 1) / kCellsThreads, kCellsThreads, 0, s,
                       b.sims, b.chunk_sim, b.npos, b.cell_capacity, b.keys_a, b.base, b.cell_u,
                       b.cell_child, b.cell_parent, b.cell_counter, b.groups, b.err);
}

cudaError_t launch_aggregate(const BatchBuffers& b, cudaStream_t s) {
    const AggArgs a{b.sims,          b.simout, b.chunk_sim, b.sbody,      b.keys_a,
                    b.cell_capacity, b.cell_u, b.cell_child, b.cell_parent,
                    b.cell_counter,  b.cell_d, b.groups};
    return launch_step(k_aggregate, (b.npos + kAggPositions - 1) / kAggPositions, kAggThreads, 0,
                       s, a, b.npos, b.base, b.err);
}

cudaError_t launch_wait_probe(const uint32_t* flags, uint32_t* err, long long limit,
                              uint32_t* out, cudaStream_t s) {
    k_wait_probe<<<1, kRadixDigits, 0, s>>>(flags, err, limit > 0 ? limit : kSpinCycles, out);
    return cudaGetLastError();
}

cudaError_t launch_refresh_mac(const BatchBuffers& b, uint32_t sim, cudaStream_t s) {
    k_refresh_mac<<<(b.cell_capacity + 255) / 256, 256, 0, s>>>(
        b.sims, b.simout, sim, b.base, b.keys_a, b.cell_capacity, b.cell_parent,
        b.cell_d, b.cell_u, b.groups);
    return cudaGetLastError();
}

template <int WARPS>
static cudaError_t traverse_launch(const BatchBuffers& b, bool compensated, bool potential,
                                   bool stats, cudaStream_t s) {
    // The compensated form keeps a residual per list entry; with it 8 warps'
    // static shared memory would pass 48 KB, so it runs at most 4 warps per
    // block (each warp does the same work at any block size).
    constexpr int CW = WARPS > 4 ? 4 : WARPS;
#define GBH_TRAVERSE(C, P, S)                                                                   \
    return launch_step(k_traverse<C, P, S, (C ? CW : WARPS)>,                                   \
                       (b.nchunks + (C ? CW : WARPS) - 1) / (C ? CW : WARPS),                   \
                       (C ? CW : WARPS) * 32, 0, s, b.sims, b.simout, b.chunk_sim, b.nchunks,  \
                       b.sbody, b.groups, b.cell_d, b.cell_capacity, b.force_stats, b.err)
    if (stats) {
        if (compensated) {
            if (potential) GBH_TRAVERSE(true, true, true);
            GBH_TRAVERSE(true, false, true);
        }
        if (potential) GBH_TRAVERSE(false, true, true);
        GBH_TRAVERSE(false, false, true);
    }
    if (compensated) {
        if (potential) GBH_TRAVERSE(true, true, false);
        GBH_TRAVERSE(true, false, false);
    }
    if (potential) GBH_TRAVERSE(false, true, false);
    GBH_TRAVERSE(false, false, false);
#undef GBH_TRAVERSE
}

static cudaError_t traverse_form(const BatchBuffers& b, bool compensated, bool potential,
                                 bool stats, cudaStream_t s) {
    if (b.trav_warps == 2) return traverse_launch<2>(b, compensated, potential, stats, s);
    if (b.trav_warps == 4) return traverse_launch<4>(b, compensated, potential, stats, s);
    return traverse_launch<kTravWarps>(b, compensated, potential, stats, s);
}

cudaError_t launch_traverse(const BatchBuffers& b, bool compensated, bool plain, bool potential,
                            bool stats, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    if (compensated) e = traverse_form(b, true, potential, stats, s);
    if (e == cudaSuccess && plain) e = traverse_form(b, false, potential, stats, s);
    return e;
}

cudaError_t launch_export(const BatchBuffers& b, uint32_t sim, GpuEntry* entries, GpuBody* bodies,
                          GpuCell* cells, cudaStream_t s) {
    if (cells)
        k_export_cells<<<(b.cell_capacity + 255) / 256, 256, 0, s>>>(
            b.sims, b.simout, sim, b.keys_a, b.base, b.cell_u, b.cell_child, b.cell_d,
            cells);
    if (entries || bodies)
        k_export_entries<<<(b.npos + 255) / 256, 256, 0, s>>>(b.sims, sim, b.keys_a, b.sbody,
                                                             entries, bodies);
    return cudaGetLastError();
}

cudaError_t launch_traverse_packed(const BhSettings* settings, const GpuBody* bodies,
                                   const GpuEntry* entries, const GpuCell* cells, uint32_t n,
                                   uint32_t ncells, float4* accel, uint32_t* err,
                                   cudaStream_t s) {
    // err[1]: set when the entries and bodies disagree (the walk then goes
    // cell by cell)
    k_check_packed<<<(n + 255) / 256, 256, 0, s>>>(bodies, entries, n, err + 1);
    const uint32_t warps = (n + 31) / 32;
    k_traverse_packed<<<(warps + kPkWarps - 1) / kPkWarps, kPkWarps * 32, 0, s>>>(
        settings, bodies, entries, cells, n, ncells, accel, err, err + 1);
    return cudaGetLastError();
}

uint32_t conservation_blocks(uint32_t n) {
    uint32_t blocks = (n + kConsThreads - 1) / kConsThreads;
    return blocks < 592u ? (blocks ? blocks : 1u) : 592u;
}

cudaError_t launch_conservation(const GpuEvolveState* state, const float* potential, uint32_t n,
                                double* partials, uint32_t nblocks, double* out,
                                cudaStream_t s) {
    k_conservation_partial<<<nblocks, kConsThreads, 0, s>>>(state, potential, n, partials);
    k_conservation_final<<<1, 32, 0, s>>>(partials, nblocks, out);
    return cudaGetLastError();
}


// ============================================================ checks ====

// The readback checks of nbody_gpu.rs:1043-1053 (states) and 1097-1101
// (accelerations), evaluated on the device copy of the records.
template <int KIND>
__global__ void __launch_bounds__(256) k_check_records(const float4* __restrict__ rec, uint32_t n,
                                                       uint32_t* first_bad) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        bool ok;
        if (KIND == 0) {
            const float4 pm = rec[2ull * i];
            const float4 v = rec[2ull * i + 1];
            ok = isfinite(pm.x) && isfinite(pm.y) && isfinite(v.x) && isfinite(v.y) &&
                 isfinite(pm.z) && pm.z > 0.f;
        } else {
            const float4 a = rec[i];
            ok = isfinite(a.x) && isfinite(a.y);
        }
        if (!ok) atomicMin(first_bad, i);
    }
}

cudaError_t launch_check_records(const void* records, int kind, uint32_t n, uint32_t* first_bad,
                                 cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const uint64_t want = (n + 255ull) / 256ull;
    const uint32_t blocks = (uint32_t)(want < 148ull * 16ull ? want : 148ull * 16ull);
    if (kind == 0)
        k_check_records<0><<<blocks, 256, 0, s>>>(static_cast<const float4*>(records), n, first_bad);
    else
        k_check_records<1><<<blocks, 256, 0, s>>>(static_cast<const float4*>(records), n, first_bad);
    return cudaGetLastError();
}

}  // namespace gbh
