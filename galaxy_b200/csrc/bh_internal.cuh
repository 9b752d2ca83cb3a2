// SPDX-License-Identifier: Apache-2.0
// Internal types shared by the engine's kernels and its host runtime.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/galaxy_bh.h"

namespace gbh {

constexpr uint32_t kNone = 0xffffffffu;
constexpr uint32_t kChunk = 32;  // positions per warp chunk; sims start on a chunk boundary
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr uint32_t kTile = kSortThreads * kSortItems;  // keys per radix tile (4096)
constexpr int kRadixDigits = 256;
constexpr int kRadixPasses = 4;
constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;  // 1024-position scan tiles: a shorter per-tile chain
constexpr uint32_t kScanTile = kScanThreads * kScanItems;  // positions per scan tile
constexpr uint32_t kMortonDepth = 16;

// Error bits accumulated in the device error word until the host reads it.
enum : uint32_t {
    kErrLookbackTimeout = 1u,
    kErrCapacity = 2u,
    kErrTraversal = 4u,
    kErrPackedStack = 8u,
    kErrPackedIndex = 16u,
};

// One simulation of a batch (the plain path is a batch of one).
struct SimDesc {
    GpuEvolveState* state;  // resident state, n records (resident order)
    float4* accel;          // resident accelerations, n records
    float* potential;       // optional per-body softened potential (n) or null
    uint32_t off;           // first position in the batch position space (multiple of 32)
    uint32_t n;
    uint32_t bucket;
    uint32_t max_depth;     // min(cfg.max_depth, 16)
    uint32_t first_tile;    // first radix tile of this simulation
    uint32_t flags;         // BH_FLAG_*
    double theta;
    float theta_f;
    float inv_theta_f;
    float eps_f;            // softening as f32 (the reference squares the f32 value)
    float g_f;
    float dt;
    float reserved;
};

// Per-simulation results of the last rebuild.
struct SimOut {
    double cx, cy, half;  // f64 root bounds (nbody/src/lib.rs:137-154)
    double reserved;
};

// Traversal record of one cell, its slot in the parent's node group
// (32 bytes, one sector):
//   f = (com_x, com_y, G*mass, hi) in f32, with the cell depth in the low 5
//       bits of hi (hi rounded up to make room, so the MAC band only widens)
//   u = (lo as f32 bits | leaf body count, start, body count, cell index or
//       kNone for a leaf)
// hi is -1 for a one-body leaf and +inf (a NaN once depth is packed) for a
// leaf of several bodies.  An empty slot has u.z == 0.
struct CellRec {
    float4 f;
    uint4 u;
};

struct Tile {
    uint32_t sim;
    uint32_t start;  // first position
    uint32_t count;  // keys in this tile (<= kTile)
    uint32_t reserved;
};

// Device buffers of one batch (all sized from the batch layout).
struct BatchBuffers {
    const SimDesc* sims;
    SimOut* simout;
    const uint32_t* chunk_sim;  // P/32 entries, kNone for unused chunks
    const Tile* tiles;
    uint32_t nsims;
    uint32_t npos;     // P, multiple of 32
    uint32_t nchunks;  // P / 32
    uint32_t ntiles;
    uint32_t nscan_tiles;
    uint32_t cell_capacity;
    uint32_t radix_bits;   // 8 (4 passes) or 4 (8 passes); results do not depend on it
    uint32_t trav_warps;   // warps per traversal block, 2, 4 or 8; results do not depend on it
    // zeroed once per rebuild (one memset): control block
    uint32_t* minmax;      // nsims * 4 (atomicMax of encoded floats; mins stored inverted)
    uint32_t* hist;        // nsims * 4 * 256
    uint32_t* counters;    // 16: radix tile counters (one per pass, <= 8), scan tile counter [8]
    uint32_t* sort_flags;  // 4 * ntiles * 256
    unsigned long long* scan_flags;  // nscan_tiles
    // transient per rebuild
    uint32_t* keys_a;
    uint32_t* keys_b;
    uint32_t* vals_a;
    uint32_t* vals_b;
    float4* sbody;      // sorted (x, y, m, body index bits)
    uint32_t* base;     // npos + 1: first cell index of each position's chain
    uint4* cell_u;      // per cell in preorder: (end, skip, start, depth) (build, export,
                        // refresh); the MAC fields live in the node-group slots
    CellRec* groups;    // node groups: children of cell k at [4k, 4k+4); simulation s's
                        // root at slot 0 of group cell_capacity + s (traversal)
    double4* cell_d;    // com_x, com_y, mass (f64), then the f32 residuals of
                        // com_x, com_y (float2 bits): com - (float)com
    uint4* cell_child;  // children (global cell indices)
    uint32_t* cell_parent;
    uint32_t* cell_counter;
    // persistent
    uint32_t* err;                   // error bits
    unsigned long long* force_stats; // 4 counters
};

// ---- launchers (bh_kernels.cu) -------------------------------------------
// mode: 0 bounds only, 1 kick_drift (+bounds), 2 final_kick, 3 final_kick+kick_drift (+bounds)
cudaError_t launch_integrate(const BatchBuffers& b, int mode, cudaStream_t s);
cudaError_t launch_morton(const BatchBuffers& b, cudaStream_t s);
cudaError_t launch_radix(const BatchBuffers& b, cudaStream_t s);
cudaError_t launch_count_scan(const BatchBuffers& b, cudaStream_t s);
cudaError_t launch_cells(const BatchBuffers& b, cudaStream_t s);
cudaError_t launch_aggregate(const BatchBuffers& b, cudaStream_t s);
// Recomputes G*m and the MAC bounds of simulation `sim` for new theta / G.
cudaError_t launch_refresh_mac(const BatchBuffers& b, uint32_t sim, cudaStream_t s);
// Bounded-wait probe: the radix look-back against kRadixDigits zeroed flags
// (a first tile that never publishes); limit in clock cycles, 0 = production.
cudaError_t launch_wait_probe(const uint32_t* flags, uint32_t* err, long long limit,
                              uint32_t* out, cudaStream_t s);
// One launch per summation form present in the batch (compensated two-sum,
// plain); each launch computes only the simulations that use its form.
cudaError_t launch_traverse(const BatchBuffers& b, bool compensated, bool plain, bool potential,
                            bool stats, cudaStream_t s);
cudaError_t launch_export(const BatchBuffers& b, uint32_t sim, GpuEntry* entries, GpuBody* bodies,
                          GpuCell* cells, cudaStream_t s);
// err: two zeroed words, the error bits and a flag the launch sets when the
// packed entries and bodies disagree.
cudaError_t launch_traverse_packed(const BhSettings* settings, const GpuBody* bodies,
                                   const GpuEntry* entries, const GpuCell* cells, uint32_t n,
                                   uint32_t ncells, float4* accel, uint32_t* err,
                                   cudaStream_t s);
// FP64 direct accelerations of nprobes probe bodies (out: 2 doubles each).
cudaError_t launch_direct_probes(const GpuEvolveState* state, uint32_t n, const uint32_t* probes,
                                 uint32_t nprobes, double eps, double g, double* out,
                                 cudaStream_t s);
// The reference's f64 flat traversal over the tree of simulation `sim` (n
// bodies): out gets (ax, ay) per body in resident order, abs_sum (or null)
// the sum of term magnitudes, stats (or null, 3 counters, pre-zeroed) the
// visited / approximated / direct counts.
cudaError_t launch_traverse_f64(const BatchBuffers& b, uint32_t sim, uint32_t n, double theta,
                                double eps, double g, double* out, double* abs_sum,
                                unsigned long long* stats, cudaStream_t s);
// FP64 conservation partial sums: out gets 9 doubles (see galaxy_bh_conservation).
cudaError_t launch_conservation(const GpuEvolveState* state, const float* potential, uint32_t n,
                                double* partials, uint32_t nblocks, double* out,
                                cudaStream_t s);
uint32_t conservation_blocks(uint32_t n);
// Record validity check: *first_bad (preset to all ones) gets the smallest
// index of a record that fails it.  kind 0: evolving states (finite position,
// velocity and mass, mass > 0); kind 1: accelerations (finite x, y).
cudaError_t launch_check_records(const void* records, int kind, uint32_t n, uint32_t* first_bad,
                                 cudaStream_t s);

// Hands state st (made on another handle of the same GPU) to device handle
// `to`, after the state's pending work (bh_engine.cu).
int state_move(bh_state* st, bh_device* to);

// Re-forms *batch over new members, or points *tree at another state,
// reusing the arena when it is large enough (bh_engine.cu); null creates,
// a failure leaves null.
int batch_reform(bh_device* dev, bh_batch** batch, bh_state* const* states,
                 const bh_config* cfgs, uint32_t count);
int tree_retarget(bh_device* dev, bh_tree** tree, bh_state* st, const bh_config* cfg);

// Sets the calling thread's last-error message (bh_engine.cu); returns status.
int set_error_message(int status, const char* message);

}  // namespace gbh
