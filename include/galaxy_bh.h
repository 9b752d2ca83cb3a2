/* SPDX-License-Identifier: Apache-2.0
 *
 * galaxy_bh.h — C ABI of the B200 (sm_100a) Barnes-Hut engine.
 *
 * Drop-in for the reference's BH evolution path: the Rust host methods of
 * NbodyGpu (runtime/src/nbody_gpu.rs) and ParallelTreeRuntime
 * (runtime/src/nbody_parallel.rs).  The frozen f32/u32 transfer records
 * (runtime/src/nbody_gpu.rs:22-83) are kept byte-for-byte.
 *
 * Conventions
 *  - Every function returns a bh_status (0 = BH_OK).  On failure the
 *    thread-local message is read with galaxy_bh_last_error().  Messages
 *    follow the reference's Result<_, String> texts where one exists.
 *  - Handles are opaque and owned by the caller; *_close / *_destroy free
 *    them (the reference frees on Drop).
 *  - One CUDA stream per device handle.  Calls are synchronous (they return
 *    after the device work finished), like the reference's
 *    queue.submit + device.poll(Maintain::Wait).  Handles are not thread-safe.
 *  - Plain pointers and sizes only: host arrays are read/written in the
 *    frozen record layouts below.
 */
#ifndef GALAXY_BH_H
#define GALAXY_BH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GALAXY_BH_ABI_VERSION 1u
#define GALAXY_BH_NO_CHILD 0xffffffffu

typedef enum {
    BH_OK = 0,
    BH_INVALID_ARG = 1,        /* bad size, config or handle */
    BH_CAPACITY_OVERFLOW = 2,  /* a device capacity check tripped */
    BH_NONFINITE = 3,          /* non-finite or non-positive-mass input/output */
    BH_OOM = 4,                /* device or host allocation failed */
    BH_TIMEOUT = 5,            /* a bounded device wait gave up */
    BH_CUDA_ERROR = 6,         /* CUDA runtime error (message has the name) */
    BH_NO_DEVICE = 7           /* no CUDA device / ordinal out of range */
} bh_status;

/* ---- frozen transfer records (runtime/src/nbody_gpu.rs:22-83) ---------- */

/* nbody_gpu.rs:24-27: info = body_count, cell_count, root_index, reserved;
 * physics = theta, softening, G, reserved. */
typedef struct { uint32_t info[4]; float physics[4]; } BhSettings;
/* nbody_gpu.rs:31-34: x, y, mass, reserved | Morton position, reserved x3. */
typedef struct { float position_mass[4]; uint32_t meta[4]; } GpuBody;
/* nbody_gpu.rs:38-40: Morton code, body index, 0, 0. */
typedef struct { uint32_t data[4]; } GpuEntry;
/* nbody_gpu.rs:44-49: cx, cy, half, mass | com_x, com_y, 0, 0 |
 * start, end, depth, reserved | children[4] (GALAXY_BH_NO_CHILD = none). */
typedef struct {
    float center_half_mass[4];
    float com[4];
    uint32_t range_depth[4];
    uint32_t children[4];
} GpuCell;
/* nbody_gpu.rs:53-55: ax, ay, 0, 0. */
typedef struct { float value[4]; } GpuAccel;
/* nbody_gpu.rs:59-62 */
typedef struct { uint32_t info[4]; float motion[4]; } EvolveSettings;
/* nbody_gpu.rs:66-69: x, y, mass, reserved | vx, vy, reserved x2. */
typedef struct { float position_mass[4]; float velocity[4]; } GpuEvolveState;
/* nbody_gpu.rs:73-76 */
typedef struct { uint32_t info[4]; float physics[4]; } TreeSettings;
/* nbody_gpu.rs:80-83.  This engine fills data = cell_count, body_count,
 * effective max_depth, status flags; bounds = root cx, cy, half (f32), 0. */
typedef struct { uint32_t data[4]; float bounds[4]; } TreeMeta;

/* ---- configuration and timings ----------------------------------------- */

/* Config of nbody/src/lib.rs:27-67 (theta, softening_kpc, g, bucket,
 * max_depth) plus engine flags. */
typedef struct {
    double theta;
    double softening;
    double g;
    uint32_t bucket;     /* 1..=1024 */
    uint32_t max_depth;  /* 1..=128; Morton topology caps it at 16 */
    uint32_t flags;      /* BH_FLAG_* */
    uint32_t reserved;
} bh_config;

#define BH_FLAG_COMPENSATED 1u /* two-sum compensated force accumulation */
#define BH_FLAG_POTENTIAL   2u /* also accumulate the softened potential */
#define BH_FLAG_NO_STATS    4u /* galaxy_bh_force skips its force statistics */

/* StageTiming of nbody_gpu.rs:125-130 (seconds). */
typedef struct {
    double transfer_seconds;
    double dispatch_seconds;
    double readback_seconds;
} bh_stage_timing;

/* ParallelTreeBuildTiming of nbody_parallel.rs:45-53 (seconds, device time
 * measured with CUDA events per stage). */
typedef struct {
    double bounds_seconds;
    double morton_seconds;
    double radix_seconds;
    double positions_seconds;
    double topology_seconds;
    double aggregate_seconds;
} bh_build_timing;

/* Traversal work counters (ForceStats of nbody/src/lib.rs:102-107). */
typedef struct {
    uint64_t visited_nodes;
    uint64_t approximated_cells;
    uint64_t direct_terms;
    uint64_t exact_mac_fallbacks; /* MAC tests decided in f64 (guard band) */
    uint64_t warp_iterations;     /* warp steps: walk pops of node groups plus the
                                     lane-by-lane tests of cells whose opening
                                     differs within a warp */
} bh_force_stats;

typedef struct bh_device bh_device;
typedef struct bh_state bh_state;
typedef struct bh_tree bh_tree;
typedef struct bh_batch bh_batch;

/* ---- errors ------------------------------------------------------------- */

/* Copies the calling thread's last error message; returns its length. */
size_t galaxy_bh_last_error(char* buf, size_t len);
/* Failure-detection probe (no reference counterpart): runs the sort's
 * bounded look-back wait against a predecessor that never publishes, with a
 * limit of spin_cycles GPU clock cycles (0 = the production limit of 2e9,
 * about one second; at most 4e9).  Returns BH_TIMEOUT with the same message a
 * stalled sort reports, and leaves the device handle usable; any other
 * status means the wait did not give up as designed. */
int galaxy_bh_wait_probe(bh_device* dev, uint64_t spin_cycles);
uint32_t galaxy_bh_abi_version(void);

/* ---- device --------------------------------------------------------------
 * Replaces NbodyGpu::new(name, allow_software) (nbody_gpu.rs:331) and
 * ParallelTreeRuntime::new(&gpu) (nbody_parallel.rs:156).  ordinal selects a
 * CUDA device.  Fails with BH_NO_DEVICE when none is present. */
int galaxy_bh_device_open(int ordinal, bh_device** out);
int galaxy_bh_device_close(bh_device* dev);
/* JSON adapter description (NbodyGpu::info, nbody_gpu.rs:298-310, 782). */
int galaxy_bh_device_info(bh_device* dev, char* buf, size_t len);
/* The device handle's CUDA stream (cudaStream_t), for external event timing. */
int galaxy_bh_device_stream(bh_device* dev, void** stream);

/* ---- persistent evolving state -------------------------------------------
 * Replaces NbodyGpu::create_evolving_state (nbody_gpu.rs:786-852).  host
 * holds n GpuEvolveState records (the host side does the f64->f32
 * checked_f32 conversion).  Requires 2 <= n, finite values and mass > 0,
 * tested on the uploaded copy: BH_NONFINITE names the smallest failing index
 * and no state is created.  The state's buffers come from a stream-ordered
 * pool of the device handle, released in order on its stream. */
int galaxy_bh_state_create(bh_device* dev, const GpuEvolveState* host, uint32_t n,
                           bh_state** out, bh_stage_timing* timing);
int galaxy_bh_state_destroy(bh_state* st);
int galaxy_bh_state_count(bh_state* st, uint32_t* n);
/* NbodyGpu::evolving_buffer_bytes (nbody_gpu.rs:1116). */
int galaxy_bh_state_bytes(bh_state* st, uint64_t* bytes);
/* NbodyGpu::kick_drift / final_kick (nbody_gpu.rs:1011-1017). */
int galaxy_bh_kick_drift(bh_device* dev, bh_state* st, double dt, bh_stage_timing* timing);
int galaxy_bh_final_kick(bh_device* dev, bh_state* st, double dt, bh_stage_timing* timing);
/* final_kick(dt) then kick_drift(dt) (nbody_gpu.rs:1011-1017, in the order
 * the reference loop calls them between two steps, galaxy-bh-gpu-tree-
 * parallel.rs:345-350) in one pass over the records, with the same two f32
 * roundings as the two calls: the results equal final_kick followed by
 * kick_drift bit for bit.  galaxy_bh_step runs this pass between steps. */
int galaxy_bh_final_kick_drift(bh_device* dev, bh_state* st, double dt,
                               bh_stage_timing* timing);
/* NbodyGpu::read_evolving_state (nbody_gpu.rs:1019-1069); fails with
 * BH_NONFINITE on non-finite values or mass <= 0 like the reference, naming
 * the first such record (checked on the device while the copy runs; `out`
 * still receives every record). */
int galaxy_bh_read_state(bh_device* dev, bh_state* st, GpuEvolveState* out, uint32_t n,
                         bh_stage_timing* timing);
/* NbodyGpu::read_evolving_accelerations (nbody_gpu.rs:1071-1114). */
int galaxy_bh_read_accel(bh_device* dev, bh_state* st, GpuAccel* out, uint32_t n,
                         bh_stage_timing* timing);
/* Overwrites the resident state (checkpoint resume).  The records are
 * uploaded to a staging buffer (allocated by the first call) and checked
 * there like galaxy_bh_state_create's input; an invalid record fails the
 * call with BH_NONFINITE, naming the first one, and leaves the resident
 * state unchanged. */
int galaxy_bh_write_state(bh_device* dev, bh_state* st, const GpuEvolveState* host, uint32_t n);

/* ---- GPU-built tree ------------------------------------------------------
 * ParallelTreeRuntime::create_tree (nbody_parallel.rs:361-493).  No 65,536
 * cap: capacity is sized from n and cfg (cells <= n + depth*n/(bucket+1)). */
int galaxy_bh_tree_create(bh_device* dev, bh_state* st, const bh_config* cfg, bh_tree** out);
int galaxy_bh_tree_destroy(bh_tree* tree);
/* ParallelTreeRuntime::rebuild (nbody_parallel.rs:555-826): bounds, Morton,
 * stable radix sort, positions, topology, aggregates — all on the device. */
int galaxy_bh_tree_rebuild(bh_device* dev, bh_state* st, bh_tree* tree, const bh_config* cfg,
                           bh_build_timing* timing);
/* ParallelTreeRuntime::force (nbody_parallel.rs:828-897): theta-MAC
 * traversal writing the state's acceleration buffer (resident order). */
int galaxy_bh_force(bh_device* dev, bh_state* st, bh_tree* tree, const bh_config* cfg,
                    bh_stage_timing* timing);
/* Counters of the last galaxy_bh_force on this tree. */
int galaxy_bh_force_stats(bh_device* dev, bh_tree* tree, bh_force_stats* out);
/* The reference's CPU flat traversal, flat_accelerations_from_tree
 * (nbody/src/flat.rs:270-371), in f64 on the device over the tree of the
 * last rebuild: the same cells in the same depth-first order, the same f64
 * aggregates, MAC and per-term arithmetic (lib.rs:247-255), so each body's
 * sum repeats the reference's additions.  accel receives ax, ay per body
 * (2n doubles, resident order, host memory); abs_sum (n doubles, or NULL)
 * the sum of each body's term magnitudes; stats (or NULL) the reference's
 * visited / approximated / direct counters.  cfg supplies theta, softening
 * and G in f64.  It states the per-body error of the f32 forces at full
 * size without a CPU pass; it does not touch the state's accelerations. */
int galaxy_bh_force_f64(bh_device* dev, bh_state* st, bh_tree* tree, const bh_config* cfg,
                        double* accel, double* abs_sum, bh_force_stats* stats);
/* ParallelTreeRuntime::read_evidence (nbody_parallel.rs:929-988): meta,
 * sorted entries (n), bodies with Morton positions (n), and the cells in
 * the reference CPU preorder (flat.rs:127-177) in the frozen 64-byte
 * layout, range_depth[3] = 0 as pack_flat_tree writes it.  Any output
 * pointer may be NULL.  *cell_count receives the cell count; cells must hold
 * cell_capacity records. */
int galaxy_bh_read_tree_evidence(bh_device* dev, bh_tree* tree, TreeMeta* meta,
                                 GpuEntry* entries, GpuBody* bodies, uint32_t n, GpuCell* cells,
                                 uint32_t cell_capacity, uint32_t* cell_count);
/* ParallelTreeRuntime::buffer_bytes (nbody_parallel.rs:990-992). */
int galaxy_bh_tree_buffer_bytes(bh_tree* tree, uint64_t* bytes);
/* Device bytes galaxy_bh_tree_buffer_bytes reports for a tree of n bodies
 * under cfg, without a device: the tree-buffer formula a receipt validator
 * checks (the engine's counterpart of bench-bh2d-hardware.py:837-853). */
int galaxy_bh_tree_footprint(uint32_t n, const bh_config* cfg, uint64_t* bytes);

/* ---- BH #2B1 host-tree path -----------------------------------------------
 * NbodyGpu::traverse (nbody_gpu.rs:640-780) over a packed flat tree
 * (pack_flat_tree, nbody_gpu.rs:175-250): uploads, traverses with the
 * reference's f32 MAC (each body's decisions and terms are the reference's;
 * their summation order differs), and reads back n accelerations. */
int galaxy_bh_traverse_packed(bh_device* dev, const BhSettings* settings, const GpuBody* bodies,
                              uint32_t n, const GpuEntry* entries, const GpuCell* cells,
                              uint32_t cell_count, GpuAccel* out, bh_stage_timing* timing);
/* NbodyGpu::force_into (nbody_gpu.rs:854-938): the same traversal writing the
 * evolving state's acceleration buffer. */
int galaxy_bh_force_into(bh_device* dev, bh_state* st, const BhSettings* settings,
                         const GpuBody* bodies, const GpuEntry* entries, const GpuCell* cells,
                         uint32_t cell_count, bh_stage_timing* timing);

/* ---- fused evolution ------------------------------------------------------
 * nsteps KDK steps exactly as the reference loop
 * (galaxy-bh-gpu-tree-parallel.rs:345-350): kick_drift, rebuild, force,
 * final_kick, with the boundary acceleration reused (call rebuild + force
 * once first).  Final kick n and kick-drift n+1 run as one kernel with the
 * same two roundings; each step is a replayed CUDA graph. */
int galaxy_bh_step(bh_device* dev, bh_state* st, bh_tree* tree, const bh_config* cfg, double dt,
                   uint32_t nsteps);

/* ---- FP64 direct-sum probes ---------------------------------------------------
 * direct_acceleration_for (nbody/src/lib.rs:315-329) on the device for
 * nprobes body indices of the resident state, in f64 with the reference's
 * per-term arithmetic (only the summation order is parallel).  out receives
 * ax, ay per probe (2*nprobes doubles, host memory); cfg supplies softening
 * and G.  The reference runs these probes on the CPU (probe_error,
 * nbody/src/lib.rs:370-395); the engine uses them to state the FP64 error of
 * every run. */
int galaxy_bh_direct_probes(bh_device* dev, bh_state* st, const bh_config* cfg,
                            const uint32_t* probes, uint32_t nprobes, double* out);

/* ---- FP64 conservation reductions ------------------------------------------
 * Deterministic f64 sums over the resident f32 state: out[0..9] = mass,
 * com_x, com_y, px, py, lz, kinetic energy, potential energy (0 unless the
 * last force ran with BH_FLAG_POTENTIAL), mass*|v| sum, total energy.  The
 * first six follow galaxy-bh-evolve.rs:252-278. */
int galaxy_bh_conservation(bh_device* dev, bh_state* st, double out[10]);

/* The same sums for callers that cannot allocate device memory — a serving
 * loop that reserved its memory budget up front, a host whose own allocator
 * owns the device memory, code handed only device buffers.  No counterpart in
 * the reference (it has no allocation-free path).  Allocates nothing: state
 * (n GpuEvolveState records) and potential (n floats, or NULL) are device
 * inputs; sums is a device output of 9 doubles — mass, sum m*x, sum m*y, px,
 * py, lz, kinetic, potential, sum m*|v| (divide 1 and 2 by 0 for the centre
 * of mass).  Work is enqueued on `stream` (a cudaStream_t of the current
 * device, BH_INVALID_ARG otherwise) and the function returns without
 * waiting.  NULL means the legacy default stream, which is NOT ordered after
 * this library's own streams (they are non-blocking): when state comes from
 * an engine call, order this call after it yourself (an event, or a
 * synchronize).  Scratch is a 73,728-byte static device array, so n is
 * limited to 4,194,304 (BH_INVALID_ARG beyond).  The first call on each
 * device looks up that array's device address with the device current; make
 * that first call before any stream capture.  The address is kept for the
 * life of the process: after a cudaDeviceReset of a device, do not call this
 * function on that device again.  All calls share the one array: calls that
 * overlap on the GPU (different streams or threads at once) race and
 * corrupt each other's sums. */
int galaxy_bh_conservation_noalloc(const GpuEvolveState* state, const float* potential,
                                   uint32_t n, double* sums, void* stream);

/* ---- batched engine --------------------------------------------------------
 * Many independent simulations of uneven n advanced together: one launch per
 * stage covers every simulation (the force stage takes one launch per
 * summation form present, plain and BH_FLAG_COMPENSATED).  Each state keeps
 * its own resident buffers; cfgs[i] applies to states[i] alone, so a
 * member's results are bit-identical to the same state advanced by itself. */
int galaxy_bh_batch_create(bh_device* dev, bh_state* const* states, const bh_config* cfgs,
                           uint32_t count, bh_batch** out);
int galaxy_bh_batch_destroy(bh_batch* batch);
/* rebuild + force for every member (the boundary solve). */
int galaxy_bh_batch_solve(bh_device* dev, bh_batch* batch);
/* nsteps fused KDK steps for every member, dts[i] per member.  Each member's
 * acceleration buffer must hold its boundary acceleration (a batch_solve,
 * force or earlier step of that state); no solve is needed when a batch is
 * re-formed from states that were already stepping. */
int galaxy_bh_batch_step(bh_device* dev, bh_batch* batch, const double* dts, uint32_t nsteps);
int galaxy_bh_batch_bytes(bh_batch* batch, uint64_t* bytes);

/* ---- native serving loop --------------------------------------------------
 * No reference counterpart (the reference has no serving path).  A server
 * owns two device handles of the GPU and two host threads running
 * continuous batching: submitted simulations are taken in arrival order by
 * a stager, which, as soon as the device-memory footprint of the active set,
 * the already staged ones and the newcomer (the galaxy_bh_batch_footprint
 * figure) fits budget_bytes, uploads and checks the newcomer's state and runs
 * its boundary solve on its own handle and stream while rounds continue;
 * the serving loop admits staged simulations, which stay resident and
 * advance together in rounds of at most round_steps fused KDK steps in one
 * batch; a round stops at the smallest remaining step count so finished
 * simulations leave and waiting ones join between rounds.  Each result
 * equals the same simulation stepped alone.  The budget counts the current
 * members; beyond it the server keeps, once grown, the batch arena of its
 * largest active set so far and the stager's tree arena of its largest
 * request (reused at every join and leave instead of reallocated).  submit
 * copies the initial
 * records; poll waits up to timeout_ms for a finished request (BH_TIMEOUT if
 * none), fills *result (status = the request's bh_status: a request that can
 * never fit the budget fails with BH_CAPACITY_OVERFLOW) and copies its final
 * records to out (capacity >= n; with less room it returns BH_INVALID_ARG,
 * sets result->request_id and result->n and keeps the result queued).
 * submit, poll and stats may be called from
 * any host thread; stop ends the loop after the current round, drops
 * unfinished requests (submitted, waiting and active ones get no result),
 * makes polls that are waiting return BH_INVALID_ARG ("server stopped"),
 * waits for them to leave and frees everything; the handle must not be used
 * after stop returns. */
typedef struct bh_server bh_server;
typedef struct {
    uint64_t budget_bytes;
    uint32_t round_steps;
    uint32_t max_members;
} bh_serve_config;
typedef struct {
    uint64_t request_id;
    uint32_t n;
    uint32_t status;
    uint32_t steps;
    uint32_t reserved;
    double submitted_s, admitted_s, finished_s;  /* seconds since serve_start */
} bh_serve_result;
/* busy_seconds: rounds of steps; the serving thread's other working time
 * splits into form (batch re-formation) and readback (finished results).
 * admit (state uploads and checks) and solve (boundary solves) are the
 * stager thread's, on its own device handle and stream, overlapping the
 * rounds.  elapsed is the time since serve_start. */
typedef struct {
    uint64_t rounds, particle_steps, completed;
    double busy_seconds, elapsed_seconds;
    double admit_seconds, solve_seconds, form_seconds, readback_seconds;
} bh_serve_stats;
int galaxy_bh_serve_start(int ordinal, const bh_serve_config* config, bh_server** out);
int galaxy_bh_serve_submit(bh_server* server, const GpuEvolveState* host, uint32_t n,
                           const bh_config* cfg, double dt, uint32_t steps, uint64_t* request_id);
int galaxy_bh_serve_poll(bh_server* server, uint32_t timeout_ms, bh_serve_result* result,
                         GpuEvolveState* out, uint32_t capacity);
int galaxy_bh_serve_stats(bh_server* server, bh_serve_stats* out);
int galaxy_bh_serve_stop(bh_server* server);

/* ---- launch-shape tuning --------------------------------------------------
 * No reference counterpart (the reference's WGSL dispatch shapes are fixed).
 * Knobs the autotuner (galaxy_b200/autotune.py) picks per batch or tree;
 * neither changes any result bit: the sort is the same stable permutation
 * at either digit width and each traversal warp does the same work at
 * either block size.  Takes effect at the next launch (graphs are
 * re-captured).  Leaf size, the third knob, is bh_config.bucket. */
typedef struct {
    uint32_t radix_bits;      /* 8 (default): 4 sort passes; 4: 8 passes */
    uint32_t traverse_warps;  /* 4 (default), 2 or 8 warps per traversal block */
    uint32_t reserved[2];
} bh_tuning;
int galaxy_bh_batch_tune(bh_batch* batch, const bh_tuning* tuning);
int galaxy_bh_tree_tune(bh_tree* tree, const bh_tuning* tuning);
/* Device bytes a batch of these sizes/configs would need (admission). */
int galaxy_bh_batch_footprint(const uint32_t* counts, const bh_config* cfgs, uint32_t count,
                              uint64_t* bytes);

#ifdef __cplusplus
}
#endif
#endif /* GALAXY_BH_H */
