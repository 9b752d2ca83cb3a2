/* SPDX-License-Identifier: Apache-2.0
 *
 * CPU oracle for the Barnes-Hut evolution path — TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the reference's f64 CPU substrate
 * (nbody/src/lib.rs, nbody/src/flat.rs) plus f32 models of the GPU stage
 * semantics (runtime/src/nbody_evolve.wgsl, runtime/src/nbody.wgsl).  It is
 * the checker for the CUDA engine: only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline / --impl reference legs may load it.  The engine
 * never calls it and has no CPU fallback through it.
 *
 * Build with -O2 -ffp-contract=off (the reference is Rust, which never
 * contracts a*b+c into an FMA), so every f64 expression rounds exactly as in
 * the reference.
 */
#ifndef GALAXY_BH_ORACLE_H
#define GALAXY_BH_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OB_NO_CHILD 0xffffffffu
#define OB_MORTON_AXIS_BITS 16u
#define OB_MORTON_TREE_DEPTH 16u

/* nbody/src/lib.rs:12-19 (field order x, y, vx, vy, mass). */
typedef struct { double x, y, vx, vy, mass; } ob_body;
/* nbody/src/lib.rs:21-25 */
typedef struct { double ax, ay; } ob_accel;
/* nbody/src/lib.rs:27-34 */
typedef struct {
    double theta;
    double softening;
    double g;
    uint64_t bucket;
    uint64_t max_depth;
} ob_config;
/* nbody/src/flat.rs:17-22 */
typedef struct { uint32_t code, body_index; } ob_entry;
/* nbody/src/flat.rs:24-37 */
typedef struct {
    double cx, cy, half, mass, com_x, com_y;
    uint32_t start, end, depth;
    uint32_t children[4];
} ob_cell;
/* nbody/src/lib.rs:89-94 */
typedef struct { uint64_t node_count, leaf_count, max_depth; } ob_tree_stats;
/* nbody/src/lib.rs:102-107 */
typedef struct { uint64_t visited_nodes, approximated_cells, direct_terms; } ob_force_stats;

typedef struct ob_flat_tree ob_flat_tree;

/* Summary of a flat tree (nbody/src/flat.rs:49-58). */
typedef struct {
    uint32_t body_count;
    uint32_t cell_count;
    uint32_t root;
    uint32_t morton_axis_bits;
    ob_tree_stats stats;
    double root_cx, root_cy, root_half;
} ob_flat_tree_info;

const char* ob_last_error(void);

int ob_validate_config(const ob_config* c);
int ob_validate_bodies(const ob_body* b, size_t n);

/* nbody/src/lib.rs:137-154 */
void ob_root_bounds(const ob_body* b, size_t n, double out[3]);
/* nbody/src/flat.rs:67-94 */
uint32_t ob_spread16(uint32_t v);
uint32_t ob_morton2(uint32_t x, uint32_t y);
uint32_t ob_quantize_axis(double value, double center, double half);
uint32_t ob_morton_key_for_point(double x, double y, double cx, double cy, double half);

/* nbody/src/flat.rs:217-268 */
int ob_flat_tree_build(const ob_body* b, size_t n, const ob_config* c, ob_flat_tree** out);
void ob_flat_tree_free(ob_flat_tree* t);
void ob_flat_tree_get_info(const ob_flat_tree* t, ob_flat_tree_info* info);
void ob_flat_tree_copy(const ob_flat_tree* t, ob_entry* entries, uint32_t* position_by_body,
                       ob_cell* cells);
/* nbody/src/flat.rs:416-433 */
uint64_t ob_flat_topology_checksum(const ob_flat_tree* t);
/* The same checksum over (code, body_index) words (entry_stride words per
 * entry) and 16-word GpuCell records. */
uint64_t ob_topology_checksum_arrays(uint32_t n, const uint32_t* entries_pairs,
                                     uint32_t entry_stride, uint32_t ncells,
                                     const uint32_t* cells16);

/* nbody/src/flat.rs:270-371.  targets==NULL: all bodies (out has n rows),
 * else out has ntargets rows.  abs_sum (optional) receives, per target, the
 * sum of the magnitudes of the individual terms (the scale of f32 rounding).
 * nthreads<=1 runs on the calling thread. */
int ob_flat_accelerations(const ob_body* b, size_t n, const ob_flat_tree* t, const ob_config* c,
                          const uint32_t* targets, size_t ntargets, ob_accel* out,
                          double* abs_sum, ob_force_stats* stats, int nthreads);

/* nbody/src/lib.rs:315-351 */
int ob_direct_acceleration_for(size_t index, const ob_body* b, size_t n, const ob_config* c,
                               ob_accel* out);
int ob_direct_accelerations(const ob_body* b, size_t n, const ob_config* c, ob_accel* out);
/* Per-target direct sums for arbitrary targets, threaded (probe oracle). */
int ob_direct_accelerations_for(const ob_body* b, size_t n, const ob_config* c,
                                const uint32_t* targets, size_t ntargets, ob_accel* out,
                                int nthreads);
/* nbody/src/lib.rs:370-395 */
int ob_probe_error(const ob_body* b, size_t n, const ob_accel* approx, const ob_config* c,
                   size_t probes, double out_rms_max[2]);

/* nbody/src/lib.rs:182-313: recursive BH #1 tree and walk. */
int ob_bh1_accelerations(const ob_body* b, size_t n, const ob_config* c, ob_accel* out,
                         ob_tree_stats* tstats, ob_force_stats* fstats);
/* nbody/src/lib.rs:397-428 */
int ob_bh1_leapfrog_step_from_acceleration(ob_body* b, size_t n, double dt, const ob_config* c,
                                           const ob_accel* first, size_t nfirst,
                                           ob_accel* second);

/* nbody/src/lib.rs:430-528 */
int ob_make_disc(size_t count, uint64_t seed, double total_mass, double scale, ob_body* out);
int ob_make_collision(size_t count, uint64_t seed, ob_body* out);
/* nbody/src/lib.rs:530-543 */
uint64_t ob_state_checksum(const ob_body* b, size_t n);

/* runtime/src/nbody_gpu.rs:175-250: frozen f32/u32 records.  settings 8
 * words, bodies 8 words each, entries 4 words each, cells 16 words each. */
int ob_pack_flat_tree(const ob_body* b, size_t n, const ob_flat_tree* t, const ob_config* c,
                      uint32_t* settings, uint32_t* bodies, uint32_t* entries, uint32_t* cells);

/* runtime/src/bin/galaxy-bh-evolve.rs:339-363 (f64 KDK on the flat tree). */
int ob_cpu_flat_evolve(ob_body* b, size_t n, size_t steps, double dt, const ob_config* c,
                       int nthreads);

/* `steps` KDK steps from the boundary acceleration acc (updated in place):
 * the loop body of galaxy-bh-evolve.rs:348-361. */
int ob_cpu_flat_steps(ob_body* b, size_t n, ob_accel* acc, size_t steps, double dt,
                      const ob_config* c, int nthreads, double* build_seconds,
                      double* force_seconds);

/* runtime/src/bin/galaxy-bh-evolve.rs:252-278: mass, com_x, com_y, px, py, lz,
 * mass_speed_scale. */
void ob_invariants(const ob_body* b, size_t n, double out[7]);

/* f32 models of runtime/src/nbody_evolve.wgsl:19-46 over GpuEvolveState
 * records (8 floats) and float4 accelerations; bit-exact semantics. */
void ob_f32_kick_drift(float* states, const float* accel, size_t n, float dt);
void ob_f32_final_kick(float* states, const float* accel, size_t n, float dt);

/* f32 model of runtime/src/nbody.wgsl:43-123 over packed records (inverseSqrt
 * modelled as 1/sqrtf).  Returns nonzero when a traversal stack overflows. */
int ob_f32_traverse_packed(const uint32_t* settings, const uint32_t* bodies,
                           const uint32_t* entries, const uint32_t* cells, size_t n,
                           float* accel_out);

#ifdef __cplusplus
}
#endif
#endif
