/* SPDX-License-Identifier: Apache-2.0
 *
 * CPU oracle for the Barnes-Hut evolution path — TEST INFRASTRUCTURE ONLY.
 * Restates, in f64 C, the reference's CPU substrate:
 *   nbody/src/lib.rs   (BH #1 recursive tree, direct sums, KDK, ICs, checksum)
 *   nbody/src/flat.rs  (BH #2A Morton / flat-cell substrate)
 *   runtime/src/nbody_gpu.rs:175-250 (pack_flat_tree, frozen f32/u32 records)
 *   runtime/src/bin/galaxy-bh-evolve.rs:252-278, 339-363 (invariants, cpu_flat_evolve)
 * plus f32 models of runtime/src/nbody_evolve.wgsl and runtime/src/nbody.wgsl.
 * Compile with -O2 -ffp-contract=off: each f64 expression below is written in
 * the reference's evaluation order and must round exactly as Rust does.
 */
#define _POSIX_C_SOURCE 200809L
#include "bh_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static __thread char g_err[512];

static int fail(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return 1;
}

const char* ob_last_error(void) { return g_err; }

static const double G_KPC3_PER_MSUN_MYR2 = 4.498502151575286e-12; /* lib.rs:6 */
static const double DEFAULT_SOFTENING_KPC = 0.05;                  /* lib.rs:8 */
static const double TAU = 6.283185307179586;

/* ---------------------------------------------------------------- config -- */

/* lib.rs:48-66 */
int ob_validate_config(const ob_config* c) {
    if (!isfinite(c->theta) || c->theta < 0.0) return fail("theta must be finite and >= 0");
    if (!isfinite(c->softening) || c->softening < 0.0)
        return fail("softening_kpc must be finite and >= 0");
    if (!isfinite(c->g) || c->g <= 0.0) return fail("g must be positive and finite");
    if (c->bucket == 0 || c->bucket > 1024) return fail("bucket must be in 1..=1024");
    if (c->max_depth == 0 || c->max_depth > 128) return fail("max_depth must be in 1..=128");
    return 0;
}

/* lib.rs:122-135 */
int ob_validate_bodies(const ob_body* b, size_t n) {
    if (n < 2) return fail("Barnes-Hut requires at least two resident bodies");
    for (size_t i = 0; i < n; ++i) {
        if (!isfinite(b[i].x) || !isfinite(b[i].y) || !isfinite(b[i].vx) || !isfinite(b[i].vy))
            return fail("body %zu contains non-finite state", i);
        if (!isfinite(b[i].mass) || b[i].mass <= 0.0)
            return fail("body %zu mass must be positive and finite", i);
    }
    return 0;
}

/* lib.rs:137-154 */
void ob_root_bounds(const ob_body* b, size_t n, double out[3]) {
    double min_x = INFINITY, min_y = INFINITY, max_x = -INFINITY, max_y = -INFINITY;
    for (size_t i = 0; i < n; ++i) {
        min_x = fmin(min_x, b[i].x);
        min_y = fmin(min_y, b[i].y);
        max_x = fmax(max_x, b[i].x);
        max_y = fmax(max_y, b[i].y);
    }
    double span = fmax(fmax(max_x - min_x, max_y - min_y), 1e-12);
    out[0] = (min_x + max_x) * 0.5;
    out[1] = (min_y + max_y) * 0.5;
    out[2] = span * 0.500000000001 + 1e-12;
}

/* lib.rs:247-255 */
static inline void add_point_mass(ob_accel* acc, double tx, double ty, double x, double y,
                                  double mass, const ob_config* c, double* abs_sum) {
    double dx = x - tx;
    double dy = y - ty;
    double r2 = dx * dx + dy * dy + c->softening * c->softening;
    double inv_r = 1.0 / sqrt(r2);
    double scale = c->g * mass * inv_r * inv_r * inv_r;
    acc->ax += dx * scale;
    acc->ay += dy * scale;
    if (abs_sum) *abs_sum += hypot(dx * scale, dy * scale);
}

/* ------------------------------------------------------------ flat tree -- */

/* flat.rs:67-75 */
uint32_t ob_spread16(uint32_t value) {
    value &= 0x0000ffffu;
    value = (value | (value << 8)) & 0x00ff00ffu;
    value = (value | (value << 4)) & 0x0f0f0f0fu;
    value = (value | (value << 2)) & 0x33333333u;
    value = (value | (value << 1)) & 0x55555555u;
    return value;
}

/* flat.rs:77-80 */
uint32_t ob_morton2(uint32_t x, uint32_t y) {
    return ob_spread16(x & 0xffffu) | (ob_spread16(y & 0xffffu) << 1);
}

/* flat.rs:82-87 */
uint32_t ob_quantize_axis(double value, double center, double half) {
    double low = center - half;
    double width = half * 2.0;
    double scaled = floor((value - low) / width * 65536.0);
    if (scaled < 0.0) scaled = 0.0;
    if (scaled > 65535.0) scaled = 65535.0;
    return (uint32_t)scaled;
}

/* flat.rs:89-94 */
uint32_t ob_morton_key_for_point(double x, double y, double cx, double cy, double half) {
    return ob_morton2(ob_quantize_axis(x, cx, half), ob_quantize_axis(y, cy, half));
}

struct ob_flat_tree {
    uint32_t n;
    ob_entry* entries;
    uint32_t* position_by_body;
    ob_cell* cells;
    uint32_t n_cells, cap_cells;
    uint32_t root;
    ob_tree_stats stats;
    double root_cx, root_cy, root_half;
};

/* flat.rs:96-103 */
static void child_bounds(double cx, double cy, double half, unsigned q, double* ox, double* oy,
                         double* oh) {
    double child_half = half * 0.5;
    *ox = cx + ((q & 1u) ? child_half : -child_half);
    *oy = cy + ((q & 2u) ? child_half : -child_half);
    *oh = child_half;
}

static int push_cell(ob_flat_tree* t, const ob_cell* c) {
    if (t->n_cells == t->cap_cells) {
        uint32_t cap = t->cap_cells ? t->cap_cells * 2u : 1024u;
        ob_cell* p = (ob_cell*)realloc(t->cells, (size_t)cap * sizeof(ob_cell));
        if (!p) return fail("out of host memory");
        t->cells = p;
        t->cap_cells = cap;
    }
    t->cells[t->n_cells++] = *c;
    return 0;
}

/* flat.rs:127-177 (recursive preorder). */
static int build_topology(ob_flat_tree* t, uint32_t start, uint32_t end, double cx, double cy,
                          double half, uint32_t depth, uint64_t bucket, uint64_t max_depth,
                          uint32_t* out_index) {
    uint32_t cell_index = t->n_cells;
    ob_cell cell;
    memset(&cell, 0, sizeof cell);
    cell.cx = cx;
    cell.cy = cy;
    cell.half = half;
    cell.start = start;
    cell.end = end;
    cell.depth = depth;
    for (int q = 0; q < 4; ++q) cell.children[q] = OB_NO_CHILD;
    if (push_cell(t, &cell)) return 1;
    t->stats.node_count += 1;
    if (depth > t->stats.max_depth) t->stats.max_depth = depth;
    *out_index = cell_index;

    if ((uint64_t)(end - start) <= bucket || (uint64_t)depth >= max_depth) {
        t->stats.leaf_count += 1;
        return 0;
    }
    uint32_t shift = 30u - 2u * depth;
    uint32_t cursor = start;
    while (cursor < end) {
        uint32_t quadrant = (t->entries[cursor].code >> shift) & 3u;
        uint32_t group_start = cursor;
        cursor += 1;
        while (cursor < end && ((t->entries[cursor].code >> shift) & 3u) == quadrant) cursor += 1;
        double ccx, ccy, ch;
        child_bounds(cx, cy, half, quadrant, &ccx, &ccy, &ch);
        uint32_t child;
        if (build_topology(t, group_start, cursor, ccx, ccy, ch, depth + 1, bucket, max_depth,
                           &child))
            return 1;
        t->cells[cell_index].children[quadrant] = child;
    }
    return 0;
}

static int cell_is_leaf(const ob_cell* c) {
    return c->children[0] == OB_NO_CHILD && c->children[1] == OB_NO_CHILD &&
           c->children[2] == OB_NO_CHILD && c->children[3] == OB_NO_CHILD;
}

/* flat.rs:179-215 (reverse index order; leaf sums in entry order, internal
 * sums over children in quadrant order). */
static void fill_aggregates(const ob_body* b, ob_flat_tree* t) {
    for (uint32_t k = t->n_cells; k-- > 0;) {
        ob_cell* cell = &t->cells[k];
        double mass = 0.0, wx = 0.0, wy = 0.0;
        if (cell_is_leaf(cell)) {
            for (uint32_t p = cell->start; p < cell->end; ++p) {
                const ob_body* body = &b[t->entries[p].body_index];
                mass += body->mass;
                wx += body->mass * body->x;
                wy += body->mass * body->y;
            }
        } else {
            for (int q = 0; q < 4; ++q) {
                uint32_t ci = cell->children[q];
                if (ci == OB_NO_CHILD) continue;
                const ob_cell* child = &t->cells[ci];
                mass += child->mass;
                wx += child->mass * child->com_x;
                wy += child->mass * child->com_y;
            }
        }
        cell->mass = mass;
        cell->com_x = wx / mass;
        cell->com_y = wy / mass;
    }
}

/* Stable LSD radix sort of (code, body_index) by code: the same permutation
 * as Rust's stable sort_by_key (flat.rs:233-234). */
static int stable_sort_entries(ob_entry* e, size_t n) {
    ob_entry* tmp = (ob_entry*)malloc(n * sizeof(ob_entry));
    if (!tmp) return fail("out of host memory");
    ob_entry *src = e, *dst = tmp;
    for (int pass = 0; pass < 4; ++pass) {
        size_t count[257];
        memset(count, 0, sizeof count);
        int sh = pass * 8;
        for (size_t i = 0; i < n; ++i) count[((src[i].code >> sh) & 255u) + 1]++;
        for (int d = 0; d < 256; ++d) count[d + 1] += count[d];
        for (size_t i = 0; i < n; ++i) dst[count[(src[i].code >> sh) & 255u]++] = src[i];
        ob_entry* s = src;
        src = dst;
        dst = s;
    }
    /* four passes: result is back in e */
    free(tmp);
    return 0;
}

int ob_flat_tree_build(const ob_body* b, size_t n, const ob_config* c, ob_flat_tree** out) {
    *out = NULL;
    if (ob_validate_bodies(b, n) || ob_validate_config(c)) return 1;
    if (n > 0xffffffffull)
        return fail("flat Barnes-Hut tree requires at most u32::MAX resident bodies");
    ob_flat_tree* t = (ob_flat_tree*)calloc(1, sizeof(ob_flat_tree));
    if (!t) return fail("out of host memory");
    t->n = (uint32_t)n;
    double rb[3];
    ob_root_bounds(b, n, rb);
    t->root_cx = rb[0];
    t->root_cy = rb[1];
    t->root_half = rb[2];
    t->entries = (ob_entry*)malloc(n * sizeof(ob_entry));
    t->position_by_body = (uint32_t*)malloc(n * sizeof(uint32_t));
    if (!t->entries || !t->position_by_body) {
        ob_flat_tree_free(t);
        return fail("out of host memory");
    }
    for (size_t i = 0; i < n; ++i) {
        t->entries[i].code = ob_morton_key_for_point(b[i].x, b[i].y, rb[0], rb[1], rb[2]);
        t->entries[i].body_index = (uint32_t)i;
    }
    if (stable_sort_entries(t->entries, n)) {
        ob_flat_tree_free(t);
        return 1;
    }
    for (size_t p = 0; p < n; ++p) t->position_by_body[t->entries[p].body_index] = (uint32_t)p;
    uint64_t max_depth = c->max_depth < OB_MORTON_TREE_DEPTH ? c->max_depth : OB_MORTON_TREE_DEPTH;
    if (build_topology(t, 0, (uint32_t)n, rb[0], rb[1], rb[2], 0, c->bucket, max_depth,
                       &t->root)) {
        ob_flat_tree_free(t);
        return 1;
    }
    fill_aggregates(b, t);
    *out = t;
    return 0;
}

void ob_flat_tree_free(ob_flat_tree* t) {
    if (!t) return;
    free(t->entries);
    free(t->position_by_body);
    free(t->cells);
    free(t);
}

void ob_flat_tree_get_info(const ob_flat_tree* t, ob_flat_tree_info* info) {
    info->body_count = t->n;
    info->cell_count = t->n_cells;
    info->root = t->root;
    info->morton_axis_bits = OB_MORTON_AXIS_BITS;
    info->stats = t->stats;
    info->root_cx = t->root_cx;
    info->root_cy = t->root_cy;
    info->root_half = t->root_half;
}

void ob_flat_tree_copy(const ob_flat_tree* t, ob_entry* entries, uint32_t* position_by_body,
                       ob_cell* cells) {
    if (entries) memcpy(entries, t->entries, (size_t)t->n * sizeof(ob_entry));
    if (position_by_body) memcpy(position_by_body, t->position_by_body, (size_t)t->n * 4);
    if (cells) memcpy(cells, t->cells, (size_t)t->n_cells * sizeof(ob_cell));
}

static void checksum_word(uint64_t* hash, uint64_t word) {
    *hash ^= word;
    *hash *= 0x00000100000001b3ull;
    *hash ^= (word << 23) | (word >> 41);
}

/* flat.rs:410-433 */
uint64_t ob_flat_topology_checksum(const ob_flat_tree* t) {
    uint64_t hash = 0xcbf29ce484222325ull;
    checksum_word(&hash, OB_MORTON_AXIS_BITS);
    checksum_word(&hash, t->n);
    for (uint32_t i = 0; i < t->n; ++i) {
        checksum_word(&hash, t->entries[i].code);
        checksum_word(&hash, t->entries[i].body_index);
    }
    for (uint32_t k = 0; k < t->n_cells; ++k) {
        const ob_cell* cell = &t->cells[k];
        checksum_word(&hash, cell->start);
        checksum_word(&hash, cell->end);
        checksum_word(&hash, cell->depth);
        for (int q = 0; q < 4; ++q) checksum_word(&hash, cell->children[q]);
    }
    return hash;
}

/* flat.rs:416-433 over arrays: entries as (code, body_index) pairs and cells
 * as frozen 16-word GpuCell records (range_depth at words 8..10, children at
 * 12..15), so a GPU-built tree can be checksummed the reference's way. */
uint64_t ob_topology_checksum_arrays(uint32_t n, const uint32_t* entries_pairs,
                                     uint32_t entry_stride, uint32_t ncells,
                                     const uint32_t* cells16) {
    uint64_t hash = 0xcbf29ce484222325ull;
    checksum_word(&hash, OB_MORTON_AXIS_BITS);
    checksum_word(&hash, n);
    for (uint32_t i = 0; i < n; ++i) {
        checksum_word(&hash, entries_pairs[(size_t)i * entry_stride + 0]);
        checksum_word(&hash, entries_pairs[(size_t)i * entry_stride + 1]);
    }
    for (uint32_t k = 0; k < ncells; ++k) {
        const uint32_t* c = cells16 + 16 * (size_t)k;
        checksum_word(&hash, c[8]);
        checksum_word(&hash, c[9]);
        checksum_word(&hash, c[10]);
        for (int q = 0; q < 4; ++q) checksum_word(&hash, c[12 + q]);
    }
    return hash;
}

/* flat.rs:270-346 */
static void flat_acceleration_for(uint32_t target_index, const ob_body* b,
                                  const ob_flat_tree* t, const ob_config* c, uint32_t* stack,
                                  ob_accel* out, double* abs_sum, ob_force_stats* st) {
    const ob_body target = b[target_index];
    uint32_t target_position = t->position_by_body[target_index];
    ob_accel acc = {0.0, 0.0};
    double s = 0.0;
    double* sp = abs_sum ? &s : NULL;
    size_t len = 0;
    stack[len++] = t->root;
    while (len) {
        const ob_cell* cell = &t->cells[stack[--len]];
        st->visited_nodes += 1;
        if (cell_is_leaf(cell)) {
            for (uint32_t p = cell->start; p < cell->end; ++p) {
                uint32_t other = t->entries[p].body_index;
                if (other == target_index) continue;
                add_point_mass(&acc, target.x, target.y, b[other].x, b[other].y, b[other].mass, c,
                               sp);
                st->direct_terms += 1;
            }
            continue;
        }
        double dx = cell->com_x - target.x;
        double dy = cell->com_y - target.y;
        double distance = hypot(dx, dy);
        double width = cell->half * 2.0;
        int contains = target_position >= cell->start && target_position < cell->end;
        if (!contains && distance > 0.0 && width / distance < c->theta) {
            add_point_mass(&acc, target.x, target.y, cell->com_x, cell->com_y, cell->mass, c, sp);
            st->approximated_cells += 1;
            continue;
        }
        for (int q = 3; q >= 0; --q)
            if (cell->children[q] != OB_NO_CHILD) stack[len++] = cell->children[q];
    }
    *out = acc;
    if (abs_sum) *abs_sum = s;
}

typedef struct {
    const ob_body* b;
    size_t n;
    const ob_flat_tree* t;
    const ob_config* c;
    const uint32_t* targets;
    size_t lo, hi;
    ob_accel* out;
    double* abs_sum;
    ob_force_stats stats;
} flat_job;

static void* flat_worker(void* arg) {
    flat_job* j = (flat_job*)arg;
    uint32_t stack[3 * 130 + 8];
    for (size_t k = j->lo; k < j->hi; ++k) {
        uint32_t ti = j->targets ? j->targets[k] : (uint32_t)k;
        flat_acceleration_for(ti, j->b, j->t, j->c, stack, &j->out[k],
                              j->abs_sum ? &j->abs_sum[k] : NULL, &j->stats);
    }
    return NULL;
}

int ob_flat_accelerations(const ob_body* b, size_t n, const ob_flat_tree* t, const ob_config* c,
                          const uint32_t* targets, size_t ntargets, ob_accel* out,
                          double* abs_sum, ob_force_stats* stats, int nthreads) {
    if (ob_validate_bodies(b, n) || ob_validate_config(c)) return 1;
    if (t->n != n) return fail("flat tree body count does not match resident bodies");
    size_t count = targets ? ntargets : n;
    if (targets)
        for (size_t k = 0; k < ntargets; ++k)
            if (targets[k] >= n) return fail("body index is out of range");
    if (nthreads < 1) nthreads = 1;
    if ((size_t)nthreads > count) nthreads = count ? (int)count : 1;
    flat_job jobs[256];
    pthread_t tid[256];
    if (nthreads > 256) nthreads = 256;
    for (int k = 0; k < nthreads; ++k) {
        jobs[k] = (flat_job){b, n, t, c, targets, count * k / nthreads, count * (k + 1) / nthreads,
                             out, abs_sum, {0, 0, 0}};
    }
    if (nthreads == 1) {
        flat_worker(&jobs[0]);
    } else {
        for (int k = 0; k < nthreads; ++k) pthread_create(&tid[k], NULL, flat_worker, &jobs[k]);
        for (int k = 0; k < nthreads; ++k) pthread_join(tid[k], NULL);
    }
    if (stats) {
        memset(stats, 0, sizeof *stats);
        for (int k = 0; k < nthreads; ++k) {
            stats->visited_nodes += jobs[k].stats.visited_nodes;
            stats->approximated_cells += jobs[k].stats.approximated_cells;
            stats->direct_terms += jobs[k].stats.direct_terms;
        }
    }
    return 0;
}

/* --------------------------------------------------------------- direct -- */

/* lib.rs:315-329 */
int ob_direct_acceleration_for(size_t index, const ob_body* b, size_t n, const ob_config* c,
                               ob_accel* out) {
    if (ob_validate_bodies(b, n) || ob_validate_config(c)) return 1;
    if (index >= n) return fail("body index is out of range");
    ob_accel acc = {0.0, 0.0};
    for (size_t j = 0; j < n; ++j)
        if (j != index) add_point_mass(&acc, b[index].x, b[index].y, b[j].x, b[j].y, b[j].mass, c, NULL);
    *out = acc;
    return 0;
}

/* lib.rs:331-351 (pairwise, i < j). */
int ob_direct_accelerations(const ob_body* b, size_t n, const ob_config* c, ob_accel* out) {
    if (ob_validate_bodies(b, n) || ob_validate_config(c)) return 1;
    memset(out, 0, n * sizeof(ob_accel));
    for (size_t i = 0; i < n; ++i) {
        for (size_t j = i + 1; j < n; ++j) {
            ob_body a = b[i], bb = b[j];
            double dx = bb.x - a.x;
            double dy = bb.y - a.y;
            double r2 = dx * dx + dy * dy + c->softening * c->softening;
            double inv_r = 1.0 / sqrt(r2);
            double common = c->g * inv_r * inv_r * inv_r;
            out[i].ax += dx * common * bb.mass;
            out[i].ay += dy * common * bb.mass;
            out[j].ax -= dx * common * a.mass;
            out[j].ay -= dy * common * a.mass;
        }
    }
    return 0;
}

typedef struct {
    const ob_body* b;
    size_t n;
    const ob_config* c;
    const uint32_t* targets;
    size_t lo, hi;
    ob_accel* out;
} direct_job;

static void* direct_worker(void* arg) {
    direct_job* j = (direct_job*)arg;
    for (size_t k = j->lo; k < j->hi; ++k) {
        size_t i = j->targets[k];
        ob_accel acc = {0.0, 0.0};
        for (size_t q = 0; q < j->n; ++q)
            if (q != i)
                add_point_mass(&acc, j->b[i].x, j->b[i].y, j->b[q].x, j->b[q].y, j->b[q].mass,
                               j->c, NULL);
        j->out[k] = acc;
    }
    return NULL;
}

int ob_direct_accelerations_for(const ob_body* b, size_t n, const ob_config* c,
                                const uint32_t* targets, size_t ntargets, ob_accel* out,
                                int nthreads) {
    if (ob_validate_bodies(b, n) || ob_validate_config(c)) return 1;
    for (size_t k = 0; k < ntargets; ++k)
        if (targets[k] >= n) return fail("body index is out of range");
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    if ((size_t)nthreads > ntargets) nthreads = ntargets ? (int)ntargets : 1;
    direct_job jobs[256];
    pthread_t tid[256];
    for (int k = 0; k < nthreads; ++k)
        jobs[k] = (direct_job){b, n, c, targets, ntargets * k / nthreads,
                               ntargets * (k + 1) / nthreads, out};
    if (nthreads == 1) {
        direct_worker(&jobs[0]);
    } else {
        for (int k = 0; k < nthreads; ++k) pthread_create(&tid[k], NULL, direct_worker, &jobs[k]);
        for (int k = 0; k < nthreads; ++k) pthread_join(tid[k], NULL);
    }
    return 0;
}

/* lib.rs:370-395 */
int ob_probe_error(const ob_body* b, size_t n, const ob_accel* approx, const ob_config* c,
                   size_t probes, double out_rms_max[2]) {
    if (probes < 1) probes = 1;
    if (probes > n) probes = n;
    double sum_sq = 0.0, max_rel = 0.0;
    size_t denom = probes > 1 ? probes - 1 : 1;
    for (size_t k = 0; k < probes; ++k) {
        size_t index = k * (n - 1) / denom;
        ob_accel e;
        if (ob_direct_acceleration_for(index, b, n, c, &e)) return 1;
        double den = fmax(hypot(e.ax, e.ay), 1e-30);
        double rel = hypot(approx[index].ax - e.ax, approx[index].ay - e.ay) / den;
        sum_sq += rel * rel;
        max_rel = fmax(max_rel, rel);
    }
    out_rms_max[0] = sqrt(sum_sq / (double)probes);
    out_rms_max[1] = max_rel;
    return 0;
}

/* ------------------------------------------------------ BH #1 recursive -- */

typedef struct {
    double cx, cy, half, mass, com_x, com_y;
    uint32_t count, depth;
    int32_t children[4];
    uint32_t* indices; /* non-NULL only for leaves */
    uint32_t nidx;
} bh1_node;

typedef struct {
    bh1_node* nodes;
    size_t n, cap;
    ob_tree_stats stats;
} bh1_tree;

static int bh1_push(bh1_tree* t, bh1_node* node, int32_t* idx) {
    if (t->n == t->cap) {
        size_t cap = t->cap ? t->cap * 2 : 1024;
        bh1_node* p = (bh1_node*)realloc(t->nodes, cap * sizeof(bh1_node));
        if (!p) return fail("out of host memory");
        t->nodes = p;
        t->cap = cap;
    }
    t->nodes[t->n] = *node;
    *idx = (int32_t)t->n++;
    return 0;
}

/* lib.rs:182-227 */
static int bh1_build(const ob_body* b, bh1_tree* t, uint32_t* indices, uint32_t count, double cx,
                     double cy, double half, uint32_t depth, const ob_config* c, int32_t* out) {
    t->stats.node_count += 1;
    if (depth > t->stats.max_depth) t->stats.max_depth = depth;
    double mass = 0.0, wx = 0.0, wy = 0.0;
    for (uint32_t k = 0; k < count; ++k) {
        const ob_body* body = &b[indices[k]];
        mass += body->mass;
        wx += body->mass * body->x;
        wy += body->mass * body->y;
    }
    bh1_node node;
    memset(&node, 0, sizeof node);
    node.cx = cx;
    node.cy = cy;
    node.half = half;
    node.mass = mass;
    node.com_x = wx / mass;
    node.com_y = wy / mass;
    node.count = count;
    node.depth = depth;
    for (int q = 0; q < 4; ++q) node.children[q] = -1;
    if ((uint64_t)count <= c->bucket || (uint64_t)depth >= c->max_depth ||
        half <= 2.220446049250313e-16 * 32.0) {
        t->stats.leaf_count += 1;
        node.indices = (uint32_t*)malloc((size_t)count * 4);
        if (!node.indices) return fail("out of host memory");
        memcpy(node.indices, indices, (size_t)count * 4);
        node.nidx = count;
        return bh1_push(t, &node, out);
    }
    int32_t self;
    if (bh1_push(t, &node, &self)) return 1;
    *out = self;
    uint32_t* groups[4];
    uint32_t gn[4] = {0, 0, 0, 0};
    for (int q = 0; q < 4; ++q) {
        groups[q] = (uint32_t*)malloc((size_t)count * 4);
        if (!groups[q]) return fail("out of host memory");
    }
    for (uint32_t k = 0; k < count; ++k) {
        const ob_body* body = &b[indices[k]];
        unsigned q = (unsigned)(body->x >= cx) | ((unsigned)(body->y >= cy) << 1);
        groups[q][gn[q]++] = indices[k];
    }
    int rc = 0;
    for (unsigned q = 0; q < 4 && !rc; ++q) {
        if (!gn[q]) continue;
        double h = half * 0.5;
        double ccx = cx + ((q & 1u) ? h : -h);
        double ccy = cy + ((q & 2u) ? h : -h);
        int32_t child;
        rc = bh1_build(b, t, groups[q], gn[q], ccx, ccy, h, depth + 1, c, &child);
        if (!rc) t->nodes[self].children[q] = child;
    }
    for (int q = 0; q < 4; ++q) free(groups[q]);
    return rc;
}

/* lib.rs:257-291 */
static void bh1_walk(uint32_t ti, const ob_body* b, const bh1_tree* t, int32_t ni,
                     const ob_config* c, ob_accel* acc, ob_force_stats* st) {
    const bh1_node* node = &t->nodes[ni];
    st->visited_nodes += 1;
    if (node->indices) {
        for (uint32_t k = 0; k < node->nidx; ++k) {
            uint32_t o = node->indices[k];
            if (o == ti) continue;
            add_point_mass(acc, b[ti].x, b[ti].y, b[o].x, b[o].y, b[o].mass, c, NULL);
            st->direct_terms += 1;
        }
        return;
    }
    double dx = node->com_x - b[ti].x;
    double dy = node->com_y - b[ti].y;
    double distance = hypot(dx, dy);
    double width = node->half * 2.0;
    int contains = b[ti].x >= node->cx - node->half && b[ti].x <= node->cx + node->half &&
                   b[ti].y >= node->cy - node->half && b[ti].y <= node->cy + node->half;
    if (!contains && distance > 0.0 && width / distance < c->theta) {
        add_point_mass(acc, b[ti].x, b[ti].y, node->com_x, node->com_y, node->mass, c, NULL);
        st->approximated_cells += 1;
        return;
    }
    for (int q = 0; q < 4; ++q)
        if (node->children[q] >= 0) bh1_walk(ti, b, t, node->children[q], c, acc, st);
}

static void bh1_free(bh1_tree* t) {
    for (size_t k = 0; k < t->n; ++k) free(t->nodes[k].indices);
    free(t->nodes);
}

/* lib.rs:229-238, 305-313 */
int ob_bh1_accelerations(const ob_body* b, size_t n, const ob_config* c, ob_accel* out,
                         ob_tree_stats* tstats, ob_force_stats* fstats) {
    if (ob_validate_bodies(b, n) || ob_validate_config(c)) return 1;
    double rb[3];
    ob_root_bounds(b, n, rb);
    bh1_tree t;
    memset(&t, 0, sizeof t);
    uint32_t* idx = (uint32_t*)malloc(n * 4);
    if (!idx) return fail("out of host memory");
    for (size_t i = 0; i < n; ++i) idx[i] = (uint32_t)i;
    int32_t root;
    int rc = bh1_build(b, &t, idx, (uint32_t)n, rb[0], rb[1], rb[2], 0, c, &root);
    free(idx);
    if (rc) {
        bh1_free(&t);
        return 1;
    }
    ob_force_stats st = {0, 0, 0};
    for (size_t i = 0; i < n; ++i) {
        ob_accel acc = {0.0, 0.0};
        bh1_walk((uint32_t)i, b, &t, root, c, &acc, &st);
        out[i] = acc;
    }
    if (tstats) *tstats = t.stats;
    if (fstats) *fstats = st;
    bh1_free(&t);
    return 0;
}

/* lib.rs:397-423 */
int ob_bh1_leapfrog_step_from_acceleration(ob_body* b, size_t n, double dt, const ob_config* c,
                                           const ob_accel* first, size_t nfirst,
                                           ob_accel* second) {
    if (!isfinite(dt) || dt <= 0.0) return fail("dt_myr must be positive and finite");
    if (ob_validate_config(c) || ob_validate_bodies(b, n)) return 1;
    if (nfirst != n) return fail("boundary acceleration count does not match bodies");
    for (size_t i = 0; i < n; ++i) {
        b[i].vx += 0.5 * dt * first[i].ax;
        b[i].vy += 0.5 * dt * first[i].ay;
        b[i].x += dt * b[i].vx;
        b[i].y += dt * b[i].vy;
    }
    if (ob_bh1_accelerations(b, n, c, second, NULL, NULL)) return 1;
    for (size_t i = 0; i < n; ++i) {
        b[i].vx += 0.5 * dt * second[i].ax;
        b[i].vy += 0.5 * dt * second[i].ay;
    }
    return 0;
}

/* --------------------------------------------------------------- ICs ----- */

typedef struct { uint64_t state; } xorshift64;

/* lib.rs:435-451 */
static uint64_t xs_next(xorshift64* r) {
    uint64_t x = r->state;
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    r->state = x;
    return x;
}

static double xs_unit(xorshift64* r) {
    return (double)(xs_next(r) >> 11) / (double)(1ull << 53);
}

/* lib.rs:454-483 */
static ob_body disc_body(xorshift64* rng, double per_body_mass, double total_mass,
                         double scale_kpc, double cx, double cy, double cvx, double cvy,
                         double direction, double spin, double softening_kpc) {
    double u = fmax(1.0 - xs_unit(rng), 1e-15);
    double r = scale_kpc * sqrt(-log(u));
    double angle = TAU * xs_unit(rng);
    double x = cx + r * cos(angle);
    double y = cy + r * sin(angle);
    double q = fmax(r / scale_kpc, 0.0);
    double enclosed = 1.0 - exp(-q) * (1.0 + q);
    if (enclosed < 0.0) enclosed = 0.0;
    if (enclosed > 1.0) enclosed = 1.0;
    double softened_r = fmax(sqrt(r * r + softening_kpc * softening_kpc), 1e-9);
    double circular = sqrt(G_KPC3_PER_MSUN_MYR2 * total_mass * enclosed / softened_r);
    ob_body body;
    body.x = x;
    body.y = y;
    body.vx = cvx - direction * spin * circular * sin(angle);
    body.vy = cvy + direction * spin * circular * cos(angle);
    body.mass = per_body_mass;
    return body;
}

/* lib.rs:485-502 */
int ob_make_disc(size_t count, uint64_t seed, double total_mass, double scale, ob_body* out) {
    if (count < 2 || count > 1000000) return fail("particle count must be in 2..=1000000");
    if (!isfinite(total_mass) || total_mass <= 0.0 || !isfinite(scale) || scale <= 0.0)
        return fail("disc mass and scale must be positive and finite");
    xorshift64 rng = {seed ? seed : 1};
    double per = total_mass / (double)count;
    for (size_t i = 0; i < count; ++i)
        out[i] = disc_body(&rng, per, total_mass, scale, 0.0, 0.0, 0.0, 0.0, 1.0, 0.88,
                           DEFAULT_SOFTENING_KPC);
    return 0;
}

/* lib.rs:504-528 */
int ob_make_collision(size_t count, uint64_t seed, ob_body* out) {
    if (count < 4 || count > 1000000)
        return fail("collision particle count must be in 4..=1000000");
    size_t left = count / 2, right = count - left;
    double total = 5.0e10, half_mass = total * 0.5;
    xorshift64 a = {seed ? seed : 1};
    uint64_t sb = seed + 1;
    xorshift64 bb = {sb ? sb : 1};
    for (size_t i = 0; i < left; ++i)
        out[i] = disc_body(&a, half_mass / (double)left, half_mass, 3.0, -7.5, -1.2, 0.030, 0.010,
                           1.0, 0.86, DEFAULT_SOFTENING_KPC);
    for (size_t i = 0; i < right; ++i)
        out[left + i] = disc_body(&bb, half_mass / (double)right, half_mass, 2.7, 7.5, 1.2, -0.030,
                                  -0.010, -1.0, 0.86, DEFAULT_SOFTENING_KPC);
    return 0;
}

static uint64_t dbits(double v) {
    uint64_t u;
    memcpy(&u, &v, 8);
    return u;
}

/* lib.rs:530-543 */
uint64_t ob_state_checksum(const ob_body* b, size_t n) {
    uint64_t hash = 0xcbf29ce484222325ull;
    for (size_t i = 0; i < n; ++i) {
        uint64_t w[5] = {dbits(b[i].x), dbits(b[i].y), dbits(b[i].vx), dbits(b[i].vy),
                         dbits(b[i].mass)};
        for (int k = 0; k < 5; ++k) checksum_word(&hash, w[k]);
    }
    return hash;
}

/* ------------------------------------------------------------ packing ---- */

static int checked_f32(double v, const char* name, uint32_t* out) {
    float f = (float)v;
    if (!isfinite(f)) return fail("%s cannot be represented as finite f32", name);
    memcpy(out, &f, 4);
    return 0;
}

/* nbody_gpu.rs:175-250 */
int ob_pack_flat_tree(const ob_body* b, size_t n, const ob_flat_tree* t, const ob_config* c,
                      uint32_t* settings, uint32_t* bodies, uint32_t* entries, uint32_t* cells) {
    if (ob_validate_config(c)) return 1;
    if (n != t->n) return fail("flat tree/body cardinality mismatch");
    if (!t->n_cells || t->root >= t->n_cells) return fail("flat tree has invalid root");
    memset(settings, 0, 32);
    settings[0] = (uint32_t)n;
    settings[1] = t->n_cells;
    settings[2] = t->root;
    if (checked_f32(c->theta, "theta", &settings[4]) ||
        checked_f32(c->softening, "softening_kpc", &settings[5]) ||
        checked_f32(c->g, "G", &settings[6]))
        return 1;
    for (size_t i = 0; i < n; ++i) {
        uint32_t* r = bodies + 8 * i;
        memset(r, 0, 32);
        if (checked_f32(b[i].x, "body.x", &r[0]) || checked_f32(b[i].y, "body.y", &r[1]) ||
            checked_f32(b[i].mass, "body.mass", &r[2]))
            return 1;
        r[4] = t->position_by_body[i];
    }
    for (size_t i = 0; i < n; ++i) {
        uint32_t* r = entries + 4 * i;
        r[0] = t->entries[i].code;
        r[1] = t->entries[i].body_index;
        r[2] = 0;
        r[3] = 0;
    }
    for (uint32_t k = 0; k < t->n_cells; ++k) {
        const ob_cell* cell = &t->cells[k];
        uint32_t* r = cells + 16 * (size_t)k;
        memset(r, 0, 64);
        if (checked_f32(cell->cx, "cell.cx", &r[0]) || checked_f32(cell->cy, "cell.cy", &r[1]) ||
            checked_f32(cell->half, "cell.half", &r[2]) ||
            checked_f32(cell->mass, "cell.mass", &r[3]) ||
            checked_f32(cell->com_x, "cell.com_x", &r[4]) ||
            checked_f32(cell->com_y, "cell.com_y", &r[5]))
            return 1;
        r[8] = cell->start;
        r[9] = cell->end;
        r[10] = cell->depth;
        for (int q = 0; q < 4; ++q) r[12 + q] = cell->children[q];
    }
    return 0;
}

/* --------------------------------------------------------- evolution ----- */

/* galaxy-bh-evolve.rs:339-363 */
int ob_cpu_flat_evolve(ob_body* b, size_t n, size_t steps, double dt, const ob_config* c,
                       int nthreads) {
    ob_accel* acc = (ob_accel*)malloc(n * sizeof(ob_accel));
    if (!acc) return fail("out of host memory");
    ob_flat_tree* t = NULL;
    int rc = ob_flat_tree_build(b, n, c, &t);
    if (!rc) rc = ob_flat_accelerations(b, n, t, c, NULL, 0, acc, NULL, NULL, nthreads);
    ob_flat_tree_free(t);
    for (size_t s = 0; s < steps && !rc; ++s) {
        for (size_t i = 0; i < n; ++i) {
            b[i].vx += 0.5 * dt * acc[i].ax;
            b[i].vy += 0.5 * dt * acc[i].ay;
            b[i].x += dt * b[i].vx;
            b[i].y += dt * b[i].vy;
        }
        t = NULL;
        rc = ob_flat_tree_build(b, n, c, &t);
        if (!rc) rc = ob_flat_accelerations(b, n, t, c, NULL, 0, acc, NULL, NULL, nthreads);
        ob_flat_tree_free(t);
        if (rc) break;
        for (size_t i = 0; i < n; ++i) {
            b[i].vx += 0.5 * dt * acc[i].ax;
            b[i].vy += 0.5 * dt * acc[i].ay;
        }
    }
    free(acc);
    return rc;
}

/* The loop body of galaxy-bh-evolve.rs:348-361: `steps` KDK steps from a
 * boundary acceleration `acc` (n rows, updated in place), so steps can be
 * timed one at a time.  build_seconds/force_seconds (optional) accumulate the
 * tree-build and traversal wall times. */
int ob_cpu_flat_steps(ob_body* b, size_t n, ob_accel* acc, size_t steps, double dt,
                      const ob_config* c, int nthreads, double* build_seconds,
                      double* force_seconds) {
    struct timespec t0, t1, t2;
    for (size_t s = 0; s < steps; ++s) {
        for (size_t i = 0; i < n; ++i) {
            b[i].vx += 0.5 * dt * acc[i].ax;
            b[i].vy += 0.5 * dt * acc[i].ay;
            b[i].x += dt * b[i].vx;
            b[i].y += dt * b[i].vy;
        }
        ob_flat_tree* t = NULL;
        clock_gettime(CLOCK_MONOTONIC, &t0);
        int rc = ob_flat_tree_build(b, n, c, &t);
        clock_gettime(CLOCK_MONOTONIC, &t1);
        if (!rc) rc = ob_flat_accelerations(b, n, t, c, NULL, 0, acc, NULL, NULL, nthreads);
        clock_gettime(CLOCK_MONOTONIC, &t2);
        ob_flat_tree_free(t);
        if (rc) return rc;
        if (build_seconds)
            *build_seconds += (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
        if (force_seconds)
            *force_seconds += (double)(t2.tv_sec - t1.tv_sec) + 1e-9 * (double)(t2.tv_nsec - t1.tv_nsec);
        for (size_t i = 0; i < n; ++i) {
            b[i].vx += 0.5 * dt * acc[i].ax;
            b[i].vy += 0.5 * dt * acc[i].ay;
        }
    }
    return 0;
}

/* galaxy-bh-evolve.rs:252-278 */
void ob_invariants(const ob_body* b, size_t n, double out[7]) {
    double mass = 0, wx = 0, wy = 0, px = 0, py = 0, lz = 0, mss = 0;
    for (size_t i = 0; i < n; ++i) {
        mass += b[i].mass;
        wx += b[i].mass * b[i].x;
        wy += b[i].mass * b[i].y;
        px += b[i].mass * b[i].vx;
        py += b[i].mass * b[i].vy;
        lz += b[i].mass * (b[i].x * b[i].vy - b[i].y * b[i].vx);
        mss += b[i].mass * hypot(b[i].vx, b[i].vy);
    }
    out[0] = mass;
    out[1] = wx / mass;
    out[2] = wy / mass;
    out[3] = px;
    out[4] = py;
    out[5] = lz;
    out[6] = mss;
}

/* ------------------------------------------------------- f32 models ------ */

/* nbody_evolve.wgsl:19-33 */
void ob_f32_kick_drift(float* s, const float* a, size_t n, float dt) {
    float hdt = 0.5f * dt;
    for (size_t i = 0; i < n; ++i) {
        float* r = s + 8 * i;
        float hvx = r[4] + hdt * a[4 * i + 0];
        float hvy = r[5] + hdt * a[4 * i + 1];
        r[0] = r[0] + dt * hvx;
        r[1] = r[1] + dt * hvy;
        r[4] = hvx;
        r[5] = hvy;
    }
}

/* nbody_evolve.wgsl:35-46 */
void ob_f32_final_kick(float* s, const float* a, size_t n, float dt) {
    float hdt = 0.5f * dt;
    for (size_t i = 0; i < n; ++i) {
        float* r = s + 8 * i;
        r[4] = r[4] + hdt * a[4 * i + 0];
        r[5] = r[5] + hdt * a[4 * i + 1];
    }
}

static float u2f(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}

/* nbody.wgsl:43-123 */
int ob_f32_traverse_packed(const uint32_t* settings, const uint32_t* bodies,
                           const uint32_t* entries, const uint32_t* cells, size_t n,
                           float* accel_out) {
    float theta = u2f(settings[4]), soft = u2f(settings[5]), g = u2f(settings[6]);
    uint32_t root = settings[2];
    int overflow = 0;
    for (size_t t = 0; t < n && t < settings[0]; ++t) {
        float tx = u2f(bodies[8 * t + 0]), ty = u2f(bodies[8 * t + 1]);
        uint32_t tpos = bodies[8 * t + 4];
        float ax = 0.0f, ay = 0.0f;
        uint32_t stack[64];
        uint32_t len = 1;
        stack[0] = root;
        while (len) {
            const uint32_t* c = cells + 16 * (size_t)stack[--len];
            int leaf = c[12] == OB_NO_CHILD && c[13] == OB_NO_CHILD && c[14] == OB_NO_CHILD &&
                       c[15] == OB_NO_CHILD;
            if (leaf) {
                for (uint32_t p = c[8]; p < c[9]; ++p) {
                    uint32_t o = entries[4 * (size_t)p + 1];
                    if (o == t) continue;
                    float dx = u2f(bodies[8 * o + 0]) - tx;
                    float dy = u2f(bodies[8 * o + 1]) - ty;
                    float r2 = dx * dx + dy * dy + soft * soft;
                    float inv_r = 1.0f / sqrtf(r2);
                    float scale = g * u2f(bodies[8 * o + 2]) * inv_r * inv_r * inv_r;
                    ax += dx * scale;
                    ay += dy * scale;
                }
                continue;
            }
            float dx = u2f(c[4]) - tx, dy = u2f(c[5]) - ty;
            float d2 = dx * dx + dy * dy;
            int contains = tpos >= c[8] && tpos < c[9];
            if (!contains && d2 > 0.0f) {
                float d = sqrtf(d2);
                if ((2.0f * u2f(c[2])) / d < theta) {
                    float r2 = dx * dx + dy * dy + soft * soft;
                    float inv_r = 1.0f / sqrtf(r2);
                    float scale = g * u2f(c[3]) * inv_r * inv_r * inv_r;
                    ax += dx * scale;
                    ay += dy * scale;
                    continue;
                }
            }
            for (int q = 3; q >= 0; --q) {
                if (c[12 + q] == OB_NO_CHILD) continue;
                if (len >= 64) {
                    overflow = 1;
                    break;
                }
                stack[len++] = c[12 + q];
            }
        }
        accel_out[4 * t + 0] = ax;
        accel_out[4 * t + 1] = ay;
        accel_out[4 * t + 2] = 0.0f;
        accel_out[4 * t + 3] = 0.0f;
    }
    return overflow;
}
