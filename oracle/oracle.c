/*
 * CPU oracle: plain-C restatement of the reference's FP64 force path.
 * TEST INFRASTRUCTURE ONLY -- see oracle.h for the rules it is used under.
 *
 * Compiled with -ffp-contract=off and without -mfma so that every expression
 * rounds exactly where the reference's does; parenthesisation below mirrors the
 * reference's C++ operator order (left to right).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* Softening (include/orrery/core/softening.hpp:83-100)                        */
/* ------------------------------------------------------------------------- */

static double softened_inverse_distance(double separation_squared, double eps2) {
    return 1.0 / sqrt(separation_squared + eps2);
}

static double softened_inverse_distance_cubed(double separation_squared, double eps2) {
    const double inverse = softened_inverse_distance(separation_squared, eps2);
    return (inverse * inverse) * inverse;
}

/* Softening stores the square of the length (softening.hpp:50-60). */
static double softening_squared(double length) { return length * length; }

/* ------------------------------------------------------------------------- */
/* Direct sum (direct_kernel_scalar.cpp:31-59, direct_solver.cpp:20-80)        */
/* ------------------------------------------------------------------------- */

static void accumulate_range(const double *x, const double *y, const double *z, const double *m,
                             double tx, double ty, double tz, size_t begin, size_t end,
                             double eps2, double out[3]) {
    double acc_x = 0.0, acc_y = 0.0, acc_z = 0.0;
    for (size_t j = begin; j < end; ++j) {
        const double dx = x[j] - tx;
        const double dy = y[j] - ty;
        const double dz = z[j] - tz;
        const double separation_squared = ((dx * dx) + (dy * dy)) + (dz * dz);
        const double factor = m[j] * softened_inverse_distance_cubed(separation_squared, eps2);
        acc_x = acc_x + (factor * dx);
        acc_y = acc_y + (factor * dy);
        acc_z = acc_z + (factor * dz);
    }
    out[0] = acc_x;
    out[1] = acc_y;
    out[2] = acc_z;
}

void oc_direct(size_t n, const double *x, const double *y, const double *z, const double *m,
               double softening, double *ax, double *ay, double *az, oc_counts *counts) {
    const double eps2 = softening_squared(softening);
    for (size_t i = 0; i < n; ++i) {
        double before[3], after[3];
        accumulate_range(x, y, z, m, x[i], y[i], z[i], 0, i, eps2, before);
        accumulate_range(x, y, z, m, x[i], y[i], z[i], i + 1, n, eps2, after);
        /* G = 1 (units.hpp:38): 1 * s is exact. */
        ax[i] = 1.0 * (before[0] + after[0]);
        ay[i] = 1.0 * (before[1] + after[1]);
        az[i] = 1.0 * (before[2] + after[2]);
    }
    if (counts != NULL) {
        counts->evaluations += 1;
        if (n > 1) {
            counts->particle_particle += (uint64_t)n * (uint64_t)(n - 1);
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Compensated reference (reference_kernel.cpp:31-104)                         */
/* ------------------------------------------------------------------------- */

typedef struct {
    double total;
    double correction;
} neumaier;

static void neumaier_add(neumaier *s, double term) {
    const double updated = s->total + term;
    if (fabs(s->total) >= fabs(term)) {
        s->correction = s->correction + ((s->total - updated) + term);
    } else {
        s->correction = s->correction + ((term - updated) + s->total);
    }
    s->total = updated;
}

static double neumaier_value(const neumaier *s) { return s->total + s->correction; }

void oc_reference_acceleration(size_t n, const double *x, const double *y, const double *z,
                               const double *m, size_t target, double softening, double out[3]) {
    const double tx = x[target], ty = y[target], tz = z[target];
    const double eps2 = softening_squared(softening);
    neumaier sx = {0, 0}, sy = {0, 0}, sz = {0, 0};
    for (size_t j = 0; j < n; ++j) {
        if (j == target) {
            continue;
        }
        const double dx = x[j] - tx;
        const double dy = y[j] - ty;
        const double dz = z[j] - tz;
        const double separation_squared = (((dx * dx) + (dy * dy)) + (dz * dz)) + eps2;
        const double inverse = 1.0 / sqrt(separation_squared);
        const double factor = ((m[j] * inverse) * inverse) * inverse;
        neumaier_add(&sx, factor * dx);
        neumaier_add(&sy, factor * dy);
        neumaier_add(&sz, factor * dz);
    }
    out[0] = 1.0 * neumaier_value(&sx);
    out[1] = 1.0 * neumaier_value(&sy);
    out[2] = 1.0 * neumaier_value(&sz);
}

/* ------------------------------------------------------------------------- */
/* Morton ordering (morton.cpp:60-197, morton.hpp:70-175)                      */
/* ------------------------------------------------------------------------- */

#define OC_MORTON_BITS 21u
#define OC_MORTON_GRID (1u << OC_MORTON_BITS)

void oc_bounding_cube(size_t n, const double *x, const double *y, const double *z,
                      double origin[3], double *size) {
    if (n == 0) {
        origin[0] = origin[1] = origin[2] = 0.0;
        *size = 0.0;
        return;
    }
    double lo[3] = {x[0], y[0], z[0]};
    double hi[3] = {x[0], y[0], z[0]};
    for (size_t i = 1; i < n; ++i) {
        /* std::min(a, b) returns a unless b < a; std::max(a, b) returns a unless a < b. */
        if (x[i] < lo[0]) lo[0] = x[i];
        if (y[i] < lo[1]) lo[1] = y[i];
        if (z[i] < lo[2]) lo[2] = z[i];
        if (hi[0] < x[i]) hi[0] = x[i];
        if (hi[1] < y[i]) hi[1] = y[i];
        if (hi[2] < z[i]) hi[2] = z[i];
    }
    const double ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
    /* std::max({ex, ey, ez}) keeps the first of equal maxima. */
    double s = ex;
    if (s < ey) s = ey;
    if (s < ez) s = ez;
    if (!(s > 0)) {
        s = 1.0;
    }
    for (int a = 0; a < 3; ++a) {
        const double centre = (lo[a] + hi[a]) / 2.0;
        origin[a] = centre - (s / 2.0);
    }
    *size = s;
}

uint64_t oc_spread_bits(uint32_t value) {
    uint64_t spread = value & 0x1fffffu;
    spread = (spread | (spread << 32)) & 0x1f00000000ffffull;
    spread = (spread | (spread << 16)) & 0x1f0000ff0000ffull;
    spread = (spread | (spread << 8)) & 0x100f00f00f00f00full;
    spread = (spread | (spread << 4)) & 0x10c30c30c30c30c3ull;
    spread = (spread | (spread << 2)) & 0x1249249249249249ull;
    return spread;
}

uint64_t oc_morton_code_grid(uint32_t gx, uint32_t gy, uint32_t gz) {
    return (oc_spread_bits(gx) << 2) | (oc_spread_bits(gy) << 1) | oc_spread_bits(gz);
}

static uint32_t to_grid(double coordinate, double origin, double scale) {
    const double cell = (coordinate - origin) * scale;
    if (!(cell > 0)) {
        return 0;
    }
    if (cell >= (double)OC_MORTON_GRID) {
        return OC_MORTON_GRID - 1;
    }
    return (uint32_t)cell;
}

uint64_t oc_morton_code(double px, double py, double pz, const double origin[3], double size) {
    if (!(size > 0)) {
        return 0;
    }
    const double scale = (double)OC_MORTON_GRID / size;
    return oc_morton_code_grid(to_grid(px, origin[0], scale), to_grid(py, origin[1], scale),
                               to_grid(pz, origin[2], scale));
}

unsigned oc_morton_octant(uint64_t code, unsigned level) {
    if (level == 0 || level > OC_MORTON_BITS) {
        return 0;
    }
    const unsigned shift = 3u * (OC_MORTON_BITS - level);
    return (unsigned)((code >> shift) & 7u);
}

typedef struct {
    uint64_t code;
    uint64_t index;
} oc_key;

static int key_compare(const void *a, const void *b) {
    const oc_key *ka = (const oc_key *)a;
    const oc_key *kb = (const oc_key *)b;
    if (ka->code != kb->code) return ka->code < kb->code ? -1 : 1;
    if (ka->index != kb->index) return ka->index < kb->index ? -1 : 1;
    return 0;
}

void oc_morton_order(size_t n, const double *x, const double *y, const double *z,
                     uint64_t *codes, uint64_t *indices, double origin[3], double *size) {
    oc_bounding_cube(n, x, y, z, origin, size);
    oc_key *keys = (oc_key *)malloc((n ? n : 1) * sizeof(oc_key));
    for (size_t i = 0; i < n; ++i) {
        keys[i].code = oc_morton_code(x[i], y[i], z[i], origin, *size);
        keys[i].index = i;
    }
    /* MortonKey's defaulted operator<=> orders by (code, index), a total order,
     * so any correct sort gives the reference's permutation (morton.hpp:155-175). */
    qsort(keys, n, sizeof(oc_key), key_compare);
    for (size_t i = 0; i < n; ++i) {
        codes[i] = keys[i].code;
        indices[i] = keys[i].index;
    }
    free(keys);
}

/* ------------------------------------------------------------------------- */
/* Octree (octree.cpp:41-387)                                                  */
/* ------------------------------------------------------------------------- */

typedef struct {
    size_t n;
    const double *x, *y, *z, *m;
    const uint64_t *codes;
    int quadrupole;
    uint64_t leaf_capacity;
    double opening_angle;
    oc_tree *tree;
    int failed;
} build_state;

static size_t push_node(build_state *s) {
    oc_tree *t = s->tree;
    if (t->node_count == t->capacity) {
        size_t grown = t->capacity ? t->capacity * 2 : 64;
        oc_node *nodes = (oc_node *)realloc(t->nodes, grown * sizeof(oc_node));
        if (nodes == NULL) {
            s->failed = 1;
            return 0;
        }
        t->nodes = nodes;
        if (s->quadrupole) {
            oc_quadrupole *q =
                (oc_quadrupole *)realloc(t->quadrupoles, grown * sizeof(oc_quadrupole));
            if (q == NULL) {
                s->failed = 1;
                return 0;
            }
            t->quadrupoles = q;
        }
        t->capacity = grown;
    }
    size_t self = t->node_count++;
    memset(&t->nodes[self], 0, sizeof(oc_node));
    if (s->quadrupole) {
        memset(&t->quadrupoles[self], 0, sizeof(oc_quadrupole));
    }
    return self;
}

/* octree.cpp:56-66 -- first index in [begin, end) whose octant at `level`
 * exceeds `octant` (std::partition_point over a sorted range). */
static size_t octant_end(const uint64_t *codes, size_t begin, size_t end, unsigned level,
                         unsigned octant) {
    size_t lo = begin, hi = end;
    while (lo < hi) {
        size_t mid = lo + (hi - lo) / 2;
        if (oc_morton_octant(codes[mid], level) <= octant) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    return lo;
}

/* octree.cpp:41-47 */
static void child_centre(const double c[3], double size, unsigned octant, double out[3]) {
    const double quarter = size / 4.0;
    out[0] = c[0] + ((octant & 4u) != 0 ? quarter : -quarter);
    out[1] = c[1] + ((octant & 2u) != 0 ? quarter : -quarter);
    out[2] = c[2] + ((octant & 1u) != 0 ? quarter : -quarter);
}

/* octree.cpp:75-84 */
static void add_displaced_moment(oc_quadrupole *q, double mass, double dx, double dy, double dz) {
    const double trace = mass * (((dx * dx) + (dy * dy)) + (dz * dz));
    q->xx = q->xx + ((((3.0 * mass) * dx) * dx) - trace);
    q->xy = q->xy + (((3.0 * mass) * dx) * dy);
    q->xz = q->xz + (((3.0 * mass) * dx) * dz);
    q->yy = q->yy + ((((3.0 * mass) * dy) * dy) - trace);
    q->yz = q->yz + (((3.0 * mass) * dy) * dz);
    q->zz = q->zz + ((((3.0 * mass) * dz) * dz) - trace);
}

/* octree.cpp:91-135 */
static void set_leaf_moments(build_state *s, size_t self) {
    oc_node *node = &s->tree->nodes[self];
    const size_t begin = node->first_particle;
    const size_t end = begin + node->particle_count;
    double mass = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
    for (size_t i = begin; i < end; ++i) {
        const double pm = s->m[i];
        mass = mass + pm;
        wx = wx + (s->x[i] * pm);
        wy = wy + (s->y[i] * pm);
        wz = wz + (s->z[i] * pm);
    }
    node->mass = mass;
    if (mass > 0) {
        node->com_x = wx / mass;
        node->com_y = wy / mass;
        node->com_z = wz / mass;
    } else {
        node->com_x = s->x[begin];
        node->com_y = s->y[begin];
        node->com_z = s->z[begin];
    }
    if (!s->quadrupole) {
        return;
    }
    oc_quadrupole *q = &s->tree->quadrupoles[self];
    memset(q, 0, sizeof(*q));
    for (size_t i = begin; i < end; ++i) {
        add_displaced_moment(q, s->m[i], s->x[i] - node->com_x, s->y[i] - node->com_y,
                             s->z[i] - node->com_z);
    }
}

/* octree.cpp:142-185 */
static void gather_moments(build_state *s, size_t index) {
    oc_node *nodes = s->tree->nodes;
    const size_t end = nodes[index].next;
    double mass = 0.0, wx = 0.0, wy = 0.0, wz = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
    size_t children = 0;
    for (size_t child = index + 1; child < end; child = nodes[child].next) {
        mass = mass + nodes[child].mass;
        wx = wx + (nodes[child].com_x * nodes[child].mass);
        wy = wy + (nodes[child].com_y * nodes[child].mass);
        wz = wz + (nodes[child].com_z * nodes[child].mass);
        mx = mx + nodes[child].com_x;
        my = my + nodes[child].com_y;
        mz = mz + nodes[child].com_z;
        ++children;
    }
    nodes[index].mass = mass;
    if (mass > 0) {
        nodes[index].com_x = wx / mass;
        nodes[index].com_y = wy / mass;
        nodes[index].com_z = wz / mass;
    } else {
        const double count = (double)(children == 0 ? 1 : children);
        nodes[index].com_x = mx / count;
        nodes[index].com_y = my / count;
        nodes[index].com_z = mz / count;
    }
    if (!s->quadrupole) {
        return;
    }
    oc_quadrupole moment;
    memset(&moment, 0, sizeof(moment));
    for (size_t child = index + 1; child < end; child = nodes[child].next) {
        const oc_quadrupole *cm = &s->tree->quadrupoles[child];
        moment.xx = moment.xx + cm->xx;
        moment.xy = moment.xy + cm->xy;
        moment.xz = moment.xz + cm->xz;
        moment.yy = moment.yy + cm->yy;
        moment.yz = moment.yz + cm->yz;
        moment.zz = moment.zz + cm->zz;
        add_displaced_moment(&moment, nodes[child].mass, nodes[child].com_x - nodes[index].com_x,
                             nodes[child].com_y - nodes[index].com_y,
                             nodes[child].com_z - nodes[index].com_z);
    }
    s->tree->quadrupoles[index] = moment;
}

/* octree.cpp:374-387 */
static double acceptance_radius_squared(double opening_angle, double size, double offset) {
    if (!(opening_angle > 0)) {
        return INFINITY;
    }
    const double radius = (size / opening_angle) + offset;
    return radius * radius;
}

/* octree.cpp:320-372 */
static void emit(build_state *s, size_t begin, size_t end, unsigned level, const double centre[3],
                 double size) {
    const size_t self = push_node(s);
    if (s->failed) return;
    const int leaf = (end - begin <= s->leaf_capacity) || level >= OC_MORTON_BITS;
    if (leaf) {
        s->tree->nodes[self].first_particle = begin;
        s->tree->nodes[self].particle_count = end - begin;
        set_leaf_moments(s, self);
        s->tree->leaf_count += 1;
        if (level > s->tree->depth) s->tree->depth = level;
        s->tree->nodes[self].next = s->tree->node_count;
    } else {
        const unsigned child_level = level + 1;
        size_t child_begin = begin;
        for (unsigned octant = 0; octant < 8; ++octant) {
            const size_t child_end = octant_end(s->codes, child_begin, end, child_level, octant);
            if (child_end > child_begin) {
                double cc[3];
                child_centre(centre, size, octant, cc);
                emit(s, child_begin, child_end, child_level, cc, size / 2.0);
                if (s->failed) return;
            }
            child_begin = child_end;
        }
        s->tree->nodes[self].next = s->tree->node_count;
        gather_moments(s, self);
    }
    oc_node *node = &s->tree->nodes[self];
    const double ox = node->com_x - centre[0];
    const double oy = node->com_y - centre[1];
    const double oz = node->com_z - centre[2];
    const double offset = sqrt(((ox * ox) + (oy * oy)) + (oz * oz));
    node->acceptance_radius_squared = acceptance_radius_squared(s->opening_angle, size, offset);
}

int oc_tree_build(size_t n, const double *sx, const double *sy, const double *sz,
                  const double *sm, const uint64_t *codes, const double origin[3], double size,
                  double opening_angle, uint64_t leaf_capacity, int quadrupole, oc_tree *tree) {
    memset(tree, 0, sizeof(*tree));
    /* corrected_parameters (octree.cpp:189-194). */
    if (opening_angle < 0) opening_angle = 0;
    if (opening_angle > 1) opening_angle = 1;
    if (leaf_capacity < 1) leaf_capacity = 1;
    tree->opening_angle = opening_angle;
    tree->leaf_capacity = leaf_capacity;
    if (n == 0) {
        return 0;
    }
    build_state s = {n, sx, sy, sz, sm, codes, quadrupole, leaf_capacity, opening_angle, tree, 0};
    /* BoundingCube::centre (morton.hpp:93-95): origin + size/2. */
    const double root_centre[3] = {origin[0] + (size / 2.0), origin[1] + (size / 2.0),
                                   origin[2] + (size / 2.0)};
    emit(&s, 0, n, 0, root_centre, size);
    return s.failed ? -1 : 0;
}

void oc_tree_free(oc_tree *tree) {
    free(tree->nodes);
    free(tree->quadrupoles);
    memset(tree, 0, sizeof(*tree));
}

/* ------------------------------------------------------------------------- */
/* Tree walk (tree_walk.cpp:20-83, tree_walk.hpp:129-181)                      */
/* ------------------------------------------------------------------------- */

void oc_walk(const oc_tree *tree, size_t n, const double *sx, const double *sy, const double *sz,
             const double *sm, size_t target, double softening, double out[3],
             uint64_t *pairs, uint64_t *cells) {
    (void)n;
    double acc_x = 0.0, acc_y = 0.0, acc_z = 0.0;
    out[0] = out[1] = out[2] = 0.0;
    if (tree->node_count == 0) {
        return;
    }
    const double eps2 = softening_squared(softening);
    const double px = sx[target], py = sy[target], pz = sz[target];
    size_t node = 0;
    while (node < tree->node_count) {
        const oc_node *cell = &tree->nodes[node];
        const double ox = cell->com_x - px;
        const double oy = cell->com_y - py;
        const double oz = cell->com_z - pz;
        const double d2 = ((ox * ox) + (oy * oy)) + (oz * oz);
        if (d2 >= cell->acceptance_radius_squared) {
            /* monopole_acceleration (tree_walk.hpp:129-139) */
            const double factor = cell->mass * softened_inverse_distance_cubed(d2, eps2);
            acc_x = acc_x + (ox * factor);
            acc_y = acc_y + (oy * factor);
            acc_z = acc_z + (oz * factor);
            if (tree->quadrupoles != NULL) {
                /* quadrupole_acceleration (tree_walk.hpp:156-181) */
                const oc_quadrupole *q = &tree->quadrupoles[node];
                const double inverse = softened_inverse_distance(d2, eps2);
                const double inv2 = inverse * inverse;
                const double inv5 = (inv2 * inv2) * inverse;
                const double inv7 = inv5 * inv2;
                const double cx = ((q->xx * ox) + (q->xy * oy)) + (q->xz * oz);
                const double cy = ((q->xy * ox) + (q->yy * oy)) + (q->yz * oz);
                const double cz = ((q->xz * ox) + (q->yz * oy)) + (q->zz * oz);
                const double quadratic = ((ox * cx) + (oy * cy)) + (oz * cz);
                const double scale = (2.5 * quadratic) * inv7;
                acc_x = acc_x + ((cx * -inv5) + (ox * scale));
                acc_y = acc_y + ((cy * -inv5) + (oy * scale));
                acc_z = acc_z + ((cz * -inv5) + (oz * scale));
            }
            *cells += 1;
            node = cell->next;
        } else if (cell->particle_count > 0) {
            const size_t begin = cell->first_particle;
            const size_t end = begin + cell->particle_count;
            double part[3];
            if (target >= begin && target < end) {
                accumulate_range(sx, sy, sz, sm, px, py, pz, begin, target, eps2, part);
                acc_x = acc_x + part[0];
                acc_y = acc_y + part[1];
                acc_z = acc_z + part[2];
                accumulate_range(sx, sy, sz, sm, px, py, pz, target + 1, end, eps2, part);
                acc_x = acc_x + part[0];
                acc_y = acc_y + part[1];
                acc_z = acc_z + part[2];
                *pairs += cell->particle_count - 1;
            } else {
                accumulate_range(sx, sy, sz, sm, px, py, pz, begin, end, eps2, part);
                acc_x = acc_x + part[0];
                acc_y = acc_y + part[1];
                acc_z = acc_z + part[2];
                *pairs += cell->particle_count;
            }
            node = cell->next;
        } else {
            node = node + 1;
        }
    }
    out[0] = acc_x;
    out[1] = acc_y;
    out[2] = acc_z;
}

int oc_barnes_hut(size_t n, const double *x, const double *y, const double *z, const double *m,
                  double softening, double opening_angle, uint64_t leaf_capacity, int quadrupole,
                  double *ax, double *ay, double *az, oc_counts *counts) {
    const size_t alloc = n ? n : 1;
    uint64_t *codes = (uint64_t *)malloc(alloc * sizeof(uint64_t));
    uint64_t *index = (uint64_t *)malloc(alloc * sizeof(uint64_t));
    double *sx = (double *)malloc(alloc * sizeof(double));
    double *sy = (double *)malloc(alloc * sizeof(double));
    double *sz = (double *)malloc(alloc * sizeof(double));
    double *sm = (double *)malloc(alloc * sizeof(double));
    int rc = 0;
    if (!codes || !index || !sx || !sy || !sz || !sm) {
        rc = -1;
        goto done;
    }
    double origin[3], size;
    oc_morton_order(n, x, y, z, codes, index, origin, &size);
    /* gather (barnes_hut_solver.cpp:41-62) */
    for (size_t i = 0; i < n; ++i) {
        sx[i] = x[index[i]];
        sy[i] = y[index[i]];
        sz[i] = z[index[i]];
        sm[i] = m[index[i]];
    }
    oc_tree tree;
    if (oc_tree_build(n, sx, sy, sz, sm, codes, origin, size, opening_angle, leaf_capacity,
                      quadrupole, &tree) != 0) {
        rc = -1;
        goto done;
    }
    uint64_t pairs = 0, cells = 0;
    for (size_t i = 0; i < n; ++i) {
        double a[3];
        oc_walk(&tree, n, sx, sy, sz, sm, i, softening, a, &pairs, &cells);
        ax[index[i]] = 1.0 * a[0];
        ay[index[i]] = 1.0 * a[1];
        az[index[i]] = 1.0 * a[2];
    }
    oc_tree_free(&tree);
    if (counts != NULL) {
        counts->evaluations += 1;
        counts->particle_particle += pairs;
        counts->particle_cell += cells;
    }
done:
    free(codes);
    free(index);
    free(sx);
    free(sy);
    free(sz);
    free(sm);
    return rc;
}

int oc_barnes_hut_targets(size_t n, const double *x, const double *y, const double *z,
                          const double *m, double softening, double opening_angle,
                          uint64_t leaf_capacity, int quadrupole, size_t count,
                          const uint64_t *targets, double *acc, uint64_t *pairs,
                          uint64_t *cells) {
    const size_t alloc = n ? n : 1;
    uint64_t *codes = (uint64_t *)malloc(alloc * sizeof(uint64_t));
    uint64_t *index = (uint64_t *)malloc(alloc * sizeof(uint64_t));
    uint64_t *where = (uint64_t *)malloc(alloc * sizeof(uint64_t));
    double *sx = (double *)malloc(alloc * sizeof(double));
    double *sy = (double *)malloc(alloc * sizeof(double));
    double *sz = (double *)malloc(alloc * sizeof(double));
    double *sm = (double *)malloc(alloc * sizeof(double));
    int rc = 0;
    if (!codes || !index || !where || !sx || !sy || !sz || !sm) {
        rc = -1;
        goto done;
    }
    double origin[3], size;
    oc_morton_order(n, x, y, z, codes, index, origin, &size);
    for (size_t i = 0; i < n; ++i) {
        sx[i] = x[index[i]];
        sy[i] = y[index[i]];
        sz[i] = z[index[i]];
        sm[i] = m[index[i]];
        where[index[i]] = i;
    }
    oc_tree tree;
    if (oc_tree_build(n, sx, sy, sz, sm, codes, origin, size, opening_angle, leaf_capacity,
                      quadrupole, &tree) != 0) {
        rc = -1;
        goto done;
    }
    for (size_t k = 0; k < count; ++k) {
        uint64_t p = 0, c = 0;
        oc_walk(&tree, n, sx, sy, sz, sm, where[targets[k]], softening, acc + 3 * k, &p, &c);
        pairs[k] = p;
        cells[k] = c;
    }
    oc_tree_free(&tree);
done:
    free(codes);
    free(index);
    free(where);
    free(sx);
    free(sy);
    free(sz);
    free(sm);
    return rc;
}

/* ------------------------------------------------------------------------- */
/* Integrators (velocity_verlet.cpp:20-72, yoshida4.cpp:24-59)                 */
/* ------------------------------------------------------------------------- */

static void kick(size_t n, double *v, const double *a, double scale) {
    for (size_t i = 0; i < n; ++i) v[i] = v[i] + (scale * a[i]);
}

static void drift(size_t n, double *p, const double *v, double scale) {
    for (size_t i = 0; i < n; ++i) p[i] = p[i] + (scale * v[i]);
}

void oc_vv_step_direct(size_t n, double *x, double *y, double *z, double *vx, double *vy,
                       double *vz, double *ax, double *ay, double *az, const double *m,
                       double softening, double dt, oc_counts *counts) {
    const double half = dt / 2.0;
    kick(n, vx, ax, half);
    kick(n, vy, ay, half);
    kick(n, vz, az, half);
    drift(n, x, vx, dt);
    drift(n, y, vy, dt);
    drift(n, z, vz, dt);
    oc_direct(n, x, y, z, m, softening, ax, ay, az, counts);
    kick(n, vx, ax, half);
    kick(n, vy, ay, half);
    kick(n, vz, az, half);
}

void oc_yoshida_weights(double *outer, double *inner) {
    const double cube_root_of_two = 1.2599210498948731647672106;
    *outer = 1.0 / (2.0 - cube_root_of_two);
    *inner = -cube_root_of_two / (2.0 - cube_root_of_two);
}

void oc_yoshida_step_direct(size_t n, double *x, double *y, double *z, double *vx, double *vy,
                            double *vz, double *ax, double *ay, double *az, const double *m,
                            double softening, double dt, oc_counts *counts) {
    double outer, inner;
    oc_yoshida_weights(&outer, &inner);
    oc_vv_step_direct(n, x, y, z, vx, vy, vz, ax, ay, az, m, softening, outer * dt, counts);
    oc_vv_step_direct(n, x, y, z, vx, vy, vz, ax, ay, az, m, softening, inner * dt, counts);
    oc_vv_step_direct(n, x, y, z, vx, vy, vz, ax, ay, az, m, softening, outer * dt, counts);
}

/* RungeKutta4::step (runge_kutta4.cpp:64-139) with the direct field: stages at
 * h/2, h/2 and h from the step's start (x0, v0), each moving the state to
 * x0 + s v and v0 + s a with the previous stage's v and a, derivative sums
 * weighted 1, 2, 2, 1, the state set to x0 + (h/6) S, and a last evaluation
 * so that the carried accelerations belong to the final positions. */
void oc_rk4_step_direct(size_t n, double *x, double *y, double *z, double *vx, double *vy,
                        double *vz, double *ax, double *ay, double *az, const double *m,
                        double softening, double dt, oc_counts *counts) {
    double *p[3] = {x, y, z}, *v[3] = {vx, vy, vz}, *a[3] = {ax, ay, az};
    double *start = malloc(sizeof(double) * 12 * (n ? n : 1));
    double *x0 = start, *v0 = start + 3 * n, *sx = start + 6 * n, *sv = start + 9 * n;
    for (int c = 0; c < 3; ++c) {
        for (size_t i = 0; i < n; ++i) {
            x0[c * n + i] = p[c][i];
            v0[c * n + i] = v[c][i];
            sx[c * n + i] = v[c][i];
            sv[c * n + i] = a[c][i];
        }
    }
    const double scales[3] = {dt / 2.0, dt / 2.0, dt};
    const double weights[3] = {2.0, 2.0, 1.0};
    for (int stage = 0; stage < 3; ++stage) {
        const double s = scales[stage];
        for (int c = 0; c < 3; ++c) {
            for (size_t i = 0; i < n; ++i) {
                const double stage_v = v[c][i];
                p[c][i] = x0[c * n + i] + (s * stage_v);
                v[c][i] = v0[c * n + i] + (s * a[c][i]);
            }
        }
        oc_direct(n, x, y, z, m, softening, ax, ay, az, counts);
        for (int c = 0; c < 3; ++c) {
            for (size_t i = 0; i < n; ++i) {
                sx[c * n + i] += weights[stage] * v[c][i];
                sv[c * n + i] += weights[stage] * a[c][i];
            }
        }
    }
    const double sixth = dt / 6.0;
    for (int c = 0; c < 3; ++c) {
        for (size_t i = 0; i < n; ++i) {
            p[c][i] = x0[c * n + i] + (sixth * sx[c * n + i]);
            v[c][i] = v0[c * n + i] + (sixth * sv[c * n + i]);
        }
    }
    oc_direct(n, x, y, z, m, softening, ax, ay, az, counts);
    free(start);
}

/* ------------------------------------------------------------------------- */
/* Energies (diagnostics.cpp:36-158)                                           */
/* ------------------------------------------------------------------------- */

double oc_kinetic_energy(size_t n, const double *vx, const double *vy, const double *vz,
                         const double *m) {
    neumaier sum = {0, 0};
    for (size_t i = 0; i < n; ++i) {
        neumaier_add(&sum, m[i] * (((vx[i] * vx[i]) + (vy[i] * vy[i])) + (vz[i] * vz[i])));
    }
    return neumaier_value(&sum) / 2.0;
}

double oc_potential_energy(size_t n, const double *x, const double *y, const double *z,
                           const double *m, double softening) {
    const double eps2 = softening_squared(softening);
    neumaier sum = {0, 0};
    for (size_t i = 0; i < n; ++i) {
        double interaction = 0.0;
        for (size_t j = i + 1; j < n; ++j) {
            const double dx = x[j] - x[i];
            const double dy = y[j] - y[i];
            const double dz = z[j] - z[i];
            interaction = interaction +
                          (m[j] * softened_inverse_distance(((dx * dx) + (dy * dy)) + (dz * dz),
                                                            eps2));
        }
        neumaier_add(&sum, (-1.0 * m[i]) * interaction);
    }
    return neumaier_value(&sum);
}
