/*
 * CPU oracle for the force-evaluation path: a plain-C restatement of the
 * reference's FP64 algorithms.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product (the `orrery_b200` package,
 * its CUDA library or its C ABI) links or calls this code. Only the tests, the
 * smoke check and the CPU-baseline leg of bench.py use it, and only as the
 * checker, never as the thing measured or shipped.
 *
 * Parity is pinned against the reference's own outputs: the recipe in
 * oracle/Makefile compiles the reference's CPU sources into oracle/_ref/, and
 * tests/test_oracle_pinning.py checks every function here bit-for-bit against
 * them (plus the reference tests' known-answer vectors).
 *
 * Every function names the reference file:line it restates. All arithmetic is
 * IEEE binary64 with no contraction (compiled with -ffp-contract=off), in the
 * same operation order as the reference, so results are bit-identical to the
 * reference's scalar kernels.
 */
#ifndef ORRERY_ORACLE_H
#define ORRERY_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* include/orrery/solvers/interaction_count.hpp:37-76 */
typedef struct oc_counts {
    uint64_t evaluations;
    uint64_t particle_particle;
    uint64_t particle_cell;
} oc_counts;

/* include/orrery/solvers/octree.hpp:104-139 (TreeNode), widened to fixed types. */
typedef struct oc_node {
    double mass;
    double com_x, com_y, com_z;
    double acceptance_radius_squared;
    uint64_t next;
    uint64_t first_particle;
    uint64_t particle_count;
} oc_node;

/* include/orrery/solvers/octree.hpp:89-96 */
typedef struct oc_quadrupole {
    double xx, xy, xz, yy, yz, zz;
} oc_quadrupole;

typedef struct oc_tree {
    oc_node *nodes;
    oc_quadrupole *quadrupoles; /* NULL unless built with quadrupoles */
    size_t node_count;
    size_t capacity;
    size_t leaf_count;
    unsigned depth;
    double opening_angle; /* after corrected_parameters */
    uint64_t leaf_capacity;
} oc_tree;

/* Direct O(N^2) sum, scalar kernel order (direct_solver.cpp:20-80,
 * direct_kernel_scalar.cpp:31-59). Writes a; adds N(N-1) pairs to counts. */
void oc_direct(size_t n, const double *x, const double *y, const double *z, const double *m,
               double softening, double *ax, double *ay, double *az, oc_counts *counts);

/* Compensated per-target FP64 sum (reference_kernel.cpp:58-104). */
void oc_reference_acceleration(size_t n, const double *x, const double *y, const double *z,
                               const double *m, size_t target, double softening, double out[3]);

/* Bounding cube (morton.cpp:60-104). */
void oc_bounding_cube(size_t n, const double *x, const double *y, const double *z,
                      double origin[3], double *size);

/* Bit dilation and interleave (morton.cpp:106-126). */
uint64_t oc_spread_bits(uint32_t value);
uint64_t oc_morton_code_grid(uint32_t gx, uint32_t gy, uint32_t gz);

/* Position to code (morton.cpp:128-164). */
uint64_t oc_morton_code(double px, double py, double pz, const double origin[3], double size);

/* Octant at a level (morton.cpp:166-178). */
unsigned oc_morton_octant(uint64_t code, unsigned level);

/* MortonOrdering::build (morton.cpp:180-197): codes and indices sorted by
 * (code, index). */
void oc_morton_order(size_t n, const double *x, const double *y, const double *z,
                     uint64_t *codes, uint64_t *indices, double origin[3], double *size);

/* Octree::build on particles already in Morton order (octree.cpp:196-468,
 * serial path). Returns 0 on success. Free with oc_tree_free. */
int oc_tree_build(size_t n, const double *sx, const double *sy, const double *sz,
                  const double *sm, const uint64_t *codes, const double origin[3], double size,
                  double opening_angle, uint64_t leaf_capacity, int quadrupole, oc_tree *tree);
void oc_tree_free(oc_tree *tree);

/* walk_tree for one sorted target (tree_walk.cpp:20-83), scalar leaves. */
void oc_walk(const oc_tree *tree, size_t n, const double *sx, const double *sy, const double *sz,
             const double *sm, size_t target, double softening, double out[3],
             uint64_t *pairs, uint64_t *cells);

/* BarnesHutSolver::evaluate (barnes_hut_solver.cpp:64-130) with the scalar
 * leaf kernel. Returns 0 on success. */
int oc_barnes_hut(size_t n, const double *x, const double *y, const double *z, const double *m,
                  double softening, double opening_angle, uint64_t leaf_capacity, int quadrupole,
                  double *ax, double *ay, double *az, oc_counts *counts);

/* BarnesHutSolver::evaluate restricted to some targets (original indices):
 * the full ordering and tree, then walk_tree for each listed target only.
 * Writes 3 accelerations and the pair and cell counts per target. */
int oc_barnes_hut_targets(size_t n, const double *x, const double *y, const double *z,
                          const double *m, double softening, double opening_angle,
                          uint64_t leaf_capacity, int quadrupole, size_t count,
                          const uint64_t *targets, double *acc, uint64_t *pairs,
                          uint64_t *cells);

/* velocity_verlet_step (velocity_verlet.cpp:59-72) with the direct field. */
void oc_vv_step_direct(size_t n, double *x, double *y, double *z, double *vx, double *vy,
                       double *vz, double *ax, double *ay, double *az, const double *m,
                       double softening, double dt, oc_counts *counts);

/* Yoshida4::step (yoshida4.cpp:45-59) with the direct field. */
void oc_yoshida_step_direct(size_t n, double *x, double *y, double *z, double *vx, double *vy,
                            double *vz, double *ax, double *ay, double *az, const double *m,
                            double softening, double dt, oc_counts *counts);

/* RungeKutta4::step (runge_kutta4.cpp:64-139) with the direct field. */
void oc_rk4_step_direct(size_t n, double *x, double *y, double *z, double *vx, double *vy,
                        double *vz, double *ax, double *ay, double *az, const double *m,
                        double softening, double dt, oc_counts *counts);

/* Yoshida-4 substep weights (yoshida4.cpp:24-30). */
void oc_yoshida_weights(double *outer, double *inner);

/* Energies (diagnostics.cpp:118-158). */
double oc_kinetic_energy(size_t n, const double *vx, const double *vy, const double *vz,
                         const double *m);
double oc_potential_energy(size_t n, const double *x, const double *y, const double *z,
                           const double *m, double softening);

#ifdef __cplusplus
}
#endif

#endif
