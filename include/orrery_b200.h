/*
 * orrery_b200 -- B200 (sm_100a) force-evaluation backend for the Orrery N-body
 * simulator, behind a plain C ABI.
 *
 * Conventions (the same ones the reference's kernel boundary uses:
 * include/orrery/solvers/cuda_kernels.hpp:102-111 returns cudaError_t and never
 * throws):
 *   - every function returns an int status, OB_OK on success;
 *   - ob_last_error() gives a message for the calling thread's last failure;
 *   - handles are opaque; arrays are plain pointers plus a count;
 *   - particle data is FP64 structure-of-arrays, like the reference's
 *     ParticleData (include/orrery/core/particle_data.hpp:43-149);
 *   - accelerations are written, never accumulated
 *     (include/orrery/integrators/acceleration_field.hpp:56-58).
 * No CUDA or torch type appears in a signature; streams are passed as void*.
 */
#ifndef ORRERY_B200_H
#define ORRERY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define OB_OK 0
#define OB_ERROR_INVALID_ARGUMENT 1
#define OB_ERROR_NO_DEVICE 2      /* no usable sm_100 device: the try_create -> null case */
#define OB_ERROR_OUT_OF_MEMORY 3
#define OB_ERROR_CUDA 4           /* a CUDA runtime error; the message names it */
#define OB_ERROR_TIMEOUT 5        /* a bounded device-side wait ran out */
#define OB_ERROR_CAPACITY 6       /* a size or budget limit was exceeded */
#define OB_ERROR_UNSUPPORTED 7
#define OB_ERROR_IO 8             /* a file could not be opened, written or read, or fails its
                                     format checks; the message names the file and the check */

/* Solver kinds: the reference's DirectSolver and BarnesHutSolver
 * (include/orrery/solvers/direct_solver.hpp:107,
 *  include/orrery/solvers/barnes_hut_solver.hpp:108). */
#define OB_SOLVER_DIRECT 0
#define OB_SOLVER_TREE 1

/* Arithmetic of the pair interactions.
 *   FP32  -- positions rounded to FP32, FP32 pair math (the plain kernel);
 *   SPLIT -- FP32 pair math on hi/lo-split FP64 positions, Kahan-compensated
 *            FP32 partials, FP64 tile accumulation (the precision form);
 *   FP64  -- FP64 pair math in the reference's order: bit-identical to the
 *            reference's scalar DirectSolver (direct solver only). */
#define OB_PRECISION_FP32 0
#define OB_PRECISION_SPLIT 1
#define OB_PRECISION_FP64 2

/* Integrators (src/integrators/velocity_verlet.cpp:59-72,
 * src/integrators/yoshida4.cpp:45-59, src/integrators/runge_kutta4.cpp:64-139).
 * RK4 takes four force evaluations a step; batches and the server run VV and
 * Yoshida-4. */
#define OB_INTEGRATOR_VV 0
#define OB_INTEGRATOR_YOSHIDA4 1
#define OB_INTEGRATOR_RK4 2

/* Solver parameters. Mirrors core::Softening (softening.hpp:50-60), which
 * stores the square of the softening length -- pass Softening::squared() so
 * FP64 results stay bit-identical -- and solvers::TreeParameters
 * (octree.hpp:147-191;
 * defaults theta 0.5, leaf 32, no quadrupole; corrected like
 * corrected_parameters, octree.cpp:189-194). */
typedef struct ob_solver_params {
    int32_t kind;           /* OB_SOLVER_* */
    int32_t precision;      /* OB_PRECISION_* */
    double softening_squared; /* epsilon^2 (>= 0) */
    double opening_angle;   /* theta, clamped to [0, 1] (tree only) */
    uint64_t leaf_capacity; /* at least 1 (tree only) */
    int32_t quadrupole;     /* nonzero: carry traceless quadrupoles (tree only) */
    int32_t reserved;
} ob_solver_params;

/* solvers::InteractionCount (interaction_count.hpp:37-76). */
typedef struct ob_counts {
    uint64_t evaluations;
    uint64_t particle_particle;
    uint64_t particle_cell;
} ob_counts;

/* Device-timed phases of the last evaluation, in milliseconds (CUDA events);
 * the counterpart of EvaluationTimings / CudaTreeTimings
 * (barnes_hut_solver.hpp:92-105, cuda_tree_solver.hpp:81-117). */
typedef struct ob_timings {
    double transfer_in_ms;  /* host -> device copies (host entry points only) */
    double ordering_ms;     /* cube, Morton encode, radix sort, gather */
    double construction_ms; /* octree layout and moments */
    double traversal_ms;    /* the force kernel (direct sum or walk) */
    double transfer_out_ms; /* device -> host copies (host entry points only) */
} ob_timings;

/* Library information and errors. */
const char *ob_version(void);
const char *ob_last_error(void);
int ob_device_count(int *count);

/* ------------------------------------------------------------------------ */
/* Solver: the ForceSolver drop-in                                           */
/* ------------------------------------------------------------------------ */
typedef struct ob_solver ob_solver;

/* Replaces CudaDirectSolver::try_create / CudaTreeSolver::try_create
 * (src/solvers/cuda_direct_solver.cpp:140-164, cuda_tree_solver.cpp:205-221):
 * returns OB_ERROR_NO_DEVICE (and *out = NULL) when no usable device exists. */
int ob_solver_create(const ob_solver_params *params, ob_solver **out);
void ob_solver_destroy(ob_solver *solver);
int ob_solver_get_params(const ob_solver *solver, ob_solver_params *params);

/* Replaces ForceSolver::evaluate on host spans
 * (include/orrery/integrators/acceleration_field.hpp:56-58): synchronous,
 * host FP64 SoA in, accelerations written to host FP64 SoA. n may be 0. */
int ob_solver_evaluate(ob_solver *solver, uint64_t n, const double *x, const double *y,
                       const double *z, const double *m, double *ax, double *ay, double *az);

/* The same evaluation on device-resident FP64 arrays, enqueued on `stream`
 * (a cudaStream_t, NULL = the default stream) without synchronising. Replaces
 * launch_cuda_direct / launch_cuda_tree (cuda_kernels.hpp:111,228). */
int ob_solver_evaluate_device(ob_solver *solver, uint64_t n, const double *x, const double *y,
                              const double *z, const double *m, double *ax, double *ay,
                              double *az, void *stream);

/* ForceSolver::interaction_count / reset_interaction_count
 * (force_solver.hpp:64-76). Tree counts are read back when asked for. */
int ob_solver_counts(ob_solver *solver, ob_counts *counts);
int ob_solver_reset_counts(ob_solver *solver);
int ob_solver_timings(const ob_solver *solver, ob_timings *timings);

/* Inspection of the last tree evaluation: the Morton order and the octree as
 * the reference lays them out (MortonOrdering::keys, Octree::nodes /
 * quadrupoles / leaf_count / depth; include/orrery/solvers/morton.hpp:182-210,
 * octree.hpp:208-248). Synchronous; for tests and tools. */
int ob_tree_stats(ob_solver *solver, uint64_t *nodes, uint64_t *leaves, uint32_t *depth);

/* reals: 5 doubles per node (mass, centre of mass x y z, acceptance radius^2);
 * idx: 3 per node (next, first particle, particle count); quads: 6 per node
 * (xx xy xz yy yz zz) or NULL. Arrays must hold ob_tree_stats' node count. */
int ob_tree_copy(ob_solver *solver, double *reals, uint64_t *idx, double *quads);

/* codes and indices of the sorted keys (n each), the cube origin (3) and size. */
int ob_tree_copy_order(ob_solver *solver, uint64_t *codes, uint32_t *indices, double *origin,
                       double *size);

/* Morton ordering (codes sorted ascending with their particle indices) of n
 * particles whose FP64 positions are in device memory, written to the
 * caller's device arrays codes[n] and indices[n], enqueued on `stream`
 * without synchronising. It allocates nothing: for callers that cannot
 * allocate device memory when they need an ordering -- services that take
 * device memory only from their own fixed pool, or that must not grow or
 * fragment the device heap once running. (Like every entry point here it
 * makes CUDA calls, so it must not be called from a stream or host callback.)
 * Every intermediate buffer lives in one fixed device array of about 17 MB
 * that each device holds from the library's loading until the process exits;
 * n above 1,048,576 is refused with OB_ERROR_CAPACITY. The first call on a
 * device looks up that array's device address, so make it before any stream
 * capture. All calls share the one array: calls whose work overlaps on the
 * GPU race and must be ordered by the caller.
 * status: a device word (or NULL) that receives, on the stream after the
 * ordering, 0 when it completed or a nonzero value when a bounded device wait
 * ran out (OB_DEVICE_STATUS_TIMEOUT): the outputs are then incomplete and
 * must not be used. With NULL such a failure cannot be detected.
 * No counterpart in the reference (its MortonOrdering allocates on the host). */
#define OB_DEVICE_STATUS_TIMEOUT 1u
int ob_morton_order_noalloc(uint64_t n, const double *x, const double *y, const double *z,
                            uint64_t *codes, uint32_t *indices, uint32_t *status,
                            void *stream);

/* Tile shape of the direct kernels: threads per CTA, targets per thread, the
 * number of CTAs (one thread-block cluster) that split the sources of a
 * target tile, and the number of thread groups of a CTA that split each
 * staged tile's sources (each group serves the CTA's targets; 0 reads as 1).
 * A CTA holds threads * targets_per_thread / groups targets. No reference
 * counterpart: the reference picks one block size
 * (src/solvers/cuda_direct_solver.cpp:46-63). */
typedef struct ob_direct_shape {
    int32_t threads;
    int32_t targets_per_thread;
    int32_t split;
    int32_t groups;
} ob_direct_shape;

/* Lists the shapes the library implements for a precision (FP32 or SPLIT);
 * *count receives the total even when it exceeds capacity. */
int ob_direct_shapes(int32_t precision, ob_direct_shape *out, int32_t capacity, int32_t *count);

/* Fixes the shape a direct solver uses for n particles. */
int ob_solver_set_direct_shape(ob_solver *solver, uint64_t n, const ob_direct_shape *shape);

/* Times every implemented shape on the device for n synthetic particles and
 * keeps the fastest for n; returns it and its time per evaluation. */
int ob_solver_autotune(ob_solver *solver, uint64_t n, ob_direct_shape *chosen, double *best_ms);

/* ------------------------------------------------------------------------ */
/* System: particle state resident in HBM, integrated on the device          */
/* ------------------------------------------------------------------------ */
typedef struct ob_system ob_system;

/* A system of n particles with its own solver. The state is FP64 SoA in HBM
 * and stays there between steps. */
int ob_system_create(const ob_solver_params *params, uint64_t n, ob_system **out);
void ob_system_destroy(ob_system *system);

/* Uploads positions, velocities and masses (velocities may be NULL = zero)
 * and evaluates the accelerations, as sim::Simulation's constructor does
 * (src/sim/simulation.cpp:16-27). */
int ob_system_set_state(ob_system *system, const double *x, const double *y, const double *z,
                        const double *vx, const double *vy, const double *vz, const double *m);

/* Overwrites the carried accelerations (as a restored checkpoint does). */
int ob_system_set_accelerations(ob_system *system, const double *ax, const double *ay,
                                const double *az);

/* Downloads any of the arrays (NULL pointers are skipped). */
int ob_system_get_state(ob_system *system, double *x, double *y, double *z, double *vx,
                        double *vy, double *vz, double *ax, double *ay, double *az);

/* Advances `steps` steps of the integrator with timestep dt (Integrator::step,
 * integrator.hpp:65), entirely on the device; one step is replayed from a CUDA
 * graph. Synchronous. */
int ob_system_step(ob_system *system, int32_t integrator, double dt, uint64_t steps);

/* The same, enqueued without waiting (sync with ob_system_synchronize). */
int ob_system_step_async(ob_system *system, int32_t integrator, double dt, uint64_t steps);

/* Integrator::step over host-resident particle data (integrator.hpp:65 with
 * ParticleData, include/orrery/core/particle_data.hpp): uploads positions,
 * velocities, carried accelerations and masses (all required), advances
 * `steps` steps on the device and writes positions, velocities and
 * accelerations back into the same arrays. Synchronous; no force evaluation
 * beyond the steps' own (the accelerations passed in are those the previous
 * step left, as the reference's integrators carry them). */
int ob_system_step_host(ob_system *system, int32_t integrator, double dt, uint64_t steps,
                        double *x, double *y, double *z, double *vx, double *vy, double *vz,
                        double *ax, double *ay, double *az, const double *m);
int ob_system_synchronize(ob_system *system);

/* Energies in FP64 on the device (core::kinetic_energy / potential_energy,
 * src/core/diagnostics.cpp:118-158); the O(N^2) potential uses the system's
 * softening. Either pointer may be NULL. */
int ob_system_energy(ob_system *system, double *kinetic, double *potential);

/* core::Diagnostics (include/orrery/core/diagnostics.hpp:52-82). */
typedef struct ob_diagnostics {
    double kinetic_energy;
    double potential_energy;
    double linear_momentum[3];
    double angular_momentum[3];
} ob_diagnostics;

/* core::measure_diagnostics (src/core/diagnostics.cpp:179-200) of the
 * system's current state: the energies as ob_system_energy computes them, and
 * the momenta as compensated sums in index order, bit-identical to the
 * reference's. Waits for the enqueued steps. */
int ob_system_diagnostics(ob_system *system, ob_diagnostics *out);

/* The device addresses of the system's ten FP64 state arrays, each of n
 * doubles: x y z vx vy vz ax ay az m (NULL when n is 0), for zero-copy views
 * (e.g. DLPack or __cuda_array_interface__). They stay valid until the
 * system is destroyed. Work on them from another stream is ordered against the
 * system's steps by the caller (ob_system_synchronize, or events on
 * ob_system_stream). */
int ob_system_device_arrays(ob_system *system, void **arrays);

/* The whole state, masses included, in a checkpoint's order (after the
 * enqueued steps; waits for them). */
int ob_system_snapshot(ob_system *system, double *m, double *x, double *y, double *z,
                       double *vx, double *vy, double *vz, double *ax, double *ay, double *az);

/* Installs a state whose accelerations already belong to its positions, as
 * sim::Simulation::restore with accelerations_are_current
 * (include/orrery/sim/simulation.hpp:101-102): no force evaluation. */
int ob_system_restore(ob_system *system, const double *m, const double *x, const double *y,
                      const double *z, const double *vx, const double *vy, const double *vz,
                      const double *ax, const double *ay, const double *az);

/* The stream the system's work is enqueued on (a cudaStream_t), for callers
 * that order their own work or events after it. */
int ob_system_stream(ob_system *system, void **stream);

/* Per-phase device timing inside graph replays: the next `steps` steps record
 * CUDA events around each evaluation's phases (0 turns it off).
 * ob_system_phase_times then gives the per-evaluation average of each phase
 * (ordering, construction, traversal) over the recorded steps, and the number
 * of evaluations averaged. Synchronises. */
int ob_system_profile(ob_system *system, uint32_t steps);
int ob_system_phase_times(ob_system *system, ob_timings *average, uint32_t *evaluations);

/* Kernel launches one step of the integrator makes (kernel nodes of the
 * captured step graph). */
int ob_system_step_kernels(ob_system *system, int32_t integrator, double dt, uint32_t *kernels);

/* Runs ob_solver_autotune for the system's direct solver at its size and uses
 * the chosen shape from the next step on (the step graph is captured again). */
int ob_system_autotune(ob_system *system, ob_direct_shape *chosen, double *best_ms);

/* Whole steps of a small system in one launch: with the FP32 direct field,
 * softening and velocity Verlet or Yoshida-4, a system whose sources fit one
 * CTA's shared memory (a few thousand particles) takes its steps -- kicks,
 * drifts and every force evaluation -- in a single cooperative kernel instead
 * of four launches per substep (on by default). The forces are the FP32
 * direct kernel's arithmetic with its own summation order (within its
 * bounds of the FP64 forces); the kicks and drifts are bit-identical.
 * enable = 0 turns it off for this system; *active (may be NULL) tells
 * whether the next velocity-Verlet step will use it. No reference
 * counterpart (the reference launches per evaluation). */
int ob_system_set_fused_steps(ob_system *system, int32_t enable, int32_t *active);

int ob_system_counts(ob_system *system, ob_counts *counts);
int ob_system_size(const ob_system *system, uint64_t *n);

/* ------------------------------------------------------------------------ */
/* Run output: checkpoints and trajectories in the reference's formats       */
/* ------------------------------------------------------------------------ */
/* ORRERYCK v1 checkpoints (sim::write_checkpoint / sim::read_checkpoint,
 * include/orrery/sim/checkpoint.hpp:85-94) and ORRERYTJ v1 trajectories
 * (sim::TrajectoryWriter, include/orrery/sim/trajectory.hpp:112-146), byte for
 * byte as the reference's double-precision build writes them, so that its
 * `orrery resume` and `orrery show` read these files and it writes files these
 * calls read. The configuration a checkpoint carries is the caller's text in
 * the reference's configuration format (sim::write_configuration); it is
 * stored and returned unparsed. A checkpoint is written to "<path>.partial"
 * and renamed over <path>. Failures are OB_ERROR_IO. */

/* A checkpoint from host arrays (n of each): masses, positions, velocities,
 * accelerations, taken after `step` steps. */
int ob_checkpoint_write(const char *path, uint64_t step, const char *configuration,
                        uint64_t configuration_bytes, uint64_t n, const double *m,
                        const double *x, const double *y, const double *z, const double *vx,
                        const double *vy, const double *vz, const double *ax, const double *ay,
                        const double *az);
/* A checkpoint's header: step, particle count, configuration length. */
int ob_checkpoint_info(const char *path, uint64_t *step, uint64_t *n,
                       uint64_t *configuration_bytes);
/* Reads a whole checkpoint of n particles and checks it (magic, version,
 * flags, sizes, checksum); `configuration` (NULL to skip) receives the text. */
int ob_checkpoint_read(const char *path, char *configuration, uint64_t configuration_capacity,
                       uint64_t n, double *m, double *x, double *y, double *z, double *vx,
                       double *vy, double *vz, double *ax, double *ay, double *az);
/* A checkpoint of a device-resident system's state as it stands after the
 * steps already enqueued (waits for them). */
int ob_system_write_checkpoint(ob_system *system, const char *path, uint64_t step,
                               const char *configuration, uint64_t configuration_bytes);
/* Restores a system of the checkpoint's size to the stored state, the
 * carried accelerations included (as sim::Simulation::restore with
 * accelerations_are_current, include/orrery/sim/simulation.hpp:101-102), so
 * that a resumed run continues bit for bit; returns the step and the text. */
int ob_system_read_checkpoint(ob_system *system, const char *path, uint64_t *step,
                              char *configuration, uint64_t configuration_capacity,
                              uint64_t *configuration_bytes);

typedef struct ob_trajectory ob_trajectory;

/* A trajectory file of n particles: the header (masses, timestep, whether
 * frames carry velocities) is written here. */
int ob_trajectory_create(const char *path, uint64_t n, const double *masses, double timestep,
                         int32_t with_velocities, ob_trajectory **out);
/* The same for a device-resident system (its masses). Its frames can then
 * be snapshots of the system taken on the device between steps and written
 * by a background thread (ob_trajectory_write_system_frame). Close the
 * trajectory before destroying the system. */
int ob_trajectory_create_for_system(const char *path, ob_system *system, double timestep,
                                    int32_t with_velocities, ob_trajectory **out);
/* A frame from host arrays (velocities ignored when the file has none). */
int ob_trajectory_write_frame(ob_trajectory *trajectory, uint64_t step, double time,
                              const double *x, const double *y, const double *z,
                              const double *vx, const double *vy, const double *vz);
/* A frame of the bound system's state at this point of its stream: a
 * device-to-device copy enqueued between the steps; returns without waiting
 * for the file (at most two frames in flight; a third waits for one). */
int ob_trajectory_write_system_frame(ob_trajectory *trajectory, uint64_t step, double time);
/* Waits until every frame given so far is in the file and flushes it; returns
 * the first failure of any of them. */
int ob_trajectory_flush(ob_trajectory *trajectory);
int ob_trajectory_frames(ob_trajectory *trajectory, uint64_t *frames);
/* Flushes, closes and frees (returns the flush's status). */
int ob_trajectory_close(ob_trajectory *trajectory);

/* ------------------------------------------------------------------------ */
/* Batch: many independent systems integrated together                       */
/* ------------------------------------------------------------------------ */
/* No reference counterpart: the reference integrates one system per
 * Simulation with one Softening per solver. A batch holds `systems` systems
 * of uneven size, each with its own squared softening (> 0), in HBM; one
 * persistent launch evaluates all their direct sums (precision form: split
 * FP32 pair arithmetic, FP64 accumulation) from a largest-first work queue of
 * (system, target tile, source chunk) items, and a step of all systems is one
 * replayed CUDA graph. */
typedef struct ob_batch ob_batch;

typedef struct ob_batch_shape {
    int32_t threads;
    int32_t targets_per_thread;
    uint32_t chunk_tiles; /* 512-source tiles per work item; 0 = a whole system */
    int32_t groups;       /* thread groups splitting each tile's sources; 0 reads as 1 */
} ob_batch_shape;

int ob_batch_create(uint32_t systems, const uint64_t *counts, const double *softening_squared,
                    ob_batch **out);
void ob_batch_destroy(ob_batch *batch);
int ob_batch_set_state(ob_batch *batch, uint32_t system, const double *x, const double *y,
                       const double *z, const double *vx, const double *vy, const double *vz,
                       const double *m);
int ob_batch_get_state(ob_batch *batch, uint32_t system, double *x, double *y, double *z,
                       double *vx, double *vy, double *vz, double *ax, double *ay, double *az);
/* Evaluates every system's accelerations from its positions (after set_state). */
int ob_batch_refresh(ob_batch *batch);
int ob_batch_step(ob_batch *batch, int32_t integrator, double dt, uint64_t steps);
int ob_batch_step_async(ob_batch *batch, int32_t integrator, double dt, uint64_t steps);
int ob_batch_synchronize(ob_batch *batch);
int ob_batch_energy(ob_batch *batch, uint32_t system, double *kinetic, double *potential);
/* Times the implemented shapes on this batch and keeps the fastest. */
int ob_batch_autotune(ob_batch *batch, ob_batch_shape *chosen, double *best_ms);
int ob_batch_set_shape(ob_batch *batch, const ob_batch_shape *shape);
/* Pair interactions of one evaluation of all systems (sum of N(N-1)),
 * evaluations so far, and work items per evaluation. */
int ob_batch_stats(ob_batch *batch, uint64_t *pairs_per_evaluation, uint64_t *evaluations,
                   uint32_t *items);
int ob_batch_stream(ob_batch *batch, void **stream);

/* ------------------------------------------------------------------------ */
/* Server: a persistent request loop with continuous batching                */
/* ------------------------------------------------------------------------ */
/* Replaces the reference service's one-CLI-process-per-job worker
 * (service/orrery_service/worker.py:262-300) and its concurrency and work
 * limits (service/orrery_service/limits.py:38-167) for the force path: jobs
 * are admitted from per-solver FIFO queues while their device memory fits the
 * HBM budget and the direct work per step stays under a cap; each job's state
 * stays on the device; all direct jobs with the same integrator and timestep
 * step together in one batched launch (members join and leave between
 * steps); each tree job steps on its own stream, overlapping the batch. */
typedef struct ob_server ob_server;

typedef struct ob_server_config {
    uint64_t hbm_budget_bytes;       /* device memory the jobs may hold */
    uint64_t direct_pairs_cap;       /* max sum N(N-1) of running direct jobs (0: none) */
    uint64_t direct_arena_particles; /* padded particles per direct batch arena */
    uint32_t max_tree_jobs;          /* tree jobs running at once */
    int32_t fake_device;             /* nonzero: no GPU; steps take modelled time */
    double fake_direct_gint_s;       /* fake mode: direct interactions per second / 1e9 */
    double fake_tree_ns_per_particle;/* fake mode: tree step time per particle */
    double max_job_work;             /* per-job ceiling in ob_work_units (0: none); above it a
                                        job is refused (OB_ERROR_CAPACITY) */
    double max_running_work;         /* max ob_work_units of the running jobs together (0:
                                        none); a job alone always runs */
} ob_server_config;

typedef struct ob_job_spec {
    int32_t kind;              /* OB_SOLVER_DIRECT (precision form) or OB_SOLVER_TREE */
    int32_t integrator;        /* OB_INTEGRATOR_* */
    uint64_t n;
    uint64_t steps;
    double dt;
    double softening_squared;
    double opening_angle;      /* tree jobs */
    uint64_t leaf_capacity;    /* tree jobs */
    int32_t quadrupole;        /* tree jobs */
    int32_t reserved;
} ob_job_spec;

#define OB_JOB_QUEUED 0
#define OB_JOB_RUNNING 1
#define OB_JOB_DONE 2
#define OB_JOB_FAILED 3
#define OB_JOB_CANCELLED 4
#define OB_JOB_REJECTED 5

typedef struct ob_job_report {
    uint64_t id;
    int32_t status;            /* OB_JOB_* */
    int32_t reserved;
    uint64_t steps_done;
    double submitted_s;        /* seconds since the server started */
    double admitted_s;
    double finished_s;
} ob_job_report;

typedef struct ob_server_summary {
    uint64_t submitted, admitted, completed, failed, cancelled, rejected;
    uint64_t queued, running;
    double elapsed_s;
    double jobs_per_s;                 /* completed / elapsed */
    double job_latency_p50_s, job_latency_p99_s;   /* finish - submit, completed jobs */
    double step_latency_p50_ms, step_latency_p99_ms; /* per advanced step, all jobs */
    uint64_t hbm_in_use, hbm_peak;
} ob_server_summary;

int ob_server_create(const ob_server_config *config, ob_server **out);
/* The reference service's cost of a run (work_units,
 * service/orrery_service/limits.py:82-111): count^2 * steps for the direct
 * solver (kind OB_SOLVER_DIRECT), count * log2(count) * steps for the tree; 0
 * below two particles. */
double ob_work_units(uint64_t count, uint64_t steps, int32_t kind);
/* Stops the loop (running jobs are cancelled) and frees everything. */
void ob_server_destroy(ob_server *server);
/* Copies the initial state (vx..vz may be NULL = zero); returns the job id. A
 * job that can never fit the budget is rejected (OB_ERROR_CAPACITY). */
int ob_server_submit(ob_server *server, const ob_job_spec *spec, const double *x,
                     const double *y, const double *z, const double *vx, const double *vy,
                     const double *vz, const double *m, uint64_t *job_id);
/* Waits up to timeout_s for the job to end (OB_ERROR_TIMEOUT otherwise), then
 * fills the report and any non-NULL output arrays (n each). A timeout that is
 * negative or NaN waits not at all; one above 1e9 s (infinity included) waits
 * 1e9 s. */
int ob_server_wait(ob_server *server, uint64_t job_id, double timeout_s, ob_job_report *report,
                   double *x, double *y, double *z, double *vx, double *vy, double *vz,
                   double *ax, double *ay, double *az);
int ob_server_cancel(ob_server *server, uint64_t job_id);
int ob_server_stats(ob_server *server, ob_server_summary *stats);
/* Waits until no job is queued or running (OB_ERROR_TIMEOUT otherwise); the
 * timeout as for ob_server_wait. */
int ob_server_drain(ob_server *server, double timeout_s);

/* Measured FP32 FFMA and SFU rsqrt lane operations per second on the current
 * device: the denominators of the direct kernel's roofline. No reference
 * counterpart in the library (the reference's probes are benchmark code,
 * benchmarks/cuda_probes.cu:15-115). */
int ob_probe_fp32(double *ffma_lane_per_s, double *rsqrt_lane_per_s);

/* Measured FMAs per second through packed FP32x2 FMA instructions (each
 * counts as two), for comparison with the scalar FFMA rate. */
int ob_probe_fp32x2(double *ffma2_flop_lanes_per_s);

/* Measured FP64 FMA lane operations per second on the current device: the
 * denominator of the FP64 (parity-mode) tree walk's roofline. */
int ob_probe_fp64(double *dfma_lane_per_s);

/* ------------------------------------------------------------------------ */
/* Test support: failure paths driven without faulting the device            */
/* ------------------------------------------------------------------------ */
/* Runs one onesweep radix-sort pass over n (<= 2^24) synthetic keys with its
 * own buffers, its tiles polling a predecessor's look-back word at most
 * poll_limit times. With skip_first_tile nonzero no CTA takes the first tile,
 * whose words therefore are never published: the waits run out, the pass sets
 * its timeout bit and OB_ERROR_TIMEOUT is returned, the device staying usable.
 * Otherwise the pass must complete and sort (OB_OK). Exercises the bounded
 * look-back wait of the Morton ordering; no reference counterpart. */
int ob_test_lookback_timeout(uint64_t n, uint32_t poll_limit, int skip_first_tile);

/* Bounds the FP32 tree walk's per-warp traversal stack of `solver` to `cap`
 * entries (0 restores the full 256) from its next evaluation on. A warp whose
 * stack fills discards its partial sums and finishes with the per-target
 * union walk (the fallback a valid tree rarely needs); a small cap forces it,
 * so tests can hold that path to the oracle. OB_ERROR_UNSUPPORTED for direct
 * or FP64 solvers. No reference counterpart. */
int ob_test_set_walk_stack_cap(ob_solver *solver, uint32_t cap);

/* Arms the next fused launch of `system` (ob_system_set_fused_steps) for a
 * test of its bounded wait: that launch polls each ready word at most
 * `poll_limit` times and its first CTA never publishes its positions, so the
 * other CTAs' waits run out, the launch sets its timeout bit and the step
 * returns OB_ERROR_TIMEOUT, the device staying usable; the launch after it
 * clears the ready words and steps normally. OB_ERROR_UNSUPPORTED when the
 * system does not take fused steps. No reference counterpart. */
int ob_test_fused_timeout(ob_system *system, uint32_t poll_limit);

#ifdef __cplusplus
}
#endif

#endif /* ORRERY_B200_H */
