/* swl_b200 -- B200-native curvilinear velocity-stress engine, C ABI.
 *
 * Drop-in compute backend for SeisWave Lab (Curvilinear).  Two levels:
 *
 *  - Engine level: replaces the reference's private CUDA engines.  The caller builds the
 *    model arrays exactly as the reference's Simulation::initialize does and hands them
 *    over as a mesh; the engine copies them to the GPU and advances RK4 steps there.
 *      2D: Seis2D::Curvilinear::CudaEngine        (src/two_d/CudaEngine2D.hpp:5-24)
 *      3D: Seis3D::Curvilinear::CudaEngine3D      (src/three_d/CudaEngine3D.hpp:7-24)
 *  - Session level: the whole Simulation (model build from parameters, dt plan, receivers,
 *    records, fault policy) with the engine underneath.
 *      2D: Seis2D::Curvilinear::Simulation        (include/Seis2D/CurvilinearSolver2D.hpp:93-123)
 *      3D: Seis3D::Curvilinear::ISimulationBackend3D (include/Seis3D/CurvilinearSolver.hpp:165-185)
 *
 * Conventions: every call returns an swl_status (0 = success) and never throws across this
 * boundary; the message of the last failure on the calling thread is available from
 * swl_last_error().  A failed step leaves a sticky fault (the reference's `fault` string)
 * that only reset or rebuild clears.  An engine is driven by one thread at a time.
 * Arrays are padded (ghost width 3), x fastest, structure of arrays.
 */
#ifndef SWL_B200_H
#define SWL_B200_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t swl_status;
enum {
    SWL_OK = 0,
    SWL_ERR_INVALID = -1,     /* bad argument or configuration */
    SWL_ERR_CUDA = -2,        /* CUDA runtime failure (message names the action) */
    SWL_ERR_MEMORY = -3,      /* allocation refused or over the memory budget */
    SWL_ERR_FAULT = -4,       /* step rejected (non-finite or energy growth); sticky */
    SWL_ERR_UNAVAILABLE = -5, /* no usable sm_100 device */
    SWL_ERR_STATE = -6        /* call out of order, or refused while an earlier rejected step is held */
};
enum { SWL_FP64 = 0, SWL_FP32 = 1 };

/* Message of the last failed call on this thread ("" when none). */
const char *swl_last_error(void);
/* Library version string. */
const char *swl_version(void);
/* Number of usable sm_100 devices (0 when none); mirrors queryBackend3D
 * (src/common/ComputeDevices.cpp:98-102). */
int32_t swl_device_count(void);

/* ---------------------------------------------------------------- engine, 2D ---- */

/* POD mirror of Point::MeshT<Real> (src/two_d/PointKernels2D.hpp:14-27).  `array_precision`
 * says whether the pointers reference double or float arrays (the reference converts its
 * StoredArrays before building the mesh); `precision` selects the compute precision.
 * Non-owning: the engine copies everything at create. */
typedef struct swl_mesh2d {
    int32_t nx, nz;  /* padded node counts (computational + 6) */
    int64_t count;   /* nx * nz */
    double h;
    const void *a, *b, *jac, *normals, *lambda, *mu, *rho, *source, *damping;
    double source_direction[3];
    const void *source_gradient[2]; /* both null for a directional force */
    int32_t mechanisms, field_count; /* GSLS mechanisms 0..3; 5 or 6+4*mechanisms fields */
    const void *cpml_x, *cpml_z;     /* (d, kappa, alpha) per computational node, or null */
    int32_t cpml_width_x, cpml_width_z;
    int64_t cpml_count;              /* compact ADE scalars, 0 without CFS-PML */
    double rates[3];
    const void *delta_p[3], *delta_s[3];
    int32_t precision, array_precision;
    int32_t segment_rule; /* 0: time the candidate stage-kernel segment lengths at creation; 1: choose by
                           * occupancy, without running steps (for engines built while others run) */
} swl_mesh2d;

/* Per-step diagnostics, mirror of the GPU-relevant part of Diagnostics
 * (include/Seis2D/CurvilinearSolver2D.hpp:75-86). */
typedef struct swl_diag2d {
    double energy, peak_energy, max_velocity, traction_relative;
    int32_t finite;
    int32_t rhs_registers;
    int64_t rhs_local_bytes;
    int64_t resident_bytes;
} swl_diag2d;

typedef struct swl2d_engine swl2d_engine;

/* CudaEngine::CudaEngine(mesh, receivers, device) (src/two_d/CudaEngine2D.cu:127-142).
 * receiver_nodes are padded node indices (i + nx*k).  device < 0 picks the device with
 * the most memory. */
swl_status swl2d_create(const swl_mesh2d *mesh, const int64_t *receiver_nodes, int32_t n_receivers, int32_t device,
                        swl2d_engine **out);
void swl2d_destroy(swl2d_engine *engine);

/* CudaEngine::step(time, dt, frequency, scale, step) (src/two_d/CudaEngine2D.cu:143-152):
 * one accepted classic-RK4 step; the Ricker force scale*ricker(t) is evaluated at
 * step*dt, (step+0.5)*dt and (step+1)*dt as the reference CPU driver does.  The previous
 * state stays resident for swl2d_rollback.  Asynchronous. */
swl_status swl2d_step(swl2d_engine *engine, double time, double dt, double frequency, double scale, int32_t step);

/* Batched form of `count` calls to step + diagnostics + sample: steps first..first+count-1
 * run from a CUDA graph; after every step the device checks finiteness and the late energy
 * growth rule of Simulation::advance (src/two_d/CurvilinearSolver2D.cpp:576-590) and, on a
 * failure, stops advancing and keeps the failed step's starting state.  Receiver samples go
 * to a device trace buffer read with swl2d_traces.  Returns SWL_ERR_FAULT when a step was
 * rejected; *accepted receives the number of accepted steps.  check_growth_after is the
 * time (s) after which the 1e4 x peak energy rule applies (3/f in the reference). */
swl_status swl2d_advance(swl2d_engine *engine, int32_t first, int32_t count, double dt, double frequency,
                         double scale, double check_growth_after, int32_t *accepted);

/* Asynchronous form of swl2d_advance for callers that overlap many shots on one device: the
 * batch is enqueued on the engine's stream and the call returns; swl2d_query reports completion
 * without blocking (*done = 0/1), swl2d_wait blocks.  Both return SWL_ERR_FAULT once a rejected
 * step has ended the batch.  Any other call on the engine first waits for the batch.  No
 * counterpart in the reference, whose AsyncSimulation moves whole advance calls onto a worker
 * thread (src/two_d/AsyncSimulation2D.cpp:30-58). */
swl_status swl2d_launch(swl2d_engine *engine, int32_t first, int32_t count, double dt, double frequency, double scale,
                        double check_growth_after);
swl_status swl2d_query(swl2d_engine *engine, int32_t *done, int32_t *accepted);
swl_status swl2d_wait(swl2d_engine *engine, int32_t *accepted);

/* Persistent multi-shot launches: the batches of n engines (one precision, one GSLS mechanism
 * count, one device) advance together in ONE kernel launch driven by a (shot, tile, stage) work
 * queue.  Each CTA takes the next item of a fixed global order, waits (bounded) until its shot has
 * finished the previous phase, and runs the same tile, verdict and receiver record that the
 * engine's own batch would, so every engine's results equal those of swl2d_launch with the same
 * arguments.  Each engine's uploads and read-backs stay on its own stream, ordered with the launch
 * (on the queue's stream) by events; after the launch each engine's batch is completed with
 * swl2d_query / swl2d_wait / swl2d_traces as after swl2d_launch.
 * swl2d_queue_query / swl2d_queue_wait report the launch itself: SWL_ERR_CUDA if a wait in it ran
 * out.  No counterpart in the reference, which steps one simulation per engine. */
typedef struct swl2d_queue swl2d_queue;
swl_status swl2d_queue_create(int32_t device, int32_t precision, swl2d_queue **out);
void swl2d_queue_destroy(swl2d_queue *queue);
swl_status swl2d_queue_launch(swl2d_queue *queue, swl2d_engine *const *engines, int32_t n, const int32_t *first,
                              const int32_t *count, const double *dt, const double *frequency, const double *scale,
                              const double *check_growth_after);
/* Resident CTAs per SM the queue's launches may use: 0 all that fit (default); n > 0 at most n;
 * n < 0 all but -n (at least one), which leaves room for other kernels beside the launch. */
swl_status swl2d_queue_limit(swl2d_queue *queue, int32_t ctas_per_sm);
/* Row blocks of 8 rows per work item (1, 2, 4 or 8), or 0 (default): per grid, the longest that
 * still cuts it into at least 64 items per stage.  Either way a shot's decomposition depends on
 * its grid only, never on the other shots of a launch. */
swl_status swl2d_queue_segment(swl2d_queue *queue, int32_t segment);
swl_status swl2d_queue_query(swl2d_queue *queue, int32_t *done);
swl_status swl2d_queue_wait(swl2d_queue *queue);

swl_status swl2d_rollback(swl2d_engine *engine);    /* CudaEngine::rollback */
swl_status swl2d_reset(swl2d_engine *engine);       /* CudaEngine::reset: zero fields, memories, traces */
swl_status swl2d_diagnostics(swl2d_engine *engine, swl_diag2d *out); /* CudaEngine::diagnostics */
/* The diagnostics of the last accepted step as the device-side acceptance verdict computed them
 * (the energy, peak |v|, traction ratio and finiteness that CudaEngine2D.cu:155-162 reads back after
 * every step), returned from the step clock that comes back with each batch: no kernel and no
 * synchronisation.  Before the first batch (or after reset/load) it equals swl2d_diagnostics. */
swl_status swl2d_step_diagnostics(swl2d_engine *engine, swl_diag2d *out);
/* CudaEngine::sample: Vx, Vz of the current state at every receiver (FP64). */
swl_status swl2d_sample(swl2d_engine *engine, double *vx, double *vz);
/* Raw per-step receiver samples recorded by swl2d_advance for steps
 * [first, first+count) of the current run: receivers x count, row-major. */
swl_status swl2d_traces(swl2d_engine *engine, int32_t first, int32_t count, double *vx, double *vz);
/* Whole padded field `field` (0..field_count-1) of the current state, as FP64; field -1
 * reads the compact CFS-PML memories (cpml_count values).  CudaEngine::snapshot. */
swl_status swl2d_snapshot(swl2d_engine *engine, int32_t field, double *out);
/* Overwrite field `field` (or -1: memories) of the current state from FP64 values. */
swl_status swl2d_load_field(swl2d_engine *engine, int32_t field, const double *values);
/* CudaEngine::probes: Vx, Vz, Sxx, Szz, Sxz at padded node indices, 5 per node. */
swl_status swl2d_probes(swl2d_engine *engine, const int64_t *nodes, int32_t n, double *out5);
int64_t swl2d_resident_bytes(const swl2d_engine *engine);

/* Kernel timing of `count` steps run one launch at a time with CUDA events around every
 * kernel (the steps are real, accepted steps of the simulation).  No counterpart in the
 * reference (its own timing is host wall time per advance, CurvilinearSolver2D.cpp:553-596). */
typedef struct swl_profile {
    double stage_ms[4]; /* mean duration of each RK-stage kernel */
    double stats_ms, verdict_ms, step_ms;
    int64_t steps, launches_per_step;
    double bytes_per_step;  /* algorithmic HBM bytes of one step: 17 F + 4 M per node (F, M: state and
                             * model bytes of a node) plus 17 words per CFS-PML memory */
    double extra_bytes_per_step; /* bytes the FP32 form moves beyond those: its Kahan compensation
                                  * terms (and, in 3D, U) in the last stage; 0 in FP64 */
} swl_profile;
swl_status swl2d_profile(swl2d_engine *engine, int32_t first, int32_t count, double dt, double frequency, double scale,
                         swl_profile *out);
/* How the stage kernels decompose the grid: CTAs walk strips of strip_width columns down
 * segments of segment_blocks blocks of block_rows rows; interior_ctas of the strips x segments
 * CTAs touch no absorber, source support or surface row and run the interior form; exact_h says
 * that x/h is formed as x*(1/h) (h a power of two, or FP32) rather than as the correctly rounded
 * quotient.  No counterpart in the reference (its kernels use one form for every node). */
typedef struct swl_layout2d {
    int32_t strip_width, block_rows, segment_blocks;
    int32_t strips, segments;
    int64_t interior_ctas;
    int32_t exact_h, precision;
} swl_layout2d;
swl_status swl2d_layout(swl2d_engine *engine, swl_layout2d *out);
/* Run the engine's work on a caller-provided cudaStream_t (NULL restores its own stream).
 * No counterpart in the reference (its engines launch on the legacy default stream). */
swl_status swl2d_set_stream(swl2d_engine *engine, void *cuda_stream);
/* Preallocate the forcing and trace tables for batches of up to `steps` steps, so that later
 * batches within that size allocate nothing and record no new CUDA graphs.  No counterpart in
 * the reference (it reads traces back every step). */
swl_status swl2d_reserve(swl2d_engine *engine, int32_t steps);

/* FP64 node geometry of the 2D terrain-following map (src/two_d/CurvilinearSolver2D.cpp:344-361),
 * built on the GPU: coordinates (2 per node), metric_a, metric_b, jacobian and normals (2 per
 * node) of the padded nx x nz grid (x fastest), written to host arrays, and the smallest
 * Jacobian and largest metric norm sqrt(1 + a^2 + b^2) over the physical nodes for the dt plan.
 * `surface` holds the surface height and slope of each padded column. */
typedef struct swl_geometry2d {
    int32_t nx, nz, ghost, offset_x; /* padded grid, ghost width, storage columns before the model */
    double spacing, flatten_depth;
    const double *surface;           /* 2 * nx values: (height, slope) per column */
} swl_geometry2d;
swl_status swl2d_build_geometry(const swl_geometry2d *geometry, int32_t device, double *coordinates, double *metric_a,
                                double *metric_b, double *jacobian, double *normals, double *min_jacobian,
                                double *max_metric);

/* FP64 node geometry of the 3D terrain-following map (src/three_d/CurvilinearSolver.cpp:146-190,
 * :330-364), built on the GPU: coordinates (3 per node), metrics (9 per node,
 * d(xi,eta,zeta)/d(x,y,z) row-major), jacobian and the top-row normals (3 per node) of the padded
 * nx x ny x nz grid (x fastest), plus the smallest Jacobian and the largest metric norm over the
 * physical nodes.  `surface` holds the terrain displacement of each padded (i, j) column. */
typedef struct swl_geometry3d {
    int32_t nx, ny, nz, ghost;
    double spacing, dz, flatten_depth;
    int32_t terrain;           /* 0: flat (identity metrics) */
    const double *surface;     /* nx * ny values, x fastest */
} swl_geometry3d;
swl_status swl3d_build_geometry(const swl_geometry3d *geometry, int32_t device, double *coordinates, double *metrics,
                                double *jacobian, double *normals, double *min_jacobian, double *max_metric_norm);

/* A 2D FP64 state held in caller-owned device memory (padded nx x nz grid, x fastest). */
typedef struct swl_state2d_view {
    int32_t nx, nz;                             /* padded node counts */
    double h;
    const double *vx, *vz, *sxx, *szz, *sxz;   /* device pointers, nx*nz values each */
    const double *lambda, *mu, *rho, *jac;     /* device pointers, nx*nz values each */
    const double *normals;                     /* device pointer, 2 values per node */
    const double *pml;                         /* device pointer to the CFS-PML memories, or null */
    int32_t cpml_width_x, cpml_width_z;        /* strip widths when pml is given */
} swl_state2d_view;

/* Diagnostics of a 2D state without allocating any memory: the energy, peak |v|, peak surface
 * traction ratio and finiteness that swl2d_diagnostics reports, computed from the caller's device
 * arrays and written to out[0..3] in device memory (out[3] = 1 when every value is finite, else 0),
 * enqueued on cuda_stream (null: the default stream).  It is meant for callers that cannot call
 * cudaMalloc: processes whose device memory is owned entirely by their own allocator or pre-sized
 * arena (a serving process that reserves the GPU up front, a framework's caching allocator), and
 * latency-critical loops where an allocation could synchronise the device.  Its per-block partial
 * sums live in one fixed device array inside this library, sized for at most 65,536 blocks of
 * 32x8 nodes (about 16.7 million physical nodes); larger states are rejected with SWL_ERR_INVALID.
 * Every GPU that loads the library holds that array (2 MiB) until the process exits.  Each call
 * that is not being captured looks up the array's device address in the current CUDA context (so a
 * device reset or another context is followed); a call made during stream capture reuses the
 * address of the last uncaptured call in the same context, so make one call before any capture.
 * All calls share the array: calls that overlap on the GPU (on different streams, or on the same
 * device from several threads) race and must be serialised by the caller.  The finiteness flag
 * covers the five wavefields and, when given, the CFS-PML memories; a GSLS state's Syy and
 * relaxation memories are not passed and not checked.  CFS-PML widths beyond the grid
 * (2*wx > nx-6 or wz > nz-6) are rejected with SWL_ERR_INVALID.
 * No counterpart in the reference. */
swl_status swl2d_stats_noalloc(const swl_state2d_view *state, double *out, void *cuda_stream);

/* ---------------------------------------------------------------- engine, 3D ---- */

/* POD mirror of Seis3D::Curvilinear::Point::Mesh (src/three_d/PointKernels3D.hpp:13-21),
 * FP64 arrays; `precision` selects the compute precision of the engine. */
typedef struct swl_mesh3d {
    int32_t nx, ny, nz;
    int64_t count;
    double h, lambda, mu, density;
    const double *metrics;  /* 9 per node: d(xi,eta,zeta)/d(x,y,z) rows */
    const double *normals;  /* 3 per node (surface row used) */
    const double *jacobian, *source, *damping;
    const double *material_lambda, *material_mu, *material_density; /* null for uniform */
    double source_direction[3], source_amplitude;
    const double *source_gradient[3];
    int32_t precision;
    /* CFS-PML ADE (no counterpart in the reference's 3D path, which has only the sponge):
     * (d, kappa, alpha) per computational index along x, y and z, the slab widths (x and y on both
     * sides, z at the bottom) and the memory count 6*(2wx*ny*nz + 2wy*nx*nz + wz*nx*ny) over the
     * computational grid; cpml_count = 0: none.  Memories are read and written as field -1. */
    const double *cpml_x, *cpml_y, *cpml_z;
    int32_t cpml_width_x, cpml_width_y, cpml_width_z;
    int64_t cpml_count;
    /* GSLS (no counterpart in the reference's 3D path): mechanisms 0..3; the fields become
     * 9 + 6*mechanisms, the memories of mechanism l (xx, yy, zz, xy, xz, yz) at 9 + 6l; relaxation
     * rates and per-node strengths (count values each) as swl_mesh2d has them. */
    int32_t mechanisms;
    double rates[3];
    const double *delta_p[3], *delta_s[3];
} swl_mesh3d;

typedef struct swl_diag3d {
    double energy, peak_energy, max_velocity, traction_rate_relative;
    double peaks[5]; /* |Vz|, |Vx|, |Vy|, |V|, |mean stress| */
    int32_t finite;
    int32_t rhs_registers;
    int64_t resident_bytes;
} swl_diag3d;

typedef struct swl3d_engine swl3d_engine;

/* CudaEngine3D::CudaEngine3D(mesh, receivers, device) (src/three_d/CudaEngine3D.cu:80-103). */
swl_status swl3d_create(const swl_mesh3d *mesh, const int64_t *receiver_nodes, int32_t n_receivers, int32_t device,
                        swl3d_engine **out);
void swl3d_destroy(swl3d_engine *engine);
/* CudaEngine3D::step(time, dt, frequency, step) (src/three_d/CudaEngine3D.cu:113-124). */
swl_status swl3d_step(swl3d_engine *engine, double time, double dt, double frequency, int32_t step);
swl_status swl3d_advance(swl3d_engine *engine, int32_t first, int32_t count, double dt, double frequency,
                         double check_growth_after, int32_t *accepted);
/* As swl2d_launch / swl2d_query / swl2d_wait (no counterpart in the reference). */
swl_status swl3d_launch(swl3d_engine *engine, int32_t first, int32_t count, double dt, double frequency,
                        double check_growth_after);
swl_status swl3d_query(swl3d_engine *engine, int32_t *done, int32_t *accepted);
swl_status swl3d_wait(swl3d_engine *engine, int32_t *accepted);
swl_status swl3d_rollback(swl3d_engine *engine);
swl_status swl3d_reset(swl3d_engine *engine);
swl_status swl3d_diagnostics(swl3d_engine *engine, swl_diag3d *out);
swl_status swl3d_step_diagnostics(swl3d_engine *engine, swl_diag3d *out); /* as swl2d_step_diagnostics */
swl_status swl3d_sample(swl3d_engine *engine, double *vx, double *vy, double *vz);
swl_status swl3d_traces(swl3d_engine *engine, int32_t first, int32_t count, double *vx, double *vy, double *vz);
swl_status swl3d_snapshot(swl3d_engine *engine, int32_t field, double *out);
swl_status swl3d_load_field(swl3d_engine *engine, int32_t field, const double *values);
int64_t swl3d_resident_bytes(const swl3d_engine *engine);
/* As swl2d_profile / swl2d_set_stream (no counterpart in the reference). */
swl_status swl3d_profile(swl3d_engine *engine, int32_t first, int32_t count, double dt, double frequency,
                         swl_profile *out);
swl_status swl3d_set_stream(swl3d_engine *engine, void *cuda_stream);
swl_status swl3d_reserve(swl3d_engine *engine, int32_t steps); /* as swl2d_reserve */

#ifdef __cplusplus
}
#endif
#endif
