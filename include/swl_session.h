/* swl_b200 session level: a whole simulation (model build, dt plan, receivers, records, fault
 * policy) over the engine of swl_b200.h.  Mirrors the reference's session classes:
 *   2D  Seis2D::Curvilinear::Simulation              (include/Seis2D/CurvilinearSolver2D.hpp:93-123)
 *   3D  Seis3D::Curvilinear::ISimulationBackend3D    (include/Seis3D/CurvilinearSolver.hpp:165-185)
 * Parameter structures are flat mirrors of Parameters (CurvilinearSolver2D.hpp:29-57) and
 * SimulationParameters (CurvilinearSolver.hpp:70-95); fill them with the *_params_default
 * functions first.  Validation failures return SWL_ERR_INVALID with the reference's message.
 */
#ifndef SWL_SESSION_H
#define SWL_SESSION_H
#include "swl_b200.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct swl_layer2d {
    double thickness, vp, vs, density, qp, qs;
} swl_layer2d;

typedef struct swl_params2d {
    int32_t precision; /* SWL_FP64 / SWL_FP32 */
    int32_t nx, nz;
    double spacing, vp, vs, density, relief, wavelength, flatten_depth, frequency, duration, cfl, force_per_length;
    int32_t source_x, source_z, max_steps;
    int32_t source_kind; /* 0 directional force, 1 isotropic moment */
    double source_direction[3];
    double moment_per_length, source_sigma_m, source_radius_m;
    int32_t absorbing, sponge_x, sponge_z;
    double sponge_strength;
    int32_t absorber; /* 0 sponge, 1 CFS-PML */
    double cpml_reflection, cpml_kappa_max, cpml_frequency;
    int32_t external_absorption;
    int32_t receiver_start, receiver_count, receiver_stride, receiver_depth;
    double sample_interval_ms;
    int32_t layered, n_layers;
    const swl_layer2d *layers;
    int32_t attenuation, mechanisms;
    double q_min_frequency, q_max_frequency, q_reference_frequency, qp, qs;
    int32_t imported_surface, n_surface;
    double surface_datum;
    const double *surface_xz; /* n_surface pairs (x, elevation) */
    int32_t device_geometry;  /* 1: build the FP64 node geometry on the session's GPU (swl2d_build_geometry) */
    int32_t segment_rule;     /* 1: the engine's segment length by occupancy rule, without timing runs (the
                               * server's choice for every shot); 0: timed at creation */
} swl_params2d;

typedef struct swl_info2d {
    int32_t nx, nz, model_offset_x, total_steps, step, field_count, receivers, completed, finite, mechanisms;
    int64_t count, samples, cpml_count, resident_bytes;
    double dt, record_dt, h, flatten_depth, max_metric, min_jacobian, max_edge, ppw, wave_dt, damping_dt, source_dt,
        relaxation_dt, cpml_dt, max_relative_q_error, energy, peak_energy, max_velocity, traction_relative, init_ms,
        total_step_ms, last_step_ms;
} swl_info2d;

typedef struct swl2d_session swl2d_session;

/* Pass as `device` to build and inspect the model without creating an engine (no GPU needed);
 * stepping calls then return SWL_ERR_STATE. */
#define SWL_MODEL_ONLY (-2)

void swl2d_params_default(swl_params2d *p);
/* Simulation::initialize (src/two_d/CurvilinearSolver2D.cpp:151-540) on the GPU backend. */
swl_status swl2d_session_create(const swl_params2d *p, int32_t device, swl2d_session **out);
void swl2d_session_destroy(swl2d_session *s);
/* Simulation::advance (:541-604): up to `count` accepted steps (stops at the planned total). */
swl_status swl2d_session_advance(swl2d_session *s, int32_t count);
swl_status swl2d_session_reset(swl2d_session *s);          /* Simulation::reset (:605-637) */
swl_status swl2d_session_info(const swl2d_session *s, swl_info2d *out);
/* Receiver records on the record axis (t = 0 included): receivers x samples, row-major. */
swl_status swl2d_session_records(const swl2d_session *s, double *vx, double *vz);
/* Receiver positions (x, z) in metres, 2 per receiver. */
swl_status swl2d_session_receiver_positions(const swl2d_session *s, double *xz);
swl_status swl2d_session_snapshot(swl2d_session *s, int32_t field, double *out);
/* FP64 model array by name ("metricA", "metricB", "jacobian", "normals", "coordinates", "lambda",
 * "mu", "density", "vp", "vs", "source", "damping", "sourceGradientX/Z", "cpmlX", "cpmlZ",
 * "deltaP0".."deltaS2"); *n receives the length (out may be null to query it). */
swl_status swl2d_session_model(const swl2d_session *s, const char *name, double *out, int64_t *n);
swl2d_engine *swl2d_session_engine(swl2d_session *s);
/* writeSnapshot (src/two_d/CurvilinearSolver2D.cpp:725-810): the current wavefield as a VTK
 * structured grid (.vts, ASCII) of the logical model, byte for byte the reference's file.
 * components: Vx, Vz, velocity magnitude, pressure, Sxx, Szz, Sxz (SnapshotExportOptions); the
 * reference's default is {1, 1, 0, 0, 1, 1, 1} with the material. */
swl_status swl2d_session_write_snapshot(swl2d_session *s, const char *path, const int32_t components[7], int32_t include_material);
/* Simulation::readProbes (:710-724): Vx, Vz, Sxx, Szz, Sxz at logical nodes (i, k), 5 per node. */
swl_status swl2d_session_read_probes(swl2d_session *s, const int32_t *nodes_ik, int32_t n, double *out5);

typedef struct swl_layer3d {
    double thickness, vp, vs, density;
} swl_layer3d;

typedef struct swl_params3d {
    int32_t precision;
    int32_t nx, ny, nz;
    double spacing, vp, vs, density;
    int32_t layered, layer_depth_mode, n_layers; /* depth mode 0 grid index, 1 below surface, 2 datum */
    const swl_layer3d *layers;
    double frequency;
    int32_t source_x, source_y, source_z, source_kind;
    double source_direction[3], source_force, source_moment, duration;
    int32_t max_steps;
    double cfl, relief, wavelength, flatten_depth;
    int32_t dem_nx, dem_ny; /* 0: analytic terrain */
    double dem_spacing, dem_origin_x, dem_origin_y, dem_datum;
    const double *dem_elevations; /* dem_ny rows of dem_nx, first row minimum y */
    int32_t receiver_kind, receiver_start_x, receiver_start_y, receiver_z, receiver_count_x, receiver_count_y,
        receiver_stride_x, receiver_stride_y, receiver_limit;
    int32_t absorbing, absorbing_cells[3];
    double absorbing_strength;
    int32_t device_geometry; /* 1: build the FP64 node geometry on the session's GPU (swl3d_build_geometry) */
    const char *const *layer_names; /* n_layers UTF-8 names (MaterialLayer3D::name), or null: unnamed */
    /* 0: the reference's sponge; 1: CFS-PML ADE slabs of absorbing_cells widths (x, y both sides, z at the
     * bottom) with the 2D profiles per axis.  No counterpart in the reference's 3D path. */
    int32_t absorber;
    double cpml_reflection, cpml_kappa_max, cpml_frequency; /* frequency 0: the source frequency */
    /* GSLS viscoelasticity with 1..3 mechanisms (the 2D settings of swl_params2d; no counterpart in
     * the reference's 3D path).  layer_q: qp, qs per layer (2 * n_layers values), or null: qp, qs. */
    int32_t attenuation, mechanisms;
    double q_min_frequency, q_max_frequency, q_reference_frequency, qp, qs;
    const double *layer_q;
} swl_params3d;

typedef struct swl_info3d {
    int32_t nx, ny, nz, total_steps, step, receivers, completed, finite;
    int64_t count, resident_bytes;
    double dt, h, flatten_depth, min_jacobian, max_metric_norm, min_cell_length, max_cell_edge, wave_dt, damping_dt,
        source_dt, ppw, energy, peak_energy, max_velocity, traction_rate_relative, init_ms, total_step_ms, last_step_ms;
} swl_info3d;

typedef struct swl3d_session swl3d_session;

void swl3d_params_default(swl_params3d *p);
/* CpuSimulation3D::initialize (src/three_d/CurvilinearSolver.cpp:301-442) on the GPU backend. */
swl_status swl3d_session_create(const swl_params3d *p, int32_t device, swl3d_session **out);
void swl3d_session_destroy(swl3d_session *s);
swl_status swl3d_session_advance(swl3d_session *s, int32_t count); /* CpuSimulation3D::advance (:445-513) */
swl_status swl3d_session_reset(swl3d_session *s);                  /* resetFields (:514-525) */
swl_status swl3d_session_info(const swl3d_session *s, swl_info3d *out);
/* Vx, Vy, Vz records per receiver, receivers x (step + 1), t = 0 included. */
swl_status swl3d_session_records(const swl3d_session *s, double *vx, double *vy, double *vz);
swl_status swl3d_session_snapshot(swl3d_session *s, int32_t field, double *out);
/* "coordinates", "metrics", "jacobian", "normals", "source", "damping", "sourceGradient0..2",
 * "materialLambda", "materialMu", "materialDensity"; with CFS-PML "cpmlX", "cpmlY", "cpmlZ" (d, kappa,
 * alpha per computational index) and "cpmlShape" (wx, wy, wz, memory count). */
swl_status swl3d_session_model(const swl3d_session *s, const char *name, double *out, int64_t *n);
swl3d_engine *swl3d_session_engine(swl3d_session *s);
/* writeVts (src/three_d/VtsWriter.cpp) of the current state: the physical nodes as a VTK
 * structured grid (.vts, ASCII), byte for byte the reference's file.  fields: Vx, Vy, Vz, |V|,
 * mean normal stress, Sxx, Syy, Szz, Sxy, Sxz, Syz (VtsExportOptions3D; default all, with the
 * material and the velocity vector). */
swl_status swl3d_session_write_snapshot(swl3d_session *s, const char *path, const int32_t fields[11], int32_t include_material,
                                        int32_t include_velocity_vector);

#ifdef __cplusplus
}
#endif
#endif
