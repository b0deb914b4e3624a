/* Test infrastructure only (the oracle): a plain-C FP64 restatement of SeisWave Lab's
 * curvilinear velocity-stress RK4 step, used by tests/ and bench.py as the checker.
 * The product never links this library.
 *
 * Layout follows the reference: padded grids with a ghost width of 3, x fastest,
 * one array per field (structure of arrays).  2D fields: Vx, Vz, Sxx, Szz, Sxz
 * [, Syy, 4 memories per GSLS mechanism]; 3D fields: Vx, Vy, Vz, Sxx, Syy, Szz, Sxy, Sxz, Syz.
 */
#ifndef SWL_ORACLE_H
#define SWL_ORACLE_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Mirror of Seis2D::Curvilinear::Point::MeshT<double> (src/two_d/PointKernels2D.hpp:14-27). */
typedef struct swlo_mesh2d {
    int32_t nx, nz;          /* padded node counts */
    int64_t count;           /* nx*nz */
    double h;
    const double *a, *b, *jac, *normals, *lambda, *mu, *rho, *source, *damping;
    double source_direction[3];
    const double *source_gradient[2]; /* null for a directional force */
    int32_t mechanisms, field_count;
    const double *cpml_x, *cpml_z;    /* 3 values (d, kappa, alpha) per computational node */
    int32_t cpml_width_x, cpml_width_z;
    int64_t cpml_count;
    double rates[3];
    const double *delta_p[3], *delta_s[3];
} swlo_mesh2d;

/* Mirror of Seis3D::Curvilinear::Point::Mesh (src/three_d/PointKernels3D.hpp:13-21). */
typedef struct swlo_mesh3d {
    int32_t nx, ny, nz;
    int64_t count;
    double h, lambda, mu, density;
    const double *metrics, *normals, *jacobian, *source, *damping;
    const double *material_lambda, *material_mu, *material_density; /* null for a uniform model */
    double source_direction[3], source_amplitude;
    const double *source_gradient[3];
    /* CFS-PML ADE in 3D (the reference has the sponge only; this build extends its 2D ADE, see
     * swl_oracle.c): (d, kappa, alpha) per computational index along x, y and z, the slab widths
     * (x and y on both sides, z at the bottom) and the compact memory count (0: no CFS-PML). */
    const double *cpml_x, *cpml_y, *cpml_z;
    int32_t cpml_width_x, cpml_width_y, cpml_width_z;
    int64_t cpml_count;
    /* GSLS in 3D (the reference's 3D path is elastic; this build extends its 2D GSLS, see
     * swl_oracle.c): mechanisms 0..3, fields 9 + 6*mechanisms (the memories of mechanism l at
     * 9 + 6l: xx, yy, zz, xy, xz, yz), relaxation rates and per-node strengths. */
    int32_t mechanisms, field_count;
    double rates[3];
    const double *delta_p[3], *delta_s[3];
} swlo_mesh3d;

int swlo_direction(int step, int stage, int axis);

/* One RHS evaluation over every physical node (2D); out/out_pml are zeroed first. */
void swlo2d_rhs(const swlo_mesh2d *g, double *const *in, const double *in_pml, double *const *out,
                double *out_pml, double forcing, int step, int stage);
/* Traction projection of row k=3. */
void swlo2d_project(const swlo_mesh2d *g, double *const *fields);
/* Advance `steps` accepted RK4 steps from step `first`.  state: field_count*count doubles,
 * pml: cpml_count doubles.  scale = force (or moment) per length / h^2.  Receivers are padded
 * node indices; traces (receivers x steps, row-major) receive Vx and Vz after each step. */
int swlo2d_run(const swlo_mesh2d *g, double *state, double *pml, int first, int steps, double dt,
               double frequency, double scale, const int64_t *receivers, int nreceivers, double *trace_vx,
               double *trace_vz);

void swlo3d_rhs(const swlo_mesh3d *g, double *const *in, const double *in_pml, double *const *out, double *out_pml,
                double source, int step, int stage);
void swlo3d_project(const swlo_mesh3d *g, double *const *fields);
/* state: field_count*count doubles (9 when field_count is 0); pml: cpml_count doubles (null
 * without CFS-PML).  traces: receivers x steps for Vx, Vy, Vz. */
int swlo3d_run(const swlo_mesh3d *g, double *state, double *pml, int first, int steps, double dt, double frequency,
               const int64_t *receivers, int nreceivers, double *trace_vx, double *trace_vy, double *trace_vz);

#ifdef __cplusplus
}
#endif
#endif
