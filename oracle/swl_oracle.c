/* Test infrastructure only (the oracle).  Plain-C FP64 restatement of the reference
 * SeisWave Lab curvilinear velocity-stress scheme: MacCormack-DRP alternating stencils,
 * metric-transformed derivatives, traction-image free surface, CFS-PML ADE memories,
 * GSLS relaxation and the classic RK4 driver.  Every function names the reference lines
 * (paths relative to the reference project) that it restates; expression order follows
 * the reference so that, compiled without FMA contraction, results match the reference
 * CPU build bit for bit.  It is the checker for tests/ and the port arm of bench.py; the
 * product never links it.
 */
#include "swl_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* include/SeisCommon/FiniteDifference.hpp:9-13 -- the 8-step MacCormack direction table,
 * flipped at every RK stage.  Axis 0 = x, 1 = y, 2 = z (2D uses 0 and 2). */
int swlo_direction(int step, int stage, int axis) {
    static const int table[8][3] = {{0, 0, 0}, {1, 1, 0}, {1, 1, 1}, {0, 0, 1},
                                    {0, 1, 0}, {1, 0, 0}, {1, 0, 1}, {0, 1, 1}};
    return (table[step % 8][axis] + stage) % 2;
}

/* include/SeisCommon/FiniteDifference.hpp:14-26 -- 5-point DRP (offsets -1..3), the
 * one-sided 2-point (depth 1) and 3-point (depth 2) near-surface velocity stencils; a
 * backward stencil negates offsets and coefficients. */
static int stencil(int dir, int depth, int *off, double *c) {
    static const double drp[5] = {-.30874, -.6326, 1.233, -.3334, .04168};
    const double low[3] = {-7.0 / 6.0, 8.0 / 6.0, -1.0 / 6.0};
    const int n = depth == 1 ? 2 : depth == 2 ? 3 : 5;
    for (int l = 0; l < n; ++l) {
        const int pos = n == 5 ? l - 1 : l;
        const double v = n == 5 ? drp[l] : n == 3 ? low[l] : (l == 0 ? -1.0 : 1.0);
        off[l] = dir ? -pos : pos;
        c[l] = dir ? -v : v;
    }
    return n;
}

/* ---------------------------------------------------------------- 2D ---------- */

/* src/two_d/PointKernels2D.hpp:38-47 */
static double d2(const double *v, const swlo_mesh2d *g, ptrdiff_t q, int axis, int dir, int depth) {
    int off[5];
    double c[5];
    const int n = stencil(dir, depth, off, c);
    const ptrdiff_t s = axis ? g->nx : 1;
    double r = 0;
    for (int l = 0; l < n; ++l) r += c[l] * v[q + off[l] * s];
    return r / g->h;
}

/* src/two_d/PointKernels2D.hpp:50-56 -- compact CFS-PML slot: x strips own
 * 4*(k*2w+j), the bottom strip follows after all side slots. */
static ptrdiff_t pml_slot(const swlo_mesh2d *g, ptrdiff_t q, int axis) {
    if (!g->cpml_count) return -1;
    const int i = (int)(q % g->nx) - 3, k = (int)(q / g->nx) - 3, nx = g->nx - 6, nz = g->nz - 6;
    if (axis == 0) {
        const int w = g->cpml_width_x;
        const int j = i < w ? i : i >= nx - w ? w + i - (nx - w) : -1;
        return j < 0 ? -1 : 4 * ((ptrdiff_t)k * 2 * w + j);
    }
    return k < nz - g->cpml_width_z ? -1
                                     : 4 * ((ptrdiff_t)(2 * g->cpml_width_x) * nz +
                                            (ptrdiff_t)(k - (nz - g->cpml_width_z)) * nx + i);
}

/* src/two_d/PointKernels2D.hpp:57-64 -- ADE memory rate and stretched derivative. */
static double stretched(const swlo_mesh2d *g, const double *in_pml, double *out_pml, ptrdiff_t q, int axis,
                        int field, double deriv) {
    const ptrdiff_t slot = pml_slot(g, q, axis);
    if (slot < 0) return deriv;
    const int at = axis ? (int)(q / g->nx) - 3 : (int)(q % g->nx) - 3;
    const double *p = (axis ? g->cpml_z : g->cpml_x) + 3 * at;
    const double d = p[0], kappa = p[1], alpha = p[2], psi = in_pml[slot + field];
    out_pml[slot + field] = -(d / kappa + alpha) * psi - d / (kappa * kappa) * deriv;
    return deriv / kappa + psi;
}

/* src/two_d/PointKernels2D.hpp:70-78 -- remove the surface traction on row k=3. */
void swlo2d_project(const swlo_mesh2d *g, double *const *f) {
    for (int i = 3; i < g->nx - 3; ++i) {
        const ptrdiff_t q = i + (ptrdiff_t)g->nx * 3;
        const double nx = g->normals[2 * q], nz = g->normals[2 * q + 1];
        const double tx = f[2][q] * nx + f[4][q] * nz, tz = f[4][q] * nx + f[3][q] * nz, nn = nx * tx + nz * tz;
        f[2][q] += -2 * nx * tx + nn * nx * nx;
        f[3][q] += -2 * nz * tz + nn * nz * nz;
        f[4][q] += -nx * tz - tx * nz + nn * nx * nz;
    }
}

/* src/two_d/PointKernels2D.hpp:79-89 -- surface eta-derivative of (Vx, Vz) implied by a
 * traction-free surface, from a local normal/tangent solve. */
static void surface_derivative(const swlo_mesh2d *g, double *const *w, ptrdiff_t q, int dir, double *res,
                               const double *xi) {
    const double c0 = g->a[q], c1 = g->b[q], c2 = c0 * c0 + c1 * c1, len = sqrt(c2);
    const double n[2] = {c0 / len, c1 / len};
    const double dx = xi ? xi[0] : d2(w[0], g, q, 0, dir, -1), dz = xi ? xi[1] : d2(w[1], g, q, 0, dir, -1);
    const double lambda = g->lambda[q], mu = g->mu[q];
    double t[2] = {(lambda + 2 * mu) * dx * c0 + mu * dz * c1, mu * dz * c0 + lambda * dx * c1};
    for (int l = 0; l < g->mechanisms; ++l) {
        const int m = 6 + 4 * l;
        t[0] -= w[m][q] * c0 + w[m + 2][q] * c1;
        t[1] -= w[m + 2][q] * c0 + w[m + 1][q] * c1;
    }
    const double normal = t[0] * n[0] + t[1] * n[1];
    for (int v = 0; v < 2; ++v) res[v] = -(t[v] - n[v] * normal) / (mu * c2) - n[v] * normal / ((lambda + 2 * mu) * c2);
}

/* src/two_d/PointKernels2D.hpp:90-93 */
static double flux(const swlo_mesh2d *g, double *const *w, ptrdiff_t q, int axis, int comp) {
    const double x = axis ? g->a[q] : 1, z = axis ? g->b[q] : 0;
    return g->jac[q] * (x * w[comp ? 4 : 2][q] + z * w[comp ? 3 : 4][q]);
}

/* src/two_d/PointKernels2D.hpp:94-120 -- conservative traction-image momentum: the
 * surface tap is dropped and taps above it are mirrored with a sign flip. */
static double momentum(const swlo_mesh2d *g, double *const *w, ptrdiff_t q, int comp, const int *dirs, int depth,
                       int only) {
    double r = 0;
    for (int axis = 0; axis < 2; ++axis) {
        if (only >= 0 && axis != only) continue;
        int off[5];
        double c[5];
        const int n = stencil(dirs[axis], -1, off, c);
        for (int l = 0; l < n; ++l) {
            int o = off[l];
            double sign = 1;
            if (axis) {
                const int k = depth + o;
                if (k == 0) continue;
                if (k < 0) {
                    o = -k - depth;
                    sign = -1;
                }
            }
            r += sign * c[l] * flux(g, w, q + (ptrdiff_t)o * (axis ? g->nx : 1), axis, comp);
        }
    }
    return r / (g->h * g->jac[q] * g->rho[q]);
}

/* src/two_d/PointKernels2D.hpp:121-172 -- the P-SV right-hand side at one node. */
static void rhs2_point(const swlo_mesh2d *g, double *const *w, const double *in_pml, double *const *out,
                       double *out_pml, ptrdiff_t q, double forcing, int step, int stage) {
    const int depth = (int)(q / g->nx) - 3;
    const int dirs[2] = {swlo_direction(step, stage, 0), swlo_direction(step, stage, 2)};
    const int cpml = g->cpml_count != 0;
    double surface[2] = {0, 0};
    if (depth == 0) {
        double xi[2] = {0, 0};
        if (cpml)
            for (int v = 0; v < 2; ++v)
                xi[v] = stretched(g, in_pml, out_pml, q, 0, v, d2(w[v], g, q, 0, dirs[0], -1));
        surface_derivative(g, w, q, dirs[0], surface, cpml ? xi : NULL);
    }
    double dx[5], dz[5], xis[5], etas[5];
    for (int f = 0; f < 5; ++f) {
        const double xi = d2(w[f], g, q, 0, dirs[0], -1);
        const double eta = f < 2 && depth == 0 ? surface[f] : d2(w[f], g, q, 1, dirs[1], f < 2 ? depth : -1);
        xis[f] = xi;
        etas[f] = eta;
        const double vx = cpml && f < 2 ? stretched(g, in_pml, out_pml, q, 0, f, xi) : xi;
        const double vz = cpml && f < 2 ? stretched(g, in_pml, out_pml, q, 1, f, eta) : eta;
        dx[f] = vx + g->a[q] * vz;
        dz[f] = g->b[q] * vz;
    }
    out[0][q] = (dx[2] + dz[4]) / g->rho[q];
    out[1][q] = (dx[4] + dz[3]) / g->rho[q];
    const int near = depth <= (dirs[1] ? 3 : 1);
    if (near)
        for (int v = 0; v < 2; ++v) out[v][q] = momentum(g, w, q, v, dirs, depth, -1);
    if (cpml)
        for (int v = 0; v < 2; ++v) {
            const int f = v ? 4 : 2, other = v ? 3 : 4;
            double x = xis[f] / g->rho[q], z = (g->a[q] * etas[f] + g->b[q] * etas[other]) / g->rho[q];
            if (near) {
                x = momentum(g, w, q, v, dirs, depth, 0);
                z = momentum(g, w, q, v, dirs, depth, 1);
            }
            out[v][q] = stretched(g, in_pml, out_pml, q, 0, 2 + v, x) + stretched(g, in_pml, out_pml, q, 1, 2 + v, z);
        }
    for (int v = 0; v < 2; ++v)
        out[v][q] += forcing *
                     (g->source_gradient[v] ? g->source_gradient[v][q] : g->source[q] * g->source_direction[v == 0 ? 0 : 2]) /
                     g->rho[q];
    const double lambda = g->lambda[q], mu = g->mu[q], div = dx[0] + dz[1];
    out[2][q] = lambda * div + 2 * mu * dx[0];
    out[3][q] = lambda * div + 2 * mu * dz[1];
    out[4][q] = mu * (dz[0] + dx[1]);
    if (g->mechanisms) {
        out[5][q] = lambda * div;
        for (int l = 0; l < g->mechanisms; ++l) {
            const int m = 6 + 4 * l;
            const double dp = g->delta_p[l][q], ds = g->delta_s[l][q], dl = dp - 2 * ds;
            const double drive[4] = {dl * div + 2 * ds * dx[0], dl * div + 2 * ds * dz[1], ds * (dz[0] + dx[1]), dl * div};
            out[2][q] -= w[m][q];
            out[3][q] -= w[m + 1][q];
            out[4][q] -= w[m + 2][q];
            out[5][q] -= w[m + 3][q];
            for (int f = 0; f < 4; ++f) out[m + f][q] = g->rates[l] * (drive[f] - w[m + f][q]);
        }
    }
    for (int f = 0; f < g->field_count; ++f) out[f][q] -= g->damping[q] * w[f][q];
}

/* src/two_d/CurvilinearSolver2D.cpp:68-78 -- zero the rates and memories, then every
 * physical node. */
void swlo2d_rhs(const swlo_mesh2d *g, double *const *in, const double *in_pml, double *const *out, double *out_pml,
                double forcing, int step, int stage) {
    for (int f = 0; f < g->field_count; ++f) memset(out[f], 0, sizeof(double) * (size_t)g->count);
    if (g->cpml_count) memset(out_pml, 0, sizeof(double) * (size_t)g->cpml_count);
    for (int k = 3; k < g->nz - 3; ++k)
        for (int i = 3; i < g->nx - 3; ++i)
            rhs2_point(g, in, in_pml, out, out_pml, i + (ptrdiff_t)g->nx * k, forcing, step, stage);
}

/* src/two_d/CurvilinearSolver2D.cpp:31-34 */
static double ricker(double t, double f) {
    const double a = 3.14159265358979323846 * f * (t - 1.5 / f);
    return (1 - 2 * a * a) * exp(-a * a);
}

/* src/two_d/CurvilinearSolver2D.cpp:80-97 -- stage or final RK combine. */
static void combine2(double *target, const double *base, const double *rate, const double *k1, const double *k2,
                     const double *k3, const double *k4, size_t n, double delta, double weight, int final) {
    for (size_t q = 0; q < n; ++q)
        target[q] = base[q] + (final ? delta * (k1[q] + 2 * k2[q] + 2 * k3[q] + k4[q]) / 6.0 : weight * rate[q]);
}

/* src/two_d/CurvilinearSolver2D.cpp:541-604 (the CPU branch at :266-276) -- the
 * seven-state classic RK4 step; inspect/rollback are host policy and not restated. */
int swlo2d_run(const swlo_mesh2d *g, double *state, double *pml, int first, int steps, double dt, double frequency,
               double scale, const int64_t *receivers, int nreceivers, double *trace_vx, double *trace_vz) {
    const size_t n = (size_t)g->count, fc = (size_t)g->field_count, np = (size_t)g->cpml_count;
    double *mem = (double *)calloc(6 * (fc * n + np + 1), sizeof(double));
    if (!mem) return -1;
    double *sets[6];
    double *psets[6];
    for (int s = 0; s < 6; ++s) {
        sets[s] = mem + (size_t)s * (fc * n + np + 1);
        psets[s] = sets[s] + fc * n;
    }
    /* sets: 0 = base, 1..4 = k1..k4, 5 = stage */
    double *F0[18], *B[18], *K[4][18], *S[18];
    for (size_t f = 0; f < fc; ++f) {
        F0[f] = state + f * n;
        B[f] = sets[0] + f * n;
        for (int s = 0; s < 4; ++s) K[s][f] = sets[1 + s] + f * n;
        S[f] = sets[5] + f * n;
    }
    for (int it = 0; it < steps; ++it) {
        const int step = first + it;
        memcpy(sets[0], state, sizeof(double) * fc * n);
        if (np) memcpy(psets[0], pml, sizeof(double) * np);
        const double t0 = step * dt, th = (step + .5) * dt, t1 = (step + 1) * dt;
        const double half = dt / 2;
        swlo2d_rhs(g, F0, pml, K[0], psets[1], scale * ricker(t0, frequency), step, 0);
        for (size_t f = 0; f < fc; ++f) combine2(S[f], B[f], K[0][f], 0, 0, 0, 0, n, dt, half, 0);
        if (np) combine2(psets[5], psets[0], psets[1], 0, 0, 0, 0, np, dt, half, 0);
        swlo2d_project(g, S);
        swlo2d_rhs(g, S, psets[5], K[1], psets[2], scale * ricker(th, frequency), step, 1);
        for (size_t f = 0; f < fc; ++f) combine2(S[f], B[f], K[1][f], 0, 0, 0, 0, n, dt, half, 0);
        if (np) combine2(psets[5], psets[0], psets[2], 0, 0, 0, 0, np, dt, half, 0);
        swlo2d_project(g, S);
        swlo2d_rhs(g, S, psets[5], K[2], psets[3], scale * ricker(th, frequency), step, 2);
        for (size_t f = 0; f < fc; ++f) combine2(S[f], B[f], K[2][f], 0, 0, 0, 0, n, dt, dt, 0);
        if (np) combine2(psets[5], psets[0], psets[3], 0, 0, 0, 0, np, dt, dt, 0);
        swlo2d_project(g, S);
        swlo2d_rhs(g, S, psets[5], K[3], psets[4], scale * ricker(t1, frequency), step, 3);
        for (size_t f = 0; f < fc; ++f) combine2(F0[f], B[f], 0, K[0][f], K[1][f], K[2][f], K[3][f], n, dt, 0, 1);
        if (np) combine2(pml, psets[0], 0, psets[1], psets[2], psets[3], psets[4], np, dt, 0, 1);
        swlo2d_project(g, F0);
        for (int r = 0; r < nreceivers; ++r) {
            if (trace_vx) trace_vx[(size_t)r * steps + it] = F0[0][receivers[r]];
            if (trace_vz) trace_vz[(size_t)r * steps + it] = F0[1][receivers[r]];
        }
    }
    free(mem);
    return 0;
}

/* ---------------------------------------------------------------- 3D ---------- */

static double lam3(const swlo_mesh3d *g, ptrdiff_t q) { return g->material_lambda ? g->material_lambda[q] : g->lambda; }
static double mu3(const swlo_mesh3d *g, ptrdiff_t q) { return g->material_mu ? g->material_mu[q] : g->mu; }
static double rho3(const swlo_mesh3d *g, ptrdiff_t q) { return g->material_density ? g->material_density[q] : g->density; }

/* src/three_d/PointKernels3D.hpp:30-35 */
static double d3(const double *v, const swlo_mesh3d *g, ptrdiff_t q, int axis, int dir, int depth) {
    const ptrdiff_t s = axis == 0 ? 1 : axis == 1 ? g->nx : (ptrdiff_t)g->nx * g->ny;
    int off[5];
    double c[5];
    const int n = stencil(dir, depth, off, c);
    double r = 0;
    for (int l = 0; l < n; ++l) r += c[l] * v[q + off[l] * s];
    return r / g->h;
}

/* src/three_d/PointKernels3D.hpp:36-51 -- tangential stress projection on k=3. */
void swlo3d_project(const swlo_mesh3d *g, double *const *f) {
    for (int j = 3; j < g->ny - 3; ++j)
        for (int i = 3; i < g->nx - 3; ++i) {
            const ptrdiff_t q = i + (ptrdiff_t)g->nx * (j + (ptrdiff_t)g->ny * 3);
            const double s[9] = {f[3][q], f[6][q], f[7][q], f[6][q], f[4][q], f[8][q], f[7][q], f[8][q], f[5][q]};
            const double *n = g->normals + 3 * q;
            double t[3] = {0, 0, 0}, o[9];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) t[a] += s[3 * a + b] * n[b];
            const double nn = t[0] * n[0] + t[1] * n[1] + t[2] * n[2];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) o[3 * a + b] = s[3 * a + b] - n[a] * t[b] - t[a] * n[b] + nn * n[a] * n[b];
            f[3][q] = o[0];
            f[4][q] = o[4];
            f[5][q] = o[8];
            f[6][q] = 0.5 * (o[1] + o[3]);
            f[7][q] = 0.5 * (o[2] + o[6]);
            f[8][q] = 0.5 * (o[5] + o[7]);
        }
}

/* ---- 3D CFS-PML (no counterpart in the reference, whose 3D path has only the quadratic sponge,
 * include/Seis3D/AbsorbingBoundary3D.hpp:17-21).  The 2D ADE of src/two_d/PointKernels2D.hpp:50-64
 * carried over axis by axis: slabs of width wx on both x sides, wy on both y sides, wz at the
 * bottom; six memories per active axis of a node -- the axis derivative of Vx, Vy, Vz (0..2) and
 * the axis part of the three momentum components (3..5).  A node in any slab sums its momentum
 * per axis (x/rho + y/rho + z/rho, each stretched where the axis is active), as the 2D ADE does;
 * a node outside every slab keeps the sponge-free form. */
static ptrdiff_t pml_slot3(const swlo_mesh3d *g, ptrdiff_t q, int axis) {
    if (!g->cpml_count) return -1;
    const ptrdiff_t plane = (ptrdiff_t)g->nx * g->ny;
    const int i = (int)(q % g->nx) - 3, j = (int)((q / g->nx) % g->ny) - 3, k = (int)(q / plane) - 3;
    const int nx = g->nx - 6, ny = g->ny - 6, nz = g->nz - 6;
    const int wx = g->cpml_width_x, wy = g->cpml_width_y, wz = g->cpml_width_z;
    const ptrdiff_t c0 = 6 * (ptrdiff_t)2 * wx * ny * nz, c1 = 6 * (ptrdiff_t)2 * wy * nx * nz;
    if (axis == 0) {
        const int s = i < wx ? i : i >= nx - wx ? wx + i - (nx - wx) : -1;
        return s < 0 ? -1 : 6 * (((ptrdiff_t)k * ny + j) * 2 * wx + s);
    }
    if (axis == 1) {
        const int s = j < wy ? j : j >= ny - wy ? wy + j - (ny - wy) : -1;
        return s < 0 ? -1 : c0 + 6 * (((ptrdiff_t)k * 2 * wy + s) * nx + i);
    }
    return k < nz - wz ? -1 : c0 + c1 + 6 * (((ptrdiff_t)(k - (nz - wz)) * ny + j) * nx + i);
}
/* psi' = -(d/kappa + alpha) psi - d/kappa^2 * derivative; returns derivative/kappa + psi
 * (PointKernels2D.hpp:57-64 per axis). */
static double stretched3(const swlo_mesh3d *g, const double *in_pml, double *out_pml, ptrdiff_t q, int axis, int field,
                         double derivative) {
    const ptrdiff_t slot = pml_slot3(g, q, axis);
    if (slot < 0) return derivative;
    const ptrdiff_t plane = (ptrdiff_t)g->nx * g->ny;
    const int at = axis == 0 ? (int)(q % g->nx) - 3 : axis == 1 ? (int)((q / g->nx) % g->ny) - 3 : (int)(q / plane) - 3;
    const double *pr = (axis == 0 ? g->cpml_x : axis == 1 ? g->cpml_y : g->cpml_z) + 3 * at;
    const double d = pr[0], kappa = pr[1], alpha = pr[2], psi = in_pml[slot + field];
    out_pml[slot + field] = -(d / kappa + alpha) * psi - d / (kappa * kappa) * derivative;
    return derivative / kappa + psi;
}
static int in_slab3(const swlo_mesh3d *g, ptrdiff_t q) {
    return g->cpml_count && (pml_slot3(g, q, 0) >= 0 || pml_slot3(g, q, 1) >= 0 || pml_slot3(g, q, 2) >= 0);
}

/* src/three_d/PointKernels3D.hpp:52-66 -- surface zeta-derivative of the velocity from
 * the local traction-free solve; `xy` (3 velocities x (xi, eta)) are the CFS-PML-stretched
 * derivatives when the node lies in a slab, else null. */
static void surface_derivative3(const swlo_mesh3d *g, double *const *w, ptrdiff_t q, double *res, int dx_dir,
                                int dy_dir, const double *xy) {
    const double *m = g->metrics + 9 * q;
    const double lambda = lam3(g, q), mu = mu3(g, q);
    const double c[3] = {m[6], m[7], m[8]};
    const double c2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2], len = sqrt(c2);
    const double n[3] = {c[0] / len, c[1] / len, c[2] / len};
    double gr[9] = {0}, t[3] = {0, 0, 0};
    for (int v = 0; v < 3; ++v) {
        const double dx = xy ? xy[2 * v] : d3(w[v], g, q, 0, dx_dir, -1), dy = xy ? xy[2 * v + 1] : d3(w[v], g, q, 1, dy_dir, -1);
        for (int a = 0; a < 3; ++a) gr[3 * v + a] = m[a] * dx + m[3 + a] * dy;
    }
    const double trace = gr[0] + gr[4] + gr[8];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) t[a] += ((a == b ? lambda * trace : 0) + mu * (gr[3 * a + b] + gr[3 * b + a])) * c[b];
    /* GSLS: the memory stresses' traction, as the 2D surfaceDerivative subtracts it
     * (src/two_d/PointKernels2D.hpp:84) */
    static const int T[3][3] = {{0, 3, 4}, {3, 1, 5}, {4, 5, 2}}; /* tensor (a, b) -> memory component */
    for (int l = 0; l < g->mechanisms; ++l) {
        const int mm = 9 + 6 * l;
        for (int a = 0; a < 3; ++a)
            t[a] -= (w[mm + T[a][0]][q] * c[0] + w[mm + T[a][1]][q] * c[1]) + w[mm + T[a][2]][q] * c[2];
    }
    const double normal = t[0] * n[0] + t[1] * n[1] + t[2] * n[2];
    for (int a = 0; a < 3; ++a) res[a] = -(t[a] - n[a] * normal) / (mu * c2) - n[a] * normal / ((lambda + 2 * mu) * c2);
}

/* src/three_d/PointKernels3D.hpp:67-72 */
static double traction_flux(const swlo_mesh3d *g, double *const *w, ptrdiff_t q, int axis, int comp) {
    static const int fields[3][3] = {{3, 6, 7}, {6, 4, 8}, {7, 8, 5}};
    const double *m = g->metrics + 9 * q + 3 * axis;
    double v = 0;
    for (int a = 0; a < 3; ++a) v += m[a] * w[fields[comp][a]][q];
    return g->jacobian[q] * v;
}

/* src/three_d/PointKernels3D.hpp:73-91; `only` >= 0: that axis's part alone (the CFS-PML split). */
static double surface_momentum(const swlo_mesh3d *g, double *const *w, ptrdiff_t q, int comp, const int *dirs, int depth,
                               int only) {
    double sum = 0;
    for (int axis = 0; axis < 3; ++axis) {
        if (only >= 0 && axis != only) continue;
        int off[5];
        double c[5];
        const int n = stencil(dirs[axis], -1, off, c);
        const ptrdiff_t s = axis == 0 ? 1 : axis == 1 ? g->nx : (ptrdiff_t)g->nx * g->ny;
        for (int l = 0; l < n; ++l) {
            int o = off[l];
            double sign = 1;
            if (axis == 2) {
                const int z = depth + o;
                if (z == 0) continue;
                if (z < 0) {
                    o = -z - depth;
                    sign = -1;
                }
            }
            sum += sign * c[l] * traction_flux(g, w, q + o * s, axis, comp);
        }
    }
    return sum / (g->h * g->jacobian[q] * rho3(g, q));
}

/* src/three_d/PointKernels3D.hpp:92-112 -- nine-field right-hand side at one node, with the
 * CFS-PML terms above for the nodes in a slab. */
static void rhs3_point(const swlo_mesh3d *g, double *const *w, const double *in_pml, double *const *out, double *out_pml,
                       ptrdiff_t q, double source, int step, int stage) {
    static const int F[3][3] = {{3, 6, 7}, {6, 4, 8}, {7, 8, 5}};
    const double lambda = lam3(g, q), mu = mu3(g, q), density = rho3(g, q);
    double gr[9][3], D[9][3];
    const double *m = g->metrics + 9 * q;
    const int depth = (int)(q / ((ptrdiff_t)g->nx * g->ny)) - 3;
    const int dirs[3] = {swlo_direction(step, stage, 0), swlo_direction(step, stage, 1), swlo_direction(step, stage, 2)};
    const int split = in_slab3(g, q);
    for (int f = 0; f < 9; ++f)
        for (int a = 0; a < 2; ++a) D[f][a] = d3(w[f], g, q, a, dirs[a], -1);
    if (split) /* the velocities' xi and eta derivatives, stretched before the surface solve */
        for (int v = 0; v < 3; ++v)
            for (int a = 0; a < 2; ++a) D[v][a] = stretched3(g, in_pml, out_pml, q, a, v, D[v][a]);
    double dzs[3] = {0, 0, 0};
    if (depth == 0) {
        const double xy[6] = {D[0][0], D[0][1], D[1][0], D[1][1], D[2][0], D[2][1]};
        surface_derivative3(g, w, q, dzs, dirs[0], dirs[1], split ? xy : 0);
    }
    for (int f = 0; f < 9; ++f) {
        D[f][2] = f < 3 && depth == 0 ? dzs[f] : d3(w[f], g, q, 2, dirs[2], f < 3 ? depth : -1);
        if (split && f < 3) D[f][2] = stretched3(g, in_pml, out_pml, q, 2, f, D[f][2]);
        for (int a = 0; a < 3; ++a) gr[f][a] = m[a] * D[f][0] + m[3 + a] * D[f][1] + m[6 + a] * D[f][2];
    }
    const int near = depth <= (dirs[2] ? 3 : 1);
    if (!split) {
        out[0][q] = (gr[3][0] + gr[6][1] + gr[7][2]) / density;
        out[1][q] = (gr[6][0] + gr[4][1] + gr[8][2]) / density;
        out[2][q] = (gr[7][0] + gr[8][1] + gr[5][2]) / density;
        if (near)
            for (int a = 0; a < 3; ++a) out[a][q] = surface_momentum(g, w, q, a, dirs, depth, -1);
    } else {
        for (int c = 0; c < 3; ++c) {
            double part[3];
            for (int a = 0; a < 3; ++a) {
                const double *ma = m + 3 * a; /* d(xi_a)/d(x, y, z) */
                part[a] = near ? surface_momentum(g, w, q, c, dirs, depth, a)
                               : (ma[0] * D[F[c][0]][a] + ma[1] * D[F[c][1]][a] + ma[2] * D[F[c][2]][a]) / density;
            }
            out[c][q] = stretched3(g, in_pml, out_pml, q, 0, 3 + c, part[0]) + stretched3(g, in_pml, out_pml, q, 1, 3 + c, part[1]) +
                        stretched3(g, in_pml, out_pml, q, 2, 3 + c, part[2]);
        }
    }
    for (int a = 0; a < 3; ++a)
        out[a][q] += source * (g->source_gradient[a] ? g->source_gradient[a][q] : g->source[q] * g->source_direction[a]) *
                     (g->density / density);
    const double div = gr[0][0] + gr[1][1] + gr[2][2];
    out[3][q] = lambda * div + 2 * mu * gr[0][0];
    out[4][q] = lambda * div + 2 * mu * gr[1][1];
    out[5][q] = lambda * div + 2 * mu * gr[2][2];
    out[6][q] = mu * (gr[0][1] + gr[1][0]);
    out[7][q] = mu * (gr[0][2] + gr[2][0]);
    out[8][q] = mu * (gr[1][2] + gr[2][1]);
    /* GSLS (the 2D form of src/two_d/PointKernels2D.hpp:161-168 with all six stress components):
     * drive = dl*div + 2 ds*e_aa on the normal components, ds*(g_ab + g_ba) on the shear ones,
     * dl = dP - 2 dS; the stresses subtract the memories; memory rate = rate_l (drive - memory). */
    for (int l = 0; l < g->mechanisms; ++l) {
        const int mm = 9 + 6 * l;
        const double dp = g->delta_p[l][q], ds = g->delta_s[l][q], dl = dp - 2 * ds;
        const double drive[6] = {dl * div + 2 * ds * gr[0][0], dl * div + 2 * ds * gr[1][1], dl * div + 2 * ds * gr[2][2],
                                 ds * (gr[0][1] + gr[1][0]),  ds * (gr[0][2] + gr[2][0]),  ds * (gr[1][2] + gr[2][1])};
        for (int c = 0; c < 6; ++c) out[3 + c][q] -= w[mm + c][q];
        for (int c = 0; c < 6; ++c) out[mm + c][q] = g->rates[l] * (drive[c] - w[mm + c][q]);
    }
    const int fc = g->field_count ? g->field_count : 9;
    for (int f = 0; f < fc; ++f) out[f][q] -= g->damping[q] * w[f][q];
}

/* src/three_d/CurvilinearSolver.cpp:70-89 */
void swlo3d_rhs(const swlo_mesh3d *g, double *const *in, const double *in_pml, double *const *out, double *out_pml,
                double source, int step, int stage) {
    const int fc = g->field_count ? g->field_count : 9;
    for (int f = 0; f < fc; ++f) memset(out[f], 0, sizeof(double) * (size_t)g->count);
    if (g->cpml_count) memset(out_pml, 0, sizeof(double) * (size_t)g->cpml_count);
    for (int k = 3; k < g->nz - 3; ++k)
        for (int j = 3; j < g->ny - 3; ++j)
            for (int i = 3; i < g->nx - 3; ++i)
                rhs3_point(g, in, in_pml, out, out_pml, i + (ptrdiff_t)g->nx * (j + (ptrdiff_t)g->ny * k), source, step, stage);
}

/* src/three_d/CurvilinearSolver.cpp:75-77 -- Ricker force/moment per unit volume. */
static double source3(const swlo_mesh3d *g, double t, double f) {
    const double scale = g->source_amplitude / (g->density * g->h * g->h * g->h);
    const double tau = 3.14159265358979323846 * f * (t - 1.5 / f);
    return scale * (1.0 - 2.0 * tau * tau) * exp(-tau * tau);
}

/* src/three_d/CurvilinearSolver.cpp:91-101 -- weighted sum in the reference's order. */
static void combine3(double *out, const double *base, const double *a, double wa, const double *b, double wb,
                     const double *c, double wc, const double *d, double wd, size_t n) {
    for (size_t q = 0; q < n; ++q)
        out[q] = base[q] + wa * a[q] + (b ? wb * b[q] : 0.0) + (c ? wc * c[q] : 0.0) + (d ? wd * d[q] : 0.0);
}

/* src/three_d/CurvilinearSolver.cpp:445-513 (CPU branch :460-473); the CFS-PML memories follow
 * the fields' RK sums. */
int swlo3d_run(const swlo_mesh3d *g, double *state, double *pml, int first, int steps, double dt, double frequency,
               const int64_t *receivers, int nreceivers, double *trace_vx, double *trace_vy, double *trace_vz) {
    const size_t n = (size_t)g->count, np = (size_t)(pml ? g->cpml_count : 0);
    const int fc = g->field_count ? g->field_count : 9;
    if ((g->cpml_count && !pml) || fc != 9 + 6 * g->mechanisms || fc > 27) return -1;
    double *mem = (double *)calloc(6 * (size_t)fc * n + 6 * (np + 1), sizeof(double));
    if (!mem) return -1;
    double *st[27], *base[27], *k[4][27], *sg[27];
    for (int f = 0; f < fc; ++f) {
        st[f] = state + f * n;
        base[f] = mem + f * n;
        for (int s = 0; s < 4; ++s) k[s][f] = mem + (size_t)(1 + s) * fc * n + f * n;
        sg[f] = mem + 5 * (size_t)fc * n + f * n;
    }
    double *pb = mem + 6 * (size_t)fc * n, *pk[4], *ps = pb + 5 * (np + 1);
    for (int s = 0; s < 4; ++s) pk[s] = pb + (size_t)(1 + s) * (np + 1);
    for (int it = 0; it < steps; ++it) {
        const int step = first + it;
        memcpy(mem, state, sizeof(double) * fc * n);
        if (np) memcpy(pb, pml, sizeof(double) * np);
        const double t = step * dt;
        swlo3d_rhs(g, st, pml, k[0], pk[0], source3(g, t, frequency), step, 0);
        for (int f = 0; f < fc; ++f) combine3(sg[f], base[f], k[0][f], 0.5 * dt, 0, 0, 0, 0, 0, 0, n);
        if (np) combine3(ps, pb, pk[0], 0.5 * dt, 0, 0, 0, 0, 0, 0, np);
        swlo3d_project(g, sg);
        swlo3d_rhs(g, sg, ps, k[1], pk[1], source3(g, t + 0.5 * dt, frequency), step, 1);
        for (int f = 0; f < fc; ++f) combine3(sg[f], base[f], k[1][f], 0.5 * dt, 0, 0, 0, 0, 0, 0, n);
        if (np) combine3(ps, pb, pk[1], 0.5 * dt, 0, 0, 0, 0, 0, 0, np);
        swlo3d_project(g, sg);
        swlo3d_rhs(g, sg, ps, k[2], pk[2], source3(g, t + 0.5 * dt, frequency), step, 2);
        for (int f = 0; f < fc; ++f) combine3(sg[f], base[f], k[2][f], dt, 0, 0, 0, 0, 0, 0, n);
        if (np) combine3(ps, pb, pk[2], dt, 0, 0, 0, 0, 0, 0, np);
        swlo3d_project(g, sg);
        swlo3d_rhs(g, sg, ps, k[3], pk[3], source3(g, t + dt, frequency), step, 3);
        for (int f = 0; f < fc; ++f)
            combine3(st[f], base[f], k[0][f], dt / 6.0, k[1][f], dt / 3.0, k[2][f], dt / 3.0, k[3][f], dt / 6.0, n);
        if (np) combine3(pml, pb, pk[0], dt / 6.0, pk[1], dt / 3.0, pk[2], dt / 3.0, pk[3], dt / 6.0, np);
        swlo3d_project(g, st);
        for (int r = 0; r < nreceivers; ++r) {
            const int64_t q = receivers[r];
            if (trace_vx) trace_vx[(size_t)r * steps + it] = st[0][q];
            if (trace_vy) trace_vy[(size_t)r * steps + it] = st[1][q];
            if (trace_vz) trace_vz[(size_t)r * steps + it] = st[2][q];
        }
    }
    free(mem);
    return 0;
}
