// FP64 curvilinear geometry built on the GPU.  2D: node coordinates, the inverse
// metrics a = d(eta)/dx and b = d(eta)/dz, the Jacobian and the unit surface normals of the
// terrain-following map x = xi, z = eta + H(xi) F(eta), with the ninth-order blend F that
// vanishes with four derivatives at both ends of [0, flatten depth]
// (src/two_d/CurvilinearSolver2D.cpp:344-356), plus the two reductions the dt plan needs (the
// smallest Jacobian and the largest metric norm sqrt(1 + a^2 + b^2) over the physical nodes,
// :357-361 and :464-479).  The surface height and slope per column come from the host (PCHIP or
// sinusoid, a one-dimensional evaluation); everything per node is computed here in FP64.
// Built without FMA contraction, like the reference; pow and hypot are CUDA's, so the arrays
// agree with the reference's host build to within a few ulp rather than bit for bit.
#include "../../include/swl_b200.h"
#include "runtime.cuh"
#include <algorithm>
#include <vector>

namespace swl::geo {

struct Range {
    double minJac, maxMetric;
};

__global__ void __launch_bounds__(256) geometry2d(int nx, int nz, int ghost, int offsetX, double h, double flatten,
                                                  const double *__restrict__ surface, double *coordinates, double *a,
                                                  double *b, double *jac, double *normals, Range *partial) {
    __shared__ Range sh[256];
    const int t = threadIdx.x;
    const long long q = blockIdx.x * 256ll + t;
    Range r{1e300, 0};
    if (q < (long long)nx * nz) {
        const int i = int(q % nx), k = int(q / nx);
        const double x = (i - ghost - offsetX) * h, eta = (k - ghost) * h;
        const double s = eta / flatten, tt = s < 0 ? 0.0 : s > 1 ? 1.0 : s;
        const double fade = 1 - pow(tt, 5) * (126 + tt * (-420 + tt * (540 + tt * (-315 + 70 * tt))));
        const double fadeDerivative = eta > 0 && eta < flatten ? -630 * pow(tt, 4) * pow(1 - tt, 4) / flatten : 0;
        const double zx = surface[2 * i + 1] * fade, j = 1 + surface[2 * i] * fadeDerivative;
        coordinates[2 * q] = x;
        coordinates[2 * q + 1] = eta + surface[2 * i] * fade;
        const double ma = -zx / j, mb = 1 / j;
        a[q] = ma, b[q] = mb, jac[q] = j;
        const double n = hypot(zx, 1.0);
        normals[2 * q] = -zx / n;
        normals[2 * q + 1] = 1 / n;
        if (i >= ghost && i < nx - ghost && k >= ghost && k < nz - ghost)
            r.minJac = j, r.maxMetric = sqrt(1 + ma * ma + mb * mb);
        if (!(j > 1e-9) || !isfinite(j)) r.minJac = -1; // reported to the host as a nonpositive Jacobian
    }
    sh[t] = r;
    __syncthreads();
    for (int stride = 128; stride > 0; stride >>= 1) {
        if (t < stride) sh[t].minJac = fmin(sh[t].minJac, sh[t + stride].minJac), sh[t].maxMetric = fmax(sh[t].maxMetric, sh[t + stride].maxMetric);
        __syncthreads();
    }
    if (t == 0) partial[blockIdx.x] = sh[0];
}

// 3D (src/three_d/CurvilinearSolver.cpp:146-190): node coordinates x, y, depth + S(x, y) F(depth)
// with the same blend, then fourth-order central differences of the coordinates, the Jacobian
// r_xi . (r_eta x r_zeta), the cofactor inverse metrics and the unit surface normal on the top
// row.  `surface` holds S per padded column (host-evaluated: DEM bilinear or the sinusoid).
__global__ void __launch_bounds__(256) coordinates3d(int nx, int ny, int nz, int ghost, double h, double dz, double ttd,
                                                     int terrain, const double *__restrict__ surface, double *coordinates) {
    const long long q = blockIdx.x * 256ll + threadIdx.x;
    const long long plane = (long long)nx * ny;
    if (q >= plane * nz) return;
    const int i = int(q % nx), j = int((q / nx) % ny), k = int(q / plane);
    const double x = (i - ghost) * h, y = (j - ghost) * h, depth = (k - ghost) * dz;
    double z = depth;
    if (terrain) {
        const double s = depth / ttd, ss = s < 0 ? 0.0 : s > 1 ? 1.0 : s;
        const double fade = depth >= ttd ? 0.0 : 1.0 - pow(ss, 5) * (126.0 + ss * (-420.0 + ss * (540.0 + ss * (-315.0 + 70.0 * ss))));
        z = depth + surface[i + (long long)nx * j] * fade;
    }
    coordinates[3 * q] = x, coordinates[3 * q + 1] = y, coordinates[3 * q + 2] = z;
}

__global__ void __launch_bounds__(256) metrics3d(int nx, int ny, int nz, int ghost, double h, int terrain,
                                                 const double *__restrict__ c, double *metrics, double *jac, double *normals,
                                                 Range *partial) {
    __shared__ Range sh[256];
    const int t = threadIdx.x;
    const long long plane = (long long)nx * ny;
    const long long q = blockIdx.x * 256ll + t;
    Range r{1e300, 0};
    if (q < plane * nz) {
        const int i = int(q % nx), j = int((q / nx) % ny), k = int(q / plane);
        if (i >= ghost && i < nx - ghost && j >= ghost && j < ny - ghost && k >= ghost && k < nz - ghost) {
            double *m = metrics + 9 * q;
            double J = 1;
            if (!terrain) {
                for (int a = 0; a < 9; ++a) m[a] = (a % 4 == 0) ? 1.0 : 0.0;
                jac[q] = 1;
                if (k == ghost) normals[3 * q] = 0, normals[3 * q + 1] = 0, normals[3 * q + 2] = 1;
            } else {
                const long long stride[3] = {1, nx, plane};
                double d[3][3]; // d[axis][component]
                for (int axis = 0; axis < 3; ++axis)
                    for (int comp = 0; comp < 3; ++comp) {
                        const long long s = stride[axis];
                        d[axis][comp] = (c[3 * (q - 2 * s) + comp] - 8.0 * c[3 * (q - s) + comp] + 8.0 * c[3 * (q + s) + comp] -
                                         c[3 * (q + 2 * s) + comp]) /
                                        (12.0 * h);
                    }
                const double *rx = d[0], *re = d[1], *rz = d[2];
                const double ez[3] = {re[1] * rz[2] - re[2] * rz[1], re[2] * rz[0] - re[0] * rz[2], re[0] * rz[1] - re[1] * rz[0]};
                const double zx[3] = {rz[1] * rx[2] - rz[2] * rx[1], rz[2] * rx[0] - rz[0] * rx[2], rz[0] * rx[1] - rz[1] * rx[0]};
                const double xe[3] = {rx[1] * re[2] - rx[2] * re[1], rx[2] * re[0] - rx[0] * re[2], rx[0] * re[1] - rx[1] * re[0]};
                J = rx[0] * ez[0] + rx[1] * ez[1] + rx[2] * ez[2];
                jac[q] = J;
                for (int a = 0; a < 3; ++a) m[a] = ez[a] / J, m[3 + a] = zx[a] / J, m[6 + a] = xe[a] / J;
                if (k == ghost) {
                    const double length = sqrt(xe[0] * xe[0] + xe[1] * xe[1] + xe[2] * xe[2]);
                    for (int a = 0; a < 3; ++a) normals[3 * q + a] = xe[a] / length;
                    if (!(length > 0) || !isfinite(length)) J = -1; // reported as a failed surface normal
                }
            }
            double norm2 = 0;
            for (int a = 0; a < 9; ++a) norm2 += m[a] * m[a];
            r.minJac = (J > 1e-10 && isfinite(J)) ? J : -1, r.maxMetric = sqrt(norm2);
        }
    }
    sh[t] = r;
    __syncthreads();
    for (int stride = 128; stride > 0; stride >>= 1) {
        if (t < stride) sh[t].minJac = fmin(sh[t].minJac, sh[t + stride].minJac), sh[t].maxMetric = fmax(sh[t].maxMetric, sh[t + stride].maxMetric);
        __syncthreads();
    }
    if (t == 0) partial[blockIdx.x] = sh[0];
}

} // namespace swl::geo

extern "C" swl_status swl3d_build_geometry(const swl_geometry3d *g, int32_t device, double *coordinates, double *metrics,
                                           double *jacobian, double *normals, double *min_jacobian, double *max_metric_norm) {
    try {
        if (!g || (g->terrain && !g->surface) || !coordinates || !metrics || !jacobian || !normals || !min_jacobian ||
            !max_metric_norm)
            throw swl::Error(SWL_ERR_INVALID, "geometry description and every output are required");
        if (g->nx < 7 || g->ny < 7 || g->nz < 7 || g->ghost < 2 || !(g->spacing > 0) || !(g->dz > 0) || !(g->flatten_depth > 0))
            throw swl::Error(SWL_ERR_INVALID, "geometry needs nx, ny, nz >= 7, ghost >= 2, positive spacings and flatten depth");
        const int dev = swl::selectDevice(device);
        if (dev < 0) throw swl::Error(SWL_ERR_UNAVAILABLE, "no usable sm_100 CUDA device");
        swl::DeviceScope scope(dev);
        const std::size_t plane = std::size_t(g->nx) * g->ny, n = plane * g->nz;
        const int blocks = int((n + 255) / 256);
        swl::DeviceBuffer surf(std::max<std::size_t>(1, plane) * sizeof(double)), coords(3 * n * sizeof(double)),
            met(9 * n * sizeof(double)), jac(n * sizeof(double)), nor(3 * n * sizeof(double)),
            part(std::size_t(blocks) * sizeof(swl::geo::Range));
        if (g->terrain) swl::check(cudaMemcpy(surf.ptr, g->surface, plane * sizeof(double), cudaMemcpyHostToDevice), "geometry surface upload");
        swl::geo::coordinates3d<<<blocks, 256>>>(g->nx, g->ny, g->nz, g->ghost, g->spacing, g->dz, g->flatten_depth, g->terrain,
                                                 surf.as<double>(), coords.as<double>());
        swl::geo::metrics3d<<<blocks, 256>>>(g->nx, g->ny, g->nz, g->ghost, g->spacing, g->terrain, coords.as<double>(),
                                             met.as<double>(), jac.as<double>(), nor.as<double>(), part.as<swl::geo::Range>());
        swl::check(cudaGetLastError(), "geometry launch");
        std::vector<swl::geo::Range> parts(blocks);
        swl::check(cudaMemcpy(parts.data(), part.ptr, part.bytes, cudaMemcpyDeviceToHost), "geometry reduction readback");
        swl::check(cudaMemcpy(coordinates, coords.ptr, coords.bytes, cudaMemcpyDeviceToHost), "geometry readback");
        swl::check(cudaMemcpy(metrics, met.ptr, met.bytes, cudaMemcpyDeviceToHost), "geometry readback");
        swl::check(cudaMemcpy(jacobian, jac.ptr, jac.bytes, cudaMemcpyDeviceToHost), "geometry readback");
        swl::check(cudaMemcpy(normals, nor.ptr, nor.bytes, cudaMemcpyDeviceToHost), "geometry readback");
        double mj = 1e300, mm = 0;
        for (const auto &p : parts) mj = std::min(mj, p.minJac), mm = std::max(mm, p.maxMetric);
        if (!(mj > 0)) throw swl::Error(SWL_ERR_INVALID, "Curvilinear mapping has a non-positive or non-finite Jacobian.");
        *min_jacobian = mj, *max_metric_norm = mm;
        return SWL_OK;
    } catch (const swl::Error &e) {
        swl::lastErrorRef() = e.what();
        return swl_status(e.status);
    } catch (const std::exception &e) {
        swl::lastErrorRef() = e.what();
        return SWL_ERR_INVALID;
    }
}

extern "C" swl_status swl2d_build_geometry(const swl_geometry2d *g, int32_t device, double *coordinates, double *metric_a,
                                           double *metric_b, double *jacobian, double *normals, double *min_jacobian,
                                           double *max_metric) {
    try {
        if (!g || !g->surface || !coordinates || !metric_a || !metric_b || !jacobian || !normals || !min_jacobian || !max_metric)
            throw swl::Error(SWL_ERR_INVALID, "geometry description and every output are required");
        if (g->nx < 7 || g->nz < 7 || g->ghost < 0 || !(g->spacing > 0) || !(g->flatten_depth > 0))
            throw swl::Error(SWL_ERR_INVALID, "geometry needs nx, nz >= 7, ghost >= 0, spacing > 0 and flatten depth > 0");
        const int dev = swl::selectDevice(device);
        if (dev < 0) throw swl::Error(SWL_ERR_UNAVAILABLE, "no usable sm_100 CUDA device");
        swl::DeviceScope scope(dev);
        const std::size_t n = std::size_t(g->nx) * g->nz;
        const int blocks = int((n + 255) / 256);
        swl::DeviceBuffer surf(2 * std::size_t(g->nx) * sizeof(double)), coords(2 * n * sizeof(double)), a(n * sizeof(double)),
            b(n * sizeof(double)), jac(n * sizeof(double)), nor(2 * n * sizeof(double)),
            part(std::size_t(blocks) * sizeof(swl::geo::Range));
        swl::check(cudaMemcpy(surf.ptr, g->surface, surf.bytes, cudaMemcpyHostToDevice), "geometry surface upload");
        swl::geo::geometry2d<<<blocks, 256>>>(g->nx, g->nz, g->ghost, g->offset_x, g->spacing, g->flatten_depth, surf.as<double>(),
                                              coords.as<double>(), a.as<double>(), b.as<double>(), jac.as<double>(),
                                              nor.as<double>(), part.as<swl::geo::Range>());
        swl::check(cudaGetLastError(), "geometry launch");
        std::vector<swl::geo::Range> parts(blocks);
        swl::check(cudaMemcpy(parts.data(), part.ptr, part.bytes, cudaMemcpyDeviceToHost), "geometry reduction readback");
        swl::check(cudaMemcpy(coordinates, coords.ptr, coords.bytes, cudaMemcpyDeviceToHost), "geometry readback");
        swl::check(cudaMemcpy(metric_a, a.ptr, a.bytes, cudaMemcpyDeviceToHost), "geometry readback");
        swl::check(cudaMemcpy(metric_b, b.ptr, b.bytes, cudaMemcpyDeviceToHost), "geometry readback");
        swl::check(cudaMemcpy(jacobian, jac.ptr, jac.bytes, cudaMemcpyDeviceToHost), "geometry readback");
        swl::check(cudaMemcpy(normals, nor.ptr, nor.bytes, cudaMemcpyDeviceToHost), "geometry readback");
        double mj = 1e300, mm = 0;
        for (const auto &p : parts) mj = std::min(mj, p.minJac), mm = std::max(mm, p.maxMetric);
        if (!(mj > 0)) throw swl::Error(SWL_ERR_INVALID, "Nonpositive curvilinear Jacobian.");
        *min_jacobian = mj, *max_metric = mm;
        return SWL_OK;
    } catch (const swl::Error &e) {
        swl::lastErrorRef() = e.what();
        return swl_status(e.status);
    } catch (const std::exception &e) {
        swl::lastErrorRef() = e.what();
        return SWL_ERR_INVALID;
    }
}
