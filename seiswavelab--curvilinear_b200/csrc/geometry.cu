// FP64 curvilinear geometry of a 2D model, built on the GPU: node coordinates, the inverse
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

} // namespace swl::geo

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
