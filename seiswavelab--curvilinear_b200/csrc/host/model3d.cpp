// 3D model construction: validateSimulationConfiguration3D, Grid3D::buildGeometry and the model
// part of CpuSimulation3D::initialize (src/three_d/CurvilinearSolver.cpp:117-190, 258-442) with the
// helpers of include/Seis3D/{AbsorbingBoundary3D,TimeStepPlan3D,MaterialModels3D,ReceiverGeometry3D}.hpp.
#include "model.hpp"
#include "../../../include/swl_b200.h"
#include <algorithm>
#include <cmath>
#include <limits>
#include <stdexcept>

namespace swl::host {
namespace {
constexpr double kPi = 3.14159265358979323846;
constexpr int ghost = 3;
using V3 = std::array<double, 3>;
void require(bool ok, const char *message) {
    if (!ok) throw std::runtime_error(message);
}
V3 cross(const V3 &a, const V3 &b) { return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]}; }
double dot(const V3 &a, const V3 &b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// include/Seis3D/ReceiverGeometry3D.hpp:30-42 (limit configurable; the reference caps 1024)
std::vector<std::array<int, 3>> receiverNodes(const Params3D &p) {
    std::vector<std::array<int, 3>> nodes;
    const int limit = p.receiverLimit;
    require(p.receiverKind >= 0 && p.receiverKind <= 3 && p.receiverZ >= 0 && p.receiverZ < p.nz,
            "Invalid receiver grid, mode, start, active stride or depth index.");
    if (p.receiverKind == 0) {
        require(p.nx - 4 <= limit, "Auto X line exceeds 1024 traces; select a custom line with a larger receiver stride.");
        for (int i = 2; i < p.nx - 2; ++i) nodes.push_back({i, p.ny / 2, p.receiverZ});
        return nodes;
    }
    const int x = p.receiverStartX == -1 ? p.nx / 2 : p.receiverStartX, y = p.receiverStartY == -1 ? p.ny / 2 : p.receiverStartY;
    require(x >= 0 && x < p.nx && y >= 0 && y < p.ny, "Invalid receiver grid, mode, start, active stride or depth index.");
    const auto capacity = [](int n, int start, int stride) { return stride > 0 ? 1 + (n - 1 - start) / stride : 0; };
    const int lx = p.receiverKind == 2 ? 1 : capacity(p.nx, x, p.receiverStrideX);
    const int ly = p.receiverKind == 1 ? 1 : capacity(p.ny, y, p.receiverStrideY);
    const int cx = p.receiverKind == 2 ? 1 : p.receiverCountX, cy = p.receiverKind == 1 ? 1 : p.receiverCountY;
    require(lx > 0 && ly > 0 && cx >= 1 && cy >= 1 && cx <= lx && cy <= ly && (long long)cx * cy <= limit,
            "Receiver counts exceed the start/stride capacity or the trace limit. Review capacity or fit counts.");
    for (int j = 0; j < cy; ++j)
        for (int i = 0; i < cx; ++i)
            nodes.push_back({x + i * (p.receiverKind == 2 ? 0 : p.receiverStrideX), y + j * (p.receiverKind == 1 ? 0 : p.receiverStrideY),
                             p.receiverZ});
    return nodes;
}
} // namespace

Model3D buildModel3D(const Params3D &p) {
    // validateSimulationConfiguration3D (src/three_d/CurvilinearSolver.cpp:258-299)
    require(p.precision == 0 || p.precision == 1, "Unknown 3D calculation precision.");
    require(std::isfinite(p.cfl) && p.cfl >= .02 && p.cfl <= .8, "CFL coefficient must be finite and in 0.02..0.8.");
    require(p.maxSteps >= 0 && p.maxSteps <= 20000, "Maximum steps must be 0 (duration) or 1..20,000.");
    require(std::isfinite(p.absorbingStrength) && p.absorbingStrength >= 0.1 && p.absorbingStrength <= 10.0,
            "Sponge strength must be in 0.1..10.");
    for (int w : p.absorbingCells) require(w >= 1 && w <= 64, "Sponge widths must be 1..64 cells.");
    require(p.absorber == 0 || p.absorber == 1, "Unknown 3D absorber (0 sponge, 1 CFS-PML).");
    if (p.absorbing && p.absorber == 1) // the 2D CFS-PML limits (CurvilinearSolver2D.cpp validation)
        require(std::isfinite(p.cpmlReflection) && p.cpmlReflection >= 1e-8 && p.cpmlReflection <= .1 &&
                    std::isfinite(p.cpmlKappaMax) && p.cpmlKappaMax >= 1 && p.cpmlKappaMax <= 20 &&
                    std::isfinite(p.cpmlFrequency) && p.cpmlFrequency >= 0 && p.cpmlFrequency <= 1e6,
                "CFS-PML reflection must be in 1e-8..0.1, kappa max in 1..20 and frequency in 0..1e6.");
    for (double v : {p.spacing, p.vp, p.vs, p.density, p.frequency, p.duration, p.relief, p.wavelength, p.flattenDepth})
        require(std::isfinite(v), "Simulation parameters must be finite.");
    require(!(p.nx < 8 || p.ny < 8 || p.nz < 8 || p.nx > 4096 || p.ny > 4096 || p.nz > 4096 || p.spacing <= 0 || p.vp <= 0 ||
              p.vs <= 0 || p.density <= 0 || p.vp * p.vp <= 4.0 * p.vs * p.vs / 3.0 || p.frequency <= 0 || p.frequency > 1e6 ||
              p.duration <= 0 || p.duration > 10 || p.wavelength <= 0 || p.flattenDepth < 0 ||
              (p.surfaceGrid.empty() && p.relief != 0 && p.wavelength < 4.0 * p.spacing)),
            "Require 8..4096 nodes per axis within the total node/memory budget, positive finite parameters and resolved topography.");
    const std::size_t points = std::size_t(p.nx + 6) * (p.ny + 6) * (p.nz + 6);
    require(points <= std::size_t(306) * 306 * 306, "Grid exceeds the 28,652,616 padded-node total budget; redistribute X/Y/Z nodes.");
    const bool moment = p.sourceKind == 1;
    require(p.sourceKind == 0 || p.sourceKind == 1, "Unknown source mechanism.");
    if (!moment) {
        const double norm = std::hypot(p.sourceDirection[0], p.sourceDirection[1], p.sourceDirection[2]);
        require(std::isfinite(norm) && norm > 0, "Force direction must be finite and nonzero.");
    }
    require(std::isfinite(p.sourceForce) && std::isfinite(p.sourceMoment) && (moment ? p.sourceMoment : p.sourceForce) > 0,
            "Source amplitudes must be finite and the active force (N) or moment (N*m) must be positive.");
    const std::array<int, 3> src{p.sourceX < 0 ? p.nx / 2 : p.sourceX, p.sourceY < 0 ? p.ny / 2 : p.sourceY, p.sourceZ};
    if (moment)
        require(!(p.nx < 11 || p.ny < 11 || p.nz < 11 || src[0] < 5 || src[0] > p.nx - 6 || src[1] < 5 || src[1] > p.ny - 6 ||
                  src[2] < 5 || src[2] > p.nz - 6),
                "Isotropic moment needs 11+ nodes per axis and source center five nodes inside each face.");
    require(!(p.sourceX < -1 || p.sourceY < -1 || src[0] < 2 || src[0] > p.nx - 3 || src[1] < 2 || src[1] > p.ny - 3 ||
              src[2] < 2 || src[2] > p.nz - 3),
            "Source must stay two nodes inside every physical face; X/Y may be -1 for center.");
    if (p.layered) { // include/Seis3D/MaterialModels3D.hpp:32-41
        require(p.layerDepthMode >= 0 && p.layerDepthMode <= 2, "Invalid layer depth coordinate mode.");
        require(p.layers.size() >= 2 && p.layers.size() <= 8, "Layered material requires 2..8 layers.");
        for (std::size_t i = 0; i < p.layers.size(); ++i) {
            const auto &l = p.layers[i];
            require(std::isfinite(l.thickness) && std::isfinite(l.vp) && std::isfinite(l.vs) && std::isfinite(l.density) && l.vp > 0 &&
                        l.vs > 0 && l.density > 0 && l.vp * l.vp > 4 * l.vs * l.vs / 3 && std::isfinite(l.density * l.vp * l.vp) &&
                        l.density * l.vs * l.vs > 0 && (i + 1 == p.layers.size() ? l.thickness == 0 : l.thickness > 0),
                    "Invalid layer: positive finite Vp/Vs/density and bulk modulus required; last thickness must be zero (auto).");
        }
    }
    const auto rnodes = receiverNodes(p);
    if (!p.surfaceGrid.empty()) {
        const auto &s = p.surfaceGrid;
        require(s.nx >= 2 && s.ny >= 2 && s.nx <= 4096 && s.ny <= 4096 && s.elevations.size() == std::size_t(s.nx) * s.ny &&
                    std::isfinite(s.spacing) && s.spacing > 0 && std::isfinite(s.datum),
                "DEM array requires 2..4096 rows/columns, at most 4 million samples, positive metre spacing and finite origin/datum.");
        for (double e : s.elevations) require(std::isfinite(e) && std::abs(e) <= 1e7, "DEM contains missing, nonfinite or unreasonable elevations.");
        require(!((p.nx - 1) * p.spacing > (s.nx - 1) * s.spacing + 1e-8 * s.spacing || (p.ny - 1) * p.spacing > (s.ny - 1) * s.spacing + 1e-8 * s.spacing),
                "Imported DEM does not cover the staged X/Y model span; reduce dimensions/spacing or export a larger region.");
    }
    Model3D g;
    g.nx = p.nx + 6, g.ny = p.ny + 6, g.nz = p.nz + 6, g.h = p.spacing;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const std::size_t plane = std::size_t(nx) * ny, count = plane * nz;
    const auto index = [&](int i, int j, int k) { return std::size_t(i) + std::size_t(nx) * (std::size_t(j) + std::size_t(ny) * std::size_t(k)); };
    const double dz = p.spacing;
    // Grid3D::validateGeometry (:117-145): transition depth
    const bool terrain = !p.surfaceGrid.empty() || p.relief != 0;
    const double bottomDepth = (nz - 2 * ghost - 1) * dz;
    double relief = std::abs(p.relief);
    if (!p.surfaceGrid.empty()) {
        relief = 0;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                relief = std::max(relief, std::abs(p.surfaceGrid.displacement((i - ghost) * p.spacing, (j - ghost) * p.spacing)));
    }
    double ttd = p.flattenDepth;
    if (ttd == 0.0) ttd = std::min(bottomDepth, std::max({0.35 * bottomDepth, 6.0 * dz, 4.0 * relief + 2.0 * dz}));
    require(!(ttd > bottomDepth || (terrain && (ttd < 4.0 * dz || ttd <= 2.6 * relief))),
            "Terrain transition must fit the model depth and exceed 2.6 times relief amplitude (at least four cells).");
    g.flattenDepth = ttd;
    // Grid3D::buildGeometry (:146-190)
    g.coordinates.assign(3 * count, 0);
    g.metrics.assign(9 * count, 0);
    g.jacobian.assign(count, 0);
    g.normals.assign(3 * count, 0);
    if (p.deviceGeometry) { // the node geometry below, computed on the GPU from the surface per column
        std::vector<double> columns(terrain ? plane : 1, 0.0);
        if (terrain)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    const double x = (i - ghost) * p.spacing, y = (j - ghost) * p.spacing;
                    const double phaseX = 2.0 * kPi * x / p.wavelength, phaseY = 2.0 * kPi * y / p.wavelength;
                    columns[i + std::size_t(nx) * j] =
                        p.surfaceGrid.empty() ? p.relief * std::cos(phaseX) * std::cos(phaseY) : p.surfaceGrid.displacement(x, y);
                }
        const swl_geometry3d geo{nx, ny, nz, ghost, p.spacing, dz, ttd, terrain ? 1 : 0, columns.data()};
        double minJ = 0, maxM = 0;
        if (swl3d_build_geometry(&geo, p.geometryDevice, g.coordinates.data(), g.metrics.data(), g.jacobian.data(),
                                 g.normals.data(), &minJ, &maxM) != SWL_OK)
            throw std::runtime_error(swl_last_error());
    } else {
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const double x = (i - ghost) * p.spacing, y = (j - ghost) * p.spacing, depth = (k - ghost) * dz;
                const std::size_t q = index(i, j, k);
                if (!terrain) {
                    g.coordinates[3 * q] = x, g.coordinates[3 * q + 1] = y, g.coordinates[3 * q + 2] = depth;
                    continue;
                }
                const double phaseX = 2.0 * kPi * x / p.wavelength, phaseY = 2.0 * kPi * y / p.wavelength;
                const double surface = p.surfaceGrid.empty() ? p.relief * std::cos(phaseX) * std::cos(phaseY) : p.surfaceGrid.displacement(x, y);
                const double s = std::clamp(depth / ttd, 0.0, 1.0);
                const double fade = depth >= ttd ? 0.0 : 1.0 - std::pow(s, 5) * (126.0 + s * (-420.0 + s * (540.0 + s * (-315.0 + 70.0 * s))));
                g.coordinates[3 * q] = x, g.coordinates[3 * q + 1] = y, g.coordinates[3 * q + 2] = depth + surface * fade;
            }
    const auto at = [&](int c, int i, int j, int k) { return g.coordinates[3 * index(i, j, k) + c]; };
    // src/three_d/CurvilinearSolver.cpp:47-54: 4th-order central difference of the coordinates
    const auto dcoord = [&](int c, int i, int j, int k, int axis) {
        const int di = axis == 0, dj = axis == 1, dk = axis == 2;
        return (at(c, i - 2 * di, j - 2 * dj, k - 2 * dk) - 8.0 * at(c, i - di, j - dj, k - dk) + 8.0 * at(c, i + di, j + dj, k + dk) -
                at(c, i + 2 * di, j + 2 * dj, k + 2 * dk)) /
               (12.0 * p.spacing);
    };
    for (int k = ghost; k < nz - ghost; ++k)
        for (int j = ghost; j < ny - ghost; ++j)
            for (int i = ghost; i < nx - ghost; ++i) {
                const std::size_t q = index(i, j, k);
                double *m = &g.metrics[9 * q];
                if (!terrain) {
                    m[0] = m[4] = m[8] = 1;
                    g.jacobian[q] = 1;
                    if (k == ghost) g.normals[3 * q + 2] = 1;
                    continue;
                }
                V3 rXi{}, rEta{}, rZeta{};
                for (int c = 0; c < 3; ++c) rXi[c] = dcoord(c, i, j, k, 0), rEta[c] = dcoord(c, i, j, k, 1), rZeta[c] = dcoord(c, i, j, k, 2);
                const V3 ez = cross(rEta, rZeta), zx = cross(rZeta, rXi), xe = cross(rXi, rEta);
                const double jac = dot(rXi, ez);
                require(jac > 1.0e-10 && std::isfinite(jac), "Curvilinear mapping has a non-positive or non-finite Jacobian.");
                g.jacobian[q] = jac;
                for (int c = 0; c < 3; ++c) m[c] = ez[c] / jac, m[3 + c] = zx[c] / jac, m[6 + c] = xe[c] / jac;
                if (k == ghost) {
                    V3 n = xe;
                    const double length = std::sqrt(dot(n, n));
                    require(length > 0.0 && std::isfinite(length), "Could not compute topographic surface normal.");
                    for (double &v : n) v /= length;
                    for (int c = 0; c < 3; ++c) g.normals[3 * q + c] = n[c];
                }
            }
    }
    // geometry diagnostics (:330-364)
    g.minJacobian = std::numeric_limits<double>::max();
    double maxMetricNorm = 0;
    for (int k = ghost; k < nz - ghost; ++k)
        for (int j = ghost; j < ny - ghost; ++j)
            for (int i = ghost; i < nx - ghost; ++i) {
                const std::size_t q = index(i, j, k);
                g.minJacobian = std::min(g.minJacobian, g.jacobian[q]);
                double norm2 = 0;
                for (int c = 0; c < 9; ++c) norm2 += g.metrics[9 * q + c] * g.metrics[9 * q + c];
                maxMetricNorm = std::max(maxMetricNorm, std::sqrt(norm2));
            }
    g.maxMetricNorm = maxMetricNorm;
    const auto coord = [&](int i, int j, int k) { const std::size_t q = index(i, j, k); return V3{g.coordinates[3 * q], g.coordinates[3 * q + 1], g.coordinates[3 * q + 2]}; };
    double minLength = !terrain ? p.spacing / std::sqrt(3.0) : std::numeric_limits<double>::max();
    if (terrain) // CFL: smallest distance from a node to its eight adjacent planes
        for (int k = ghost; k < nz - ghost; ++k)
            for (int j = ghost; j < ny - ghost; ++j)
                for (int i = ghost; i < nx - ghost; ++i) {
                    const V3 center = coord(i, j, k);
                    for (int sk : {-1, 1})
                        for (int sj : {-1, 1})
                            for (int si : {-1, 1}) {
                                const V3 a = coord(i + si, j, k), b = coord(i, j + sj, k), c = coord(i, j, k + sk);
                                V3 ab{}, ac{}, ap{};
                                for (int x = 0; x < 3; ++x) ab[x] = b[x] - a[x], ac[x] = c[x] - a[x], ap[x] = center[x] - a[x];
                                const V3 normal = cross(ab, ac);
                                const double length = std::sqrt(dot(normal, normal));
                                const double distance = std::abs(dot(ap, normal)) / length;
                                require(std::isfinite(distance) && distance > 0, "Degenerate adjacent cell plane in CFL geometry.");
                                minLength = std::min(minLength, distance);
                            }
                }
    g.minCellLength = minLength;
    double maxEdge = !terrain ? p.spacing : 0;
    if (terrain)
        for (int k = ghost; k < nz - ghost; ++k)
            for (int j = ghost; j < ny - ghost; ++j)
                for (int i = ghost; i < nx - ghost; ++i) {
                    const V3 a = coord(i, j, k);
                    for (int axis = 0; axis < 3; ++axis) {
                        const int ni = i + (axis == 0), nj = j + (axis == 1), nk = k + (axis == 2);
                        if (ni >= nx - ghost || nj >= ny - ghost || nk >= nz - ghost) continue;
                        const V3 b = coord(ni, nj, nk);
                        V3 d{};
                        for (int c = 0; c < 3; ++c) d[c] = b[c] - a[c];
                        maxEdge = std::max(maxEdge, std::sqrt(dot(d, d)));
                    }
                }
    g.maxCellEdge = maxEdge;
    g.lambda = p.density * (p.vp * p.vp - 2.0 * p.vs * p.vs);
    g.mu = p.density * p.vs * p.vs;
    g.density = p.density;
    require(std::isfinite(g.lambda) && std::isfinite(g.mu) && g.mu > 0 && std::isfinite(maxMetricNorm),
            "Derived elastic coefficients or grid metrics are out of range.");
    double maxVp = p.vp, minVs = p.vs;
    // GSLS: one fit per layer (or for the uniform model); the moduli become the unrelaxed ones
    validateGsls(p.attenuation);
    const int L = p.attenuation.enabled ? p.attenuation.mechanisms : 0;
    std::vector<GslsMaterial> rheology;
    if (L) {
        auto q = [&](double v, double fallback) { return v >= 0 ? v : fallback; };
        if (p.layered)
            for (const auto &l : p.layers)
                rheology.push_back(fitGsls(l.vp, l.vs, l.density, q(l.qp, p.attenuation.qp), q(l.qs, p.attenuation.qs), p.attenuation));
        else
            rheology.push_back(fitGsls(p.vp, p.vs, p.density, p.attenuation.qp, p.attenuation.qs, p.attenuation));
        g.mechanisms = L;
        g.rates = rheology.front().rates;
        g.gslsRates.assign(g.rates.begin(), g.rates.begin() + L);
        for (int l = 0; l < L; ++l) g.deltaP[l].assign(count, 0), g.deltaS[l].assign(count, 0);
        for (const auto &r : rheology) g.maxRelativeQError = std::max(g.maxRelativeQError, r.maxRelativeQError);
        g.relaxationDt = .25 / g.rates[L - 1];
    } else {
        g.relaxationDt = std::numeric_limits<double>::max();
    }
    if (p.layered || L) { // include/Seis3D/MaterialModels3D.hpp:19-31 (uniform: one layer)
        const std::vector<Layer3D> uniform{Layer3D{0, p.vp, p.vs, p.density}};
        const auto &layers = p.layered ? p.layers : uniform;
        maxVp = 0, minVs = std::numeric_limits<double>::max();
        for (std::size_t l = 0; l < layers.size(); ++l) {
            maxVp = std::max(maxVp, L ? std::sqrt(rheology[l].pUnrelaxed / layers[l].density) : layers[l].vp);
            minVs = std::min(minVs, L ? std::sqrt(rheology[l].sRelaxed / layers[l].density) : layers[l].vs);
        }
        g.materialLambda.resize(count), g.materialMu.resize(count), g.materialDensity.resize(count);
        for (std::size_t q = 0; q < count; ++q) {
            if (!p.layered) { // uniform model with GSLS: the fitted unrelaxed moduli everywhere
                const auto &r = rheology.front();
                g.materialLambda[q] = r.pUnrelaxed - 2 * r.sUnrelaxed, g.materialMu[q] = r.sUnrelaxed;
                g.materialDensity[q] = p.density;
                for (int l = 0; l < L; ++l) g.deltaP[l][q] = r.deltaP[l], g.deltaS[l][q] = r.deltaS[l];
                continue;
            }
            double depth;
            if (p.layerDepthMode == 0) depth = (static_cast<int>(q / plane) - ghost) * dz;
            else if (p.layerDepthMode == 2) depth = g.coordinates[3 * q + 2];
            else depth = g.coordinates[3 * q + 2] - g.coordinates[3 * (std::size_t(ghost) * plane + q % plane) + 2];
            int id = int(p.layers.size()) - 1;
            double bottom = 0;
            for (std::size_t l = 0; l + 1 < p.layers.size(); ++l) {
                bottom += p.layers[l].thickness;
                if (depth < bottom) {
                    id = int(l);
                    break;
                }
            }
            const auto &l = p.layers[id];
            g.materialLambda[q] = l.density * (l.vp * l.vp - 2 * l.vs * l.vs);
            g.materialMu[q] = l.density * l.vs * l.vs;
            g.materialDensity[q] = l.density;
            if (L) {
                const auto &r = rheology[id];
                g.materialLambda[q] = r.pUnrelaxed - 2 * r.sUnrelaxed, g.materialMu[q] = r.sUnrelaxed;
                for (int k = 0; k < L; ++k) g.deltaP[k][q] = r.deltaP[k], g.deltaS[k][q] = r.deltaS[k];
            }
        }
    }
    // sponge (include/Seis3D/AbsorbingBoundary3D.hpp:6-21)
    g.damping.assign(count, 0);
    double maxDamping = 0;
    std::array<int, 3> widths{};
    const int nodes[3]{p.nx, p.ny, p.nz};
    if (p.absorbing)
        for (int a = 0; a < 3; ++a) widths[a] = std::min(p.absorbingCells[a], nodes[a] / 3);
    const bool cpml = p.absorbing && p.absorber == 1;
    if (cpml) { // CFS-PML slabs instead of the sponge: x and y on both sides, z at the bottom
        const double frequency = p.cpmlFrequency > 0 ? p.cpmlFrequency : p.frequency;
        g.cpmlX = cpmlProfile(p.nx, widths[0], p.spacing, maxVp, p.cpmlReflection, p.cpmlKappaMax, frequency, true);
        g.cpmlY = cpmlProfile(p.ny, widths[1], p.spacing, maxVp, p.cpmlReflection, p.cpmlKappaMax, frequency, true);
        g.cpmlZ = cpmlProfile(p.nz, widths[2], p.spacing, maxVp, p.cpmlReflection, p.cpmlKappaMax, frequency, false);
        g.cpmlWidth = widths;
        // six memories per active axis: 2wx*ny*nz x slots, 2wy*nx*nz y slots, wz*nx*ny z slots
        g.cpmlCount = 6 * (2 * std::int64_t(widths[0]) * p.ny * p.nz + 2 * std::int64_t(widths[1]) * p.nx * p.nz +
                           std::int64_t(widths[2]) * p.nx * p.ny);
        const double rate = std::max({cpmlRate(g.cpmlX), cpmlRate(g.cpmlY), cpmlRate(g.cpmlZ)});
        g.cpmlDt = rate > 0 ? .5 / rate : std::numeric_limits<double>::max();
        widths = {0, 0, 0}; // no sponge
    } else {
        g.cpmlDt = std::numeric_limits<double>::max();
    }
    g.cpmlShape = {double(g.cpmlWidth[0]), double(g.cpmlWidth[1]), double(g.cpmlWidth[2]), double(g.cpmlCount)};
    for (int k = ghost; k < nz - ghost; ++k)
        for (int j = ghost; j < ny - ghost; ++j)
            for (int i = ghost; i < nx - ghost; ++i) {
                const int ii = i - ghost, jj = j - ghost, kk = k - ghost;
                const int dist[3]{std::min(ii, p.nx - 1 - ii), std::min(jj, p.ny - 1 - jj), p.nz - 1 - kk};
                double rate = 0;
                for (int a = 0; a < 3; ++a)
                    if (widths[a] > 0) {
                        const double f = std::clamp(1.0 - static_cast<double>(dist[a]) / widths[a], 0.0, 1.0);
                        rate += p.absorbingStrength * maxVp / (widths[a] * p.spacing) * f * f;
                    }
                g.damping[index(i, j, k)] = rate;
                maxDamping = std::max(maxDamping, rate);
            }
    // include/Seis3D/TimeStepPlan3D.hpp:8-20
    g.waveDt = p.cfl * std::min(p.spacing / maxMetricNorm, minLength) / maxVp;
    g.dampingDt = maxDamping > 0 ? .5 / maxDamping : std::numeric_limits<double>::max();
    g.sourceDt = 1 / (50 * p.frequency);
    const double safe = std::min({g.waveDt, g.dampingDt, g.sourceDt, g.cpmlDt, g.relaxationDt});
    const double durationSteps = std::max(1.0, std::ceil(p.duration / safe));
    require(std::isfinite(durationSteps) && !(p.maxSteps == 0 && durationSteps > 20000),
            "Time-step limit: at most 20,000 steps. Set a maximum step cap.");
    g.dt = p.duration / durationSteps;
    g.total = static_cast<int>(p.maxSteps > 0 ? std::min(durationSteps, double(p.maxSteps)) : durationSteps);
    g.ppw = minVs / (2.5 * p.frequency * maxEdge);
    // source weights (:397-412): normalised 5^3 Gaussian divided by J
    g.source.assign(count, 0);
    double sourceSum = 0;
    for (int k = -2; k <= 2; ++k)
        for (int j = -2; j <= 2; ++j)
            for (int i = -2; i <= 2; ++i) sourceSum += std::exp(-0.5 * (i * i + j * j + k * k));
    for (int k = -2; k <= 2; ++k)
        for (int j = -2; j <= 2; ++j)
            for (int i = -2; i <= 2; ++i) {
                const std::size_t q = index(ghost + src[0] + i, ghost + src[1] + j, ghost + src[2] + k);
                g.source[q] = std::exp(-0.5 * (i * i + j * j + k * k)) / (sourceSum * g.jacobian[q]);
            }
    if (moment) { // include/SeisCommon/SourceMechanism.hpp:43-56
        for (auto &v : g.sourceGradient) v.assign(count, 0);
        const auto flux = [&](std::ptrdiff_t q, int axis, int component) {
            return g.jacobian[q] * g.metrics[9 * q + 3 * axis + component] * g.source[q];
        };
        const std::ptrdiff_t strides[3] = {1, nx, std::ptrdiff_t(plane)};
        for (int k = src[2] - 4; k <= src[2] + 4; ++k)
            for (int j = src[1] - 4; j <= src[1] + 4; ++j)
                for (int i = src[0] - 4; i <= src[0] + 4; ++i) {
                    const auto q = static_cast<std::ptrdiff_t>(index(i + ghost, j + ghost, k + ghost));
                    double force[3] = {0, 0, 0};
                    for (int c = 0; c < 3; ++c)
                        for (int a = 0; a < 3; ++a) {
                            const auto s = strides[a];
                            force[c] -= (flux(q - 2 * s, a, c) - 8 * flux(q - s, a, c) + 8 * flux(q + s, a, c) - flux(q + 2 * s, a, c)) /
                                        (12 * p.spacing * g.jacobian[q]);
                        }
                    for (int a = 0; a < 3; ++a) g.sourceGradient[a][q] = force[a];
                }
        g.sourceDirection = {0, 0, 0};
    } else {
        const auto &d = p.sourceDirection;
        const double norm = std::hypot(d[0], d[1], d[2]);
        g.sourceDirection = {d[0] / norm, d[1] / norm, d[2] / norm};
    }
    g.sourceAmplitude = moment ? p.sourceMoment : p.sourceForce;
    for (const auto &n : rnodes) {
        const std::size_t q = index(n[0] + ghost, n[1] + ghost, n[2] + ghost);
        g.receiverNodes.push_back(std::int64_t(q));
        g.receiverPositions.push_back({g.coordinates[3 * q], g.coordinates[3 * q + 1], g.coordinates[3 * q + 2]});
    }
    return g;
}

} // namespace swl::host
