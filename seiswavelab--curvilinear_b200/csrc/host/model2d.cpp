// 2D model construction: Simulation::initialize of src/two_d/CurvilinearSolver2D.cpp:151-481
// (validation, absorber layout, terrain, FP64 geometry and metrics, layers, GSLS moduli,
// sponge / CFS-PML profiles, source kernel and moment pattern, dt plan, receivers).  The
// arithmetic follows the reference expression by expression so the arrays are identical.
#include "model.hpp"
#include "../../../include/swl_b200.h"
#include <algorithm>
#include <cmath>
#include <limits>
#include <stdexcept>

namespace swl::host {
namespace {
constexpr double pi = 3.14159265358979323846;
constexpr int ghost = 3;
void require(bool ok, const char *message) {
    if (!ok) throw std::runtime_error(message);
}
bool material(double vp, double vs, double rho) {
    return std::isfinite(vp) && std::isfinite(vs) && std::isfinite(rho) && vp > 0 && vs > 0 && rho > 0 &&
           vp * vp > 4 * vs * vs / 3 && std::isfinite(rho * vp * vp);
}
} // namespace

// src/two_d/CfsPml2D.hpp:31-41
std::vector<double> cpmlProfile(int nodes, int width, double h, double vp, double reflection, double kappa, double frequency,
                                bool both) {
    std::vector<double> out(3 * std::size_t(nodes));
    const double d0 = -3 * vp * std::log(reflection) / (2 * width * h);
    for (int i = 0; i < nodes; ++i) {
        const int distance = both ? std::min(i, nodes - 1 - i) : nodes - 1 - i;
        const double t = std::clamp(1. - double(distance) / width, 0., 1.);
        out[3 * i] = d0 * t * t;
        out[3 * i + 1] = 1 + (kappa - 1) * t * t;
        out[3 * i + 2] = t > 0 ? pi * frequency * (1 - t) : 0;
    }
    return out;
}
double cpmlRate(const std::vector<double> &profile) {
    double rate = 0;
    for (std::size_t i = 0; i < profile.size(); i += 3) rate = std::max(rate, profile[i] / profile[i + 1] + profile[i + 2]);
    return rate;
}


Model2D buildModel2D(const Params2D &requested) {
    Params2D p = requested;
    require(p.precision == 0 || p.precision == 1, "Unknown 2D calculation precision.");
    require(p.nx >= 8 && p.nz >= 8 && p.nx <= 16384 && p.nz <= 16384, "2D dimensions must be in 8..16384 (subject to RAM/VRAM).");
    const Params2D logical = p;
    for (double v : {p.spacing, p.relief, p.wavelength, p.flattenDepth, p.frequency, p.duration, p.cfl, p.forcePerLength,
                     p.momentPerLength, p.spongeStrength, p.surfaceDatum, p.sampleIntervalMs})
        require(std::isfinite(v), "2D parameters must be finite.");
    const bool explosive = p.sourceKind == 1;
    require(p.spacing > 0 && p.frequency > 0 && p.frequency <= 1e6 && p.duration > 0 && p.duration <= 10 && p.cfl >= .02 &&
                p.cfl <= .8 && p.wavelength > 0 && p.flattenDepth >= 0 && (explosive ? p.momentPerLength : p.forcePerLength) > 0,
            "Invalid 2D spacing, frequency, duration, CFL or source amplitude.");
    require(material(p.vp, p.vs, p.density), "Require positive material values and positive elastic bulk modulus.");
    require(p.sampleIntervalMs == 0 || (p.sampleIntervalMs >= .01 && p.sampleIntervalMs <= 1000),
            "Record interval must be 0 (each step) or 0.01..1000 ms.");
    require(p.maxSteps >= 0 && p.maxSteps <= 200000, "Step cap must be 0..200000 (0 = full duration).");
    require(p.sourceKind == 0 || p.sourceKind == 1, "Unknown source mechanism.");
    if (!explosive) { // include/SeisCommon/SourceMechanism.hpp:19-31
        const auto &d = p.sourceDirection;
        const double norm = std::hypot(d[0], d[1], d[2]);
        require(std::isfinite(norm) && norm > 0 && d[1] == 0, "2D force direction must be finite, nonzero and inside the X-Z plane.");
    }
    require(std::isfinite(p.sourceSigmaM) && std::isfinite(p.sourceRadiusM) &&
                ((p.sourceSigmaM == 0 && p.sourceRadiusM == 0) || (!explosive && p.sourceSigmaM > 0 && p.sourceRadiusM >= p.sourceSigmaM)),
            "Physical source kernel requires a directional force and 0 < sigma <= radius, or both zero for legacy.");
    int sx = p.sourceX < 0 ? p.nx / 2 : p.sourceX;
    if (explosive)
        require(p.nx >= 11 && p.nz >= 11 && sx >= 5 && sx <= p.nx - 6 && p.sourceZ >= 5 && p.sourceZ <= p.nz - 6,
                "Isotropic moment needs 11+ nodes per axis and source center five nodes inside each face.");
    require(p.sourceX >= -1 && sx >= 2 && sx <= p.nx - 3 && p.sourceZ >= 0 && p.sourceZ <= p.nz - 3,
            "2D force source may be on the free surface; keep two cells from the sides and bottom.");
    require(p.receiverStart >= 0 && p.receiverCount > 0 && p.receiverCount <= 1024 && p.receiverStride > 0 &&
                p.receiverDepth >= 0 && p.receiverDepth < p.nz &&
                (long long)p.receiverStart + ((long long)p.receiverCount - 1) * p.receiverStride < p.nx,
            "Receiver line is outside the 2D model or exceeds 1024 positions.");
    require(p.spongeX >= 1 && p.spongeX <= 512 && p.spongeZ >= 1 && p.spongeZ <= 512 && p.spongeStrength >= .1 &&
                p.spongeStrength <= 10,
            "Sponge widths must be 1..512 cells (effective width <= axis nodes / 3) and strength 0.1..10.");
    require(p.absorber == 0 || p.absorber == 1, "Unknown 2D absorber.");
    require(std::isfinite(p.cpmlReflection) && p.cpmlReflection >= 1e-8 && p.cpmlReflection <= .1 && std::isfinite(p.cpmlKappaMax) &&
                p.cpmlKappaMax >= 1 && p.cpmlKappaMax <= 20 && std::isfinite(p.cpmlFrequency) && p.cpmlFrequency >= 0 &&
                p.cpmlFrequency <= 1e6,
            "CFS-PML requires R in 1e-8..0.1, kappa in 1..20, frequency in 0..1e6 Hz.");
    if (p.layered) {
        require(!p.layers.empty() && p.layers.size() <= 16, "Require 1..16 material layers.");
        for (std::size_t l = 0; l < p.layers.size(); ++l) {
            const auto &L = p.layers[l];
            require(material(L.vp, L.vs, L.density) && std::isfinite(L.thickness) && L.thickness >= 0 &&
                        (l + 1 == p.layers.size() || L.thickness > 0),
                    "Invalid layer thickness or material.");
        }
    }
    validateGsls(p.attenuation);
    std::vector<GslsMaterial> rheology;
    if (p.attenuation.enabled) {
        if (p.layered)
            for (const auto &L : p.layers) rheology.push_back(fitGsls(L.vp, L.vs, L.density, L.qp, L.qs, p.attenuation));
        else
            rheology.push_back(fitGsls(p.vp, p.vs, p.density, p.attenuation.qp, p.attenuation.qs, p.attenuation));
    }
    // absorber layout (src/two_d/CfsPml2D.hpp:10-14): external strips widen the grid
    const int widthX = std::clamp(logical.spongeX, 1, std::max(1, logical.nx / 3));
    const int widthZ = std::clamp(logical.spongeZ, 1, std::max(1, logical.nz / 3));
    int offsetX = 0, dnx = logical.nx, dnz = logical.nz;
    if (logical.absorbing && logical.externalAbsorption) offsetX = widthX, dnx += 2 * widthX, dnz += widthZ;
    require(dnx <= 16384 && dnz <= 16384,
            "2D computational dimensions including external absorbing strips must not exceed 16384 per axis.");
    p.nx = dnx, p.nz = dnz, p.spongeX = widthX, p.spongeZ = widthZ, p.externalAbsorption = false;
    sx += offsetX;
    p.sourceX = sx;
    p.receiverStart += offsetX;

    Model2D g;
    g.nx = p.nx + 6, g.nz = p.nz + 6, g.modelOffsetX = offsetX, g.h = p.spacing;
    g.logicalNx = logical.nx, g.logicalNz = logical.nz;
    const std::size_t count = std::size_t(g.nx) * g.nz;
    const auto index = [&](int i, int k) { return i + std::size_t(g.nx) * k; };
    const double bottom = (logical.nz - 1) * p.spacing;
    std::vector<std::array<double, 2>> surface(g.nx);
    double relief = std::abs(p.relief);
    if (p.importedSurface) {
        const SurfaceProfile profile(p.surfaceSamples);
        require(p.surfaceSamples.front()[0] <= 0 && p.surfaceSamples.back()[0] >= (logical.nx - 1) * p.spacing,
                "Imported terrain must cover x=0 through the full physical model span.");
        relief = 0;
        for (int i = 0; i < g.nx; ++i) {
            const auto value = profile.sample((i - ghost - offsetX) * p.spacing);
            surface[i] = {p.surfaceDatum - value[0], -value[1]};
            if (i >= offsetX && i < offsetX + logical.nx + 2 * ghost) relief = std::max(relief, std::abs(surface[i][0]));
        }
    } else {
        for (int i = 0; i < g.nx; ++i) {
            const double phase = 2 * pi * (i - ghost - offsetX) * p.spacing / p.wavelength;
            surface[i] = {p.relief * std::cos(phase), -p.relief * 2 * pi / p.wavelength * std::sin(phase)};
        }
    }
    g.flattenDepth = p.flattenDepth > 0 ? p.flattenDepth : std::min(bottom, std::max({.35 * bottom, 6 * p.spacing, 4 * relief + 2 * p.spacing}));
    require(g.flattenDepth <= bottom && (relief == 0 || ((p.importedSurface || p.wavelength >= 4 * p.spacing) &&
                                                         g.flattenDepth >= 4 * p.spacing && g.flattenDepth > 2.6 * relief)),
            "Terrain must be resolved and flatten depth must exceed 2.6 times relief within the model.");
    if (offsetX) { // C1 continuation of the edge height/slope into the external strips
        for (int side = 0; side < 2; ++side) {
            const int edge = ghost + offsetX + (side ? logical.nx - 1 : 0);
            const double z = surface[edge][0], slope = surface[edge][1];
            const double length = std::min(widthX * p.spacing / 3., .5 * (g.flattenDepth / 2.6 - std::abs(z)) / std::max(std::abs(slope), 1e-30));
            for (int i = side ? edge + 1 : 0; i < (side ? g.nx : edge); ++i) {
                const double distance = std::abs(i - edge) * p.spacing, decay = std::exp(-distance / length);
                surface[i] = {z + (side ? 1. : -1.) * slope * length * (1 - decay), slope * decay};
            }
        }
    }
    for (auto *v : {&g.metricA, &g.metricB, &g.jacobian, &g.vp, &g.vs, &g.density, &g.lambda, &g.mu, &g.source, &g.damping})
        v->assign(count, 0);
    g.coordinates.assign(2 * count, 0);
    g.normals.assign(2 * count, 0);
    const int L = p.attenuation.enabled ? p.attenuation.mechanisms : 0;
    if (L) {
        g.qp.assign(count, 0), g.qs.assign(count, 0);
        for (int l = 0; l < L; ++l) g.deltaP[l].assign(count, 0), g.deltaS[l].assign(count, 0);
    }
    if (p.deviceGeometry) { // the per-node geometry below, computed on the GPU
        std::vector<double> columns(2 * std::size_t(g.nx));
        for (int i = 0; i < g.nx; ++i) columns[2 * i] = surface[i][0], columns[2 * i + 1] = surface[i][1];
        const swl_geometry2d geo{g.nx, g.nz, ghost, offsetX, p.spacing, g.flattenDepth, columns.data()};
        double minJ = 0, maxM = 0;
        if (swl2d_build_geometry(&geo, p.geometryDevice, g.coordinates.data(), g.metricA.data(), g.metricB.data(),
                                 g.jacobian.data(), g.normals.data(), &minJ, &maxM) != SWL_OK)
            throw std::runtime_error(swl_last_error());
    }
    g.minJacobian = std::numeric_limits<double>::max();
    double maxVp = 0, minVs = std::numeric_limits<double>::max(), maxSigma = 0;
    for (int k = 0; k < g.nz; ++k)
        for (int i = 0; i < g.nx; ++i) {
            const auto q = index(i, k);
            const double eta = (k - ghost) * p.spacing;
            double j;
            if (p.deviceGeometry) {
                j = g.jacobian[q];
            } else {
                const double x = (i - ghost - offsetX) * p.spacing, t = std::clamp(eta / g.flattenDepth, 0.0, 1.0);
                // ninth-order blend with four vanishing derivatives at both ends
                const double fade = 1 - std::pow(t, 5) * (126 + t * (-420 + t * (540 + t * (-315 + 70 * t))));
                const double fadeDerivative =
                    eta > 0 && eta < g.flattenDepth ? -630 * std::pow(t, 4) * std::pow(1 - t, 4) / g.flattenDepth : 0;
                const double zx = surface[i][1] * fade;
                j = 1 + surface[i][0] * fadeDerivative;
                g.coordinates[2 * q] = x;
                g.coordinates[2 * q + 1] = eta + surface[i][0] * fade;
                g.metricA[q] = -zx / j;
                g.metricB[q] = 1 / j;
                g.jacobian[q] = j;
                const double n = std::hypot(zx, 1.0);
                g.normals[2 * q] = -zx / n;
                g.normals[2 * q + 1] = 1 / n;
            }
            require(j > 1e-9 && std::isfinite(j), "Nonpositive curvilinear Jacobian.");
            double vp = p.vp, vs = p.vs, rho = p.density;
            std::size_t materialIndex = 0;
            if (p.layered) {
                double boundary = 0;
                const double depth = offsetX ? std::clamp(eta, 0., bottom) : std::max(0., eta);
                for (std::size_t l = 0; l < p.layers.size(); ++l) {
                    boundary += p.layers[l].thickness;
                    if (l + 1 == p.layers.size() || depth < boundary) {
                        vp = p.layers[l].vp, vs = p.layers[l].vs, rho = p.layers[l].density, materialIndex = l;
                        break;
                    }
                }
            }
            g.vp[q] = vp, g.vs[q] = vs, g.density[q] = rho;
            g.mu[q] = rho * vs * vs;
            g.lambda[q] = rho * vp * vp - 2 * g.mu[q];
            double speedMax = vp, speedMin = vs;
            if (L) {
                const auto &m = rheology[materialIndex];
                g.mu[q] = m.sUnrelaxed;
                g.lambda[q] = m.pUnrelaxed - 2 * m.sUnrelaxed;
                g.qp[q] = p.layered ? p.layers[materialIndex].qp : p.attenuation.qp;
                g.qs[q] = p.layered ? p.layers[materialIndex].qs : p.attenuation.qs;
                for (int l = 0; l < m.mechanisms; ++l) g.deltaP[l][q] = m.deltaP[l], g.deltaS[l][q] = m.deltaS[l];
                speedMax = std::sqrt(m.pUnrelaxed / rho);
                speedMin = std::sqrt(m.sRelaxed / rho);
            }
            if (i >= ghost && i < g.nx - ghost && k >= ghost && k < g.nz - ghost) {
                g.minJacobian = std::min(g.minJacobian, j);
                g.maxMetric = std::max(g.maxMetric, std::sqrt(1 + g.metricA[q] * g.metricA[q] + g.metricB[q] * g.metricB[q]));
                maxVp = std::max(maxVp, speedMax);
                minVs = std::min(minVs, speedMin);
            }
        }
    const bool sponge = p.absorbing && p.absorber == 0;
    for (int k = 0; k < p.nz; ++k)
        for (int i = 0; i < p.nx; ++i) {
            const auto q = index(i + ghost, k + ghost);
            if (i + 1 < p.nx)
                g.maxEdge = std::max(g.maxEdge, std::hypot(g.coordinates[2 * (q + 1)] - g.coordinates[2 * q],
                                                           g.coordinates[2 * (q + 1) + 1] - g.coordinates[2 * q + 1]));
            if (k + 1 < p.nz) g.maxEdge = std::max(g.maxEdge, g.coordinates[2 * (q + g.nx) + 1] - g.coordinates[2 * q + 1]);
            if (sponge) {
                const int wx = std::min(p.spongeX, p.nx / 3), wz = std::min(p.spongeZ, p.nz / 3);
                const double xs = std::max(0.0, 1.0 - std::min(i, p.nx - 1 - i) / static_cast<double>(wx)),
                             zs = std::max(0.0, 1.0 - (p.nz - 1 - k) / static_cast<double>(wz));
                g.damping[q] = p.spongeStrength * maxVp / p.spacing * (xs * xs / wx + zs * zs / wz);
                maxSigma = std::max(maxSigma, g.damping[q]);
            }
        }
    double cpmlMaxRate = 0;
    const bool cpml = p.absorbing && p.absorber == 1;
    if (cpml) {
        const int wx = std::min(p.spongeX, p.nx / 3), wz = std::min(p.spongeZ, p.nz / 3);
        const double frequency = p.cpmlFrequency > 0 ? p.cpmlFrequency : p.frequency;
        g.cpmlX = cpmlProfile(p.nx, wx, p.spacing, maxVp, p.cpmlReflection, p.cpmlKappaMax, frequency, true);
        g.cpmlZ = cpmlProfile(p.nz, wz, p.spacing, maxVp, p.cpmlReflection, p.cpmlKappaMax, frequency, false);
        cpmlMaxRate = std::max(cpmlRate(g.cpmlX), cpmlRate(g.cpmlZ));
        g.cpmlWidthX = wx, g.cpmlWidthZ = wz;
        const int ex = std::clamp(p.spongeX, 1, std::max(1, p.nx / 3)), ez = std::clamp(p.spongeZ, 1, std::max(1, p.nz / 3));
        g.cpmlCount = 4 * (2 * std::int64_t(ex) * p.nz + std::int64_t(ez) * p.nx);
    }
    // source kernel: normalised 5x5 Gaussian, or a physical Gaussian of sigma within a radius
    double weight = 0;
    const auto coord = [&](std::size_t q) { return std::array<double, 2>{g.coordinates[2 * q], g.coordinates[2 * q + 1]}; };
    if (p.sourceSigmaM > 0) {
        const auto center = coord(index(sx + ghost, p.sourceZ + ghost));
        double boundaryDistance = std::numeric_limits<double>::infinity();
        for (int k = 0; k < p.nz; ++k)
            for (int i = 0; i < p.nx; ++i) {
                const auto q = index(i + ghost, k + ghost);
                const auto r = coord(q);
                const double distance = std::hypot(r[0] - center[0], r[1] - center[1]);
                if (k == 0 || k == p.nz - 1 || i == 0 || i == p.nx - 1) boundaryDistance = std::min(boundaryDistance, distance);
                if (distance <= p.sourceRadiusM) {
                    g.source[q] = std::exp(-.5 * distance * distance / (p.sourceSigmaM * p.sourceSigmaM));
                    weight += g.source[q] * g.jacobian[q];
                }
            }
        require(boundaryDistance > p.sourceRadiusM, "Physical source support intersects a physical computational boundary.");
        require(weight > 0 && std::isfinite(weight), "Invalid physical source normalization.");
    } else {
        for (int dk = -2; dk <= 2; ++dk)
            for (int di = -2; di <= 2; ++di) {
                if (p.sourceZ + dk < 0) continue; // surface sources keep only physical nodes
                const auto q = index(sx + ghost + di, p.sourceZ + ghost + dk);
                g.source[q] = std::exp(-.5 * (di * di + dk * dk));
                weight += g.source[q] * g.jacobian[q];
            }
    }
    for (auto &s : g.source) s = s / weight;
    if (explosive) { // include/SeisCommon/SourceMechanism.hpp:43-56 with J * metric * w fluxes
        for (auto &v : g.sourceGradient) v.assign(count, 0);
        const auto flux = [&](std::ptrdiff_t q, int axis, int component) {
            const double metric = axis == 0 ? (component == 0 ? 1. : 0.) : (component == 0 ? g.metricA[q] : g.metricB[q]);
            return g.jacobian[q] * metric * g.source[q];
        };
        for (int k = p.sourceZ - 4; k <= p.sourceZ + 4; ++k)
            for (int i = sx - 4; i <= sx + 4; ++i) {
                const auto q = static_cast<std::ptrdiff_t>(index(i + ghost, k + ghost));
                const std::ptrdiff_t strides[2] = {1, g.nx};
                double force[2] = {0, 0};
                for (int c = 0; c < 2; ++c)
                    for (int a = 0; a < 2; ++a) {
                        const auto s = strides[a];
                        force[c] -= (flux(q - 2 * s, a, c) - 8 * flux(q - s, a, c) + 8 * flux(q + s, a, c) - flux(q + 2 * s, a, c)) /
                                    (12 * p.spacing * g.jacobian[q]);
                    }
                g.sourceGradient[0][q] = force[0];
                g.sourceGradient[1][q] = force[1];
            }
    }
    if (p.sourceSigmaM > 0 || p.sourceZ < 2) {
        const auto center = coord(index(sx + ghost, p.sourceZ + ghost));
        double second = 0;
        for (std::size_t q = 0; q < count; ++q)
            if (g.source[q] > 0) {
                const auto r = coord(q);
                const double w = g.source[q] * g.jacobian[q];
                g.sourceWeightSum += w;
                second += w * ((r[0] - center[0]) * (r[0] - center[0]) + (r[1] - center[1]) * (r[1] - center[1]));
            }
        g.sourceRmsRadiusM = std::sqrt(second / g.sourceWeightSum);
    }
    // dt plan (src/two_d/CurvilinearSolver2D.cpp:165-182)
    g.ppw = minVs / (2.5 * p.frequency * g.maxEdge);
    g.waveDt = p.cfl * p.spacing / (maxVp * g.maxMetric);
    g.dampingDt = maxSigma > 0 ? .5 / maxSigma : std::numeric_limits<double>::infinity();
    g.sourceDt = 1 / (50 * p.frequency);
    g.cpmlDt = cpmlMaxRate > 0 ? .5 / cpmlMaxRate : std::numeric_limits<double>::infinity();
    g.relaxationDt = L ? .25 / rheology.front().rates[L - 1] : std::numeric_limits<double>::infinity();
    for (const auto &m : rheology) g.maxRelativeQError = std::max(g.maxRelativeQError, m.maxRelativeQError);
    g.mechanisms = L;
    g.fieldCount = L ? 6 + 4 * L : 5;
    if (L)
        for (int l = 0; l < L; ++l) g.rates[l] = rheology.front().rates[l];
    const double safe = std::min({g.waveDt, g.dampingDt, g.sourceDt, g.relaxationDt, g.cpmlDt});
    const double full = std::ceil(p.duration / safe);
    require(std::isfinite(full) && full <= 10000000, "Requested duration needs too many steps; increase spacing or lower frequency.");
    g.dt = p.duration / full;
    g.total = p.maxSteps ? std::min(static_cast<int>(full), p.maxSteps) : static_cast<int>(full);
    require(g.total <= 200000,
            "2D session exceeds 200000 accepted steps; set an explicit cap or shorter duration. A cap ends before the requested duration.");
    g.recordDt = p.sampleIntervalMs > 0 ? p.sampleIntervalMs * .001 : g.dt;
    g.recordSamples = static_cast<std::size_t>(std::floor(g.total * g.dt / g.recordDt)) + 1;
    for (int r = 0; r < p.receiverCount; ++r) {
        const int x = logical.receiverStart + r * p.receiverStride, z = p.receiverDepth;
        const auto q = index(x + ghost + offsetX, z + ghost);
        g.receiverNodes.push_back(std::int64_t(q));
        g.receiverPositions.push_back(coord(q));
    }
    if (explosive) g.sourceDirection = {0, 0, 0};
    else {
        const auto &d = p.sourceDirection;
        const double norm = std::hypot(d[0], d[1], d[2]);
        g.sourceDirection = {d[0] / norm, d[1] / norm, d[2] / norm};
    }
    g.scale = (explosive ? p.momentPerLength : p.forcePerLength) / (p.spacing * p.spacing);
    g.sourceX = sx, g.sourceZ = p.sourceZ;
    if (p.precision == 1) { // src/two_d/CurvilinearSolver2D.cpp:498-504 quantised-model checks
        for (std::size_t q = 0; q < count; ++q) {
            const float mu = float(g.mu[q]), lam = float(g.lambda[q]);
            require(mu > 0 && lam + 2 * mu / 3 > 0 && float(g.density[q]) > 0 && float(g.vp[q]) > 0 && float(g.vs[q]) > 0 &&
                        float(g.jacobian[q]) > 0 && float(g.metricB[q]) > 0,
                    "Invalid quantized material or geometry; select FP64 or revise model.");
        }
        require(std::isfinite(float(p.spacing)) && float(p.spacing) > 0 && std::isfinite(float(g.dt)) && float(g.dt) > 0,
                "FP32 spacing/time step is not representable; select FP64.");
    }
    return g;
}

} // namespace swl::host
