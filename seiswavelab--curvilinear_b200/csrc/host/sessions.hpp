// Session classes shared by the session ABI (session.cpp) and the server (server.cpp): the C++20
// host of one simulation over the engine C ABI.
#pragma once
#include "../../../include/swl_session.h"
#include "../runtime.cuh"
#include "model.hpp"
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace swl::host {

struct Failure : std::runtime_error {
    int status;
    Failure(int s, const std::string &m) : std::runtime_error(m), status(s) {}
};
inline void ok(swl_status s) {
    if (s != SWL_OK) throw Failure(s, swl_last_error());
}
template <class F> inline swl_status guard(F &&f) {
    std::string &sessionError = swl::lastErrorRef();
    try {
        sessionError.clear();
        f();
        return SWL_OK;
    } catch (const Failure &e) {
        sessionError = e.what();
        return e.status;
    } catch (const std::bad_alloc &) {
        sessionError = "host allocation failed";
        return SWL_ERR_MEMORY;
    } catch (const std::exception &e) {
        sessionError = e.what();
        return SWL_ERR_INVALID;
    }
}
inline double millis(std::chrono::steady_clock::time_point a) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
}
constexpr int maxBatch = 2048; // steps per engine batch (bounds the device trace table)

// ---------------------------------------------------------------------------------------- 2D
struct Session2D {
    Params2D params;
    Model2D model;
    swl2d_engine *engine{};
    int step{};
    std::string fault;
    std::vector<std::vector<double>> vx, vz; // records per receiver
    std::vector<std::array<double, 2>> previous;
    swl_diag2d diag{};
    double initMs{}, totalMs{}, lastMs{};
    ~Session2D() {
        if (engine) swl2d_destroy(engine);
    }
    void clearRecords() {
        const std::size_t n = model.receiverNodes.size();
        vx.assign(n, std::vector<double>(1, 0.0));
        vz.assign(n, std::vector<double>(1, 0.0));
        for (auto &v : vx) v.reserve(model.recordSamples);
        for (auto &v : vz) v.reserve(model.recordSamples);
        previous.assign(n, {0, 0});
    }
    // Simulation::Impl::sample (src/two_d/CurvilinearSolver2D.cpp:120-147) for one accepted step.
    void record(int s, const double *cx, const double *cz, std::size_t stride, std::size_t col) {
        const double dt = model.dt, interval = model.recordDt;
        const double end = (s + 1) * dt;
        for (std::size_t n = vx.front().size(); n * interval <= end + 1e-9 * dt; ++n) {
            const double a = std::clamp((n * interval - s * dt) / dt, 0.0, 1.0);
            for (std::size_t r = 0; r < vx.size(); ++r) {
                vx[r].push_back(std::lerp(previous[r][0], cx[r * stride + col], a));
                vz[r].push_back(std::lerp(previous[r][1], cz[r * stride + col], a));
            }
        }
        for (std::size_t r = 0; r < vx.size(); ++r) previous[r] = {cx[r * stride + col], cz[r * stride + col]};
    }
    void create(int device) {
        const auto t0 = std::chrono::steady_clock::now();
        if (params.deviceGeometry) {
            if (device == SWL_MODEL_ONLY) throw Failure(SWL_ERR_INVALID, "device geometry needs a CUDA device");
            params.geometryDevice = device;
        }
        model = buildModel2D(params);
        clearRecords();
        if (device != SWL_MODEL_ONLY) {
            swl_mesh2d m{};
            m.nx = model.nx, m.nz = model.nz, m.count = int64_t(model.nx) * model.nz, m.h = model.h;
            m.a = model.metricA.data(), m.b = model.metricB.data(), m.jac = model.jacobian.data(), m.normals = model.normals.data();
            m.lambda = model.lambda.data(), m.mu = model.mu.data(), m.rho = model.density.data();
            m.source = model.source.data(), m.damping = model.damping.data();
            for (int a = 0; a < 3; ++a) m.source_direction[a] = model.sourceDirection[a];
            if (!model.sourceGradient[0].empty()) m.source_gradient[0] = model.sourceGradient[0].data(), m.source_gradient[1] = model.sourceGradient[1].data();
            m.mechanisms = model.mechanisms, m.field_count = model.fieldCount;
            if (model.cpmlCount) {
                m.cpml_x = model.cpmlX.data(), m.cpml_z = model.cpmlZ.data();
                m.cpml_width_x = model.cpmlWidthX, m.cpml_width_z = model.cpmlWidthZ, m.cpml_count = model.cpmlCount;
            }
            for (int l = 0; l < model.mechanisms; ++l)
                m.rates[l] = model.rates[l], m.delta_p[l] = model.deltaP[l].data(), m.delta_s[l] = model.deltaS[l].data();
            m.precision = params.precision, m.array_precision = SWL_FP64;
            m.segment_rule = params.segmentRule ? 1 : 0;
            ok(swl2d_create(&m, model.receiverNodes.data(), int32_t(model.receiverNodes.size()), device, &engine));
            ok(swl2d_reserve(engine, std::min(model.total, maxBatch))); // batch tables sized once, at creation
            ok(swl2d_diagnostics(engine, &diag));
        }
        initMs = millis(t0);
    }
    // One asynchronous batch (at most n steps, bounded by the planned total); false if nothing to do.
    int inflight{};
    std::chrono::steady_clock::time_point batchStart;
    bool launchBatch(int n) {
        if (!engine) throw Failure(SWL_ERR_STATE, "Initialize the 2D model on a device first.");
        if (!fault.empty()) throw Failure(SWL_ERR_STATE, fault);
        n = std::max(0, std::min({n, model.total - step, maxBatch}));
        if (n == 0) return false;
        batchStart = std::chrono::steady_clock::now();
        ok(swl2d_launch(engine, step, n, model.dt, params.frequency, model.scale, 3 / params.frequency));
        inflight = n;
        return true;
    }
    // The arguments of one batch that a persistent multi-shot launch will run (swl2d_queue_launch),
    // at most n steps; the batch counts as in flight from here.  0: nothing to do.
    int queueBatch(int n, int32_t &first, double &dt, double &frequency, double &scale, double &growthAfter) {
        if (!engine) throw Failure(SWL_ERR_STATE, "Initialize the 2D model on a device first.");
        if (!fault.empty()) throw Failure(SWL_ERR_STATE, fault);
        n = std::max(0, std::min({n, model.total - step, maxBatch}));
        if (n == 0) return 0;
        batchStart = std::chrono::steady_clock::now();
        first = step, dt = model.dt, frequency = params.frequency, scale = model.scale, growthAfter = 3 / params.frequency;
        inflight = n;
        return n;
    }
    // Completion of the in-flight batch: records of the accepted steps (Simulation::Impl::sample),
    // and the sticky fault of a rejected step.  Returns false while the batch is still running.
    bool pollBatch(bool block) {
        if (!inflight) return true;
        int32_t done = 1, accepted = 0;
        const swl_status st = block ? swl2d_wait(engine, &accepted) : swl2d_query(engine, &done, &accepted);
        if (st != SWL_OK && st != SWL_ERR_FAULT) ok(st);
        if (!done) return false;
        std::vector<double> tx(std::size_t(accepted) * vx.size()), tz(tx.size());
        if (accepted && !vx.empty()) ok(swl2d_traces(engine, step, accepted, tx.data(), tz.data()));
        for (int j = 0; j < accepted; ++j) record(step + j, tx.data(), tz.data(), std::size_t(accepted), std::size_t(j));
        step += accepted;
        lastMs = millis(batchStart) / std::max(1, accepted);
        totalMs += millis(batchStart);
        inflight = 0;
        ok(swl2d_step_diagnostics(engine, &diag));
        if (st == SWL_ERR_FAULT) {
            fault = "2D step rejected: nonfinite fields or excessive late energy growth. Rebuild the session.";
            throw Failure(SWL_ERR_FAULT, fault);
        }
        return true;
    }
    // Simulation::advance (:541-604): batches on the device, records on the host.
    void advance(int count) {
        count = std::max(0, std::min(count, model.total - step));
        while (count > 0) {
            const int before = step;
            if (!launchBatch(count)) break;
            pollBatch(true);
            count -= step - before;
        }
    }
    bool completed() const { return step >= model.total; }
    int64_t estimateBytes() const {
        // four state sets, six in FP32 (the Kahan compensation of the state and accumulator)
        const double s = params.precision == SWL_FP32 ? 4 : 8, n = double(model.nx) * model.nz, sets = s == 4 ? 6 : 4;
        return int64_t(n * s * (sets * model.fieldCount + 12 + 2 * model.mechanisms) + sets * s * model.cpmlCount) + (64 << 20);
    }
    void reset() {
        if (engine) ok(swl2d_reset(engine)), ok(swl2d_diagnostics(engine, &diag));
        step = 0, fault.clear(), totalMs = lastMs = 0;
        clearRecords();
    }
    const std::vector<double> *array(const std::string &n) const {
        const Model2D &m = model;
        if (n == "metricA") return &m.metricA;
        if (n == "metricB") return &m.metricB;
        if (n == "jacobian") return &m.jacobian;
        if (n == "normals") return &m.normals;
        if (n == "coordinates") return &m.coordinates;
        if (n == "lambda") return &m.lambda;
        if (n == "mu") return &m.mu;
        if (n == "density") return &m.density;
        if (n == "vp") return &m.vp;
        if (n == "vs") return &m.vs;
        if (n == "source") return &m.source;
        if (n == "damping") return &m.damping;
        if (n == "sourceGradientX") return &m.sourceGradient[0];
        if (n == "sourceGradientZ") return &m.sourceGradient[1];
        if (n == "cpmlX") return &m.cpmlX;
        if (n == "cpmlZ") return &m.cpmlZ;
        if (n == "qp") return &m.qp;
        if (n == "qs") return &m.qs;
        for (int l = 0; l < 3; ++l) {
            if (n == "deltaP" + std::to_string(l)) return &m.deltaP[l];
            if (n == "deltaS" + std::to_string(l)) return &m.deltaS[l];
        }
        return nullptr;
    }
};

inline Params2D toParams(const swl_params2d &c) {
    Params2D p;
    p.precision = c.precision, p.nx = c.nx, p.nz = c.nz;
    p.spacing = c.spacing, p.vp = c.vp, p.vs = c.vs, p.density = c.density, p.relief = c.relief, p.wavelength = c.wavelength;
    p.flattenDepth = c.flatten_depth, p.frequency = c.frequency, p.duration = c.duration, p.cfl = c.cfl;
    p.forcePerLength = c.force_per_length, p.sourceX = c.source_x, p.sourceZ = c.source_z, p.maxSteps = c.max_steps;
    p.sourceKind = c.source_kind;
    for (int a = 0; a < 3; ++a) p.sourceDirection[a] = c.source_direction[a];
    p.momentPerLength = c.moment_per_length, p.sourceSigmaM = c.source_sigma_m, p.sourceRadiusM = c.source_radius_m;
    p.absorbing = c.absorbing != 0, p.spongeX = c.sponge_x, p.spongeZ = c.sponge_z, p.spongeStrength = c.sponge_strength;
    p.absorber = c.absorber, p.cpmlReflection = c.cpml_reflection, p.cpmlKappaMax = c.cpml_kappa_max, p.cpmlFrequency = c.cpml_frequency;
    p.externalAbsorption = c.external_absorption != 0;
    p.receiverStart = c.receiver_start, p.receiverCount = c.receiver_count, p.receiverStride = c.receiver_stride;
    p.receiverDepth = c.receiver_depth, p.sampleIntervalMs = c.sample_interval_ms;
    p.layered = c.layered != 0;
    if (c.n_layers < 0 || (c.n_layers && !c.layers)) throw std::runtime_error("Invalid layer list.");
    if (c.n_layers) {
        p.layers.clear();
        for (int l = 0; l < c.n_layers; ++l)
            p.layers.push_back({c.layers[l].thickness, c.layers[l].vp, c.layers[l].vs, c.layers[l].density, c.layers[l].qp, c.layers[l].qs});
    }
    p.attenuation.enabled = c.attenuation != 0, p.attenuation.mechanisms = c.mechanisms;
    p.attenuation.minFrequency = c.q_min_frequency, p.attenuation.maxFrequency = c.q_max_frequency;
    p.attenuation.referenceFrequency = c.q_reference_frequency, p.attenuation.qp = c.qp, p.attenuation.qs = c.qs;
    p.importedSurface = c.imported_surface != 0, p.surfaceDatum = c.surface_datum;
    if (c.n_surface < 0 || (c.n_surface && !c.surface_xz)) throw std::runtime_error("Invalid surface sample list.");
    for (int i = 0; i < c.n_surface; ++i) p.surfaceSamples.push_back({c.surface_xz[2 * i], c.surface_xz[2 * i + 1]});
    p.deviceGeometry = c.device_geometry != 0;
    p.segmentRule = c.segment_rule != 0;
    return p;
}

// ---------------------------------------------------------------------------------------- 3D
struct Session3D {
    Params3D params;
    Model3D model;
    swl3d_engine *engine{};
    int step{};
    std::string fault;
    std::vector<std::vector<double>> rec[3];
    swl_diag3d diag{};
    double initMs{}, totalMs{}, lastMs{};
    ~Session3D() {
        if (engine) swl3d_destroy(engine);
    }
    void clearRecords() {
        for (auto &c : rec) {
            c.assign(model.receiverNodes.size(), std::vector<double>(1, 0.0));
            for (auto &v : c) v.reserve(std::size_t(model.total) + 1);
        }
    }
    void create(int device) {
        const auto t0 = std::chrono::steady_clock::now();
        if (params.deviceGeometry) {
            if (device == SWL_MODEL_ONLY) throw Failure(SWL_ERR_INVALID, "device geometry needs a CUDA device");
            params.geometryDevice = device;
        }
        model = buildModel3D(params);
        clearRecords();
        if (device != SWL_MODEL_ONLY) {
            swl_mesh3d m{};
            m.nx = model.nx, m.ny = model.ny, m.nz = model.nz, m.count = int64_t(model.nx) * model.ny * model.nz;
            m.h = model.h, m.lambda = model.lambda, m.mu = model.mu, m.density = model.density;
            m.metrics = model.metrics.data(), m.normals = model.normals.data(), m.jacobian = model.jacobian.data();
            m.source = model.source.data(), m.damping = model.damping.data();
            if (!model.materialLambda.empty())
                m.material_lambda = model.materialLambda.data(), m.material_mu = model.materialMu.data(),
                m.material_density = model.materialDensity.data();
            for (int a = 0; a < 3; ++a) {
                m.source_direction[a] = model.sourceDirection[a];
                if (!model.sourceGradient[a].empty()) m.source_gradient[a] = model.sourceGradient[a].data();
            }
            m.source_amplitude = model.sourceAmplitude;
            m.precision = params.precision;
            m.mechanisms = model.mechanisms;
            for (int l = 0; l < model.mechanisms; ++l)
                m.rates[l] = model.rates[l], m.delta_p[l] = model.deltaP[l].data(), m.delta_s[l] = model.deltaS[l].data();
            if (model.cpmlCount) {
                m.cpml_x = model.cpmlX.data(), m.cpml_y = model.cpmlY.data(), m.cpml_z = model.cpmlZ.data();
                m.cpml_width_x = model.cpmlWidth[0], m.cpml_width_y = model.cpmlWidth[1], m.cpml_width_z = model.cpmlWidth[2];
                m.cpml_count = model.cpmlCount;
            }
            ok(swl3d_create(&m, model.receiverNodes.data(), int32_t(model.receiverNodes.size()), device, &engine));
            ok(swl3d_reserve(engine, std::min(model.total, maxBatch))); // batch tables sized once, at creation
            ok(swl3d_diagnostics(engine, &diag));
        }
        initMs = millis(t0);
    }
    int inflight{};
    std::chrono::steady_clock::time_point batchStart;
    bool launchBatch(int n) {
        if (!engine) throw Failure(SWL_ERR_STATE, "Initialize a model on a device before stepping.");
        if (!fault.empty()) throw Failure(SWL_ERR_STATE, fault);
        n = std::max(0, std::min({n, model.total - step, maxBatch}));
        if (n == 0) return false;
        batchStart = std::chrono::steady_clock::now();
        ok(swl3d_launch(engine, step, n, model.dt, params.frequency, 3.0 / params.frequency));
        inflight = n;
        return true;
    }
    bool pollBatch(bool block) {
        if (!inflight) return true;
        int32_t done = 1, accepted = 0;
        const swl_status st = block ? swl3d_wait(engine, &accepted) : swl3d_query(engine, &done, &accepted);
        if (st != SWL_OK && st != SWL_ERR_FAULT) ok(st);
        if (!done) return false;
        const std::size_t R = model.receiverNodes.size();
        std::vector<double> t[3];
        for (auto &v : t) v.resize(std::size_t(accepted) * R);
        if (accepted && R) ok(swl3d_traces(engine, step, accepted, t[0].data(), t[1].data(), t[2].data()));
        for (std::size_t r = 0; r < R; ++r)
            for (int j = 0; j < accepted; ++j)
                for (int c = 0; c < 3; ++c) rec[c][r].push_back(t[c][r * accepted + j]);
        step += accepted;
        lastMs = millis(batchStart) / std::max(1, accepted);
        totalMs += millis(batchStart);
        inflight = 0;
        ok(swl3d_step_diagnostics(engine, &diag));
        if (st == SWL_ERR_FAULT) {
            fault = "Non-finite RK4 step or energy growth above 10,000 times the source-window peak rejected. "
                    "Last accepted step retained; rebuild with smaller CFL or gentler terrain.";
            throw Failure(SWL_ERR_FAULT, fault);
        }
        return true;
    }
    // CpuSimulation3D::advance (src/three_d/CurvilinearSolver.cpp:445-513)
    void advance(int count) {
        if (count < 0 || count > 20000) throw Failure(SWL_ERR_INVALID, "Invalid step batch.");
        count = std::min(count, model.total - step);
        while (count > 0) {
            const int before = step;
            if (!launchBatch(count)) break;
            pollBatch(true);
            count -= step - before;
        }
    }
    bool completed() const { return step >= model.total; }
    int64_t estimateBytes() const {
        // the engine pitches rows to a multiple of four nodes
        const double s = params.precision == SWL_FP32 ? 4 : 8, n = double((model.nx + 3) / 4 * 4) * model.ny * model.nz;
        const double fields = (s == 4 ? 6 : 4) * 9; // state sets, with the FP32 compensation sets
        return int64_t(n * s * (fields + 9 + 2 + (model.materialLambda.empty() ? 0 : 3) + (model.sourceGradient[0].empty() ? 0 : 3))) + (64 << 20);
    }
    void reset() {
        if (engine) ok(swl3d_reset(engine)), ok(swl3d_diagnostics(engine, &diag));
        step = 0, fault.clear(), totalMs = lastMs = 0;
        clearRecords();
    }
    const std::vector<double> *array(const std::string &n) const {
        const Model3D &m = model;
        if (n == "coordinates") return &m.coordinates;
        if (n == "metrics") return &m.metrics;
        if (n == "jacobian") return &m.jacobian;
        if (n == "normals") return &m.normals;
        if (n == "source") return &m.source;
        if (n == "damping") return &m.damping;
        if (n == "materialLambda") return &m.materialLambda;
        if (n == "materialMu") return &m.materialMu;
        if (n == "materialDensity") return &m.materialDensity;
        if (n == "cpmlX") return &m.cpmlX;
        if (n == "cpmlY") return &m.cpmlY;
        if (n == "cpmlZ") return &m.cpmlZ;
        if (n == "cpmlShape") return &m.cpmlShape;
        if (n == "gslsRates") return &m.gslsRates;
        for (int l = 0; l < 3; ++l) {
            if (n == "deltaP" + std::to_string(l)) return &m.deltaP[l];
            if (n == "deltaS" + std::to_string(l)) return &m.deltaS[l];
        }
        for (int a = 0; a < 3; ++a)
            if (n == "sourceGradient" + std::to_string(a)) return &m.sourceGradient[a];
        return nullptr;
    }
};

inline Params3D toParams(const swl_params3d &c) {
    Params3D p;
    p.precision = c.precision, p.nx = c.nx, p.ny = c.ny, p.nz = c.nz;
    p.spacing = c.spacing, p.vp = c.vp, p.vs = c.vs, p.density = c.density;
    p.layered = c.layered != 0, p.layerDepthMode = c.layer_depth_mode;
    if (c.n_layers < 0 || (c.n_layers && !c.layers)) throw std::runtime_error("Invalid layer list.");
    for (int l = 0; l < c.n_layers; ++l) p.layers.push_back({c.layers[l].thickness, c.layers[l].vp, c.layers[l].vs, c.layers[l].density});
    p.frequency = c.frequency, p.sourceX = c.source_x, p.sourceY = c.source_y, p.sourceZ = c.source_z, p.sourceKind = c.source_kind;
    for (int a = 0; a < 3; ++a) p.sourceDirection[a] = c.source_direction[a];
    p.sourceForce = c.source_force, p.sourceMoment = c.source_moment, p.duration = c.duration, p.maxSteps = c.max_steps;
    p.cfl = c.cfl, p.relief = c.relief, p.wavelength = c.wavelength, p.flattenDepth = c.flatten_depth;
    if (c.dem_nx || c.dem_ny) {
        if (c.dem_nx < 2 || c.dem_ny < 2 || !c.dem_elevations) throw std::runtime_error("Invalid DEM description.");
        p.surfaceGrid.nx = c.dem_nx, p.surfaceGrid.ny = c.dem_ny, p.surfaceGrid.spacing = c.dem_spacing;
        p.surfaceGrid.originX = c.dem_origin_x, p.surfaceGrid.originY = c.dem_origin_y, p.surfaceGrid.datum = c.dem_datum;
        p.surfaceGrid.elevations.assign(c.dem_elevations, c.dem_elevations + std::size_t(c.dem_nx) * c.dem_ny);
    }
    p.receiverKind = c.receiver_kind, p.receiverStartX = c.receiver_start_x, p.receiverStartY = c.receiver_start_y;
    p.receiverZ = c.receiver_z, p.receiverCountX = c.receiver_count_x, p.receiverCountY = c.receiver_count_y;
    p.receiverStrideX = c.receiver_stride_x, p.receiverStrideY = c.receiver_stride_y, p.receiverLimit = c.receiver_limit;
    p.absorbing = c.absorbing != 0;
    for (int a = 0; a < 3; ++a) p.absorbingCells[a] = c.absorbing_cells[a];
    p.absorbingStrength = c.absorbing_strength;
    p.absorber = c.absorber;
    p.cpmlReflection = c.cpml_reflection, p.cpmlKappaMax = c.cpml_kappa_max, p.cpmlFrequency = c.cpml_frequency;
    p.attenuation.enabled = c.attenuation != 0, p.attenuation.mechanisms = c.mechanisms;
    p.attenuation.minFrequency = c.q_min_frequency, p.attenuation.maxFrequency = c.q_max_frequency;
    p.attenuation.referenceFrequency = c.q_reference_frequency, p.attenuation.qp = c.qp, p.attenuation.qs = c.qs;
    if (c.layer_q)
        for (int l = 0; l < c.n_layers; ++l) p.layers[l].qp = c.layer_q[2 * l], p.layers[l].qs = c.layer_q[2 * l + 1];
    p.deviceGeometry = c.device_geometry != 0;
    if (c.layer_names)
        for (int l = 0; l < c.n_layers; ++l) p.layerNames.push_back(c.layer_names[l] ? c.layer_names[l] : "");
    return p;
}

} // namespace swl::host

// The C-ABI session handles (include/swl_session.h) are the session classes themselves.
struct swl2d_session : swl::host::Session2D {};
struct swl3d_session : swl::host::Session3D {};
