// Session level (include/swl_session.h): the C++20 host of a simulation.  It builds the FP64
// model on the host, hands it to the GPU engine through the engine C ABI, advances in batches
// (one host synchronisation per batch, the acceptance rule applied on the device) and keeps the
// receiver records exactly as the reference sessions do.
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
namespace {

struct Failure : std::runtime_error {
    int status;
    Failure(int s, const std::string &m) : std::runtime_error(m), status(s) {}
};
void ok(swl_status s) {
    if (s != SWL_OK) throw Failure(s, swl_last_error());
}
template <class F> swl_status guard(F &&f) {
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
double millis(std::chrono::steady_clock::time_point a) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
}
constexpr int maxBatch = 2048; // steps per engine batch (bounds the device trace table)
} // namespace

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
            ok(swl2d_create(&m, model.receiverNodes.data(), int32_t(model.receiverNodes.size()), device, &engine));
            ok(swl2d_diagnostics(engine, &diag));
        }
        initMs = millis(t0);
    }
    // Simulation::advance (:541-604): batches on the device, records on the host.
    void advance(int count) {
        if (!engine) throw Failure(SWL_ERR_STATE, "Initialize the 2D model on a device first.");
        if (!fault.empty()) throw Failure(SWL_ERR_STATE, fault);
        count = std::max(0, std::min(count, model.total - step));
        std::vector<double> tx, tz;
        while (count > 0) {
            const int n = std::min(count, maxBatch);
            const auto t0 = std::chrono::steady_clock::now();
            int32_t accepted = 0;
            const swl_status st = swl2d_advance(engine, step, n, model.dt, params.frequency, model.scale, 3 / params.frequency, &accepted);
            if (st != SWL_OK && st != SWL_ERR_FAULT) ok(st);
            tx.resize(std::size_t(accepted) * vx.size()), tz.resize(tx.size());
            if (accepted && !vx.empty()) ok(swl2d_traces(engine, step, accepted, tx.data(), tz.data()));
            for (int j = 0; j < accepted; ++j) record(step + j, tx.data(), tz.data(), std::size_t(accepted), std::size_t(j));
            step += accepted;
            lastMs = millis(t0) / std::max(1, accepted);
            totalMs += millis(t0);
            count -= n;
            ok(swl2d_diagnostics(engine, &diag));
            if (st == SWL_ERR_FAULT) {
                fault = "2D step rejected: nonfinite fields or excessive late energy growth. Rebuild the session.";
                throw Failure(SWL_ERR_FAULT, fault);
            }
        }
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

Params2D toParams(const swl_params2d &c) {
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
            ok(swl3d_create(&m, model.receiverNodes.data(), int32_t(model.receiverNodes.size()), device, &engine));
            ok(swl3d_diagnostics(engine, &diag));
        }
        initMs = millis(t0);
    }
    void advance(int count) {
        if (!engine) throw Failure(SWL_ERR_STATE, "Initialize a model on a device before stepping.");
        if (!fault.empty()) throw Failure(SWL_ERR_STATE, fault);
        if (count < 0 || count > 20000) throw Failure(SWL_ERR_INVALID, "Invalid step batch.");
        count = std::min(count, model.total - step);
        std::vector<double> t[3];
        while (count > 0) {
            const int n = std::min(count, maxBatch);
            const auto t0 = std::chrono::steady_clock::now();
            int32_t accepted = 0;
            const swl_status st = swl3d_advance(engine, step, n, model.dt, params.frequency, 3.0 / params.frequency, &accepted);
            if (st != SWL_OK && st != SWL_ERR_FAULT) ok(st);
            const std::size_t R = model.receiverNodes.size();
            for (auto &v : t) v.resize(std::size_t(accepted) * R);
            if (accepted && R) ok(swl3d_traces(engine, step, accepted, t[0].data(), t[1].data(), t[2].data()));
            for (std::size_t r = 0; r < R; ++r)
                for (int j = 0; j < accepted; ++j)
                    for (int c = 0; c < 3; ++c) rec[c][r].push_back(t[c][r * accepted + j]);
            step += accepted;
            lastMs = millis(t0) / std::max(1, accepted);
            totalMs += millis(t0);
            count -= n;
            ok(swl3d_diagnostics(engine, &diag));
            if (st == SWL_ERR_FAULT) {
                fault = "Non-finite RK4 step or energy growth above 10,000 times the source-window peak rejected. "
                        "Last accepted step retained; rebuild with smaller CFL or gentler terrain.";
                throw Failure(SWL_ERR_FAULT, fault);
            }
        }
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
        for (int a = 0; a < 3; ++a)
            if (n == "sourceGradient" + std::to_string(a)) return &m.sourceGradient[a];
        return nullptr;
    }
};

Params3D toParams(const swl_params3d &c) {
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
    return p;
}

} // namespace swl::host

using swl::host::guard;
struct swl2d_session : swl::host::Session2D {};
struct swl3d_session : swl::host::Session3D {};

namespace {
void needSession(const void *s) {
    if (!s) throw swl::host::Failure(SWL_ERR_INVALID, "session is null");
}
template <class S> swl_status modelArray(const S *s, const char *name, double *out, int64_t *n) {
    return guard([&] {
        needSession(s);
        if (!name || !n) throw swl::host::Failure(SWL_ERR_INVALID, "name and n are required");
        const auto *v = s->array(name);
        if (!v) throw swl::host::Failure(SWL_ERR_INVALID, std::string("unknown model array ") + name);
        *n = int64_t(v->size());
        if (out && !v->empty()) std::memcpy(out, v->data(), v->size() * sizeof(double));
    });
}
} // namespace

extern "C" {

void swl2d_params_default(swl_params2d *c) {
    if (!c) return;
    const swl::host::Params2D p;
    std::memset(c, 0, sizeof(*c));
    c->precision = p.precision, c->nx = p.nx, c->nz = p.nz, c->spacing = p.spacing, c->vp = p.vp, c->vs = p.vs;
    c->density = p.density, c->relief = p.relief, c->wavelength = p.wavelength, c->flatten_depth = p.flattenDepth;
    c->frequency = p.frequency, c->duration = p.duration, c->cfl = p.cfl, c->force_per_length = p.forcePerLength;
    c->source_x = p.sourceX, c->source_z = p.sourceZ, c->max_steps = p.maxSteps, c->source_kind = p.sourceKind;
    for (int a = 0; a < 3; ++a) c->source_direction[a] = p.sourceDirection[a];
    c->moment_per_length = p.momentPerLength, c->absorbing = p.absorbing, c->sponge_x = p.spongeX, c->sponge_z = p.spongeZ;
    c->sponge_strength = p.spongeStrength, c->absorber = p.absorber, c->cpml_reflection = p.cpmlReflection;
    c->cpml_kappa_max = p.cpmlKappaMax, c->cpml_frequency = p.cpmlFrequency, c->receiver_start = p.receiverStart;
    c->receiver_count = p.receiverCount, c->receiver_stride = p.receiverStride, c->receiver_depth = p.receiverDepth;
    c->mechanisms = p.attenuation.mechanisms, c->q_min_frequency = p.attenuation.minFrequency;
    c->q_max_frequency = p.attenuation.maxFrequency, c->q_reference_frequency = p.attenuation.referenceFrequency;
    c->qp = p.attenuation.qp, c->qs = p.attenuation.qs;
    c->layered = 0, c->n_layers = 0, c->layers = nullptr; // the reference's default three layers apply when layered
}

swl_status swl2d_session_create(const swl_params2d *c, int32_t device, swl2d_session **out) {
    return guard([&] {
        if (!c || !out) throw swl::host::Failure(SWL_ERR_INVALID, "params and out are required");
        *out = nullptr;
        auto s = std::make_unique<swl2d_session>();
        s->params = swl::host::toParams(*c);
        s->create(device);
        *out = s.release();
    });
}
void swl2d_session_destroy(swl2d_session *s) { delete s; }
swl_status swl2d_session_advance(swl2d_session *s, int32_t count) {
    return guard([&] {
        needSession(s);
        s->advance(count);
    });
}
swl_status swl2d_session_reset(swl2d_session *s) {
    return guard([&] {
        needSession(s);
        s->reset();
    });
}
swl_status swl2d_session_info(const swl2d_session *s, swl_info2d *o) {
    return guard([&] {
        needSession(s);
        if (!o) throw swl::host::Failure(SWL_ERR_INVALID, "out is null");
        const auto &m = s->model;
        *o = swl_info2d{};
        o->nx = m.nx, o->nz = m.nz, o->model_offset_x = m.modelOffsetX, o->total_steps = m.total, o->step = s->step;
        o->field_count = m.fieldCount, o->receivers = int32_t(m.receiverNodes.size()), o->completed = s->step >= m.total;
        o->finite = s->diag.finite, o->mechanisms = m.mechanisms;
        o->count = int64_t(m.nx) * m.nz, o->samples = s->vx.empty() ? 0 : int64_t(s->vx.front().size());
        o->cpml_count = m.cpmlCount, o->resident_bytes = s->engine ? swl2d_resident_bytes(s->engine) : 0;
        o->dt = m.dt, o->record_dt = m.recordDt, o->h = m.h, o->flatten_depth = m.flattenDepth, o->max_metric = m.maxMetric;
        o->min_jacobian = m.minJacobian, o->max_edge = m.maxEdge, o->ppw = m.ppw, o->wave_dt = m.waveDt, o->damping_dt = m.dampingDt;
        o->source_dt = m.sourceDt, o->relaxation_dt = m.relaxationDt, o->cpml_dt = m.cpmlDt, o->max_relative_q_error = m.maxRelativeQError;
        o->energy = s->diag.energy, o->peak_energy = s->diag.peak_energy, o->max_velocity = s->diag.max_velocity;
        o->traction_relative = s->diag.traction_relative, o->init_ms = s->initMs, o->total_step_ms = s->totalMs, o->last_step_ms = s->lastMs;
    });
}
swl_status swl2d_session_records(const swl2d_session *s, double *vx, double *vz) {
    return guard([&] {
        needSession(s);
        if (!vx || !vz) throw swl::host::Failure(SWL_ERR_INVALID, "record buffers are required");
        std::size_t at = 0;
        for (std::size_t r = 0; r < s->vx.size(); ++r) {
            std::copy(s->vx[r].begin(), s->vx[r].end(), vx + at);
            std::copy(s->vz[r].begin(), s->vz[r].end(), vz + at);
            at += s->vx[r].size();
        }
    });
}
swl_status swl2d_session_receiver_positions(const swl2d_session *s, double *xz) {
    return guard([&] {
        needSession(s);
        if (!xz) throw swl::host::Failure(SWL_ERR_INVALID, "buffer is null");
        for (std::size_t r = 0; r < s->model.receiverPositions.size(); ++r)
            xz[2 * r] = s->model.receiverPositions[r][0], xz[2 * r + 1] = s->model.receiverPositions[r][1];
    });
}
swl_status swl2d_session_snapshot(swl2d_session *s, int32_t field, double *out) {
    return guard([&] {
        needSession(s);
        if (!s->engine) throw swl::host::Failure(SWL_ERR_STATE, "no engine (model-only session)");
        swl::host::ok(swl2d_snapshot(s->engine, field, out));
    });
}
swl_status swl2d_session_model(const swl2d_session *s, const char *name, double *out, int64_t *n) { return modelArray(s, name, out, n); }
swl2d_engine *swl2d_session_engine(swl2d_session *s) { return s ? s->engine : nullptr; }

void swl3d_params_default(swl_params3d *c) {
    if (!c) return;
    const swl::host::Params3D p;
    std::memset(c, 0, sizeof(*c));
    c->precision = p.precision, c->nx = p.nx, c->ny = p.ny, c->nz = p.nz, c->spacing = p.spacing, c->vp = p.vp, c->vs = p.vs;
    c->density = p.density, c->frequency = p.frequency, c->source_x = p.sourceX, c->source_y = p.sourceY, c->source_z = p.sourceZ;
    for (int a = 0; a < 3; ++a) c->source_direction[a] = p.sourceDirection[a];
    c->source_force = p.sourceForce, c->source_moment = p.sourceMoment, c->duration = p.duration, c->max_steps = p.maxSteps;
    c->cfl = p.cfl, c->relief = p.relief, c->wavelength = p.wavelength, c->flatten_depth = p.flattenDepth;
    c->receiver_kind = p.receiverKind, c->receiver_start_x = p.receiverStartX, c->receiver_start_y = p.receiverStartY;
    c->receiver_z = p.receiverZ, c->receiver_count_x = p.receiverCountX, c->receiver_count_y = p.receiverCountY;
    c->receiver_stride_x = p.receiverStrideX, c->receiver_stride_y = p.receiverStrideY, c->receiver_limit = p.receiverLimit;
    c->absorbing = p.absorbing;
    for (int a = 0; a < 3; ++a) c->absorbing_cells[a] = p.absorbingCells[a];
    c->absorbing_strength = p.absorbingStrength;
}
swl_status swl3d_session_create(const swl_params3d *c, int32_t device, swl3d_session **out) {
    return guard([&] {
        if (!c || !out) throw swl::host::Failure(SWL_ERR_INVALID, "params and out are required");
        *out = nullptr;
        auto s = std::make_unique<swl3d_session>();
        s->params = swl::host::toParams(*c);
        s->create(device);
        *out = s.release();
    });
}
void swl3d_session_destroy(swl3d_session *s) { delete s; }
swl_status swl3d_session_advance(swl3d_session *s, int32_t count) {
    return guard([&] {
        needSession(s);
        s->advance(count);
    });
}
swl_status swl3d_session_reset(swl3d_session *s) {
    return guard([&] {
        needSession(s);
        s->reset();
    });
}
swl_status swl3d_session_info(const swl3d_session *s, swl_info3d *o) {
    return guard([&] {
        needSession(s);
        if (!o) throw swl::host::Failure(SWL_ERR_INVALID, "out is null");
        const auto &m = s->model;
        *o = swl_info3d{};
        o->nx = m.nx, o->ny = m.ny, o->nz = m.nz, o->total_steps = m.total, o->step = s->step;
        o->receivers = int32_t(m.receiverNodes.size()), o->completed = s->step >= m.total, o->finite = s->diag.finite;
        o->count = int64_t(m.nx) * m.ny * m.nz, o->resident_bytes = s->engine ? swl3d_resident_bytes(s->engine) : 0;
        o->dt = m.dt, o->h = m.h, o->flatten_depth = m.flattenDepth, o->min_jacobian = m.minJacobian, o->max_metric_norm = m.maxMetricNorm;
        o->min_cell_length = m.minCellLength, o->max_cell_edge = m.maxCellEdge, o->wave_dt = m.waveDt, o->damping_dt = m.dampingDt;
        o->source_dt = m.sourceDt, o->ppw = m.ppw, o->energy = s->diag.energy, o->peak_energy = s->diag.peak_energy;
        o->max_velocity = s->diag.max_velocity, o->traction_rate_relative = s->diag.traction_rate_relative;
        o->init_ms = s->initMs, o->total_step_ms = s->totalMs, o->last_step_ms = s->lastMs;
    });
}
swl_status swl3d_session_records(const swl3d_session *s, double *vx, double *vy, double *vz) {
    return guard([&] {
        needSession(s);
        if (!vx || !vy || !vz) throw swl::host::Failure(SWL_ERR_INVALID, "record buffers are required");
        double *dst[3] = {vx, vy, vz};
        for (int c = 0; c < 3; ++c) {
            std::size_t at = 0;
            for (const auto &v : s->rec[c]) std::copy(v.begin(), v.end(), dst[c] + at), at += v.size();
        }
    });
}
swl_status swl3d_session_snapshot(swl3d_session *s, int32_t field, double *out) {
    return guard([&] {
        needSession(s);
        if (!s->engine) throw swl::host::Failure(SWL_ERR_STATE, "no engine (model-only session)");
        swl::host::ok(swl3d_snapshot(s->engine, field, out));
    });
}
swl_status swl3d_session_model(const swl3d_session *s, const char *name, double *out, int64_t *n) { return modelArray(s, name, out, n); }
swl3d_engine *swl3d_session_engine(swl3d_session *s) { return s ? s->engine : nullptr; }

} // extern "C"
