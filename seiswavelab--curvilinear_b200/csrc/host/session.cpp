// Session level (include/swl_session.h): the C++20 host of a simulation.  It builds the FP64
// model on the host, hands it to the GPU engine through the engine C ABI, advances in batches
// (one host synchronisation per batch, the acceptance rule applied on the device) and keeps the
// receiver records exactly as the reference sessions do.
#include "sessions.hpp"
#include "records.hpp"
#include "../../../include/swl_records.h"
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <locale>


using swl::host::guard;

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
// include/SeisCommon/SourceMechanism.hpp:32-38: the unit force direction (zero for a moment)
std::array<double, 3> unitDirection(int kind, const std::array<double, 3> &d) {
    if (kind == 1) return {0, 0, 0};
    const double norm = std::hypot(d[0], d[1], d[2]);
    return {d[0] / norm, d[1] / norm, d[2] / norm};
}
const char *const kBackend = "swl_b200 CUDA sm_100a";

// The record set of a 2D session as src/two_d/ui/Workbench2D.cpp:251-268 builds it: components Vz,
// Vx; receivers at (x, 0, z); the source node's coordinates (x, 0, z); the record axis's dt.
swl::records::RecordSet records2d(const swl::host::Session2D &s) {
    const auto &m = s.model;
    const auto &p = s.params;
    swl::records::RecordSet rec;
    rec.dt = m.recordDt;
    rec.components = {"Vz", "Vx"};
    rec.samples = s.vx.empty() ? 0 : s.vx.front().size();
    const int sx = (p.sourceX < 0 ? p.nx / 2 : p.sourceX) + 3 + m.modelOffsetX, sz = p.sourceZ + 3; // Grid::modelIndex
    const std::size_t node = std::size_t(sx) + std::size_t(m.nx) * std::size_t(sz);
    const double srcX = m.coordinates[2 * node], srcZ = m.coordinates[2 * node + 1];
    for (std::size_t r = 0; r < s.vx.size(); ++r) {
        swl::records::Trace t;
        t.position = {m.receiverPositions[r][0], 0, m.receiverPositions[r][1]};
        t.source = {srcX, 0, srcZ};
        t.channel = {s.vz[r].data(), s.vx[r].data(), nullptr};
        rec.traces.push_back(t);
    }
    return rec;
}
// src/three_d/ui/RecordView3D.cpp:5-6: components Vz, Vx, Vy; the solver's dt.
swl::records::RecordSet records3d(const swl::host::Session3D &s) {
    swl::records::RecordSet rec;
    rec.dt = s.model.dt;
    rec.components = {"Vz", "Vx", "Vy"};
    rec.samples = s.rec[2].empty() ? 0 : s.rec[2].front().size();
    for (std::size_t r = 0; r < s.rec[2].size(); ++r) {
        swl::records::Trace t;
        t.position = s.model.receiverPositions[r];
        t.channel = {s.rec[2][r].data(), s.rec[0][r].data(), s.rec[1][r].data()};
        rec.traces.push_back(t);
    }
    return rec;
}
swl::records::SegyOptions segyOptions(const swl_segy_options *o) {
    if (!o) throw swl::host::Failure(SWL_ERR_INVALID, "options are required");
    return {o->profile, o->sample_gain, o->sample_interval_s};
}
std::ofstream csvFile(const char *path, const char *emptyName, const char *cannotCreate) {
    if (!path) throw swl::host::Failure(SWL_ERR_INVALID, "path is null");
    const std::filesystem::path file(path);
    if (file.empty() || file.filename().empty()) throw swl::host::Failure(SWL_ERR_INVALID, emptyName);
    if (!file.parent_path().empty()) std::filesystem::create_directories(file.parent_path());
    std::ofstream out(file);
    if (!out) throw swl::host::Failure(SWL_ERR_INVALID, cannotCreate);
    out.imbue(std::locale::classic());
    out << std::setprecision(17);
    return out;
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
    c->absorber = p.absorber;
    c->cpml_reflection = p.cpmlReflection, c->cpml_kappa_max = p.cpmlKappaMax, c->cpml_frequency = p.cpmlFrequency;
    c->attenuation = p.attenuation.enabled, c->mechanisms = p.attenuation.mechanisms;
    c->q_min_frequency = p.attenuation.minFrequency, c->q_max_frequency = p.attenuation.maxFrequency;
    c->q_reference_frequency = p.attenuation.referenceFrequency, c->qp = p.attenuation.qp, c->qs = p.attenuation.qs;
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


// ------------------------------------------------------------------------- record output
swl_status swl2d_session_write_segy(const swl2d_session *s, int32_t component, const char *path, const swl_segy_options *o) {
    return guard([&] {
        needSession(s);
        if (!path) throw swl::host::Failure(SWL_ERR_INVALID, "path is null");
        swl::records::writeSegy(records2d(*s), component, path, segyOptions(o));
    });
}
swl_status swl3d_session_write_segy(const swl3d_session *s, int32_t component, const char *path, const swl_segy_options *o) {
    return guard([&] {
        needSession(s);
        if (!path) throw swl::host::Failure(SWL_ERR_INVALID, "path is null");
        swl::records::writeSegy(records3d(*s), component, path, segyOptions(o));
    });
}
// writeReceivers (src/two_d/CurvilinearSolver2D.cpp:811-855): the run's metadata as comment lines,
// then one row per receiver and record sample.
swl_status swl2d_session_write_receivers(const swl2d_session *s, const char *path) {
    return guard([&] {
        needSession(s);
        const auto &p = s->params;
        const auto &m = s->model;
        auto out = csvFile(path, "Choose a receiver CSV file name.", "Cannot create 2D receiver CSV.");
        const char *precision = p.precision == SWL_FP32 ? "FP32" : "FP64";
        const auto dir = unitDirection(p.sourceKind, p.sourceDirection);
        const auto &q = p.attenuation;
        out << "# P-SV plane strain; x,z in m; velocity in m/s; t=0 included\n# dt=" << m.recordDt << "\n# solver_dt=" << m.dt
            << "\n# backend=" << kBackend;
        out << "\n# calculation_precision=" << precision << "; model_precision=" << precision
            << "; record_storage=Float64; values_sampled_from=" << precision;
        out << "\n# external_absorption=" << p.externalAbsorption << "; computational_NXZ=" << m.nx - 6 << ',' << m.nz - 6;
        out << "\n# absorption_enabled=" << p.absorbing << "; absorber=" << (p.absorber == 1 ? "CFS-PML_ADE" : "sponge")
            << "; effective_width_XZ=" << std::min(p.spongeX, p.nx / 3) << ',' << std::min(p.spongeZ, p.nz / 3)
            << "; PML_target_R=" << p.cpmlReflection << "; kappa=" << p.cpmlKappaMax
            << "; PML_Hz=" << (p.cpmlFrequency > 0 ? p.cpmlFrequency : p.frequency);
        out << "\n# GSLS=" << q.enabled << "; mechanisms=" << q.mechanisms << "; reference_Hz=" << q.referenceFrequency
            << "; fit_band_Hz=" << q.minFrequency << ':' << q.maxFrequency;
        if (p.layered) {
            for (std::size_t i = 0; i < p.layers.size(); ++i) out << "\n# layer_" << i << "_Qp_Qs=" << p.layers[i].qp << ',' << p.layers[i].qs;
        } else {
            out << "; Qp=" << q.qp << "; Qs=" << q.qs;
        }
        out << "\n# source_kind=" << p.sourceKind << " (0=directional_force,1=isotropic_moment); force_per_length_N_per_m="
            << p.forcePerLength << "; diagonal_moment_per_length_N=" << p.momentPerLength << "; direction_XZ=" << dir[0] << ','
            << dir[2] << "; Ricker_f0_Hz=" << p.frequency << "\nreceiver,x_m,z_m,time_s,vx_m_s,vz_m_s\n";
        for (std::size_t r = 0; r < s->vx.size(); ++r)
            for (std::size_t t = 0; t < s->vx[r].size(); ++t)
                out << r << ',' << m.receiverPositions[r][0] << ',' << m.receiverPositions[r][1] << ',' << t * m.recordDt << ','
                    << s->vx[r][t] << ',' << s->vz[r][t] << '\n';
        if (!out) throw swl::host::Failure(SWL_ERR_INVALID, "2D receiver write failed.");
    });
}
// writeReceiversCsv (src/three_d/ReceiverIo.cpp): header comments, then one row per time sample with
// the selected components of every receiver.
swl_status swl3d_session_write_receivers(const swl3d_session *s, const char *path, const int32_t selected[3]) {
    return guard([&] {
        needSession(s);
        if (!selected || !(selected[0] || selected[1] || selected[2]))
            throw swl::host::Failure(SWL_ERR_INVALID, "Select at least one receiver component.");
        const auto &p = s->params;
        const auto &m = s->model;
        auto out = csvFile(path, "Could not open receiver CSV.", "Could not open receiver CSV.");
        static const char *const names[3] = {"Vx", "Vy", "Vz"};
        out << "# ";
        bool comma = false;
        for (int c = 0; c < 3; ++c)
            if (selected[c]) out << (comma ? "," : "") << names[c], comma = true;
        out << " in m/s; time in seconds; coordinates in metres; depth positive down\n";
        const auto dir = unitDirection(p.sourceKind, p.sourceDirection);
        out << "# source_kind=" << p.sourceKind << " (0=directional_force,1=isotropic_moment); force_N=" << p.sourceForce
            << "; diagonal_moment_Nm=" << p.sourceMoment << "; direction=" << dir[0] << ',' << dir[1] << ',' << dir[2]
            << "; Ricker_f0_Hz=" << p.frequency << '\n';
        const int si = p.sourceX < 0 ? p.nx / 2 : p.sourceX, sj = p.sourceY < 0 ? p.ny / 2 : p.sourceY, sk = p.sourceZ;
        const std::size_t node = std::size_t(si + 3) + std::size_t(m.nx) * (std::size_t(sj + 3) + std::size_t(m.ny) * std::size_t(sk + 3));
        out << "# source XYZ (m): " << m.coordinates[3 * node] << ',' << m.coordinates[3 * node + 1] << ',' << m.coordinates[3 * node + 2]
            << "; grid IJK (zero-based): " << si << ',' << sj << ',' << sk << '\n';
        const std::size_t R = m.receiverPositions.size();
        for (std::size_t r = 0; r < R; ++r)
            out << "# receiver " << r + 1 << ": " << m.receiverPositions[r][0] << ',' << m.receiverPositions[r][1] << ','
                << m.receiverPositions[r][2] << '\n';
        out << "time_s";
        for (std::size_t r = 0; r < R; ++r)
            for (int c = 0; c < 3; ++c)
                if (selected[c]) out << ",receiver_" << r + 1 << '_' << names[c];
        out << '\n';
        for (int t = 0; t <= s->step; ++t) {
            out << t * m.dt;
            for (std::size_t r = 0; r < R; ++r)
                for (int c = 0; c < 3; ++c)
                    if (selected[c]) out << ',' << s->rec[c][r].at(std::size_t(t));
            out << '\n';
        }
        if (!out.good()) throw swl::host::Failure(SWL_ERR_INVALID, "Receiver CSV write failed.");
    });
}


// -------------------------------------------------------------------- snapshots and probes
// writeSnapshot (src/two_d/CurvilinearSolver2D.cpp:725-810): a VTK structured grid of the logical
// model with the run's metadata as field data, the selected wavefield components (and material)
// as point data in the session precision, and the node coordinates.
swl_status swl2d_session_write_snapshot(swl2d_session *s, const char *path, const int32_t components[7], int32_t include_material) {
    return guard([&] {
        needSession(s);
        if (!components || std::none_of(components, components + 7, [](int32_t v) { return v != 0; }))
            throw swl::host::Failure(SWL_ERR_INVALID, "Select at least one wavefield export component.");
        if (!path) throw swl::host::Failure(SWL_ERR_INVALID, "path is null");
        const auto &p = s->params;
        const auto &m = s->model;
        const std::size_t count = std::size_t(m.nx) * m.nz;
        // the current state (zero before the first step, and without an engine)
        std::vector<double> fields[6];
        const int nf = m.mechanisms ? 6 : 5;
        for (int f = 0; f < nf; ++f) {
            fields[f].assign(count, 0.0);
            if (s->engine) swl::host::ok(swl2d_snapshot(s->engine, f, fields[f].data()));
        }
        std::ofstream out(path);
        if (!out) throw swl::host::Failure(SWL_ERR_INVALID, "Cannot create 2D VTS file.");
        out.imbue(std::locale::classic());
        const bool fp32 = p.precision == SWL_FP32;
        const char *pointType = fp32 ? "Float32" : "Float64";
        out << std::setprecision(17) << "<?xml version=\"1.0\"?>\n<VTKFile type=\"StructuredGrid\" version=\"0.1\" "
               "byte_order=\"LittleEndian\"><StructuredGrid WholeExtent=\"0 " << p.nx - 1 << " 0 0 0 " << p.nz - 1 << "\">\n";
        const auto dir = unitDirection(p.sourceKind, p.sourceDirection);
        out << "<FieldData>";
        const auto scalar = [&](const char *name, double value) {
            out << "<DataArray type=\"Float64\" Name=\"" << name << "\" NumberOfTuples=\"1\" format=\"ascii\">" << value << "</DataArray>";
        };
        const auto &q = p.attenuation;
        scalar("CalculationPrecisionBits", fp32 ? 32 : 64);
        scalar("ExternalAbsorption", p.externalAbsorption);
        scalar("ComputationalNodesX", m.nx - 6);
        scalar("ComputationalNodesZ", m.nz - 6);
        scalar("LogicalModelOffsetXCells", m.modelOffsetX);
        scalar("AbsorptionEnabled", p.absorbing);
        scalar("AbsorberKind", p.absorber);
        scalar("AbsorberWidthXCells", std::min(p.spongeX, p.nx / 3));
        scalar("AbsorberWidthZCells", std::min(p.spongeZ, p.nz / 3));
        scalar("CfsPmlTargetReflection", p.cpmlReflection);
        scalar("CfsPmlKappaMax", p.cpmlKappaMax);
        scalar("CfsPmlFrequencyHz", p.cpmlFrequency > 0 ? p.cpmlFrequency : p.frequency);
        scalar("SourceKind", p.sourceKind);
        scalar("SourceForcePerLengthNPerM", p.forcePerLength);
        scalar("SourceMomentPerLengthN", p.momentPerLength);
        scalar("SourceFrequencyHz", p.frequency);
        scalar("SourceDirectionX", dir[0]);
        scalar("SourceDirectionZ", dir[2]);
        scalar("SimulationDt", m.dt);
        scalar("RecordIntervalSeconds", m.recordDt);
        scalar("SimulationStep", s->step);
        scalar("TIME_VALUE", s->step * m.dt);
        scalar("AttenuationGSLS", q.enabled);
        scalar("QReferenceFrequencyHz", q.referenceFrequency);
        scalar("QBandMinHz", q.minFrequency);
        scalar("QBandMaxHz", q.maxFrequency);
        scalar("RelaxationMechanisms", q.enabled ? q.mechanisms : 0);
        static const char *const names[10] = {"Vx", "Vz", "VelocityMagnitude", "Pressure", "Sxx", "Szz", "Sxz", "Vp", "Vs", "Density"};
        const int first = int(std::find_if(components, components + 7, [](int32_t v) { return v != 0; }) - components);
        out << "</FieldData><Piece Extent=\"0 " << p.nx - 1 << " 0 0 0 " << p.nz - 1 << "\"><PointData Scalars=\"" << names[first] << "\">\n";
        const auto node = [&](int i, int k) { return std::size_t(i + 3 + m.modelOffsetX) + std::size_t(m.nx) * std::size_t(k + 3); };
        for (int f = 0; f < 10; ++f) {
            if (f < 7 ? !components[f] : !include_material) continue;
            out << "<DataArray type=\"" << pointType << "\" Name=\"" << names[f] << "\" format=\"ascii\">\n";
            for (int k = 0; k < p.nz; ++k)
                for (int i = 0; i < p.nx; ++i) {
                    const std::size_t n = node(i, k);
                    double v;
                    if (f < 2) v = fields[f][n];
                    else if (f == 2) v = std::sqrt(fields[0][n] * fields[0][n] + fields[1][n] * fields[1][n]);
                    else if (f == 3) { // pressure -tr(S)/3; plane strain Syy = lambda (Sxx + Szz) / (2 (lambda + mu)) without GSLS
                        const double mu = m.density[n] * m.vs[n] * m.vs[n];
                        const double lambda = m.density[n] * m.vp[n] * m.vp[n] - 2 * mu;
                        v = q.enabled ? -(fields[2][n] + fields[3][n] + fields[5][n]) / 3
                                      : -(1 + lambda / (2 * (lambda + mu))) * (fields[2][n] + fields[3][n]) / 3;
                    } else if (f < 7) v = fields[f - 2][n];
                    else v = f == 7 ? m.vp[n] : f == 8 ? m.vs[n] : m.density[n];
                    out << (fp32 ? double(static_cast<float>(v)) : v) << ' ';
                }
            out << "\n</DataArray>\n";
        }
        if (q.enabled) {
            const auto array = [&](const char *name, const std::vector<double> &values) {
                out << "<DataArray type=\"" << pointType << "\" Name=\"" << name << "\" format=\"ascii\">\n";
                for (int k = 0; k < p.nz; ++k)
                    for (int i = 0; i < p.nx; ++i) out << values[node(i, k)] << ' ';
                out << "\n</DataArray>\n";
            };
            if (include_material) array("Qp", m.qp), array("Qs", m.qs);
            if (components[3] || components[4] || components[5]) array("Syy", fields[5]);
        }
        out << "</PointData><Points><DataArray type=\"" << pointType << "\" NumberOfComponents=\"3\" format=\"ascii\">\n";
        for (int k = 0; k < p.nz; ++k)
            for (int i = 0; i < p.nx; ++i) {
                const std::size_t n = node(i, k);
                out << m.coordinates[2 * n] << " 0 " << m.coordinates[2 * n + 1] << ' ';
            }
        out << "</DataArray></Points></Piece></StructuredGrid></VTKFile>\n";
        if (!out) throw swl::host::Failure(SWL_ERR_INVALID, "2D VTS write failed.");
    });
}
// Simulation::readProbes (src/two_d/CurvilinearSolver2D.cpp:710-724): Vx, Vz, Sxx, Szz, Sxz at
// logical model nodes (i, k), 5 values per node, read on the device.
swl_status swl2d_session_read_probes(swl2d_session *s, const int32_t *nodes_ik, int32_t n, double *out5) {
    return guard([&] {
        if (!s) throw swl::host::Failure(SWL_ERR_INVALID, "Initialize before probe readback.");
        if (n > 1000000) throw swl::host::Failure(SWL_ERR_INVALID, "Too many probe nodes.");
        if (n < 0 || (n && (!nodes_ik || !out5))) throw swl::host::Failure(SWL_ERR_INVALID, "nodes and out are required");
        if (!s->engine) throw swl::host::Failure(SWL_ERR_STATE, "no engine (model-only session)");
        const auto &m = s->model;
        std::vector<int64_t> idx(static_cast<std::size_t>(n));
        for (int32_t r = 0; r < n; ++r) {
            const int i = nodes_ik[2 * r], k = nodes_ik[2 * r + 1];
            if (i < 0 || i >= m.logicalNx || k < 0 || k >= m.logicalNz) throw swl::host::Failure(SWL_ERR_INVALID, "Probe outside logical model.");
            idx[std::size_t(r)] = int64_t(i + 3 + m.modelOffsetX) + int64_t(m.nx) * int64_t(k + 3);
        }
        if (n) swl::host::ok(swl2d_probes(s->engine, idx.data(), n, out5));
    });
}


// writeVts (src/three_d/VtsWriter.cpp) of the session's current state (CpuSimulation3D::snapshot,
// src/three_d/CurvilinearSolver.cpp:648-687): the physical nodes as a VTK structured grid with the
// run's metadata, the selected fields, the material (and layer ids) and the velocity vector.
// fields: Vx, Vy, Vz, |V|, mean normal stress, Sxx, Syy, Szz, Sxy, Sxz, Syz.
swl_status swl3d_session_write_snapshot(swl3d_session *s, const char *path, const int32_t fields[11], int32_t include_material,
                                        int32_t include_velocity_vector) {
    return guard([&] {
        needSession(s);
        if (!path || !fields) throw swl::host::Failure(SWL_ERR_INVALID, "path and fields are required");
        if (!include_velocity_vector && std::none_of(fields, fields + 11, [](int32_t v) { return v != 0; }))
            throw swl::host::Failure(SWL_ERR_INVALID, "Select at least one wavefield component.");
        const auto &p = s->params;
        const auto &m = s->model;
        const int nx = m.nx - 6, ny = m.ny - 6, nz = m.nz - 6;
        const std::size_t count = std::size_t(m.nx) * m.ny * m.nz, plane = std::size_t(m.nx) * m.ny;
        std::vector<double> f[9];
        for (int c = 0; c < 9; ++c) {
            f[c].assign(count, 0.0);
            if (s->engine) swl::host::ok(swl3d_snapshot(s->engine, c, f[c].data()));
        }
        bool finite = true;
        if (s->engine) {
            swl_diag3d d{};
            swl::host::ok(swl3d_diagnostics(s->engine, &d));
            finite = d.finite != 0;
        }
        if (!finite) throw swl::host::Failure(SWL_ERR_INVALID, "Refusing to export non-finite simulation fields.");
        const bool layered = !m.materialLambda.empty();
        std::vector<double> vp, vs;
        std::vector<int> layer;
        if (layered) {
            vp.resize(count), vs.resize(count), layer.resize(count);
            for (std::size_t q = 0; q < count; ++q) {
                vp[q] = std::sqrt((m.materialLambda[q] + 2 * m.materialMu[q]) / m.materialDensity[q]);
                vs[q] = std::sqrt(m.materialMu[q] / m.materialDensity[q]);
                // materialDepth3D / materialLayerAtDepth3D (include/Seis3D/MaterialModels3D.hpp:19-31)
                double depth;
                if (p.layerDepthMode == 0) depth = (static_cast<int>(q / plane) - 3) * m.h;
                else if (p.layerDepthMode == 2) depth = m.coordinates[3 * q + 2];
                else depth = m.coordinates[3 * q + 2] - m.coordinates[3 * (3 * plane + q % plane) + 2];
                double bottom = 0;
                int id = static_cast<int>(p.layers.size()) - 1;
                for (std::size_t i = 0; i + 1 < p.layers.size(); ++i) {
                    bottom += p.layers[i].thickness;
                    if (depth < bottom) {
                        id = static_cast<int>(i);
                        break;
                    }
                }
                layer[q] = id;
            }
        }
        const int si = p.sourceX < 0 ? p.nx / 2 : p.sourceX, sj = p.sourceY < 0 ? p.ny / 2 : p.sourceY, sk = p.sourceZ;
        const std::size_t sq = std::size_t(si + 3) + std::size_t(m.nx) * (std::size_t(sj + 3) + std::size_t(m.ny) * std::size_t(sk + 3));
        const double *source = &m.coordinates[3 * sq];
        const auto dir = unitDirection(p.sourceKind, p.sourceDirection);
        const std::filesystem::path file(path);
        if (!file.parent_path().empty()) std::filesystem::create_directories(file.parent_path());
        std::ofstream out(file, std::ios::binary);
        if (!out) throw swl::host::Failure(SWL_ERR_INVALID, std::string("Could not open VTS output file: ") + file.string());
        out.imbue(std::locale::classic());
        out << std::setprecision(17);
        const auto meta = [&](const char *type, const char *name, auto value) {
            out << "<DataArray type=\"" << type << "\" Name=\"" << name << "\" NumberOfTuples=\"1\" format=\"ascii\">" << value << "</DataArray>";
        };
        out << "<?xml version=\"1.0\"?>\n<VTKFile type=\"StructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\">\n"
            << "  <StructuredGrid WholeExtent=\"0 " << nx - 1 << " 0 " << ny - 1 << " 0 " << nz - 1 << "\">\n    <FieldData>";
        meta("Float64", "TIME_VALUE", s->step * m.dt);
        meta("Float64", "SimulationDt", m.dt);
        meta("Int32", "SimulationStep", s->step);
        meta("Float64", "SourceX", source[0]);
        meta("Float64", "SourceY", source[1]);
        meta("Float64", "SourceZ", source[2]);
        meta("Int32", "SourceKind", p.sourceKind);
        meta("Float64", "SourceForceN", p.sourceForce);
        meta("Float64", "SourceMomentNm", p.sourceMoment);
        meta("Float64", "SourceFrequencyHz", p.frequency);
        meta("Float64", "SourceDirectionX", dir[0]);
        meta("Float64", "SourceDirectionY", dir[1]);
        meta("Float64", "SourceDirectionZ", dir[2]);
        meta("Float64", "GridSpacing", m.h);
        meta("Float64", "TerrainTransitionDepth", m.flattenDepth);
        out << "</FieldData>\n    <Piece Extent=\"0 " << nx - 1 << " 0 " << ny - 1 << " 0 " << nz - 1 << "\">\n      <PointData";
        static const char *const names[11] = {"Vx", "Vy", "Vz", "VelocityMagnitude", "MeanNormalStress", "Sxx", "Syy", "Szz", "Sxy", "Sxz", "Syz"};
        for (int c = 0; c < 11; ++c)
            if (fields[c]) {
                out << " Scalars=\"" << names[c] << "\"";
                break;
            }
        if (include_velocity_vector) out << " Vectors=\"Velocity\"";
        out << ">\n";
        // physical nodes, x fastest; `perLine` values and then a line break
        const auto each = [&](int perLine, auto &&write) {
            std::size_t written = 0;
            for (int k = 3; k < m.nz - 3; ++k)
                for (int j = 3; j < m.ny - 3; ++j)
                    for (int i = 3; i < m.nx - 3; ++i) {
                        write(std::size_t(i) + std::size_t(m.nx) * (std::size_t(j) + std::size_t(m.ny) * std::size_t(k)));
                        if (++written % perLine == 0) out << "\n          ";
                    }
        };
        const auto scalar = [&](const char *name, auto valueAt) {
            out << "        <DataArray type=\"Float64\" Name=\"" << name << "\" format=\"ascii\">\n          ";
            each(6, [&](std::size_t q) { out << valueAt(q) << ' '; });
            out << "\n        </DataArray>\n";
        };
        for (int c = 0; c < 3; ++c)
            if (fields[c]) scalar(names[c], [&](std::size_t q) { return f[c][q]; });
        if (include_material) {
            scalar("Vp", [&](std::size_t q) { return layered ? vp[q] : p.vp; });
            scalar("Vs", [&](std::size_t q) { return layered ? vs[q] : p.vs; });
            scalar("Density", [&](std::size_t q) { return layered ? m.materialDensity[q] : p.density; });
            if (layered) scalar("LayerId", [&](std::size_t q) { return layer[q]; });
        }
        if (fields[3]) scalar(names[3], [&](std::size_t q) { return std::hypot(f[0][q], f[1][q], f[2][q]); });
        if (fields[4]) scalar(names[4], [&](std::size_t q) { return -(f[3][q] + f[4][q] + f[5][q]) / 3.; });
        for (int c = 0; c < 6; ++c)
            if (fields[5 + c]) scalar(names[5 + c], [&](std::size_t q) { return f[3 + c][q]; });
        if (include_velocity_vector) {
            out << "        <DataArray type=\"Float64\" Name=\"Velocity\" NumberOfComponents=\"3\" format=\"ascii\">\n          ";
            each(2, [&](std::size_t q) { out << f[0][q] << ' ' << f[1][q] << ' ' << f[2][q] << ' '; });
            out << "\n        </DataArray>\n";
        }
        out << "      </PointData>\n      <CellData/>\n      <Points>\n"
            << "        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n          ";
        each(2, [&](std::size_t q) { out << m.coordinates[3 * q] << ' ' << m.coordinates[3 * q + 1] << ' ' << m.coordinates[3 * q + 2] << ' '; });
        out << "\n        </DataArray>\n      </Points>\n    </Piece>\n  </StructuredGrid>\n</VTKFile>\n";
        if (!out.good()) throw swl::host::Failure(SWL_ERR_INVALID, std::string("Failed while writing VTS output: ") + file.string());
    });
}

} // extern "C"
