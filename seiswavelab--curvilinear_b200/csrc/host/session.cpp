// Session level (include/swl_session.h): the C++20 host of a simulation.  It builds the FP64
// model on the host, hands it to the GPU engine through the engine C ABI, advances in batches
// (one host synchronisation per batch, the acceptance rule applied on the device) and keeps the
// receiver records exactly as the reference sessions do.
#include "sessions.hpp"


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
