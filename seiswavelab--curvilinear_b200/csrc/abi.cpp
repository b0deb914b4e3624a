// The C ABI (include/swl_b200.h): argument checks, error capture, no exceptions across the
// boundary.  Each entry point names the reference interface it stands in for in the header.
#include "../../include/swl_b200.h"
#include "engine2d.cuh"
#include "engine3d.cuh"
#include <cstring>
#include <string>
#include <vector>

namespace swl {
std::string &lastErrorRef() {
    thread_local std::string message;
    return message;
}
} // namespace swl

namespace {
#define lastError (swl::lastErrorRef())

template <class F> swl_status guarded(F &&f) {
    try {
        lastError.clear();
        f();
        return SWL_OK;
    } catch (const swl::Error &e) {
        lastError = e.what();
        return e.status;
    } catch (const std::bad_alloc &) {
        lastError = "host allocation failed";
        return SWL_ERR_MEMORY;
    } catch (const std::exception &e) {
        lastError = e.what();
        return SWL_ERR_INVALID;
    } catch (...) {
        lastError = "unknown failure";
        return SWL_ERR_INVALID;
    }
}
int device(int requested) {
    const int d = swl::selectDevice(requested);
    if (d < 0)
        throw swl::Error(SWL_ERR_UNAVAILABLE, requested >= 0 ? "CUDA device " + std::to_string(requested) +
                                                                   " is not a usable sm_100 device"
                                                             : std::string("no usable sm_100 CUDA device"));
    return d;
}
void need(const void *p, const char *what) {
    if (!p) throw swl::Error(SWL_ERR_INVALID, std::string(what) + " is null");
}
} // namespace

struct swl2d_engine {
    std::unique_ptr<swl::Engine2D> impl;
};
struct swl3d_engine {
    std::unique_ptr<swl::Engine3D> impl;
};
struct swl2d_queue {
    std::unique_ptr<swl::Queue2D> impl;
};

extern "C" {

const char *swl_last_error(void) { return lastError.c_str(); }
const char *swl_version(void) { return "swl_b200 0.1.0 (sm_100a)"; }
int32_t swl_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int usable = 0;
    for (int d = 0; d < n; ++d) {
        cudaDeviceProp p{};
        if (cudaGetDeviceProperties(&p, d) == cudaSuccess && p.major == 10) ++usable;
    }
    return usable;
}

// ----------------------------------------------------------------------------- 2D
swl_status swl2d_create(const swl_mesh2d *mesh, const int64_t *receivers, int32_t n, int32_t dev, swl2d_engine **out) {
    return guarded([&] {
        need(mesh, "mesh");
        need(out, "out");
        *out = nullptr;
        if (mesh->precision != SWL_FP64 && mesh->precision != SWL_FP32)
            throw swl::Error(SWL_ERR_INVALID, "Unknown 2D calculation precision.");
        if (mesh->array_precision != SWL_FP64 && mesh->array_precision != SWL_FP32)
            throw swl::Error(SWL_ERR_INVALID, "Unknown 2D mesh array precision.");
        const int d = device(dev);
        auto e = std::make_unique<swl2d_engine>();
        e->impl = mesh->precision == SWL_FP64 ? swl::makeEngine2D64(*mesh, receivers, n, d)
                                              : swl::makeEngine2D32(*mesh, receivers, n, d);
        *out = e.release();
    });
}
void swl2d_destroy(swl2d_engine *e) { delete e; }

#define ENGINE(e)                                                                                                      \
    need(e, "engine");                                                                                                 \
    auto &E = *(e)->impl

swl_status swl2d_step(swl2d_engine *e, double, double dt, double frequency, double scale, int32_t step) {
    return guarded([&] {
        ENGINE(e);
        if (E.faulted()) throw swl::Error(SWL_ERR_STATE, "2D engine holds a rejected step; reset or rebuild it");
        if (!(dt > 0) || step < 0) throw swl::Error(SWL_ERR_INVALID, "step needs dt > 0 and step >= 0");
        E.step(dt, frequency, scale, step);
    });
}
swl_status swl2d_advance(swl2d_engine *e, int32_t first, int32_t count, double dt, double frequency, double scale,
                         double growthAfter, int32_t *accepted) {
    int done = 0;
    swl_status s = guarded([&] {
        ENGINE(e);
        if (E.faulted()) throw swl::Error(SWL_ERR_STATE, "2D engine holds a rejected step; reset or rebuild it");
        if (!(dt > 0) || first < 0 || count < 0) throw swl::Error(SWL_ERR_INVALID, "advance needs dt > 0, first >= 0, count >= 0");
        done = E.advance(first, count, dt, frequency, scale, growthAfter);
        if (done < count)
            throw swl::Error(SWL_ERR_FAULT, "2D step rejected: nonfinite fields or excessive late energy growth. Rebuild the session.");
    });
    if (accepted) *accepted = done;
    return s;
}
swl_status swl2d_launch(swl2d_engine *e, int32_t first, int32_t count, double dt, double frequency, double scale,
                        double growthAfter) {
    return guarded([&] {
        ENGINE(e);
        if (E.faulted()) throw swl::Error(SWL_ERR_STATE, "2D engine holds a rejected step; reset or rebuild it");
        if (!(dt > 0) || first < 0 || count < 0) throw swl::Error(SWL_ERR_INVALID, "launch needs dt > 0, first >= 0, count >= 0");
        E.launch(first, count, dt, frequency, scale, growthAfter);
    });
}
swl_status swl2d_query(swl2d_engine *e, int32_t *done, int32_t *accepted) {
    return guarded([&] {
        ENGINE(e);
        need(done, "done");
        int acc = 0;
        *done = E.query(acc) ? 1 : 0;
        if (accepted) *accepted = acc;
        if (*done && E.faulted())
            throw swl::Error(SWL_ERR_FAULT, "2D step rejected: nonfinite fields or excessive late energy growth. Rebuild the session.");
    });
}
swl_status swl2d_wait(swl2d_engine *e, int32_t *accepted) {
    return guarded([&] {
        ENGINE(e);
        const int acc = E.finish();
        if (accepted) *accepted = acc;
        if (E.faulted())
            throw swl::Error(SWL_ERR_FAULT, "2D step rejected: nonfinite fields or excessive late energy growth. Rebuild the session.");
    });
}
swl_status swl2d_queue_create(int32_t dev, int32_t precision, swl2d_queue **out) {
    return guarded([&] {
        need(out, "out");
        *out = nullptr;
        if (precision != SWL_FP64 && precision != SWL_FP32) throw swl::Error(SWL_ERR_INVALID, "precision must be SWL_FP64 or SWL_FP32");
        const int d = device(dev);
        auto q = std::make_unique<swl2d_queue>();
        q->impl = precision == SWL_FP64 ? swl::makeQueue2D64(d) : swl::makeQueue2D32(d);
        *out = q.release();
    });
}
void swl2d_queue_destroy(swl2d_queue *q) {
    if (!q) return;
    try {
        delete q;
    } catch (...) {
    }
}
swl_status swl2d_queue_launch(swl2d_queue *q, swl2d_engine *const *engines, int32_t n, const int32_t *first, const int32_t *count,
                              const double *dt, const double *frequency, const double *scale, const double *growthAfter) {
    return guarded([&] {
        need(q, "queue");
        if (n < 0) throw swl::Error(SWL_ERR_INVALID, "engine count must be >= 0");
        if (n == 0) return;
        need(engines, "engines"), need(first, "first"), need(count, "count"), need(dt, "dt"), need(frequency, "frequency");
        need(scale, "scale"), need(growthAfter, "check_growth_after");
        std::vector<swl::Engine2D *> e(n);
        for (int i = 0; i < n; ++i) {
            need(engines[i], "engine");
            e[i] = engines[i]->impl.get();
        }
        const std::vector<int> f(first, first + n), c(count, count + n);
        q->impl->launch(e.data(), n, f.data(), c.data(), dt, frequency, scale, growthAfter);
    });
}
swl_status swl2d_queue_limit(swl2d_queue *q, int32_t ctasPerSm) {
    return guarded([&] {
        need(q, "queue");
        q->impl->limit(ctasPerSm);
    });
}
swl_status swl2d_queue_segment(swl2d_queue *q, int32_t segment) {
    return guarded([&] {
        need(q, "queue");
        q->impl->segment(segment);
    });
}
swl_status swl2d_queue_query(swl2d_queue *q, int32_t *done) {
    return guarded([&] {
        need(q, "queue"), need(done, "done");
        *done = 0;
        *done = q->impl->query() ? 1 : 0;
    });
}
swl_status swl2d_queue_wait(swl2d_queue *q) {
    return guarded([&] {
        need(q, "queue");
        q->impl->finish();
    });
}
swl_status swl2d_rollback(swl2d_engine *e) { return guarded([&] { ENGINE(e); E.rollback(); }); }
swl_status swl2d_reset(swl2d_engine *e) { return guarded([&] { ENGINE(e); E.reset(); }); }
swl_status swl2d_diagnostics(swl2d_engine *e, swl_diag2d *out) {
    return guarded([&] {
        ENGINE(e);
        need(out, "out");
        E.diagnostics(*out);
    });
}
swl_status swl2d_step_diagnostics(swl2d_engine *e, swl_diag2d *out) {
    return guarded([&] {
        ENGINE(e);
        need(out, "out");
        E.stepDiagnostics(*out);
    });
}
swl_status swl2d_sample(swl2d_engine *e, double *vx, double *vz) {
    return guarded([&] {
        ENGINE(e);
        need(vx, "vx");
        need(vz, "vz");
        E.sample(vx, vz);
    });
}
swl_status swl2d_traces(swl2d_engine *e, int32_t first, int32_t count, double *vx, double *vz) {
    return guarded([&] {
        ENGINE(e);
        need(vx, "vx");
        need(vz, "vz");
        E.traces(first, count, vx, vz);
    });
}
swl_status swl2d_snapshot(swl2d_engine *e, int32_t field, double *out) {
    return guarded([&] {
        ENGINE(e);
        need(out, "out");
        E.snapshot(field, out);
    });
}
swl_status swl2d_load_field(swl2d_engine *e, int32_t field, const double *values) {
    return guarded([&] {
        ENGINE(e);
        need(values, "values");
        E.load(field, values);
    });
}
swl_status swl2d_probes(swl2d_engine *e, const int64_t *nodes, int32_t n, double *out5) {
    return guarded([&] {
        ENGINE(e);
        if (n < 0 || n > 1000000) throw swl::Error(SWL_ERR_INVALID, "Too many probe nodes.");
        if (n) need(nodes, "nodes"), need(out5, "out5");
        E.probes(nodes, n, out5);
    });
}
int64_t swl2d_resident_bytes(const swl2d_engine *e) { return e && e->impl ? e->impl->residentBytes() : 0; }
swl_status swl2d_layout(swl2d_engine *e, swl_layout2d *out) {
    return guarded([&] {
        ENGINE(e);
        need(out, "out");
        E.layout(*out);
    });
}
swl_status swl2d_profile(swl2d_engine *e, int32_t first, int32_t count, double dt, double frequency, double scale,
                         swl_profile *out) {
    return guarded([&] {
        ENGINE(e);
        need(out, "out");
        if (E.faulted()) throw swl::Error(SWL_ERR_STATE, "2D engine holds a rejected step; reset or rebuild it");
        if (!(dt > 0) || first < 0 || count <= 0 || count > 4096)
            throw swl::Error(SWL_ERR_INVALID, "profile needs dt > 0, first >= 0 and 1..4096 steps");
        E.profile(first, count, dt, frequency, scale, *out);
    });
}
swl_status swl2d_set_stream(swl2d_engine *e, void *stream) {
    return guarded([&] { ENGINE(e); E.setStream(static_cast<cudaStream_t>(stream)); });
}
swl_status swl2d_reserve(swl2d_engine *e, int32_t steps) {
    return guarded([&] { ENGINE(e); E.reserve(steps); });
}

// ----------------------------------------------------------------------------- 3D
swl_status swl3d_create(const swl_mesh3d *mesh, const int64_t *receivers, int32_t n, int32_t dev, swl3d_engine **out) {
    return guarded([&] {
        need(mesh, "mesh");
        need(out, "out");
        *out = nullptr;
        if (mesh->precision != SWL_FP64 && mesh->precision != SWL_FP32)
            throw swl::Error(SWL_ERR_INVALID, "Unknown 3D calculation precision.");
        const int d = device(dev);
        auto e = std::make_unique<swl3d_engine>();
        e->impl = mesh->precision == SWL_FP64 ? swl::makeEngine3D64(*mesh, receivers, n, d)
                                              : swl::makeEngine3D32(*mesh, receivers, n, d);
        *out = e.release();
    });
}
void swl3d_destroy(swl3d_engine *e) { delete e; }
swl_status swl3d_step(swl3d_engine *e, double, double dt, double frequency, int32_t step) {
    return guarded([&] {
        ENGINE(e);
        if (E.faulted()) throw swl::Error(SWL_ERR_STATE, "3D engine holds a rejected step; reset or rebuild it");
        if (!(dt > 0) || step < 0) throw swl::Error(SWL_ERR_INVALID, "step needs dt > 0 and step >= 0");
        E.step(dt, frequency, step);
    });
}
swl_status swl3d_advance(swl3d_engine *e, int32_t first, int32_t count, double dt, double frequency, double growthAfter,
                         int32_t *accepted) {
    int done = 0;
    swl_status s = guarded([&] {
        ENGINE(e);
        if (E.faulted()) throw swl::Error(SWL_ERR_STATE, "3D engine holds a rejected step; reset or rebuild it");
        if (!(dt > 0) || first < 0 || count < 0) throw swl::Error(SWL_ERR_INVALID, "advance needs dt > 0, first >= 0, count >= 0");
        done = E.advance(first, count, dt, frequency, growthAfter);
        if (done < count)
            throw swl::Error(SWL_ERR_FAULT, "Non-finite RK4 step or energy growth rejected. Last accepted fields retained.");
    });
    if (accepted) *accepted = done;
    return s;
}
swl_status swl3d_launch(swl3d_engine *e, int32_t first, int32_t count, double dt, double frequency, double growthAfter) {
    return guarded([&] {
        ENGINE(e);
        if (E.faulted()) throw swl::Error(SWL_ERR_STATE, "3D engine holds a rejected step; reset or rebuild it");
        if (!(dt > 0) || first < 0 || count < 0) throw swl::Error(SWL_ERR_INVALID, "launch needs dt > 0, first >= 0, count >= 0");
        E.launch(first, count, dt, frequency, growthAfter);
    });
}
swl_status swl3d_query(swl3d_engine *e, int32_t *done, int32_t *accepted) {
    return guarded([&] {
        ENGINE(e);
        need(done, "done");
        int acc = 0;
        *done = E.query(acc) ? 1 : 0;
        if (accepted) *accepted = acc;
        if (*done && E.faulted()) throw swl::Error(SWL_ERR_FAULT, "Non-finite RK4 step or energy growth rejected.");
    });
}
swl_status swl3d_wait(swl3d_engine *e, int32_t *accepted) {
    return guarded([&] {
        ENGINE(e);
        const int acc = E.finish();
        if (accepted) *accepted = acc;
        if (E.faulted()) throw swl::Error(SWL_ERR_FAULT, "Non-finite RK4 step or energy growth rejected.");
    });
}
swl_status swl3d_rollback(swl3d_engine *e) { return guarded([&] { ENGINE(e); E.rollback(); }); }
swl_status swl3d_reset(swl3d_engine *e) { return guarded([&] { ENGINE(e); E.reset(); }); }
swl_status swl3d_diagnostics(swl3d_engine *e, swl_diag3d *out) {
    return guarded([&] {
        ENGINE(e);
        need(out, "out");
        E.diagnostics(*out);
    });
}
swl_status swl3d_step_diagnostics(swl3d_engine *e, swl_diag3d *out) {
    return guarded([&] {
        ENGINE(e);
        need(out, "out");
        E.stepDiagnostics(*out);
    });
}
swl_status swl3d_sample(swl3d_engine *e, double *vx, double *vy, double *vz) {
    return guarded([&] {
        ENGINE(e);
        need(vx, "vx"), need(vy, "vy"), need(vz, "vz");
        E.sample(vx, vy, vz);
    });
}
swl_status swl3d_traces(swl3d_engine *e, int32_t first, int32_t count, double *vx, double *vy, double *vz) {
    return guarded([&] {
        ENGINE(e);
        need(vx, "vx"), need(vy, "vy"), need(vz, "vz");
        E.traces(first, count, vx, vy, vz);
    });
}
swl_status swl3d_snapshot(swl3d_engine *e, int32_t field, double *out) {
    return guarded([&] {
        ENGINE(e);
        need(out, "out");
        E.snapshot(field, out);
    });
}
swl_status swl3d_load_field(swl3d_engine *e, int32_t field, const double *values) {
    return guarded([&] {
        ENGINE(e);
        need(values, "values");
        E.load(field, values);
    });
}
int64_t swl3d_resident_bytes(const swl3d_engine *e) { return e && e->impl ? e->impl->residentBytes() : 0; }
swl_status swl3d_profile(swl3d_engine *e, int32_t first, int32_t count, double dt, double frequency, swl_profile *out) {
    return guarded([&] {
        ENGINE(e);
        need(out, "out");
        if (E.faulted()) throw swl::Error(SWL_ERR_STATE, "3D engine holds a rejected step; reset or rebuild it");
        if (!(dt > 0) || first < 0 || count <= 0 || count > 4096)
            throw swl::Error(SWL_ERR_INVALID, "profile needs dt > 0, first >= 0 and 1..4096 steps");
        E.profile(first, count, dt, frequency, *out);
    });
}
swl_status swl3d_set_stream(swl3d_engine *e, void *stream) {
    return guarded([&] { ENGINE(e); E.setStream(static_cast<cudaStream_t>(stream)); });
}
swl_status swl3d_reserve(swl3d_engine *e, int32_t steps) {
    return guarded([&] { ENGINE(e); E.reserve(steps); });
}

} // extern "C"
