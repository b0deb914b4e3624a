// Host side of the 3D engine (the B200 replacement of src/three_d/CudaEngine3D.cu:68-150).
// Same state scheme as the 2D engine: two alternating state/accumulator sets and two stage
// sets of nine fields, CUDA-graph batches of eight steps, a device-side acceptance verdict.
#pragma once
#include "../../include/swl_b200.h"
#include "runtime.cuh"
#include "stage3d.cuh"
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <memory>
#include <vector>

namespace swl {

class Engine3D {
  public:
    virtual ~Engine3D() = default;
    virtual void step(double dt, double frequency, int step) = 0;
    virtual int advance(int first, int count, double dt, double frequency, double growthAfter) = 0;
    virtual void rollback() = 0;
    virtual void reset() = 0;
    virtual void diagnostics(swl_diag3d &) = 0;
    // Diagnostics of the last accepted step as the device verdict recorded them (read back with
    // the batch): no kernel and no synchronisation.  Before any step, the same as diagnostics().
    virtual void stepDiagnostics(swl_diag3d &) = 0;
    virtual void sample(double *vx, double *vy, double *vz) = 0;
    virtual void traces(int first, int count, double *vx, double *vy, double *vz) = 0;
    virtual void snapshot(int field, double *out) = 0;
    virtual void load(int field, const double *in) = 0;
    virtual int64_t residentBytes() const = 0;
    virtual bool faulted() const = 0;
    virtual void profile(int first, int count, double dt, double frequency, swl_profile &out) = 0;
    virtual void setStream(cudaStream_t stream) = 0;
    // Preallocate the forcing and trace tables for batches of up to `steps` steps, so that such
    // batches record no new CUDA graphs.
    virtual void reserve(int steps) = 0;
    virtual void launch(int first, int count, double dt, double frequency, double growthAfter) = 0;
    virtual bool query(int &accepted) = 0;
    virtual int finish() = 0;
};

std::unique_ptr<Engine3D> makeEngine3D64(const swl_mesh3d &, const int64_t *, int, int);
std::unique_ptr<Engine3D> makeEngine3D32(const swl_mesh3d &, const int64_t *, int, int);

namespace detail3 {
template <class Real> struct Launch {
    template <int DX, int DY, int DZ, bool CPML>
    static void stc(int stage, dim3 g, dim3 b, cudaStream_t s, const k3::StageArgs<Real> &a) {
        switch (stage) {
        case 0: k3::stage3d<Real, DX, DY, DZ, 0, CPML><<<g, b, 0, s>>>(a); break;
        case 1: k3::stage3d<Real, DX, DY, DZ, 1, CPML><<<g, b, 0, s>>>(a); break;
        case 2: k3::stage3d<Real, DX, DY, DZ, 2, CPML><<<g, b, 0, s>>>(a); break;
        default: k3::stage3d<Real, DX, DY, DZ, 3, CPML><<<g, b, 0, s>>>(a); break;
        }
    }
    template <int DX, int DY, int DZ>
    static void st(int stage, dim3 g, dim3 b, cudaStream_t s, const k3::StageArgs<Real> &a) {
        if (a.m.cpml || a.m.mech) stc<DX, DY, DZ, true>(stage, g, b, s, a);
        else stc<DX, DY, DZ, false>(stage, g, b, s, a);
    }
    static void stage(int dx, int dy, int dz, int stage, dim3 g, dim3 b, cudaStream_t s, const k3::StageArgs<Real> &a) {
        switch (dx * 4 + dy * 2 + dz) {
        case 0: st<0, 0, 0>(stage, g, b, s, a); break;
        case 1: st<0, 0, 1>(stage, g, b, s, a); break;
        case 2: st<0, 1, 0>(stage, g, b, s, a); break;
        case 3: st<0, 1, 1>(stage, g, b, s, a); break;
        case 4: st<1, 0, 0>(stage, g, b, s, a); break;
        case 5: st<1, 0, 1>(stage, g, b, s, a); break;
        case 6: st<1, 1, 0>(stage, g, b, s, a); break;
        default: st<1, 1, 1>(stage, g, b, s, a); break;
        }
    }
};
} // namespace detail3

template <class Real> class TypedEngine3D final : public Engine3D {
    int device_{};
    cudaStream_t stream_{}, ownStream_{};
    k3::Mesh<Real> m_{};
    long long count_{};         // nodes of one pitched field (px*ny*nz)
    long long dense_{};         // nodes of one field in the API's dense layout (nx*ny*nz)
    std::vector<DeviceBuffer> model_;
    DeviceBuffer sets_, recIdx_, traces_, forcing_, clock_, partials_, surfRate_;
    // Sets 0-1: state / accumulator (roles u_, a_); 2-3: stage states; FP32 only, 4-5: the Kahan
    // compensation of sets 0-1 (set 4 + r compensates set r, so a role swap moves both).
    static constexpr int kSets = k2::kahan<Real>() ? 6 : 4;
    Real *set_[6]{};
    // CFS-PML memories: the same sets and roles as the fields (pcount_ values each)
    DeviceBuffer psets_;
    Real *pset_[6]{};
    long long pcount_{0};
    int fc_{9}; // fields per set: 9, plus 6 GSLS memories per mechanism
    int u_{0}, a_{1};
    bool previous_{false};
    int nrec_{}, traceCap_{}, forcingCap_{};
    dim3 grid_, block_{32, 8, 1};
    dim3 statsGrid_; // stats3d: CTAs of 32 x 8 columns over k3::STATS_LAYERS z layers
    int nparts_{};
    k2::Clock hostClock_{};
    PinnedBuffer pinnedForcing_, pinnedClock_, pinnedTraces_;
    int pinnedRows_{0};     // trace rows of the last launched batch copied to pinnedTraces_ with it
    bool clockStats_{false}; // the host clock holds a verdict's diagnostics
    std::map<int, cudaGraphExec_t> graphs_;
    bool faulted_{false};
    int registers_{};
    double dt_{}, amplitudeScale_{};
    double hostDensity_{}, hostH_{}, amplitude_{};
    cudaEvent_t done_{}; // completion of the in-flight batch
    bool inflight_{false};
    int batchU0_{0};
    void settle() {
        if (inflight_) finish();
    }

    Real *upload(const std::vector<Real> &v) {
        model_.emplace_back(std::max<std::size_t>(1, v.size()) * sizeof(Real));
        if (!v.empty())
            check(cudaMemcpy(model_.back().ptr, v.data(), v.size() * sizeof(Real), cudaMemcpyHostToDevice), "upload model");
        return model_.back().template as<Real>();
    }
    // Pitched position of dense node d = i + nx*(j + ny*k).
    long long pitched(long long d) const {
        const long long i = d % m_.nx, r = d / m_.nx;
        return i + (long long)m_.px * r;
    }
    // A dense per-node array (value of node d at src[d*stride + offset]) in the engine precision,
    // pitched; the pad columns hold zero.
    std::vector<Real> conv(const double *src, std::size_t stride = 1, std::size_t offset = 0) const {
        std::vector<Real> out(std::size_t(count_), Real(0));
        const std::size_t nx = std::size_t(m_.nx), rows = std::size_t(m_.ny) * m_.nz;
        for (std::size_t r = 0; r < rows; ++r)
            for (std::size_t i = 0; i < nx; ++i) {
                const Real v = static_cast<Real>(src[(i + nx * r) * stride + offset]);
                if (!std::isfinite(double(v))) throw Error(SWL_ERR_INVALID, "3D mesh value is not finite in the engine precision");
                out[i + std::size_t(m_.px) * r] = v;
            }
        return out;
    }
    void dropGraphs() {
        for (auto &g : graphs_) cudaGraphExecDestroy(g.second);
        graphs_.clear();
    }
    k3::StageArgs<Real> args(int stage) const {
        k3::StageArgs<Real> p{};
        p.m = m_;
        Real *U = set_[u_], *A = set_[a_], *S1 = set_[2], *S2 = set_[3];
        p.base = U;
        p.acc = A;
        switch (stage) {
        case 0: p.in = U, p.out = S1; break;
        case 1: p.in = S1, p.out = S2; break;
        case 2: p.in = S2, p.out = S1; break;
        default: p.in = S1, p.out = nullptr; break;
        }
        p.forcing = forcing_.as<Real>();
        p.clock = clock_.as<k2::Clock>();
        p.weight = stage == 2 ? static_cast<Real>(dt_) : static_cast<Real>(0.5 * dt_);
        p.w6 = static_cast<Real>(dt_ / 6.0);
        p.w3 = static_cast<Real>(dt_ / 3.0);
        p.surfRate = surfRate_.as<double>();
        if (k2::kahan<Real>()) p.cin = set_[4 + u_], p.cout = set_[4 + a_];
        if (pcount_) {
            Real *PU = pset_[u_], *PA = pset_[a_], *PS1 = pset_[2], *PS2 = pset_[3];
            p.pbase = PU, p.pacc = PA;
            switch (stage) {
            case 0: p.pin = PU, p.pout = PS1; break;
            case 1: p.pin = PS1, p.pout = PS2; break;
            case 2: p.pin = PS2, p.pout = PS1; break;
            default: p.pin = PS1, p.pout = nullptr; break;
            }
            if (k2::kahan<Real>()) p.pcin = pset_[4 + u_], p.pcout = pset_[4 + a_];
        }
        return p;
    }
    void enqueueStep(int step, bool verdict, cudaEvent_t *ev = nullptr) {
        if (ev) check(cudaEventRecord(ev[0], stream_), "record event");
        for (int s = 0; s < 4; ++s) {
            detail3::Launch<Real>::stage(direction(step, s, 0), direction(step, s, 1), direction(step, s, 2), s, grid_, block_,
                                         stream_, args(s));
            if (ev) check(cudaEventRecord(ev[1 + s], stream_), "record event");
        }
        check(cudaGetLastError(), "3D stage launch");
        if (verdict) {
            Real *fresh = set_[a_];
            k3::stats3d<Real><<<statsGrid_, block_, 0, stream_>>>(m_, fresh, surfRate_.as<double>(), clock_.as<k2::Clock>(),
                                                             partials_.as<k3::Partial>());
            if (ev) check(cudaEventRecord(ev[5], stream_), "record event");
            k3::verdict3d<Real><<<1, 512, 0, stream_>>>(partials_.as<k3::Partial>(), nparts_, fresh, count_,
                                                         recIdx_.as<long long>(), nrec_, traces_.as<double>(), clock_.as<k2::Clock>());
            if (ev) check(cudaEventRecord(ev[6], stream_), "record event");
            check(cudaGetLastError(), "3D verdict launch");
        }
        std::swap(u_, a_);
    }
    // Algorithmic HBM bytes of one step, the fused classic-RK4 count 17 F + 4 M per physical node;
    // M = nine metrics plus lambda, mu, rho when the material varies.  The FP64 kernels move one F
    // less (the accumulator carries the partial state sum, so the last stage does not read U).
    double bytesPerStep() const {
        const double s = sizeof(Real), points = double(m_.nx - 6) * (m_.ny - 6) * (m_.nz - 6);
        const double F = 9 * s, M = (m_.mlambda ? 12 : 9) * s;
        return points * (17 * F * fc_ / 9 + 4 * (M + 2 * m_.mech * s)) + double(pcount_) * 17 * s;
    }
    // FP32 only: the last stage's compensation terms read and written (2 F); it also reads U, which
    // the count above already holds.
    double extraBytesPerStep() const {
        if (!k2::kahan<Real>()) return 0;
        const double s = sizeof(Real), points = double(m_.nx - 6) * (m_.ny - 6) * (m_.nz - 6);
        return points * 2 * fc_ * s + double(pcount_) * 2 * s;
    }
    void ensureCapacity(int steps) {
        if (steps > forcingCap_) {
            forcing_.allocate(std::size_t(steps) * 3 * sizeof(Real));
            forcingCap_ = steps;
            dropGraphs();
        }
        if (steps > traceCap_) {
            traces_.allocate(std::max<std::size_t>(1, std::size_t(steps) * nrec_ * 3) * sizeof(double));
            traceCap_ = steps;
            dropGraphs();
        }
        pinnedForcing_.reserve(std::size_t(steps) * 3 * sizeof(Real));
        pinnedTraces_.reserve(std::max<std::size_t>(1, std::size_t(traceCap_) * nrec_ * 3) * sizeof(double));
    }
    // src/three_d/CurvilinearSolver.cpp:75-77 (scale = amplitude / (rho0 h^3)).
    double source(double t, double f) const {
        const double scale = amplitude_ / (hostDensity_ * hostH_ * hostH_ * hostH_);
        const double tau = 3.14159265358979323846 * f * (t - 1.5 / f);
        return scale * (1.0 - 2.0 * tau * tau) * std::exp(-tau * tau);
    }
    void fillForcing(int first, int count, double dt, double frequency) {
        Real *f = pinnedForcing_.as<Real>();
        for (int j = 0; j < count; ++j) {
            const double t = (first + j) * dt;
            f[3 * j] = static_cast<Real>(source(t, frequency));
            f[3 * j + 1] = static_cast<Real>(source(t + 0.5 * dt, frequency));
            f[3 * j + 2] = static_cast<Real>(source(t + dt, frequency));
        }
        check(cudaMemcpyAsync(forcing_.ptr, f, std::size_t(count) * 3 * sizeof(Real), cudaMemcpyHostToDevice, stream_),
              "upload source");
    }
    void pushClock() {
        *pinnedClock_.as<k2::Clock>() = hostClock_;
        check(cudaMemcpyAsync(clock_.ptr, pinnedClock_.ptr, sizeof(k2::Clock), cudaMemcpyHostToDevice, stream_), "set clock");
    }
    void pullClock() {
        check(cudaMemcpyAsync(pinnedClock_.ptr, clock_.ptr, sizeof(k2::Clock), cudaMemcpyDeviceToHost, stream_), "read clock");
        check(cudaStreamSynchronize(stream_), "3D batch completion");
        hostClock_ = *pinnedClock_.as<k2::Clock>();
    }

  public:
    TypedEngine3D(const swl_mesh3d &g, const int64_t *rec, int nrec, int device) : device_(device) {
        DeviceScope scope(device_);
        if (g.nx < 14 || g.ny < 14 || g.nz < 14 || g.count != int64_t(g.nx) * g.ny * g.nz)
            throw Error(SWL_ERR_INVALID, "3D mesh needs nx, ny, nz >= 14 padded nodes and count = nx*ny*nz");
        if (!g.metrics || !g.jacobian || !g.source || !g.damping || !g.normals)
            throw Error(SWL_ERR_INVALID, "3D mesh arrays (metrics, jacobian, source, damping, normals) are required");
        if (nrec < 0 || (nrec && !rec)) throw Error(SWL_ERR_INVALID, "receiver list is invalid");
        check(cudaStreamCreateWithFlags(&ownStream_, cudaStreamNonBlocking), "create stream");
        stream_ = ownStream_;
        m_.nx = g.nx, m_.ny = g.ny, m_.nz = g.nz;
        m_.px = (g.nx + 3) / 4 * 4;
        m_.plane = (long long)m_.px * g.ny;
        m_.count = m_.plane * g.nz;
        count_ = m_.count;
        dense_ = g.count;
        const std::size_t n = std::size_t(count_);
        nrec_ = nrec;
        hostDensity_ = g.density, hostH_ = g.h, amplitude_ = g.source_amplitude;
        m_.h = static_cast<Real>(g.h);
        {
            // x/h equals x*(1/h) bit for bit when h is a power of two; otherwise the kernels form
            // the correctly rounded quotient from RN(1/h).  FP32 always multiplies.
            if (!(g.h >= 0x1p-20 && g.h <= 0x1p+20)) throw Error(SWL_ERR_INVALID, "3D grid spacing must lie in [2^-20, 2^20]");
            int e2 = 0;
            const bool pow2 = std::frexp(g.h, &e2) == 0.5;
            m_.hinv = static_cast<Real>(1.0 / g.h);
            m_.hinvExact = (pow2 || sizeof(Real) == 4) ? 1 : 0;
        }
        m_.lambda = static_cast<Real>(g.lambda), m_.mu = static_cast<Real>(g.mu), m_.density = static_cast<Real>(g.density);
        for (int c = 0; c < 9; ++c) m_.metric[c] = upload(conv(g.metrics, 9, c));
        m_.jac = upload(conv(g.jacobian));
        const auto damping = conv(g.damping);
        m_.damping = upload(damping);
        const auto src = conv(g.source);
        m_.source = upload(src);
        std::vector<Real> sg[3];
        const bool moment = g.source_gradient[0] != nullptr;
        for (int a = 0; a < 3; ++a) {
            if (moment) {
                if (!g.source_gradient[a]) throw Error(SWL_ERR_INVALID, "moment source needs three gradient arrays");
                sg[a] = conv(g.source_gradient[a]);
                m_.sg[a] = upload(sg[a]);
            }
            m_.sdir[a] = static_cast<Real>(g.source_direction[a]);
        }
        if (g.material_lambda || g.material_mu || g.material_density) {
            if (!g.material_lambda || !g.material_mu || !g.material_density)
                throw Error(SWL_ERR_INVALID, "layered material needs lambda, mu and density arrays");
            m_.mlambda = upload(conv(g.material_lambda));
            m_.mmu = upload(conv(g.material_mu));
            m_.mdensity = upload(conv(g.material_density));
        }
        {
            // divBy's correctly rounded quotient needs a divisor in [2^-20, 2^20]; only the
            // computational nodes' densities are divisors
            auto inRange = [](Real r) { return r >= Real(0x1p-20) && r <= Real(0x1p+20); };
            bool ok = inRange(m_.density);
            if (g.material_density) {
                const auto rho = conv(g.material_density);
                for (int k = 3; ok && k < g.nz - 3; ++k)
                    for (int j = 3; ok && j < g.ny - 3; ++j)
                        for (int i = 3; i < g.nx - 3; ++i)
                            if (!inRange(rho[i + std::size_t(m_.px) * j + std::size_t(m_.plane) * k])) {
                                ok = false;
                                break;
                            }
            }
            m_.rhoRecip = ok ? 1 : 0;
        }
        {
            std::vector<Real> nrm(3 * std::size_t(m_.plane), Real(0));
            const std::size_t nx = std::size_t(g.nx), top = std::size_t(3) * nx * g.ny;
            for (std::size_t j = 0; j < std::size_t(g.ny); ++j)
                for (std::size_t i = 0; i < nx; ++i)
                    for (int c = 0; c < 3; ++c)
                        nrm[3 * (i + std::size_t(m_.px) * j) + c] = static_cast<Real>(g.normals[3 * (top + i + nx * j) + c]);
            m_.normals = upload(nrm);
        }
        // boxes of the source support and of the zero sponge rate
        int b[6] = {g.nx, 0, g.ny, 0, g.nz, 0};
        for (int k = 0; k < g.nz; ++k)
            for (int j = 0; j < g.ny; ++j)
                for (int i = 0; i < g.nx; ++i) {
                    const std::size_t q = i + std::size_t(m_.px) * (j + std::size_t(g.ny) * k);
                    const bool nz = moment ? (sg[0][q] != Real(0) || sg[1][q] != Real(0) || sg[2][q] != Real(0)) : src[q] != Real(0);
                    if (nz)
                        b[0] = std::min(b[0], i), b[1] = std::max(b[1], i + 1), b[2] = std::min(b[2], j), b[3] = std::max(b[3], j + 1),
                        b[4] = std::min(b[4], k), b[5] = std::max(b[5], k + 1);
                }
        m_.src_i0 = b[0], m_.src_i1 = b[1], m_.src_j0 = b[2], m_.src_j1 = b[3], m_.src_k0 = b[4], m_.src_k1 = b[5];
        {
            auto D = [&](int i, int j, int k) { return damping[i + std::size_t(m_.px) * (j + std::size_t(g.ny) * k)]; };
            const int jm = g.ny / 2, im = g.nx / 2;
            int i0 = 3, i1 = g.nx - 3, j0 = 3, j1 = g.ny - 3, kk = 3;
            while (i0 < i1 && D(i0, jm, 3) != Real(0)) ++i0;
            while (i1 > i0 && D(i1 - 1, jm, 3) != Real(0)) --i1;
            while (j0 < j1 && D(im, j0, 3) != Real(0)) ++j0;
            while (j1 > j0 && D(im, j1 - 1, 3) != Real(0)) --j1;
            if (i0 < i1 && j0 < j1)
                while (kk < g.nz - 3 && D((i0 + i1) / 2, (j0 + j1) / 2, kk) == Real(0)) ++kk;
            bool ok = i0 < i1 && j0 < j1;
            for (int k = 0; ok && k < kk; ++k)
                for (int j = j0; ok && j < j1; ++j)
                    for (int i = i0; i < i1; ++i)
                        if (D(i, j, k) != Real(0)) {
                            ok = false;
                            break;
                        }
            if (ok) m_.dmp_i0 = i0, m_.dmp_i1 = i1, m_.dmp_j0 = j0, m_.dmp_j1 = j1, m_.dmp_k1 = kk >= g.nz - 3 ? g.nz : kk;
        }
        if (g.mechanisms < 0 || g.mechanisms > 3) throw Error(SWL_ERR_INVALID, "3D GSLS needs 0..3 mechanisms");
        if (g.mechanisms) { // GSLS: the strengths, and 6 memory fields per mechanism beside the nine
            for (int l = 0; l < g.mechanisms; ++l) {
                if (!g.delta_p[l] || !g.delta_s[l] || !(g.rates[l] > 0)) throw Error(SWL_ERR_INVALID, "3D GSLS needs rates and strengths");
                m_.rates[l] = static_cast<Real>(g.rates[l]);
                m_.dP[l] = upload(conv(g.delta_p[l]));
                m_.dS[l] = upload(conv(g.delta_s[l]));
            }
            m_.mech = g.mechanisms;
        }
        fc_ = 9 + 6 * g.mechanisms;
        sets_.allocate(kSets * std::size_t(fc_) * n * sizeof(Real));
        for (int s = 0; s < kSets; ++s) set_[s] = sets_.as<Real>() + std::size_t(s) * fc_ * n;
        if (g.cpml_count) { // CFS-PML slabs (swl_mesh3d)
            const int NX = g.nx - 6, NY = g.ny - 6, NZ = g.nz - 6;
            if (g.cpml_width_x < 0 || g.cpml_width_y < 0 || g.cpml_width_z < 0 || 2 * g.cpml_width_x > NX ||
                2 * g.cpml_width_y > NY || g.cpml_width_z > NZ || !g.cpml_x || !g.cpml_y || !g.cpml_z ||
                g.cpml_count != 6 * (2 * int64_t(g.cpml_width_x) * NY * NZ + 2 * int64_t(g.cpml_width_y) * NX * NZ +
                                     int64_t(g.cpml_width_z) * NX * NY))
                throw Error(SWL_ERR_INVALID, "3D CFS-PML needs widths within the grid, three profiles and "
                                             "cpml_count = 6*(2wx*ny*nz + 2wy*nx*nz + wz*nx*ny) over the computational grid");
            auto prof = [&](const double *src, int len) {
                std::vector<Real> v(3 * std::size_t(len));
                for (std::size_t q = 0; q < v.size(); ++q) v[q] = static_cast<Real>(src[q]);
                return upload(v);
            };
            m_.cpml = 1, m_.wx = g.cpml_width_x, m_.wy = g.cpml_width_y, m_.wz = g.cpml_width_z;
            m_.cpx = prof(g.cpml_x, NX), m_.cpy = prof(g.cpml_y, NY), m_.cpz = prof(g.cpml_z, NZ);
            pcount_ = g.cpml_count;
            psets_.allocate(kSets * std::size_t(pcount_) * sizeof(Real));
            for (int s = 0; s < kSets; ++s) pset_[s] = psets_.as<Real>() + std::size_t(s) * pcount_;
        }
        surfRate_.allocate(2 * std::size_t(m_.plane) * sizeof(double));
        std::vector<long long> idx(nrec);
        for (int r = 0; r < nrec; ++r) {
            if (rec[r] < 0 || rec[r] >= g.count) throw Error(SWL_ERR_INVALID, "receiver node outside the padded grid");
            idx[r] = pitched(rec[r]);
        }
        recIdx_.allocate(std::max(1, nrec) * sizeof(long long));
        if (nrec) check(cudaMemcpy(recIdx_.ptr, idx.data(), nrec * sizeof(long long), cudaMemcpyHostToDevice), "upload receivers");
        // CTA shape: 256 nodes of one z layer, 32 x 8 unless SWL_3D_BLOCK names another width (16, 64 or 128)
        if (const char *e = std::getenv("SWL_3D_BLOCK")) {
            const int bx = std::atoi(e);
            if (bx == 16 || bx == 32 || bx == 64 || bx == 128) block_ = dim3(bx, 256 / bx, 1);
        }
        grid_ = dim3((g.nx - 6 + block_.x - 1) / block_.x, (g.ny - 6 + block_.y - 1) / block_.y, g.nz - 6);
        statsGrid_ = dim3(grid_.x, grid_.y, (g.nz - 6 + k3::STATS_LAYERS - 1) / k3::STATS_LAYERS);
        nparts_ = statsGrid_.x * statsGrid_.y * statsGrid_.z;
        partials_.allocate(std::size_t(nparts_) * sizeof(k3::Partial));
        clock_.allocate(sizeof(k2::Clock));
        pinnedClock_.reserve(sizeof(k2::Clock));
        check(cudaEventCreateWithFlags(&done_, cudaEventDisableTiming), "create batch event");
        ensureCapacity(8);
        cudaFuncAttributes attr{};
        check(cudaFuncGetAttributes(&attr, k3::stage3d<Real, 0, 0, 0, 1, false>), "3D kernel compatibility");
        registers_ = attr.numRegs;
    }
    ~TypedEngine3D() override {
        if (done_) cudaEventSynchronize(done_), cudaEventDestroy(done_);
        if (stream_) cudaStreamSynchronize(stream_);
        dropGraphs();
        if (ownStream_) cudaStreamDestroy(ownStream_);
    }
    bool faulted() const override { return faulted_; }
    void reserve(int steps) override {
        settle();
        DeviceScope scope(device_);
        if (steps < 0) throw Error(SWL_ERR_INVALID, "reserve needs steps >= 0");
        ensureCapacity(steps);
    }
    void setStream(cudaStream_t s) override {
        settle();
        DeviceScope scope(device_);
        check(cudaStreamSynchronize(stream_), "drain stream");
        stream_ = s ? s : ownStream_;
    }
    void profile(int first, int count, double dt, double frequency, swl_profile &out) override {
        pinnedRows_ = 0, clockStats_ = false;
        settle();
        DeviceScope scope(device_);
        if (count <= 0) throw Error(SWL_ERR_INVALID, "profile needs count > 0");
        if (dt != dt_) dropGraphs(), dt_ = dt;
        ensureCapacity(count);
        hostClock_.step = hostClock_.first = first;
        hostClock_.faulted = 0, hostClock_.fault_step = -1, hostClock_.accepted = 0;
        hostClock_.trace_steps = traceCap_, hostClock_.dt = dt, hostClock_.growth_after = 3 / frequency;
        pushClock();
        fillForcing(first, count, dt, frequency);
        std::vector<cudaEvent_t> ev(7 * std::size_t(count));
        for (auto &e : ev) check(cudaEventCreate(&e), "create event");
        const int u0 = u_;
        for (int j = 0; j < count; ++j) enqueueStep(first + j, true, ev.data() + 7 * j);
        pullClock();
        out = swl_profile{};
        for (int j = 0; j < count; ++j) {
            float ms;
            const cudaEvent_t *e = ev.data() + 7 * j;
            for (int s = 0; s < 4; ++s) check(cudaEventElapsedTime(&ms, e[s], e[s + 1]), "event time"), out.stage_ms[s] += ms / count;
            check(cudaEventElapsedTime(&ms, e[4], e[5]), "event time"), out.stats_ms += ms / count;
            check(cudaEventElapsedTime(&ms, e[5], e[6]), "event time"), out.verdict_ms += ms / count;
            check(cudaEventElapsedTime(&ms, e[0], e[6]), "event time"), out.step_ms += ms / count;
        }
        for (auto &e : ev) cudaEventDestroy(e);
        out.steps = hostClock_.accepted;
        out.launches_per_step = 6;
        out.bytes_per_step = bytesPerStep();
        out.extra_bytes_per_step = extraBytesPerStep();
        const int accepted = hostClock_.accepted;
        u_ = (accepted % 2 == 0) ? u0 : 1 - u0;
        a_ = 1 - u_;
        previous_ = accepted > 0;
        faulted_ = hostClock_.faulted != 0;
    }
    void step(double dt, double frequency, int step) override {
        settle();
        DeviceScope scope(device_);
        dt_ = dt;
        ensureCapacity(1);
        hostClock_.step = hostClock_.first = step;
        hostClock_.faulted = 0;
        hostClock_.accepted = 0;
        hostClock_.trace_steps = traceCap_;
        pushClock();
        fillForcing(step, 1, dt, frequency);
        enqueueStep(step, false);
        previous_ = true;
        pinnedRows_ = 0, clockStats_ = false;
        check(cudaStreamSynchronize(stream_), "3D step completion");
    }
    int advance(int first, int count, double dt, double frequency, double growthAfter) override {
        launch(first, count, dt, frequency, growthAfter);
        return finish();
    }
    void finalize() {
        hostClock_ = *pinnedClock_.as<k2::Clock>();
        const int accepted = hostClock_.accepted;
        u_ = (accepted % 2 == 0) ? batchU0_ : 1 - batchU0_;
        a_ = 1 - u_;
        previous_ = accepted > 0;
        faulted_ = hostClock_.faulted != 0;
        inflight_ = false;
    }
    int finish() override {
        if (!inflight_) return hostClock_.accepted;
        DeviceScope scope(device_);
        check(cudaEventSynchronize(done_), "3D batch completion");
        finalize();
        return hostClock_.accepted;
    }
    bool query(int &accepted) override {
        if (inflight_) {
            DeviceScope scope(device_);
            const cudaError_t e = cudaEventQuery(done_);
            if (e == cudaErrorNotReady) return false;
            check(e, "3D batch query");
            finalize();
        }
        accepted = hostClock_.accepted;
        return true;
    }
    void launch(int first, int count, double dt, double frequency, double growthAfter) override {
        DeviceScope scope(device_);
        if (inflight_) throw Error(SWL_ERR_STATE, "a batch is already in flight on this engine");
        if (count <= 0) {
            hostClock_.accepted = 0;
            return;
        }
        if (dt != dt_) dropGraphs(), dt_ = dt;
        ensureCapacity(count);
        hostClock_.step = hostClock_.first = first;
        hostClock_.faulted = 0;
        hostClock_.fault_step = -1;
        hostClock_.accepted = 0;
        hostClock_.trace_steps = traceCap_;
        hostClock_.dt = dt;
        hostClock_.growth_after = growthAfter;
        pushClock();
        fillForcing(first, count, dt, frequency);
        const int u0 = u_;
        int done = 0;
        while (count - done >= 8) {
            const int key = ((first + done) % 8) * 2 + (u_ == 0 ? 0 : 1);
            auto it = graphs_.find(key);
            if (it == graphs_.end()) {
                cudaGraph_t graph;
                const int su = u_, sa = a_;
                check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin graph capture");
                for (int j = 0; j < 8; ++j) enqueueStep(first + done + j, true);
                check(cudaStreamEndCapture(stream_, &graph), "end graph capture");
                u_ = su, a_ = sa;
                cudaGraphExec_t exec;
                check(cudaGraphInstantiate(&exec, graph, 0), "instantiate step graph");
                cudaGraphDestroy(graph);
                it = graphs_.emplace(key, exec).first;
            }
            check(cudaGraphLaunch(it->second, stream_), "launch step graph");
            done += 8;
        }
        for (; done < count; ++done) enqueueStep(first + done, true);
        // the batch's trace rows and clock come back with it, so that reading them needs no copy
        if (nrec_)
            check(cudaMemcpyAsync(pinnedTraces_.ptr, traces_.ptr, std::size_t(count) * nrec_ * 3 * sizeof(double),
                                  cudaMemcpyDeviceToHost, stream_),
                  "read traces");
        pinnedRows_ = count;
        clockStats_ = true;
        check(cudaMemcpyAsync(pinnedClock_.ptr, clock_.ptr, sizeof(k2::Clock), cudaMemcpyDeviceToHost, stream_), "read clock");
        check(cudaEventRecord(done_, stream_), "record batch completion");
        batchU0_ = u0;
        u_ = u0, a_ = 1 - u0;
        inflight_ = true;
    }
    void rollback() override {
        settle();
        DeviceScope scope(device_);
        check(cudaStreamSynchronize(stream_), "3D rollback");
        if (previous_) std::swap(u_, a_), previous_ = false;
    }
    void reset() override {
        settle();
        DeviceScope scope(device_);
        check(cudaMemsetAsync(sets_.ptr, 0, sets_.bytes, stream_), "3D reset");
        if (psets_.ptr) check(cudaMemsetAsync(psets_.ptr, 0, psets_.bytes, stream_), "3D memory reset");
        if (traces_.ptr) check(cudaMemsetAsync(traces_.ptr, 0, traces_.bytes, stream_), "3D trace reset");
        check(cudaMemsetAsync(surfRate_.ptr, 0, surfRate_.bytes, stream_), "3D surface reset");
        hostClock_ = k2::Clock{};
        pinnedRows_ = 0, clockStats_ = false;
        pushClock();
        check(cudaStreamSynchronize(stream_), "3D clear completion");
        u_ = 0, a_ = 1, previous_ = false, faulted_ = false;
    }
    void diagnostics(swl_diag3d &d) override {
        settle();
        DeviceScope scope(device_);
        k3::stats3d<Real><<<statsGrid_, block_, 0, stream_>>>(m_, set_[u_], surfRate_.as<double>(), nullptr, partials_.as<k3::Partial>());
        check(cudaGetLastError(), "3D diagnostics");
        std::vector<k3::Partial> parts(nparts_);
        check(cudaMemcpyAsync(parts.data(), partials_.ptr, parts.size() * sizeof(k3::Partial), cudaMemcpyDeviceToHost, stream_),
              "3D diagnostics readback");
        check(cudaStreamSynchronize(stream_), "3D diagnostics completion");
        double norm = 0, traction = 0;
        d = swl_diag3d{};
        d.finite = 1;
        for (const auto &p : parts) {
            d.energy += p.energy;
            d.max_velocity = std::max(d.max_velocity, p.velocity);
            for (int c = 0; c < 5; ++c) d.peaks[c] = std::max(d.peaks[c], p.peak[c]);
            norm = std::max(norm, p.rateNorm);
            traction = std::max(traction, p.rateTraction);
            d.finite &= !p.bad;
        }
        d.traction_rate_relative = traction / std::max(norm, 1e-30);
        d.peak_energy = hostClock_.peak_energy;
        d.rhs_registers = registers_;
        d.resident_bytes = residentBytes();
    }
    void stepDiagnostics(swl_diag3d &d) override {
        settle();
        if (!clockStats_) return diagnostics(d);
        d.energy = hostClock_.energy, d.max_velocity = hostClock_.max_velocity;
        d.traction_rate_relative = hostClock_.traction;
        for (int c = 0; c < 5; ++c) d.peaks[c] = hostClock_.peaks[c];
        d.finite = hostClock_.finite;
        d.peak_energy = hostClock_.peak_energy;
        d.rhs_registers = registers_;
        d.resident_bytes = residentBytes();
    }
    void sample(double *vx, double *vy, double *vz) override {
        settle();
        DeviceScope scope(device_);
        if (!nrec_) return;
        std::vector<long long> idx(nrec_);
        check(cudaMemcpy(idx.data(), recIdx_.ptr, nrec_ * sizeof(long long), cudaMemcpyDeviceToHost), "receiver index readback");
        DeviceBuffer out(std::size_t(nrec_) * 3 * sizeof(double));
        k2::gather2d<Real><<<(nrec_ + 127) / 128, 128, 0, stream_>>>(set_[u_], count_, recIdx_.as<long long>(), nrec_, 3,
                                                                     out.as<double>());
        check(cudaGetLastError(), "3D receiver launch");
        std::vector<double> v(std::size_t(nrec_) * 3);
        check(cudaMemcpyAsync(v.data(), out.ptr, v.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_), "3D receiver readback");
        check(cudaStreamSynchronize(stream_), "3D receiver completion");
        for (int r = 0; r < nrec_; ++r) vx[r] = v[3 * r], vy[r] = v[3 * r + 1], vz[r] = v[3 * r + 2];
    }
    void traces(int first, int count, double *vx, double *vy, double *vz) override {
        settle();
        DeviceScope scope(device_);
        const int row0 = first - hostClock_.first;
        if (count < 0 || row0 < 0 || row0 + count > hostClock_.accepted)
            throw Error(SWL_ERR_INVALID, "requested trace rows were not recorded by the last advance");
        std::vector<double> copy;
        const double *buf = pinnedTraces_.as<double>() + std::size_t(row0) * nrec_ * 3;
        if (row0 + count > pinnedRows_) { // rows recorded outside an asynchronous batch
            copy.resize(std::size_t(count) * nrec_ * 3);
            if (!copy.empty())
                check(cudaMemcpy(copy.data(), traces_.as<double>() + std::size_t(row0) * nrec_ * 3, copy.size() * sizeof(double),
                                 cudaMemcpyDeviceToHost),
                      "trace readback");
            buf = copy.data();
        }
        for (int r = 0; r < nrec_; ++r)
            for (int j = 0; j < count; ++j) {
                const std::size_t at = (std::size_t(j) * nrec_ + r) * 3, to = std::size_t(r) * count + j;
                vx[to] = buf[at], vy[to] = buf[at + 1], vz[to] = buf[at + 2];
            }
    }
    void snapshot(int field, double *out) override {
        settle();
        DeviceScope scope(device_);
        if (field == -1 && pcount_) { // the CFS-PML memories
            check(cudaStreamSynchronize(stream_), "snapshot ordering");
            std::vector<Real> tmp(pcount_);
            check(cudaMemcpy(tmp.data(), pset_[u_], pcount_ * sizeof(Real), cudaMemcpyDeviceToHost), "memory download");
            for (long long q = 0; q < pcount_; ++q) out[q] = double(tmp[q]);
            return;
        }
        if (field < 0 || field >= fc_) throw Error(SWL_ERR_INVALID, "snapshot field out of range");
        check(cudaStreamSynchronize(stream_), "snapshot ordering");
        std::vector<Real> tmp(count_);
        check(cudaMemcpy(tmp.data(), set_[u_] + std::size_t(field) * count_, count_ * sizeof(Real), cudaMemcpyDeviceToHost),
              "snapshot download");
        const long long rows = (long long)m_.ny * m_.nz;
        for (long long r = 0; r < rows; ++r)
            for (int i = 0; i < m_.nx; ++i) out[i + m_.nx * r] = double(tmp[i + m_.px * r]);
    }
    void load(int field, const double *in) override {
        settle();
        DeviceScope scope(device_);
        if (field == -1 && pcount_) {
            clockStats_ = false;
            check(cudaStreamSynchronize(stream_), "load ordering");
            std::vector<Real> tmp(pcount_);
            for (long long q = 0; q < pcount_; ++q) tmp[q] = static_cast<Real>(in[q]);
            check(cudaMemcpy(pset_[u_], tmp.data(), pcount_ * sizeof(Real), cudaMemcpyHostToDevice), "memory upload");
            if (k2::kahan<Real>()) check(cudaMemset(pset_[4 + u_], 0, pcount_ * sizeof(Real)), "clear compensation");
            previous_ = false;
            return;
        }
        if (field < 0 || field >= fc_) throw Error(SWL_ERR_INVALID, "load field out of range");
        clockStats_ = false;
        check(cudaStreamSynchronize(stream_), "load ordering");
        std::vector<Real> tmp(count_, Real(0));
        const long long rows = (long long)m_.ny * m_.nz;
        for (long long r = 0; r < rows; ++r)
            for (int i = 0; i < m_.nx; ++i) tmp[i + m_.px * r] = static_cast<Real>(in[i + m_.nx * r]);
        check(cudaMemcpy(set_[u_] + std::size_t(field) * count_, tmp.data(), count_ * sizeof(Real), cudaMemcpyHostToDevice),
              "field upload");
        if (k2::kahan<Real>()) // a loaded value starts without a compensation term
            check(cudaMemset(set_[4 + u_] + std::size_t(field) * count_, 0, count_ * sizeof(Real)), "clear compensation");
        previous_ = false;
    }
    int64_t residentBytes() const override {
        int64_t b = 0;
        for (const auto &x : model_) b += x.bytes;
        for (const auto *x : {&sets_, &psets_, &recIdx_, &traces_, &forcing_, &clock_, &partials_, &surfRate_}) b += x->bytes;
        return b;
    }
};

} // namespace swl
