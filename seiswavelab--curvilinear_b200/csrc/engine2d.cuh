// Host side of the 2D engine (the B200 replacement of src/two_d/CudaEngine2D.cu:107-184).
//
// State layout in HBM: four structure-of-arrays sets of field_count*count values -- two
// alternating "state / accumulator" sets and two stage sets -- plus the same four sets of
// compact CFS-PML memories.  A step reads the state set and leaves the new state in the
// accumulator set; the sets then swap roles, so the state at the start of the last step stays
// resident and rollback is a role swap (no per-step D2D copy).
//
// A batch of steps (swl2d_advance) is recorded once per (step phase mod 8, role parity) into a
// CUDA graph of eight steps; each step is 4 fused stage kernels + a diagnostics reduction +
// a one-block verdict that applies the reference's acceptance rule on the device, records the
// receivers and advances a device-resident step clock.  The host synchronises once per batch.
#pragma once
#include "../../include/swl_b200.h"
#include "runtime.cuh"
#include "launch2d.cuh"
#include "launchq2d.cuh"
#include "stage2d.cuh"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <cstddef>
#include <tuple>
#include <vector>

namespace swl {

class Engine2D {
  public:
    virtual ~Engine2D() = default;
    virtual void step(double dt, double frequency, double scale, int step) = 0;
    virtual int advance(int first, int count, double dt, double frequency, double scale, double growthAfter) = 0;
    virtual void rollback() = 0;
    virtual void reset() = 0;
    virtual void diagnostics(swl_diag2d &) = 0;
    // Diagnostics of the last accepted step as the device verdict recorded them (read back with
    // the batch): no kernel and no synchronisation.  Before any step, the same as diagnostics().
    virtual void stepDiagnostics(swl_diag2d &) = 0;
    virtual void sample(double *vx, double *vz) = 0;
    virtual void traces(int first, int count, double *vx, double *vz) = 0;
    virtual void snapshot(int field, double *out) = 0;
    virtual void load(int field, const double *in) = 0;
    virtual void probes(const int64_t *nodes, int n, double *out5) = 0;
    virtual int64_t residentBytes() const = 0;
    virtual bool faulted() const = 0;
    virtual void profile(int first, int count, double dt, double frequency, double scale, swl_profile &out) = 0;
    virtual void setStream(cudaStream_t stream) = 0;
    // Preallocate the forcing and trace tables for batches of up to `steps` steps, so that such
    // batches record no new CUDA graphs.
    virtual void reserve(int steps) = 0;
    // Asynchronous batches: launch returns once the batch is enqueued; query polls and finish
    // waits; both return the accepted step count of the batch.
    virtual void launch(int first, int count, double dt, double frequency, double scale, double growthAfter) = 0;
    virtual bool query(int &accepted) = 0;
    virtual int finish() = 0;
    // How the stage kernels decompose the grid, and how many CTAs take each compiled form.
    virtual void layout(swl_layout2d &) const = 0;
};

std::unique_ptr<Engine2D> makeEngine2D64(const swl_mesh2d &, const int64_t *, int, int);
std::unique_ptr<Engine2D> makeEngine2D32(const swl_mesh2d &, const int64_t *, int, int);

// Persistent multi-shot launches (queue2d.cuh): the batches of several engines of one precision
// and one GSLS mechanism count advance together in one launch on the queue's stream.  After the
// launch each engine's batch completes like one of its own (query / finish).
class Queue2D {
  public:
    virtual ~Queue2D() = default;
    virtual void launch(Engine2D *const *engines, int n, const int *first, const int *count, const double *dt,
                        const double *frequency, const double *scale, const double *growthAfter) = 0;
    virtual bool query() = 0; // true once the launch completed; throws if a wait in it ran out
    virtual void finish() = 0;
    virtual int blocks() const = 0; // CTAs of the last launch
    // Resident CTAs per SM a launch may use: 0 all that fit; n > 0 at most n; n < 0 all but -n
    // (at least one), leaving room for other shots' kernels beside the persistent launch.
    virtual void limit(int ctasPerSm) = 0;
    // Row blocks per work item (1, 2, 4 or 8), or 0: chosen per grid (queueSegment).
    virtual void segment(int seg) = 0;
};
std::unique_ptr<Queue2D> makeQueue2D64(int device);
std::unique_ptr<Queue2D> makeQueue2D32(int device);

namespace detail2 {

// Dispatch on the GSLS mechanism count to the separately compiled stage instantiations.
template <class Real> struct Launch {
    static void stage(int dx, int dz, int mech, int stage, dim3 g, dim3 b, cudaStream_t s, const k2::StageArgs<Real> &a) {
        switch (mech) {
        case 0: launchStage2D<Real, 0>(dx, dz, stage, g, b, s, a); break;
        case 1: launchStage2D<Real, 1>(dx, dz, stage, g, b, s, a); break;
        case 2: launchStage2D<Real, 2>(dx, dz, stage, g, b, s, a); break;
        default: launchStage2D<Real, 3>(dx, dz, stage, g, b, s, a); break;
        }
    }
    static void prepare(int mech) {
        switch (mech) {
        case 0: prepareStages2D<Real, 0>(); break;
        case 1: prepareStages2D<Real, 1>(); break;
        case 2: prepareStages2D<Real, 2>(); break;
        default: prepareStages2D<Real, 3>(); break;
        }
    }
    static cudaFuncAttributes attributes(int mech) {
        switch (mech) {
        case 0: return stageAttributes2D<Real, 0>();
        case 1: return stageAttributes2D<Real, 1>();
        case 2: return stageAttributes2D<Real, 2>();
        default: return stageAttributes2D<Real, 3>();
        }
    }
};

template <class Real> std::vector<Real> convert(const void *src, std::size_t n, int arrayPrecision, const char *name) {
    std::vector<Real> out(n);
    if (!src) throw Error(SWL_ERR_INVALID, std::string("mesh array ") + name + " is null");
    if (arrayPrecision == SWL_FP32) {
        const float *s = static_cast<const float *>(src);
        for (std::size_t i = 0; i < n; ++i) out[i] = static_cast<Real>(s[i]);
    } else {
        const double *s = static_cast<const double *>(src);
        for (std::size_t i = 0; i < n; ++i) out[i] = static_cast<Real>(s[i]);
    }
    for (std::size_t i = 0; i < n; ++i)
        if (!std::isfinite(static_cast<double>(out[i])))
            throw Error(SWL_ERR_INVALID, std::string("mesh array ") + name +
                                             " is not finite in the engine precision; select FP64 or revise the model");
    return out;
}

} // namespace detail2

template <class Real> class TypedEngine2D final : public Engine2D {
    int device_{};
    cudaStream_t stream_{}, ownStream_{};
    k2::Mesh<Real> m_{};
    int mech_{}, fc_{};
    bool segmentRule_{false}; // choose the segment by occupancy instead of timing
    long long count_{}, pcount_{};
    bool cpml_{};
    std::vector<DeviceBuffer> model_;
    DeviceBuffer pack_; // a, b, lambda, mu, rho, J: six consecutive pitched arrays (one tensor map)
    DeviceBuffer sets_, psets_, recIdx_, traces_, forcing_, clock_, partials_;
    int pitch_{}, nx_{}, nz_{};
    // tensor maps of the streaming kernel: stage-input ring boxes of sets 0-3, word boxes of the
    // state / accumulator sets 0-1 and of their compensation sets 4-5, model words without / with J
    CUtensorMap ringMap_[4]{}, pwMap_[2]{}, compMap_[2]{}, modelMap_[2]{};
    CUtensorMap gslsIn_[4]{}, gslsComp_[2]{}, strengthMap_{}; // GSLS L2 prefetch boxes (per set)
    int gslsLead_{2}; // GSLS prefetch lead in row blocks (SWL_GSLS_PREFETCH overrides: 0 off, 1, 2, 3)
    DeviceBuffer strengths_;
    // Sets 0-1: state / accumulator (roles u_, a_); 2-3: stage states; FP32 only, 4-5: the Kahan
    // compensation of sets 0-1 (set 4 + r compensates set r, so a role swap moves both).
    static constexpr int kSets = k2::kahan<Real>() ? 6 : 4;
    Real *set_[6]{}, *pset_[6]{};
    int u_{0}, a_{1};       // state / accumulator roles among set 0 and 1
    bool previous_{false};  // set a_ holds the state before the last step
    int nrec_{}, traceCap_{}, forcingCap_{};
    dim3 grid_, block_{32, 8};                               // one node per thread (diagnostics kernel)
    dim3 stageGrid_, stageBlock_{32, 8}; // strips of 32 columns x segments of 8*seg rows
    int nparts_{};
    k2::Clock hostClock_{};
    PinnedBuffer pinnedForcing_, pinnedClock_, pinnedTraces_;
    int pinnedRows_{0};     // trace rows of the last launched batch copied to pinnedTraces_ with it
    bool clockStats_{false}; // the host clock holds a verdict's diagnostics
    std::map<int, cudaGraphExec_t> graphs_;
    bool faulted_{false};
    int registers_{};
    int64_t localBytes_{};
    cudaEvent_t done_{};    // completion of the in-flight batch
    cudaEvent_t queued_{};  // the uploads of a queued batch (Queue2D)
    bool inflight_{false};
    int batchU0_{0};
    void settle() {
        if (inflight_) finish();
    }

    // Memory offset of padded node q = i + nx k of the caller's layout.
    long long memIndex(long long q) const { return q % nx_ + 1 + (long long)pitch_ * (q / nx_); }
    // The caller's nx x nz layout (`per` values per node) in the pitched layout.
    std::vector<Real> pitched(const std::vector<Real> &v, int per) const {
        std::vector<Real> out(std::size_t(count_) * per, Real(0));
        for (int k = 0; k < nz_; ++k)
            std::copy(v.begin() + std::size_t(k) * nx_ * per, v.begin() + std::size_t(k + 1) * nx_ * per,
                      out.begin() + (std::size_t(k) * pitch_ + 1) * per);
        return out;
    }
    Real *upload(const std::vector<Real> &v) {
        model_.emplace_back(v.size() * sizeof(Real));
        check(cudaMemcpy(model_.back().ptr, v.data(), v.size() * sizeof(Real), cudaMemcpyHostToDevice), "upload model");
        return model_.back().template as<Real>();
    }
    void dropGraphs() {
        for (auto &g : graphs_) cudaGraphExecDestroy(g.second);
        graphs_.clear();
    }
    k2::StageArgs<Real> args(int stage) const {
        k2::StageArgs<Real> p{};
        p.m = m_;
        Real *U = set_[u_], *A = set_[a_], *S1 = set_[2], *S2 = set_[3];
        Real *PU = pset_[u_], *PA = pset_[a_], *PS1 = pset_[2], *PS2 = pset_[3];
        p.base = U;
        p.acc = A;
        p.pbase = PU;
        p.pacc = PA;
        switch (stage) {
        case 0: p.in = U, p.out = S1, p.pin = PU, p.pout = PS1; break;
        case 1: p.in = S1, p.out = S2, p.pin = PS1, p.pout = PS2; break;
        case 2: p.in = S2, p.out = S1, p.pin = PS2, p.pout = PS1; break;
        default: p.in = S1, p.out = nullptr, p.pin = PS1, p.pout = nullptr; break;
        }
        p.forcing = forcing_.as<Real>();
        p.clock = clock_.as<k2::Clock>();
        p.weight = stage == 2 ? static_cast<Real>(dt_) : static_cast<Real>(dt_ / 2);
        p.delta = static_cast<Real>(dt_);
        p.partials = nullptr;
        if (k2::kahan<Real>()) p.cin = set_[4 + u_], p.cout = set_[4 + a_], p.pcin = pset_[4 + u_], p.pcout = pset_[4 + a_];
        {
            const int in = stage == 0 ? u_ : stage == 2 ? 3 : 2;
            p.ringMap = ringMap_[in];
            p.uMap = pwMap_[u_];
            p.aMap = pwMap_[a_];
            p.modelMap = modelMap_[stage == 3 ? 1 : 0];
            p.compMap = compMap_[u_];
            if (mech_) {
                p.gslsInMap = gslsIn_[in];
                p.gslsUMap = gslsIn_[u_];
                p.gslsAMap = gslsIn_[a_];
                p.gslsCompMap = gslsComp_[u_];
                p.strengthMap = strengthMap_;
                p.gslsPrefetch = gslsLead_;
            }
        }
        return p;
    }
    double dt_{};
    // Enqueue one step: 4 stages (+ diagnostics and verdict when `verdict`).  Swaps roles.
    // `ev`, when given, receives 7 events: before stage 0, after each stage, after stats, after verdict.
    void enqueueStep(int step, bool verdict, cudaEvent_t *ev = nullptr) {
        if (ev) check(cudaEventRecord(ev[0], stream_), "record event");
        for (int s = 0; s < 4; ++s) {
            auto a = args(s);
            if (s == 3 && verdict) a.partials = partials_.as<k2::Partial>(); // diagnostics fused into stage 3
            detail2::Launch<Real>::stage(direction(step, s, 0), direction(step, s, 2), mech_, s, stageGrid_, stageBlock_, stream_, a);
            if (ev) check(cudaEventRecord(ev[1 + s], stream_), "record event");
        }
        check(cudaGetLastError(), "2D stage launch");
        if (verdict) {
            Real *fresh = set_[a_];
            if (ev) check(cudaEventRecord(ev[5], stream_), "record event");
            k2::verdict2d<Real><<<1, 1024, 0, stream_>>>(partials_.as<k2::Partial>(), int(stageGrid_.x * stageGrid_.y), fresh, count_,
                                                         recIdx_.as<long long>(), nrec_, traces_.as<double>(), clock_.as<k2::Clock>(), 1);
            if (ev) check(cudaEventRecord(ev[6], stream_), "record event");
            check(cudaGetLastError(), "2D verdict launch");
        }
        std::swap(u_, a_);
    }
    // Algorithmic HBM bytes of the four stage kernels of one step: 17 F + 4 M per physical
    // node (stage reads/writes of U, A, S and the per-node model arrays a, b, rho, lambda, mu
    // and the GSLS strengths) plus 17 values per CFS-PML memory.
    // Algorithmic HBM bytes of one step: 17 F + 4 M per physical node (stage 0 reads U and writes
    // S and A: 3F; stages 1-2 read S, U, A and write S, A: 5F each; stage 3 reads S, U, A and writes
    // the new state: 4F; every stage reads the model words M), plus 17 words per ADE memory.
    double bytesPerStep() const {
        const double s = sizeof(Real), points = double(m_.nx - 6) * (m_.nz - 6);
        const double F = fc_ * s, M = (5 + 2 * mech_) * s;
        return points * (17 * F + 4 * M) + double(pcount_) * 17 * s;
    }
    // FP32 only: the compensation terms read and written by stage 3 (2 F, and 2 words per memory).
    double extraBytesPerStep() const {
        if (!k2::kahan<Real>()) return 0;
        const double s = sizeof(Real), points = double(m_.nx - 6) * (m_.nz - 6);
        return points * 2 * fc_ * s + double(pcount_) * 2 * s;
    }
    void ensureCapacity(int steps) {
        if (steps > forcingCap_) {
            forcing_.allocate(std::size_t(steps) * 3 * sizeof(Real));
            forcingCap_ = steps;
            dropGraphs();
        }
        if (steps > traceCap_) {
            traces_.allocate(std::max<std::size_t>(1, std::size_t(steps) * nrec_ * 2) * sizeof(double));
            traceCap_ = steps;
            dropGraphs();
        }
        pinnedForcing_.reserve(std::size_t(steps) * 3 * sizeof(Real));
        pinnedTraces_.reserve(std::max<std::size_t>(1, std::size_t(traceCap_) * nrec_ * 2) * sizeof(double));
    }
    void fillForcing(int first, int count, double dt, double frequency, double scale) {
        Real *f = pinnedForcing_.as<Real>();
        for (int j = 0; j < count; ++j) {
            const int s = first + j;
            // src/two_d/CurvilinearSolver2D.cpp:73,268-274: Real(amplitude/h^2 * ricker(t))
            f[3 * j] = static_cast<Real>(scale * ricker(s * dt, frequency));
            f[3 * j + 1] = static_cast<Real>(scale * ricker((s + .5) * dt, frequency));
            f[3 * j + 2] = static_cast<Real>(scale * ricker((s + 1) * dt, frequency));
        }
        check(cudaMemcpyAsync(forcing_.ptr, f, std::size_t(count) * 3 * sizeof(Real), cudaMemcpyHostToDevice, stream_),
              "upload forcing");
    }
    void pushClock() {
        *pinnedClock_.as<k2::Clock>() = hostClock_;
        check(cudaMemcpyAsync(clock_.ptr, pinnedClock_.ptr, sizeof(k2::Clock), cudaMemcpyHostToDevice, stream_), "set clock");
    }
    void pullClock() {
        check(cudaMemcpyAsync(pinnedClock_.ptr, clock_.ptr, sizeof(k2::Clock), cudaMemcpyDeviceToHost, stream_), "read clock");
        check(cudaStreamSynchronize(stream_), "2D batch completion");
        hostClock_ = *pinnedClock_.as<k2::Clock>();
        checkStalled();
    }
    // A stage kernel whose bounded copy wait ran out flags the clock; report it as a CUDA error.
    void checkStalled() {
        if (!hostClock_.stalled) return;
        hostClock_.stalled = 0;
        throw Error(SWL_ERR_CUDA, "CUDA 2D stage: a tensor-copy wait ran out");
    }

  public:
    TypedEngine2D(const swl_mesh2d &g, const int64_t *rec, int nrec, int device) : device_(device) {
        DeviceScope scope(device_);
        if (g.nx < 14 || g.nz < 14 || g.count != int64_t(g.nx) * g.nz)
            throw Error(SWL_ERR_INVALID, "2D mesh needs nx, nz >= 14 padded nodes and count = nx*nz");
        if (g.mechanisms < 0 || g.mechanisms > 3 || g.field_count != (g.mechanisms ? 6 + 4 * g.mechanisms : 5))
            throw Error(SWL_ERR_INVALID, "2D mesh field_count must be 5 (elastic) or 6 + 4*mechanisms (GSLS)");
        if (nrec < 0 || (nrec && !rec)) throw Error(SWL_ERR_INVALID, "receiver list is invalid");
        check(cudaStreamCreateWithFlags(&ownStream_, cudaStreamNonBlocking), "create stream");
        stream_ = ownStream_;
        nx_ = g.nx, nz_ = g.nz;
        pitch_ = (g.nx + 1 + 7) / 8 * 8;
        count_ = (long long)pitch_ * g.nz;
        const std::size_t n = std::size_t(count_), nu = std::size_t(g.count); // device and caller node counts
        mech_ = g.mechanisms;
        segmentRule_ = g.segment_rule != 0;
        fc_ = g.field_count;
        nrec_ = nrec;
        const int ap = g.array_precision;
        auto arr = [&](const void *src, std::size_t len, const char *name) { // non-node arrays
            return upload(detail2::convert<Real>(src, len, ap, name));
        };
        auto node = [&](const void *src, int per, const char *name) { // per-node arrays, pitched
            return upload(pitched(detail2::convert<Real>(src, nu * per, ap, name), per));
        };
        m_.nx = g.nx;
        m_.nz = g.nz;
        m_.pitch = pitch_;
        m_.xoff = 1;
        m_.count = count_;
        m_.h = static_cast<Real>(g.h);
        {
            // x/h equals x*(1/h) bit for bit when h is a power of two; the FP32 form always
            // multiplies by the reciprocal.
            int e2 = 0;
            const bool pow2 = g.h > 0 && std::frexp(g.h, &e2) == 0.5;
            if (!(g.h >= 0x1p-20 && g.h <= 0x1p+20)) throw Error(SWL_ERR_INVALID, "2D grid spacing must lie in [2^-20, 2^20]");
            m_.hinv = static_cast<Real>(1.0 / g.h);
            m_.hinvExact = (pow2 || sizeof(Real) == 4) ? 1 : 0;
        }
        {
            // divBy's correctly rounded quotient needs a divisor in [2^-20, 2^20] (the densities of
            // the computational nodes; ghost nodes are never divisors)
            const auto rho = detail2::convert<Real>(g.rho, nu, ap, "rho");
            bool ok = true;
            for (int k = 3; ok && k < g.nz - 3; ++k)
                for (int i = 3; i < g.nx - 3; ++i) {
                    const Real r = rho[i + std::size_t(g.nx) * k];
                    if (!(r >= Real(0x1p-20) && r <= Real(0x1p+20))) {
                        ok = false;
                        break;
                    }
                }
            m_.rhoRecip = ok ? 1 : 0;
        }
        {
            pack_.allocate(6 * n * sizeof(Real));
            const void *src[6] = {g.a, g.b, g.lambda, g.mu, g.rho, g.jac};
            const char *names[6] = {"a", "b", "lambda", "mu", "rho", "jac"};
            Real *dst[6];
            for (int w = 0; w < 6; ++w) {
                dst[w] = pack_.as<Real>() + w * n;
                const auto v = pitched(detail2::convert<Real>(src[w], nu, ap, names[w]), 1);
                check(cudaMemcpy(dst[w], v.data(), n * sizeof(Real), cudaMemcpyHostToDevice), "upload model");
            }
            m_.a = dst[0], m_.b = dst[1], m_.lambda = dst[2], m_.mu = dst[3], m_.rho = dst[4], m_.jac = dst[5];
        }
        m_.normals = node(g.normals, 2, "normals");
        const auto damping = detail2::convert<Real>(g.damping, nu, ap, "damping");
        m_.damping = upload(pitched(damping, 1));
        const auto source = detail2::convert<Real>(g.source, nu, ap, "source");
        m_.source = upload(pitched(source, 1));
        std::vector<Real> sg[2];
        if (g.source_gradient[0] || g.source_gradient[1]) {
            sg[0] = detail2::convert<Real>(g.source_gradient[0], nu, ap, "source_gradient[0]");
            sg[1] = detail2::convert<Real>(g.source_gradient[1], nu, ap, "source_gradient[1]");
            m_.sgx = upload(pitched(sg[0], 1));
            m_.sgz = upload(pitched(sg[1], 1));
        }
        m_.sdx = static_cast<Real>(g.source_direction[0]);
        m_.sdz = static_cast<Real>(g.source_direction[2]);
        // Box of the source support (the force is exactly zero outside).
        int i0 = g.nx, i1 = 0, k0 = g.nz, k1 = 0;
        for (int k = 0; k < g.nz; ++k)
            for (int i = 0; i < g.nx; ++i) {
                const std::size_t q = i + std::size_t(g.nx) * k;
                const bool nz = m_.sgx ? (sg[0][q] != Real(0) || sg[1][q] != Real(0)) : source[q] != Real(0);
                if (nz) i0 = std::min(i0, i), i1 = std::max(i1, i + 1), k0 = std::min(k0, k), k1 = std::max(k1, k + 1);
            }
        m_.src_i0 = i0, m_.src_i1 = i1, m_.src_k0 = k0, m_.src_k1 = k1;
        // Box [i0,i1) x [0,k1) in which the sponge rate is exactly zero (verified).
        {
            auto D = [&](int i, int k) { return damping[i + std::size_t(g.nx) * k]; };
            int a0 = 3, a1 = g.nx - 3;
            while (a0 < a1 && D(a0, 3) != Real(0)) ++a0;
            while (a1 > a0 && D(a1 - 1, 3) != Real(0)) --a1;
            int kk = 3;
            const int mid = (a0 + a1) / 2;
            if (a0 < a1)
                while (kk < g.nz - 3 && D(mid, kk) == Real(0)) ++kk;
            bool ok = a0 < a1;
            for (int k = 0; ok && k < kk; ++k)
                for (int i = a0; i < a1; ++i)
                    if (D(i, k) != Real(0)) {
                        ok = false;
                        break;
                    }
            if (ok) m_.dmp_i0 = a0, m_.dmp_i1 = a1, m_.dmp_k1 = (kk >= g.nz - 3 ? g.nz : kk);
            else m_.dmp_i0 = m_.dmp_i1 = m_.dmp_k1 = 0;
        }
        cpml_ = g.cpml_count > 0;
        pcount_ = g.cpml_count;
        if (cpml_) {
            if (g.cpml_width_x < 0 || g.cpml_width_z < 1 ||
                g.cpml_count != 4 * (2 * int64_t(g.cpml_width_x) * (g.nz - 6) + int64_t(g.cpml_width_z) * (g.nx - 6)))
                throw Error(SWL_ERR_INVALID, "CFS-PML count must be 4*(2*wx*(nz-6) + wz*(nx-6))");
            m_.cpx = arr(g.cpml_x, 3 * std::size_t(g.nx - 6), "cpml_x");
            m_.cpz = arr(g.cpml_z, 3 * std::size_t(g.nz - 6), "cpml_z");
            m_.wx = g.cpml_width_x;
            m_.wz = g.cpml_width_z;
        }
        // GSLS relaxation strengths: one allocation of 2L pitched arrays (dP0, dS0, dP1, ...), so one
        // tensor box covers a row block's strengths
        if (mech_) strengths_.allocate(2 * std::size_t(mech_) * n * sizeof(Real));
        if (const char *e = std::getenv("SWL_GSLS_PREFETCH")) gslsLead_ = std::clamp(std::atoi(e), 0, 3);
        for (int l = 0; l < mech_; ++l) {
            m_.rates[l] = static_cast<Real>(g.rates[l]);
            Real *dp = strengths_.as<Real>() + std::size_t(2 * l) * n, *ds = dp + n;
            const auto vp = pitched(detail2::convert<Real>(g.delta_p[l], nu, ap, "delta_p"), 1);
            const auto vs = pitched(detail2::convert<Real>(g.delta_s[l], nu, ap, "delta_s"), 1);
            check(cudaMemcpy(dp, vp.data(), n * sizeof(Real), cudaMemcpyHostToDevice), "upload model");
            check(cudaMemcpy(ds, vs.data(), n * sizeof(Real), cudaMemcpyHostToDevice), "upload model");
            m_.dP[l] = dp;
            m_.dS[l] = ds;
        }
        m_.fc = fc_;
        sets_.allocate(kSets * std::size_t(fc_) * n * sizeof(Real));
        for (int s = 0; s < kSets; ++s) set_[s] = sets_.as<Real>() + std::size_t(s) * fc_ * n;
        psets_.allocate(kSets * std::size_t(std::max<long long>(pcount_, 1)) * sizeof(Real));
        for (int s = 0; s < kSets; ++s) pset_[s] = psets_.as<Real>() + std::size_t(s) * std::max<long long>(pcount_, 1);
        std::vector<long long> idx(nrec);
        for (int r = 0; r < nrec; ++r) {
            if (rec[r] < 0 || rec[r] >= g.count) throw Error(SWL_ERR_INVALID, "receiver node outside the padded grid");
            idx[r] = memIndex(rec[r]);
        }
        recIdx_.allocate(std::max(1, nrec) * sizeof(long long));
        if (nrec) check(cudaMemcpy(recIdx_.ptr, idx.data(), nrec * sizeof(long long), cudaMemcpyHostToDevice), "upload receivers");
        grid_ = dim3((g.nx - 6 + block_.x - 1) / block_.x, (g.nz - 6 + block_.y - 1) / block_.y);
        setSegment(k2::MAX_SEG);
        nparts_ = grid_.x * grid_.y;
        const std::size_t most = std::size_t(stageGrid_.x) * ((g.nz - 6 + k2::SB - 1) / k2::SB); // one-block segments
        partials_.allocate(std::max<std::size_t>(nparts_, most) * sizeof(k2::Partial));
        detail2::Launch<Real>::prepare(mech_);
        {
            const bool f64 = sizeof(Real) == 8;
            const uint64_t d5[3] = {uint64_t(pitch_), uint64_t(nz_), 5}, d6[3] = {uint64_t(pitch_), uint64_t(nz_), 6};
            const uint64_t st[2] = {uint64_t(pitch_) * sizeof(Real), uint64_t(n) * sizeof(Real)};
            const uint32_t ring[3] = {k2::RC, k2::SB, 5}, w5[3] = {k2::SW, k2::SB, 5}, w6[3] = {k2::SW, k2::SB, 6};
            for (int s = 0; s < 4; ++s) encodeTensorMap3D(&ringMap_[s], f64, set_[s], d5, st, ring);
            for (int r = 0; r < 2; ++r) encodeTensorMap3D(&pwMap_[r], f64, set_[r], d5, st, w5);
            if (k2::kahan<Real>())
                for (int r = 0; r < 2; ++r) encodeTensorMap3D(&compMap_[r], f64, set_[4 + r], d5, st, w5);
            encodeTensorMap3D(&modelMap_[0], f64, pack_.ptr, d6, st, w5);
            encodeTensorMap3D(&modelMap_[1], f64, pack_.ptr, d6, st, w6);
            if (mech_) { // L2 prefetch boxes of the GSLS words (fields 5 .. 5+4L) and the strengths
                const uint32_t gm = uint32_t(4 * mech_ + 1), gs = uint32_t(2 * mech_);
                const uint64_t dg[3] = {uint64_t(pitch_), uint64_t(nz_), gm}, dst2[3] = {uint64_t(pitch_), uint64_t(nz_), gs};
                const uint32_t bg[3] = {k2::SW, k2::SB, gm}, bs[3] = {k2::SW, k2::SB, gs};
                for (int t = 0; t < 4; ++t) encodeTensorMap3D(&gslsIn_[t], f64, set_[t] + 5 * n, dg, st, bg);
                if (k2::kahan<Real>())
                    for (int r = 0; r < 2; ++r) encodeTensorMap3D(&gslsComp_[r], f64, set_[4 + r] + 5 * n, dg, st, bg);
                encodeTensorMap3D(&strengthMap_, f64, strengths_.ptr, dst2, st, bs);
            }
        }
        clock_.allocate(sizeof(k2::Clock));
        pinnedClock_.reserve(sizeof(k2::Clock));
        check(cudaEventCreateWithFlags(&done_, cudaEventDisableTiming), "create batch event");
        ensureCapacity(8);
        const cudaFuncAttributes attr = detail2::Launch<Real>::attributes(mech_);
        registers_ = attr.numRegs;
        localBytes_ = attr.localSizeBytes;
        tune();
    }
    // Streaming segment length: `seg` row blocks of 8 rows per CTA.
    void setSegment(int seg) {
        m_.seg = seg;
        stageGrid_ = dim3((nx_ - 6 + k2::SW - 1) / k2::SW, (nz_ - 6 + k2::SB * seg - 1) / (k2::SB * seg));
        dropGraphs(); // the graphs hold the launch shape
    }
    // The segment length for this grid.  By default it is picked by timing an 8-step graph per
    // candidate on the fresh (zero, unforced) state: long segments stream more rows per CTA and
    // re-read fewer halo rows; short ones put more CTAs in flight and shorten each CTA's chain of
    // row blocks, which is what a small grid needs.  The state and the clock are reset afterwards.
    // With segment_rule set it follows an occupancy rule instead (see below).  The choice is kept
    // per grid shape for the life of the process, so that identical shots always run the same
    // decomposition (FP32 rounding differs slightly between the interior and the boundary forms
    // of a node, which the decomposition decides).
    void tune() {
        static std::mutex mutex;
        static std::map<std::tuple<int, int, int, int, int, int, int, bool>, int> chosen;
        const auto key = std::make_tuple(device_, nx_, nz_, mech_, m_.wx, m_.wz, m_.dmp_k1, segmentRule_);
        {
            std::lock_guard<std::mutex> g(mutex);
            const auto it = chosen.find(key);
            if (it != chosen.end()) {
                setSegment(it->second);
                return;
            }
        }
        int best = k2::MAX_SEG;
        const bool timed = !segmentRule_;
        if (!timed) {
            // An engine built while others run (a server's shots) cannot time fairly and should not
            // stall for it: the shortest segment that keeps the grid within eight waves of resident
            // CTAs.  Short segments shorten each CTA's chain of row blocks, which bounds a small
            // grid's step; past a few waves, longer ones save re-read halo rows.
            int sms = 0;
            check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_), "query SM count");
            const long long waves8 = 8LL * sms * k2::streamBlocks<Real>();
            for (best = 1;; best *= 2) {
                setSegment(best);
                if ((long long)stageGrid_.x * stageGrid_.y <= waves8 || best == k2::MAX_SEG) break;
            }
        } else {
            // Each candidate is timed as an 8-step CUDA graph, the form a batch runs in: timing eager
            // steps would measure the host's launch gaps, which dominate a small grid's step.  The
            // best of three replays counts, so that a clock ramp or a neighbour's burst during one
            // replay does not decide the segment.
            cudaEvent_t e0{}, e1{};
            check(cudaEventCreate(&e0), "create event");
            check(cudaEventCreate(&e1), "create event");
            double bestMs = 0;
            for (int seg = k2::MAX_SEG; seg >= 1; seg /= 2) {
                setSegment(seg);
                launch(0, 8, 1e-6, 10.0, 0.0, 0.3); // records this segment's graph (and loads modules)
                finish();
                float ms = 0;
                for (int rep = 0; rep < 3; ++rep) {
                    check(cudaEventRecord(e0, stream_), "record event");
                    launch(0, 8, 1e-6, 10.0, 0.0, 0.3);
                    check(cudaEventRecord(e1, stream_), "record event");
                    finish();
                    check(cudaEventSynchronize(e1), "tuning completion");
                    float one = 0;
                    check(cudaEventElapsedTime(&one, e0, e1), "event time");
                    ms = rep == 0 ? one : std::min(ms, one);
                }
                if (seg == k2::MAX_SEG || ms < 0.99 * bestMs) best = seg, bestMs = ms; // shorter only if faster by 1 %
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
        }
        {
            std::lock_guard<std::mutex> g(mutex);
            best = chosen.emplace(key, best).first->second; // a concurrent creation may have decided first
        }
        setSegment(best);
        if (timed) reset();
    }
    ~TypedEngine2D() override {
        if (done_) cudaEventSynchronize(done_), cudaEventDestroy(done_);
        if (queued_) cudaEventDestroy(queued_);
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
    void profile(int first, int count, double dt, double frequency, double scale, swl_profile &out) override {
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
        fillForcing(first, count, dt, frequency, scale);
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
        out.launches_per_step = 5;
        out.bytes_per_step = bytesPerStep();
        out.extra_bytes_per_step = extraBytesPerStep();
        const int accepted = hostClock_.accepted;
        u_ = (accepted % 2 == 0) ? u0 : 1 - u0;
        a_ = 1 - u_;
        previous_ = accepted > 0;
        faulted_ = hostClock_.faulted != 0;
    }

    void step(double dt, double frequency, double scale, int step) override {
        settle();
        DeviceScope scope(device_);
        dt_ = dt;
        ensureCapacity(1);
        hostClock_.step = step;
        hostClock_.first = step;
        hostClock_.faulted = 0;
        hostClock_.accepted = 0;
        hostClock_.trace_steps = traceCap_;
        pushClock();
        fillForcing(step, 1, dt, frequency, scale);
        enqueueStep(step, false);
        previous_ = true;
        pinnedRows_ = 0, clockStats_ = false;
        check(cudaStreamSynchronize(stream_), "2D step completion");
    }

    int advance(int first, int count, double dt, double frequency, double scale, double growthAfter) override {
        launch(first, count, dt, frequency, scale, growthAfter);
        return finish();
    }
    // Completion of an in-flight batch: roles after `accepted` steps (a rejected step leaves its
    // starting state current).
    void finalize() {
        hostClock_ = *pinnedClock_.as<k2::Clock>();
        const int accepted = hostClock_.accepted;
        u_ = (accepted % 2 == 0) ? batchU0_ : 1 - batchU0_;
        a_ = 1 - u_;
        previous_ = accepted > 0;
        faulted_ = hostClock_.faulted != 0;
        inflight_ = false;
        checkStalled();
    }
    int finish() override {
        if (!inflight_) return hostClock_.accepted;
        DeviceScope scope(device_);
        check(cudaEventSynchronize(done_), "2D batch completion");
        finalize();
        return hostClock_.accepted;
    }
    bool query(int &accepted) override {
        if (inflight_) {
            DeviceScope scope(device_);
            const cudaError_t e = cudaEventQuery(done_);
            if (e == cudaErrorNotReady) return false;
            check(e, "2D batch query");
            finalize();
        }
        accepted = hostClock_.accepted;
        return true;
    }
    // Enqueue a batch of steps on the engine's stream and return immediately.
    void launch(int first, int count, double dt, double frequency, double scale, double growthAfter) override {
        DeviceScope scope(device_);
        if (inflight_) throw Error(SWL_ERR_STATE, "a batch is already in flight on this engine");
        if (count <= 0) {
            hostClock_.accepted = 0;
            return;
        }
        if (dt != dt_) dropGraphs(), dt_ = dt;
        ensureCapacity(count);
        hostClock_.step = first;
        hostClock_.first = first;
        hostClock_.faulted = 0;
        hostClock_.fault_step = -1;
        hostClock_.accepted = 0;
        hostClock_.trace_steps = traceCap_;
        hostClock_.dt = dt;
        hostClock_.growth_after = growthAfter;
        pushClock();
        fillForcing(first, count, dt, frequency, scale);
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
            done += 8; // eight role swaps: roles are back where they started
        }
        for (; done < count; ++done) enqueueStep(first + done, true);
        // the batch's trace rows and clock come back with it, so that reading them needs no copy
        if (nrec_)
            check(cudaMemcpyAsync(pinnedTraces_.ptr, traces_.ptr, std::size_t(count) * nrec_ * 2 * sizeof(double),
                                  cudaMemcpyDeviceToHost, stream_),
                  "read traces");
        pinnedRows_ = count;
        clockStats_ = true;
        check(cudaMemcpyAsync(pinnedClock_.ptr, clock_.ptr, sizeof(k2::Clock), cudaMemcpyDeviceToHost, stream_), "read clock");
        check(cudaEventRecord(done_, stream_), "record batch completion");
        batchU0_ = u0;
        u_ = u0, a_ = 1 - u0; // the host view of the roles is settled by finalize()
        inflight_ = true;
    }
    void rollback() override {
        settle();
        DeviceScope scope(device_);
        check(cudaStreamSynchronize(stream_), "2D rollback");
        if (previous_) std::swap(u_, a_), previous_ = false;
    }
    void reset() override {
        settle();
        DeviceScope scope(device_);
        check(cudaMemsetAsync(sets_.ptr, 0, sets_.bytes, stream_), "2D reset");
        check(cudaMemsetAsync(psets_.ptr, 0, psets_.bytes, stream_), "2D PML reset");
        if (traces_.ptr) check(cudaMemsetAsync(traces_.ptr, 0, traces_.bytes, stream_), "2D trace reset");
        hostClock_ = k2::Clock{};
        pinnedRows_ = 0, clockStats_ = false;
        pushClock();
        check(cudaStreamSynchronize(stream_), "2D clear completion");
        u_ = 0, a_ = 1, previous_ = false, faulted_ = false;
    }
    int segment() const { return m_.seg; }
    void layout(swl_layout2d &out) const override {
        out = swl_layout2d{};
        out.strip_width = k2::SW;
        out.block_rows = k2::SB;
        out.segment_blocks = m_.seg;
        out.strips = int32_t(stageGrid_.x);
        out.segments = int32_t(stageGrid_.y);
        for (unsigned by = 0; by < stageGrid_.y; ++by)
            for (unsigned bx = 0; bx < stageGrid_.x; ++bx)
                out.interior_ctas += k2::interiorBlock(m_, 3 + int(bx) * k2::SW, 3 + int(by) * (k2::SB * m_.seg)) ? 1 : 0;
        out.exact_h = m_.hinvExact;
        out.precision = sizeof(Real) == 8 ? SWL_FP64 : SWL_FP32;
    }

    // ---- queued batches (Queue2D): the two halves of launch() around the persistent kernel
    int mechanisms() const { return mech_; }
    int deviceId() const { return device_; }
    cudaStream_t stream() const { return stream_; }
    // The clock and forcing tables of `count` steps from `first`, enqueued on the engine's stream,
    // and the kernel's description of the batch.
    // Row blocks per work item of a queued batch when the queue leaves it to the grid: the longest
    // segment that still cuts the grid into at least kQueueItems items per stage.  Long items amortise the
    // ticket, wait and fences of an item (measured: full 64-row segments run a launch of 24 shots
    // fastest); a tiny grid still gets enough items to spread over the SMs.  It depends on the grid
    // only, never on the other shots of a launch.
    static constexpr long long kQueueItems = 64; // 128 measured 0.85x / 1.00x of own streams for 8 / 24 shots, 64 gives 0.62x / 1.10x
    int queueSegment() const {
        const int qx = (nx_ - 6 + k2::SW - 1) / k2::SW;
        int seg = k2::MAX_SEG;
        while (seg > 1 && (long long)qx * ((nz_ - 6 + k2::SB * seg - 1) / (k2::SB * seg)) < kQueueItems) seg /= 2;
        return seg;
    }
    long long queueTiles(int qseg) const {
        if (qseg <= 0) qseg = queueSegment();
        return (long long)((nx_ - 6 + k2::SW - 1) / k2::SW) * ((nz_ - 6 + k2::SB * qseg - 1) / (k2::SB * qseg));
    }
    void queueBegin(int first, int count, double dt, double frequency, double scale, double growthAfter, int qseg,
                    k2::QueueShot<Real> &shot) {
        DeviceScope scope(device_);
        if (inflight_) throw Error(SWL_ERR_STATE, "a batch is already in flight on this engine");
        if (faulted_) throw Error(SWL_ERR_STATE, "2D engine holds a rejected step; reset or rebuild it");
        if (dt != dt_) dropGraphs(), dt_ = dt;
        ensureCapacity(count);
        hostClock_.step = first;
        hostClock_.first = first;
        hostClock_.faulted = 0;
        hostClock_.fault_step = -1;
        hostClock_.accepted = 0;
        hostClock_.trace_steps = traceCap_;
        hostClock_.dt = dt;
        hostClock_.growth_after = growthAfter;
        pushClock();
        fillForcing(first, count, dt, frequency, scale);
        // The queued form cuts the grid into work items of `qseg` row blocks (0: queueSegment()).
        if (qseg <= 0) qseg = queueSegment();
        const int su = u_, sa = a_;
        for (int r = 0; r < 2; ++r) {
            u_ = r, a_ = 1 - r;
            for (int k = 0; k < 4; ++k) shot.stage[r][k] = args(k), shot.stage[r][k].m.seg = qseg, shot.stage[r][k].gslsPrefetch = 0;
            shot.stage[r][3].partials = partials_.as<k2::Partial>(); // diagnostics fused into stage 3
        }
        u_ = su, a_ = sa;
        const int qx = (nx_ - 6 + k2::SW - 1) / k2::SW, qy = (nz_ - 6 + k2::SB * qseg - 1) / (k2::SB * qseg);
        shot.partials = partials_.as<k2::Partial>();
        shot.receivers = recIdx_.as<long long>();
        shot.traces = traces_.as<double>();
        shot.clock = clock_.as<k2::Clock>();
        shot.sets[0] = set_[0], shot.sets[1] = set_[1];
        shot.count = count_;
        shot.nrec = nrec_;
        shot.tiles = qx * qy; // the partials buffer holds at least one per one-block segment
        shot.tilesX = qx;
        shot.u0 = u_;
        shot.steps = count;
        shot.first = first;
    }
    // The uploads of queueBegin, for the queue's stream to wait on.
    cudaEvent_t queueReady() {
        DeviceScope scope(device_);
        if (!queued_) check(cudaEventCreateWithFlags(&queued_, cudaEventDisableTiming), "create queue event");
        check(cudaEventRecord(queued_, stream_), "record queue uploads");
        return queued_;
    }
    // After the kernel (`kernel`: its completion on the queue's stream): the trace rows and the clock
    // come back with the batch on the engine's stream; its completion event.
    void queueEnd(int count, cudaEvent_t kernel) {
        DeviceScope scope(device_);
        check(cudaStreamWaitEvent(stream_, kernel, 0), "order after the queued launch");
        if (nrec_)
            check(cudaMemcpyAsync(pinnedTraces_.ptr, traces_.ptr, std::size_t(count) * nrec_ * 2 * sizeof(double),
                                  cudaMemcpyDeviceToHost, stream_),
                  "read traces");
        pinnedRows_ = count;
        clockStats_ = true;
        check(cudaMemcpyAsync(pinnedClock_.ptr, clock_.ptr, sizeof(k2::Clock), cudaMemcpyDeviceToHost, stream_), "read clock");
        check(cudaEventRecord(done_, stream_), "record batch completion");
        batchU0_ = u_;
        inflight_ = true;
    }
    void diagnostics(swl_diag2d &d) override {
        settle();
        DeviceScope scope(device_);
        k2::stats2d<Real><<<grid_, block_, 0, stream_>>>(m_, set_[u_], pset_[u_], nullptr, partials_.as<k2::Partial>());
        check(cudaGetLastError(), "2D diagnostics");
        std::vector<k2::Partial> parts(nparts_);
        check(cudaMemcpyAsync(parts.data(), partials_.ptr, nparts_ * sizeof(k2::Partial), cudaMemcpyDeviceToHost, stream_),
              "2D diagnostics readback");
        check(cudaStreamSynchronize(stream_), "2D diagnostics completion");
        d.energy = d.max_velocity = d.traction_relative = 0;
        d.finite = 1;
        for (const auto &p : parts) {
            d.energy += p.energy;
            d.max_velocity = std::max(d.max_velocity, p.velocity);
            d.traction_relative = std::max(d.traction_relative, p.traction);
            d.finite &= !p.bad;
        }
        d.finite &= std::isfinite(d.energy) ? 1 : 0;
        d.peak_energy = hostClock_.peak_energy;
        d.rhs_registers = registers_;
        d.rhs_local_bytes = localBytes_;
        d.resident_bytes = residentBytes();
    }
    void stepDiagnostics(swl_diag2d &d) override {
        settle();
        if (!clockStats_) return diagnostics(d);
        d.energy = hostClock_.energy, d.max_velocity = hostClock_.max_velocity, d.traction_relative = hostClock_.traction;
        d.finite = hostClock_.finite;
        d.peak_energy = hostClock_.peak_energy;
        d.rhs_registers = registers_;
        d.rhs_local_bytes = localBytes_;
        d.resident_bytes = residentBytes();
    }
    void gather(const int64_t *nodes, int n, int fields, double *out) {
        if (n <= 0) return;
        std::vector<long long> idx(nodes, nodes + n);
        for (auto q : idx)
            if (q < 0 || q >= count_) throw Error(SWL_ERR_INVALID, "probe node outside the padded grid");
        DeviceBuffer dIdx(n * sizeof(long long)), dOut(std::size_t(n) * fields * sizeof(double));
        check(cudaMemcpyAsync(dIdx.ptr, idx.data(), n * sizeof(long long), cudaMemcpyHostToDevice, stream_), "probe upload");
        k2::gather2d<Real><<<(n + 127) / 128, 128, 0, stream_>>>(set_[u_], count_, dIdx.as<long long>(), n, fields, dOut.as<double>());
        check(cudaGetLastError(), "probe launch");
        check(cudaMemcpyAsync(out, dOut.ptr, std::size_t(n) * fields * sizeof(double), cudaMemcpyDeviceToHost, stream_), "probe readback");
        check(cudaStreamSynchronize(stream_), "probe completion");
    }
    void sample(double *vx, double *vz) override {
        settle();
        DeviceScope scope(device_);
        if (!nrec_) return;
        std::vector<int64_t> idx(nrec_);
        check(cudaMemcpy(idx.data(), recIdx_.ptr, nrec_ * sizeof(long long), cudaMemcpyDeviceToHost), "receiver index readback");
        std::vector<double> v(2 * std::size_t(nrec_));
        gather(idx.data(), nrec_, 2, v.data());
        for (int r = 0; r < nrec_; ++r) vx[r] = v[2 * r], vz[r] = v[2 * r + 1];
    }
    void traces(int first, int count, double *vx, double *vz) override {
        settle();
        DeviceScope scope(device_);
        const int row0 = first - hostClock_.first;
        if (count < 0 || row0 < 0 || row0 + count > hostClock_.accepted)
            throw Error(SWL_ERR_INVALID, "requested trace rows were not recorded by the last advance");
        std::vector<double> copy;
        const double *buf = pinnedTraces_.as<double>() + std::size_t(row0) * nrec_ * 2;
        if (row0 + count > pinnedRows_) { // rows recorded outside an asynchronous batch
            copy.resize(std::size_t(count) * nrec_ * 2);
            if (!copy.empty())
                check(cudaMemcpy(copy.data(), traces_.as<double>() + std::size_t(row0) * nrec_ * 2, copy.size() * sizeof(double),
                                 cudaMemcpyDeviceToHost),
                      "trace readback");
            buf = copy.data();
        }
        for (int r = 0; r < nrec_; ++r)
            for (int j = 0; j < count; ++j) {
                vx[std::size_t(r) * count + j] = buf[(std::size_t(j) * nrec_ + r) * 2];
                vz[std::size_t(r) * count + j] = buf[(std::size_t(j) * nrec_ + r) * 2 + 1];
            }
    }
    void snapshot(int field, double *out) override {
        settle();
        DeviceScope scope(device_);
        check(cudaStreamSynchronize(stream_), "snapshot ordering");
        const Real *src;
        std::size_t len;
        if (field == -1) src = pset_[u_], len = std::size_t(pcount_);
        else if (field >= 0 && field < fc_) src = set_[u_] + std::size_t(field) * count_, len = std::size_t(count_);
        else throw Error(SWL_ERR_INVALID, "snapshot field out of range");
        std::vector<Real> tmp(len);
        if (len) check(cudaMemcpy(tmp.data(), src, len * sizeof(Real), cudaMemcpyDeviceToHost), "snapshot download");
        if (field == -1) {
            for (std::size_t i = 0; i < len; ++i) out[i] = double(tmp[i]);
        } else { // pitched rows -> the caller's nx x nz layout
            for (int k = 0; k < nz_; ++k)
                for (int i = 0; i < nx_; ++i) out[std::size_t(k) * nx_ + i] = double(tmp[std::size_t(k) * pitch_ + 1 + i]);
        }
    }
    void load(int field, const double *in) override {
        settle();
        DeviceScope scope(device_);
        clockStats_ = false;
        check(cudaStreamSynchronize(stream_), "load ordering");
        Real *dst;
        std::size_t len;
        if (field == -1) dst = pset_[u_], len = std::size_t(pcount_);
        else if (field >= 0 && field < fc_) dst = set_[u_] + std::size_t(field) * count_, len = std::size_t(count_);
        else throw Error(SWL_ERR_INVALID, "load field out of range");
        std::vector<Real> tmp = field == -1 ? std::vector<Real>(in, in + len)
                                            : pitched(std::vector<Real>(in, in + std::size_t(nx_) * nz_), 1);
        if (len) check(cudaMemcpy(dst, tmp.data(), len * sizeof(Real), cudaMemcpyHostToDevice), "field upload");
        if (k2::kahan<Real>() && len) { // a loaded value starts without a compensation term
            Real *comp = field == -1 ? pset_[4 + u_] : set_[4 + u_] + std::size_t(field) * count_;
            check(cudaMemset(comp, 0, len * sizeof(Real)), "clear compensation");
        }
        previous_ = false;
    }
    void probes(const int64_t *nodes, int n, double *out5) override {
        settle();
        DeviceScope scope(device_);
        std::vector<int64_t> idx(nodes, nodes + std::max(n, 0));
        for (auto &q : idx) {
            if (q < 0 || q >= (long long)nx_ * nz_) throw Error(SWL_ERR_INVALID, "probe node outside the padded grid");
            q = memIndex(q);
        }
        gather(idx.data(), n, 5, out5);
    }
    int64_t residentBytes() const override {
        int64_t b = 0;
        for (const auto &x : model_) b += x.bytes;
        for (const auto *x : {&pack_, &strengths_, &sets_, &psets_, &recIdx_, &traces_, &forcing_, &clock_, &partials_}) b += x->bytes;
        return b;
    }
};


// The persistent multi-shot launch of engines of precision Real (Queue2D).  One device block
// holds the queue header, the shot descriptions and the order tables; it is written from pinned
// memory with one copy before the kernel, on the queue's own stream.  Each engine's uploads
// (clock, forcing) and read-backs (traces, clock) stay on the engine's stream, ordered with the
// kernel by events, so an engine outlives the queue and keeps working on its own afterwards.
template <class Real> class TypedQueue2D final : public Queue2D {
    int device_{}, sms_{}, blocks_{}, limit_{0}, seg_{0};
    cudaStream_t stream_{};
    cudaEvent_t done_{}, kernel_{};
    DeviceBuffer dev_;
    PinnedBuffer host_;
    bool inflight_{false};
    static std::size_t up(std::size_t n) { return (n + 63) / 64 * 64; }
    int occupancy(int mech) const {
        switch (mech) {
        case 0: return detail2::queueOccupancy2D<Real, 0>();
        case 1: return detail2::queueOccupancy2D<Real, 1>();
        case 2: return detail2::queueOccupancy2D<Real, 2>();
        default: return detail2::queueOccupancy2D<Real, 3>();
        }
    }
    void run(int mech, int blocks, k2::QueueHeader *h, const k2::QueueShot<Real> *shots) {
        switch (mech) {
        case 0: detail2::launchQueue2D<Real, 0>(blocks, stream_, h, shots); break;
        case 1: detail2::launchQueue2D<Real, 1>(blocks, stream_, h, shots); break;
        case 2: detail2::launchQueue2D<Real, 2>(blocks, stream_, h, shots); break;
        default: detail2::launchQueue2D<Real, 3>(blocks, stream_, h, shots); break;
        }
    }

  public:
    explicit TypedQueue2D(int device) : device_(device) {
        DeviceScope scope(device_);
        check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "create queue stream");
        check(cudaEventCreateWithFlags(&done_, cudaEventDisableTiming), "create queue event");
        check(cudaEventCreateWithFlags(&kernel_, cudaEventDisableTiming), "create queue event");
        check(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_), "query SM count");
    }
    ~TypedQueue2D() override {
        if (done_) cudaEventSynchronize(done_), cudaEventDestroy(done_);
        if (kernel_) cudaEventDestroy(kernel_);
        if (stream_) cudaStreamSynchronize(stream_), cudaStreamDestroy(stream_);
    }
    int blocks() const override { return blocks_; }
    void limit(int ctasPerSm) override { limit_ = ctasPerSm; }
    void segment(int seg) override {
        if (seg != 0 && seg != 1 && seg != 2 && seg != 4 && seg != 8) throw Error(SWL_ERR_INVALID, "queue segment must be 0, 1, 2, 4 or 8");
        seg_ = seg;
    }
    void launch(Engine2D *const *engines, int n, const int *first, const int *count, const double *dt, const double *frequency,
                const double *scale, const double *growthAfter) override {
        DeviceScope scope(device_);
        if (inflight_) throw Error(SWL_ERR_STATE, "a queued launch is already in flight");
        if (n <= 0) return;
        if (n > k2::kQueueMaxShots) throw Error(SWL_ERR_INVALID, "a queued launch takes at most 256 engines");
        std::vector<TypedEngine2D<Real> *> e(n);
        for (int i = 0; i < n; ++i) {
            e[i] = dynamic_cast<TypedEngine2D<Real> *>(engines[i]);
            if (!e[i]) throw Error(SWL_ERR_INVALID, "queued engines must share the queue's precision");
            if (e[i]->deviceId() != device_) throw Error(SWL_ERR_INVALID, "queued engines must live on the queue's device");
            if (e[i]->mechanisms() != e[0]->mechanisms()) throw Error(SWL_ERR_INVALID, "queued engines must share one GSLS mechanism count");
            if (count[i] <= 0 || !(dt[i] > 0) || first[i] < 0) throw Error(SWL_ERR_INVALID, "queued batches need count > 0, dt > 0, first >= 0");
            for (int k = 0; k < i; ++k)
                if (e[k] == e[i]) throw Error(SWL_ERR_INVALID, "an engine appears twice in one queued launch");
        }
        // shots in the order of their batch length, longest first: the shots stepping at step j
        // are then a prefix of the order
        std::vector<int> order(n);
        for (int i = 0; i < n; ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return count[a] > count[b]; });
        const int maxSteps = count[order[0]];
        const std::size_t oShots = up(sizeof(k2::QueueHeader)), oDone = oShots + up(sizeof(k2::QueueShot<Real>) * n);
        const std::size_t oStart = oDone + up(sizeof(int) * n), oActive = oStart + up(sizeof(long long) * (maxSteps + 1));
        long long allTiles = 0;
        for (int i = 0; i < n; ++i) allTiles += e[i]->queueTiles(seg_);
        const std::size_t oPrefix = oActive + up(sizeof(int) * maxSteps), oProgress = oPrefix + up(sizeof(long long) * (n + 1));
        const std::size_t oAbort = oProgress + up(sizeof(int) * std::size_t(allTiles));
        const std::size_t bytes = oAbort + 64;
        if (dev_.bytes < bytes) dev_.allocate(bytes);
        host_.reserve(bytes);
        std::memset(host_.ptr, 0, bytes);
        auto *hb = host_.as<unsigned char>();
        auto *db = static_cast<unsigned char *>(dev_.ptr);
        auto *shots = reinterpret_cast<k2::QueueShot<Real> *>(hb + oShots);
        for (int s = 0; s < n; ++s) {
            const int i = order[s];
            new (shots + s) k2::QueueShot<Real>{};
            e[i]->queueBegin(first[i], count[i], dt[i], frequency[i], scale[i], growthAfter[i], seg_, shots[s]);
            check(cudaStreamWaitEvent(stream_, e[i]->queueReady(), 0), "order the queued launch after the uploads");
        }
        auto *prefix = reinterpret_cast<long long *>(hb + oPrefix);
        for (int s = 0; s < n; ++s) prefix[s + 1] = prefix[s] + shots[s].tiles;
        auto *start = reinterpret_cast<long long *>(hb + oStart);
        auto *active = reinterpret_cast<int *>(hb + oActive);
        for (int j = 0, a = n; j < maxSteps; ++j) {
            while (a > 0 && count[order[a - 1]] <= j) --a;
            active[j] = a;
            start[j + 1] = start[j] + 4 * prefix[a] + a;
        }
        auto *h = reinterpret_cast<k2::QueueHeader *>(hb);
        h->head = 0;
        h->total = (unsigned long long)start[maxSteps];
        h->abort = 0;
        h->nshots = n;
        h->maxSteps = maxSteps;
        h->done = reinterpret_cast<int *>(db + oDone);
        h->progress = reinterpret_cast<int *>(db + oProgress);
        if (prefix[n] != allTiles) throw Error(SWL_ERR_STATE, "queued tile count mismatch");
        h->stepStart = reinterpret_cast<const long long *>(db + oStart);
        h->active = reinterpret_cast<const int *>(db + oActive);
        h->tilePrefix = reinterpret_cast<const long long *>(db + oPrefix);
        check(cudaMemcpyAsync(dev_.ptr, host_.ptr, oAbort, cudaMemcpyHostToDevice, stream_), "upload queue");
        const int mech = e[0]->mechanisms();
        const int occ = occupancy(mech);
        const int perSm = limit_ > 0 ? std::min(limit_, occ) : limit_ < 0 ? std::max(1, occ + limit_) : occ;
        blocks_ = int(std::min<long long>((long long)perSm * sms_, (long long)h->total));
        run(mech, blocks_, reinterpret_cast<k2::QueueHeader *>(db), reinterpret_cast<const k2::QueueShot<Real> *>(db + oShots));
        check(cudaEventRecord(kernel_, stream_), "record queued launch");
        for (int i = 0; i < n; ++i) e[i]->queueEnd(count[i], kernel_);
        check(cudaMemcpyAsync(hb + oAbort, db + offsetof(k2::QueueHeader, abort), sizeof(int), cudaMemcpyDeviceToHost, stream_),
              "read queue status");
        check(cudaEventRecord(done_, stream_), "record queue completion");
        abortAt_ = oAbort;
        inflight_ = true;
    }
    std::size_t abortAt_{};
    void settled() {
        inflight_ = false;
        const int abort = *reinterpret_cast<const int *>(host_.as<unsigned char>() + abortAt_);
        if (abort == 1) throw Error(SWL_ERR_CUDA, "CUDA 2D queue: a tensor-copy wait ran out");
        if (abort) throw Error(SWL_ERR_CUDA, "CUDA 2D queue: a stage dependency wait ran out");
    }
    bool query() override {
        if (!inflight_) return true;
        DeviceScope scope(device_);
        const cudaError_t st = cudaEventQuery(done_);
        if (st == cudaErrorNotReady) return false;
        check(st, "2D queue query");
        settled();
        return true;
    }
    void finish() override {
        if (!inflight_) return;
        DeviceScope scope(device_);
        check(cudaEventSynchronize(done_), "2D queue completion");
        settled();
    }
};
} // namespace swl
