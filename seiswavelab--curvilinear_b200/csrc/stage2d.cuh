// 2D P-SV / GSLS device code: one fused kernel per classic-RK4 stage.
//
// Each thread owns one physical node.  It evaluates the MacCormack-DRP derivatives of the
// stage input, the metric-transformed right-hand side (src/two_d/PointKernels2D.hpp:121-172)
// with the traction-image surface rows, CFS-PML ADE memories and GSLS relaxation, and then
// immediately performs its part of the RK combine and the free-surface projection -- the
// rates never touch HBM.  Three state sets stay resident beside the stage outputs:
//   U (state at the start of the step), A (running RK accumulator), S (stage state).
// Stage 0 writes A = k1 and S = U + dt/2 k1; stages 1-2 add 2k to A and write
// S = U + w k; stage 3 writes U + dt (A + k4) / 6 over A.  The sums are formed in the
// reference's order (src/two_d/CurvilinearSolver2D.cpp:80-97), so with FMA contraction off
// the FP64 results equal the reference CPU build's.
#pragma once
#include "runtime.cuh"
#include <cstdint>

namespace swl::k2 {

// Device view of the model (Point::MeshT, src/two_d/PointKernels2D.hpp:14-27), plus the
// boxes outside which the sparse source and sponge arrays are exactly zero.
template <class Real> struct Mesh {
    int nx, nz; // padded
    long long count;
    Real h;
    const Real *a, *b, *jac, *normals, *lambda, *mu, *rho, *damping, *source, *sgx, *sgz;
    Real sdx, sdz;             // unit force direction (x, z)
    int src_i0, src_i1, src_k0, src_k1; // source support box [i0,i1) x [k0,k1), padded indices
    int dmp_i0, dmp_i1, dmp_k1;         // damping is zero for i in [i0,i1) and k < k1
    const Real *cpx, *cpz;              // CFS-PML (d, kappa, alpha) per computational column / row
    int wx, wz;                         // CFS-PML widths (both 0 without CFS-PML)
    Real rates[3];
    const Real *dP[3], *dS[3];
    int fc; // field count
};

// Device-resident step clock: the step kernels of a batch read the step number here, and
// the per-step verdict kernel advances it.  A rejected step freezes the clock and turns
// every later kernel of the batch into a no-op.
struct Clock {
    int step;        // step being computed
    int first;       // first step of the current batch (forcing/trace tables start here)
    int faulted;     // set by the verdict on a rejected step
    int fault_step;  // the rejected step
    int trace_steps; // capacity of the trace table in steps
    int pad;
    double peak_energy;
    double energy, max_velocity, traction;
    int finite;
    int accepted;    // steps accepted in this batch
    double dt, growth_after; // energy-growth rule applies when (step+1)*dt > growth_after
};

template <class Real> struct StageArgs {
    Mesh<Real> m;
    const Real *in;   // stage input state (stencil reads)
    Real *out;        // stage output state S (stages 0-2)
    const Real *base; // U
    Real *acc;        // A; stage 3 writes the new state here
    const Real *pin;
    Real *pout;
    const Real *pbase;
    Real *pacc;
    const Real *forcing; // 3 values per step of the batch: t, t+dt/2, t+dt
    const Clock *clock;
    Real weight;         // dt/2, dt/2, dt for stages 0..2
    Real delta;          // dt
};

template <class Real> __device__ __forceinline__ Real ld(const Real *p) { return __ldg(p); }

// 5-point DRP derivative (include/SeisCommon/FiniteDifference.hpp:14-26, PointKernels2D.hpp:38-47):
// forward taps at offsets -1..3, backward at +1..-3 with negated coefficients.
template <class Real, int DIR>
__device__ __forceinline__ Real drp5(const Real *__restrict__ v, long long q, long long s, Real h) {
    Real r = Real(0);
    if (DIR == 0) {
        r += Real(-.30874) * ld(v + q - s);
        r += Real(-.6326) * ld(v + q);
        r += Real(1.233) * ld(v + q + s);
        r += Real(-.3334) * ld(v + q + 2 * s);
        r += Real(.04168) * ld(v + q + 3 * s);
    } else {
        r += -Real(-.30874) * ld(v + q + s);
        r += -Real(-.6326) * ld(v + q);
        r += -Real(1.233) * ld(v + q - s);
        r += -Real(-.3334) * ld(v + q - 2 * s);
        r += -Real(.04168) * ld(v + q - 3 * s);
    }
    return r / h;
}
// One-sided near-surface velocity stencils: 2 points at depth 1, 3 points at depth 2.
template <class Real, int DIR>
__device__ __forceinline__ Real near2(const Real *__restrict__ v, long long q, long long s, Real h) {
    Real r = Real(0);
    if (DIR == 0) {
        r += Real(-1) * ld(v + q);
        r += Real(1) * ld(v + q + s);
    } else {
        r += -Real(-1) * ld(v + q);
        r += -Real(1) * ld(v + q - s);
    }
    return r / h;
}
template <class Real, int DIR>
__device__ __forceinline__ Real near3(const Real *__restrict__ v, long long q, long long s, Real h) {
    const Real c0 = Real(-7) / Real(6), c1 = Real(8) / Real(6), c2 = Real(-1) / Real(6);
    Real r = Real(0);
    if (DIR == 0) {
        r += c0 * ld(v + q);
        r += c1 * ld(v + q + s);
        r += c2 * ld(v + q + 2 * s);
    } else {
        r += -c0 * ld(v + q);
        r += -c1 * ld(v + q - s);
        r += -c2 * ld(v + q - 2 * s);
    }
    return r / h;
}

// Traction flux J (x sigma_a + z sigma_b) at node qq (PointKernels2D.hpp:90-93).
template <class Real>
__device__ __forceinline__ Real flux(const Mesh<Real> &m, const Real *__restrict__ w, long long qq, int axis, int comp) {
    const long long n = m.count;
    const Real x = axis ? ld(m.a + qq) : Real(1), z = axis ? ld(m.b + qq) : Real(0);
    return ld(m.jac + qq) * (x * ld(w + (comp ? 4 : 2) * n + qq) + z * ld(w + (comp ? 3 : 4) * n + qq));
}

// Conservative traction-image momentum near the surface (PointKernels2D.hpp:94-120):
// the surface tap is dropped and taps above it mirror with a sign flip.  only = -1: both axes.
template <class Real, int DX, int DZ>
__device__ Real momentum(const Mesh<Real> &m, const Real *__restrict__ w, long long q, int comp, int depth, int only) {
    const Real C[5] = {Real(-.30874), Real(-.6326), Real(1.233), Real(-.3334), Real(.04168)};
    Real r = Real(0);
    for (int axis = 0; axis < 2; ++axis) {
        if (only >= 0 && axis != only) continue;
        const int dir = axis ? DZ : DX;
        for (int l = 0; l < 5; ++l) {
            const int pos = l - 1;
            int off = dir ? -pos : pos;
            const Real c = dir ? -C[l] : C[l];
            Real sign = Real(1);
            if (axis) {
                const int kk = depth + off;
                if (kk == 0) continue;
                if (kk < 0) {
                    off = -kk - depth;
                    sign = Real(-1);
                }
            }
            r += sign * c * flux(m, w, q + (long long)off * (axis ? m.nx : 1), axis, comp);
        }
    }
    return r / (m.h * ld(m.jac + q) * ld(m.rho + q));
}

// CFS-PML ADE (PointKernels2D.hpp:57-64): returns d/kappa + psi, rate -(d/k+a) psi - d/k^2 d.
template <class Real>
__device__ __forceinline__ Real stretch(const Real *prof, Real psi, Real d, Real &rate) {
    const Real dd = prof[0], kappa = prof[1], alpha = prof[2];
    rate = -(dd / kappa + alpha) * psi - dd / (kappa * kappa) * d;
    return d / kappa + psi;
}

// The fused stage.  DX/DZ: MacCormack directions of this (step, stage); MECH: GSLS
// mechanisms; STAGE: 0..3.  The CFS-PML branch is uniform across the launch.
template <class Real, int DX, int DZ, int MECH, int STAGE>
__global__ void __launch_bounds__(256) stage2d(const StageArgs<Real> p) {
    const Mesh<Real> &m = p.m;
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = 3 + blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= m.nx - 3 || k >= m.nz - 3) return;
    const Clock *clk = p.clock;
    if (clk->faulted) return;
    const bool CPML = m.wz > 0;
    constexpr int FC = MECH ? 6 + 4 * MECH : 5;
    const long long n = m.count, nx = m.nx, q = i + nx * k;
    const int depth = k - 3;
    const Real *__restrict__ w = p.in;
    const Real h = m.h;

    // --- derivatives along xi (x) of the five stencil fields
    Real xi[5], eta[5];
#pragma unroll
    for (int f = 0; f < 5; ++f) xi[f] = drp5<Real, DX>(w + f * n, q, 1, h);
    // --- CFS-PML slots of this node (src/two_d/PointKernels2D.hpp:50-56)
    long long slot0 = -1, slot1 = -1;
    const Real *prof0 = nullptr, *prof1 = nullptr;
    if (CPML) {
        const int ic = i - 3, kc = k - 3, nxc = m.nx - 6, nzc = m.nz - 6;
        const int j = ic < m.wx ? ic : ic >= nxc - m.wx ? m.wx + ic - (nxc - m.wx) : -1;
        if (j >= 0) slot0 = 4 * ((long long)kc * 2 * m.wx + j), prof0 = m.cpx + 3 * ic;
        if (kc >= nzc - m.wz)
            slot1 = 4 * ((long long)(2 * m.wx) * nzc + (long long)(kc - (nzc - m.wz)) * nxc + ic), prof1 = m.cpz + 3 * kc;
    }
    Real prate0[4] = {0, 0, 0, 0}, prate1[4] = {0, 0, 0, 0};
    Real vxs[2] = {xi[0], xi[1]}; // stretched xi of Vx, Vz
    if (CPML && slot0 >= 0)
        for (int v = 0; v < 2; ++v) vxs[v] = stretch(prof0, ld(p.pin + slot0 + v), xi[v], prate0[v]);

    // --- derivatives along eta (z); velocities use the one-sided / traction stencils near the surface
#pragma unroll
    for (int f = 2; f < 5; ++f) eta[f] = drp5<Real, DZ>(w + f * n, q, nx, h);
    if (depth == 0) {
        // surface eta-derivative from the traction-free condition (PointKernels2D.hpp:79-89)
        const Real c0 = ld(m.a + q), c1 = ld(m.b + q), c2 = c0 * c0 + c1 * c1, len = sqrt(c2);
        const Real nn[2] = {c0 / len, c1 / len};
        const Real dx = vxs[0], dz = vxs[1], lam = ld(m.lambda + q), mu = ld(m.mu + q);
        Real t[2] = {(lam + 2 * mu) * dx * c0 + mu * dz * c1, mu * dz * c0 + lam * dx * c1};
#pragma unroll
        for (int l = 0; l < MECH; ++l) {
            const int mm = 6 + 4 * l;
            t[0] -= ld(w + mm * n + q) * c0 + ld(w + (mm + 2) * n + q) * c1;
            t[1] -= ld(w + (mm + 2) * n + q) * c0 + ld(w + (mm + 1) * n + q) * c1;
        }
        const Real normal = t[0] * nn[0] + t[1] * nn[1];
        for (int v = 0; v < 2; ++v)
            eta[v] = -(t[v] - nn[v] * normal) / (mu * c2) - nn[v] * normal / ((lam + 2 * mu) * c2);
    } else if (depth == 1) {
        eta[0] = near2<Real, DZ>(w, q, nx, h);
        eta[1] = near2<Real, DZ>(w + n, q, nx, h);
    } else if (depth == 2) {
        eta[0] = near3<Real, DZ>(w, q, nx, h);
        eta[1] = near3<Real, DZ>(w + n, q, nx, h);
    } else {
        eta[0] = drp5<Real, DZ>(w, q, nx, h);
        eta[1] = drp5<Real, DZ>(w + n, q, nx, h);
    }
    const Real a = ld(m.a + q), b = ld(m.b + q), rho = ld(m.rho + q);
    Real dxv[5], dzv[5];
#pragma unroll
    for (int f = 0; f < 5; ++f) {
        Real vx = xi[f], vz = eta[f];
        if (CPML && f < 2) {
            vx = vxs[f];
            if (slot1 >= 0) vz = stretch(prof1, ld(p.pin + slot1 + f), eta[f], prate1[f]);
        }
        dxv[f] = vx + a * vz;
        dzv[f] = b * vz;
    }

    // --- velocity rates
    Real r[FC];
    const bool near = depth <= (DZ ? 3 : 1);
    if (!CPML) {
        if (near) {
            r[0] = momentum<Real, DX, DZ>(m, w, q, 0, depth, -1);
            r[1] = momentum<Real, DX, DZ>(m, w, q, 1, depth, -1);
        } else {
            r[0] = (dxv[2] + dzv[4]) / rho;
            r[1] = (dxv[4] + dzv[3]) / rho;
        }
    } else {
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            const int f = v ? 4 : 2, o = v ? 3 : 4;
            Real X, Z;
            if (near) {
                X = momentum<Real, DX, DZ>(m, w, q, v, depth, 0);
                Z = momentum<Real, DX, DZ>(m, w, q, v, depth, 1);
            } else {
                X = xi[f] / rho;
                Z = (a * eta[f] + b * eta[o]) / rho;
            }
            if (slot0 >= 0) X = stretch(prof0, ld(p.pin + slot0 + 2 + v), X, prate0[2 + v]);
            if (slot1 >= 0) Z = stretch(prof1, ld(p.pin + slot1 + 2 + v), Z, prate1[2 + v]);
            r[v] = X + Z;
        }
    }
    if (i >= m.src_i0 && i < m.src_i1 && k >= m.src_k0 && k < m.src_k1) {
        const Real forcing = p.forcing[3 * (clk->step - clk->first) + (STAGE == 0 ? 0 : STAGE == 3 ? 2 : 1)];
        if (m.sgx) {
            r[0] += forcing * ld(m.sgx + q) / rho;
            r[1] += forcing * ld(m.sgz + q) / rho;
        } else {
            const Real s = ld(m.source + q);
            r[0] += forcing * (s * m.sdx) / rho;
            r[1] += forcing * (s * m.sdz) / rho;
        }
    }
    // --- stress rates (and GSLS memories)
    const Real lam = ld(m.lambda + q), mu = ld(m.mu + q), div = dxv[0] + dzv[1];
    r[2] = lam * div + 2 * mu * dxv[0];
    r[3] = lam * div + 2 * mu * dzv[1];
    r[4] = mu * (dzv[0] + dxv[1]);
    Real wc[FC]; // stage input at the node (pointwise fields and damping)
#pragma unroll
    for (int f = 0; f < FC; ++f) wc[f] = ld(w + f * n + q);
    if (MECH) {
        r[5] = lam * div;
#pragma unroll
        for (int l = 0; l < MECH; ++l) {
            const int mm = 6 + 4 * l;
            const Real dp = ld(m.dP[l] + q), ds = ld(m.dS[l] + q), dl = dp - 2 * ds;
            const Real drive[4] = {dl * div + 2 * ds * dxv[0], dl * div + 2 * ds * dzv[1], ds * (dzv[0] + dxv[1]), dl * div};
            r[2] -= wc[mm];
            r[3] -= wc[mm + 1];
            r[4] -= wc[mm + 2];
            r[5] -= wc[mm + 3];
#pragma unroll
            for (int f = 0; f < 4; ++f) r[mm + f] = m.rates[l] * (drive[f] - wc[mm + f]);
        }
    }
    if (!(i >= m.dmp_i0 && i < m.dmp_i1 && k < m.dmp_k1)) {
        const Real d = ld(m.damping + q);
#pragma unroll
        for (int f = 0; f < FC; ++f) r[f] -= d * wc[f];
    }

    // --- RK combine (+ projection of the surface row), fields then ADE memories
    Real o[FC];
#pragma unroll
    for (int f = 0; f < FC; ++f) {
        const Real u = ld(p.base + f * n + q);
        if (STAGE == 0) {
            p.acc[f * n + q] = r[f];
            o[f] = u + p.weight * r[f];
        } else if (STAGE < 3) {
            p.acc[f * n + q] = p.acc[f * n + q] + 2 * r[f];
            o[f] = u + p.weight * r[f];
        } else {
            o[f] = u + p.delta * (p.acc[f * n + q] + r[f]) / Real(6);
        }
    }
    if (depth == 0) { // PointKernels2D.hpp:70-78
        const Real nx_ = ld(m.normals + 2 * q), nz_ = ld(m.normals + 2 * q + 1);
        const Real tx = o[2] * nx_ + o[4] * nz_, tz = o[4] * nx_ + o[3] * nz_, nn = nx_ * tx + nz_ * tz;
        o[2] += -2 * nx_ * tx + nn * nx_ * nx_;
        o[3] += -2 * nz_ * tz + nn * nz_ * nz_;
        o[4] += -nx_ * tz - tx * nz_ + nn * nx_ * nz_;
    }
    Real *dst = STAGE == 3 ? p.acc : p.out;
#pragma unroll
    for (int f = 0; f < FC; ++f) dst[f * n + q] = o[f];
    if (CPML) {
#pragma unroll
        for (int ax = 0; ax < 2; ++ax) {
            const long long s = ax ? slot1 : slot0;
            if (s < 0) continue;
            const Real *pr = ax ? prate1 : prate0;
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                const long long at = s + f;
                const Real u = ld(p.pbase + at);
                if (STAGE == 0) {
                    p.pacc[at] = pr[f];
                    p.pout[at] = u + p.weight * pr[f];
                } else if (STAGE < 3) {
                    p.pacc[at] = p.pacc[at] + 2 * pr[f];
                    p.pout[at] = u + p.weight * pr[f];
                } else {
                    p.pacc[at] = u + p.delta * (p.pacc[at] + pr[f]) / Real(6);
                }
            }
        }
    }
}

// ---------------------------------------------------------------- diagnostics ------------
struct Partial {
    double energy, velocity, traction;
    int bad, pad;
};

// Per-block energy / peak velocity / surface traction / finiteness of a state
// (src/two_d/CudaEngine2D.cu:43-78 semantics, PointKernels2D.hpp:181-184 energy).
template <class Real>
__global__ void __launch_bounds__(256) stats2d(const Mesh<Real> m, const Real *__restrict__ w, const Real *__restrict__ pml,
                                               const Clock *clk, Partial *out) {
    __shared__ Partial sh[256];
    const int t = threadIdx.x + blockDim.x * threadIdx.y;
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = 3 + blockIdx.y * blockDim.y + threadIdx.y;
    Partial s{0, 0, 0, 0, 0};
    if (i < m.nx - 3 && k < m.nz - 3 && !(clk && clk->faulted)) {
        const long long n = m.count, q = i + (long long)m.nx * k;
        for (int f = 0; f < m.fc; ++f)
            if (!isfinite(ld(w + f * n + q))) s.bad = 1;
        if (m.wx || m.wz) {
            const int ic = i - 3, kc = k - 3, nxc = m.nx - 6, nzc = m.nz - 6;
            const int j = ic < m.wx ? ic : ic >= nxc - m.wx ? m.wx + ic - (nxc - m.wx) : -1;
            long long slots[2] = {j >= 0 ? 4 * ((long long)kc * 2 * m.wx + j) : -1,
                                  kc >= nzc - m.wz ? 4 * ((long long)(2 * m.wx) * nzc + (long long)(kc - (nzc - m.wz)) * nxc + ic) : -1};
            for (int a = 0; a < 2; ++a)
                if (slots[a] >= 0)
                    for (int f = 0; f < 4; ++f)
                        if (!isfinite(ld(pml + slots[a] + f))) s.bad = 1;
        }
        const double l = ld(m.lambda + q), mu = ld(m.mu + q), xx = ld(w + 2 * n + q), zz = ld(w + 3 * n + q),
                     xz = ld(w + 4 * n + q), vx = ld(w + q), vz = ld(w + n + q);
        s.energy = (.5 * double(ld(m.rho + q)) * (vx * vx + vz * vz) +
                    ((l + 2 * mu) * (xx * xx + zz * zz) - 2 * l * xx * zz) / (8 * mu * (l + mu)) + xz * xz / (2 * mu)) *
                   double(ld(m.jac + q)) * double(m.h) * double(m.h);
        const Real wx_ = ld(w + q), wz_ = ld(w + n + q);
        s.velocity = double(sqrt(wx_ * wx_ + wz_ * wz_));
        if (!isfinite(s.energy) || !isfinite(s.velocity)) s.bad = 1;
        if (k == 3) {
            const double nx_ = ld(m.normals + 2 * q), nz_ = ld(m.normals + 2 * q + 1);
            const double tx = xx * nx_ + xz * nz_, tz = xz * nx_ + zz * nz_, norm = sqrt(xx * xx + zz * zz + 2 * xz * xz);
            s.traction = sqrt(tx * tx + tz * tz) / fmax(norm, 1e-25);
        }
    }
    sh[t] = s;
    __syncthreads();
    for (int stride = 128; stride > 0; stride >>= 1) {
        if (t < stride) {
            Partial &x = sh[t];
            const Partial y = sh[t + stride];
            x.energy += y.energy;
            x.velocity = fmax(x.velocity, y.velocity);
            x.traction = fmax(x.traction, y.traction);
            x.bad |= y.bad;
        }
        __syncthreads();
    }
    if (t == 0) out[blockIdx.x + gridDim.x * blockIdx.y] = sh[0];
}

// Reduce the partials, apply the acceptance rule of Simulation::advance
// (src/two_d/CurvilinearSolver2D.cpp:576-590), record the receivers of an accepted step and
// advance the clock.  One block.
template <class Real>
__global__ void __launch_bounds__(1024) verdict2d(const Partial *__restrict__ parts, int nparts, const Real *__restrict__ w,
                                                  long long count, const long long *__restrict__ receivers, int nrec,
                                                  double *__restrict__ traces, Clock *clk, int check) {
    __shared__ Partial sh[1024];
    __shared__ int accept;
    const int t = threadIdx.x;
    if (clk->faulted) return;
    Partial s{0, 0, 0, 0, 0};
    if (check) {
        for (int b = t; b < nparts; b += blockDim.x) {
            const Partial y = parts[b];
            s.energy += y.energy;
            s.velocity = fmax(s.velocity, y.velocity);
            s.traction = fmax(s.traction, y.traction);
            s.bad |= y.bad;
        }
    }
    sh[t] = s;
    __syncthreads();
    for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
        if (t < stride) {
            Partial &x = sh[t];
            const Partial y = sh[t + stride];
            x.energy += y.energy;
            x.velocity = fmax(x.velocity, y.velocity);
            x.traction = fmax(x.traction, y.traction);
            x.bad |= y.bad;
        }
        __syncthreads();
    }
    if (t == 0) {
        int ok = 1;
        if (check) {
            const Partial tot = sh[0];
            const bool finite = !tot.bad && isfinite(tot.energy);
            const bool growth = (clk->step + 1) * clk->dt > clk->growth_after && clk->peak_energy > 0 &&
                                tot.energy > clk->peak_energy * 10000;
            ok = finite && !growth;
            clk->finite = finite;
            if (ok) {
                clk->energy = tot.energy;
                clk->max_velocity = tot.velocity;
                clk->traction = tot.traction;
                clk->peak_energy = fmax(clk->peak_energy, tot.energy);
            }
        }
        accept = ok;
    }
    __syncthreads();
    if (!accept) {
        if (t == 0) {
            clk->faulted = 1;
            clk->fault_step = clk->step;
        }
        return;
    }
    const int row = clk->step - clk->first;
    if (row < clk->trace_steps)
        for (int r = t; r < nrec; r += blockDim.x) {
            const long long qq = receivers[r];
            traces[((long long)row * nrec + r) * 2] = double(w[qq]);
            traces[((long long)row * nrec + r) * 2 + 1] = double(w[count + qq]);
        }
    __syncthreads();
    if (t == 0) {
        clk->step += 1;
        clk->accepted += 1;
    }
}

// Gathers for sample / probes (CudaEngine2D.cu:79-89).
template <class Real>
__global__ void gather2d(const Real *__restrict__ w, long long count, const long long *__restrict__ nodes, int n,
                         int fields, double *__restrict__ out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n)
        for (int f = 0; f < fields; ++f) out[(long long)fields * r + f] = double(w[f * count + nodes[r]]);
}

} // namespace swl::k2
