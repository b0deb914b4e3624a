// 3D nine-field elastic device code: one fused kernel per classic-RK4 stage.
//
// Each thread owns one physical node: 27 MacCormack-DRP derivatives of the stage input, the
// metric transform to physical gradients, the nine rates of src/three_d/PointKernels3D.hpp:92-112
// (traction-image momentum near the surface, traction-free surface derivative on the top
// row, sponge damping, force or moment source), then its part of the RK combine and the
// tangential-stress projection.  The 3D reference sums the RK stages as
// (((base + dt/6 k1) + dt/3 k2) + dt/3 k3) + dt/6 k4 (src/three_d/CurvilinearSolver.cpp:91-101),
// so the accumulator here carries the partial state sum: A = U + dt/6 k1, A += dt/3 k2,
// A += dt/3 k3, new state = A + dt/6 k4 written over A.
//
// Layout: every field is a pitched (x, y, z) array; node (i, j, k) sits at i + px*j + px*ny*k
// with the row pitch px a multiple of four nodes, so that every row starts on a 16-byte
// boundary.  Metrics are nine separate arrays (structure of arrays) so that every load of a
// warp is coalesced; the surface normals and the traction-rate diagnostics only exist for the
// top row.
//
// The stencil taps are read through L1: a CTA of 32 x 8 nodes of one z layer re-reads its x/y
// neighbours from L1 and the z layers above and below from L2.  A z-marching form that stages
// halo'd planes in shared memory by TMA was measured slower: its ring of planes (207 KB FP64,
// 104 KB FP32 per CTA) leaves 8 or 16 resident warps per SM, too few to hide the point loads
// (metrics, material, base, accumulator) that every node still makes, while this form keeps 32.
#pragma once
#include "runtime.cuh"
#include "stage2d.cuh"
#include <cstdint>

namespace swl::k3 {

template <class Real> struct Mesh {
    int nx, ny, nz;
    int px;                         // row pitch in nodes (multiple of 4, >= nx)
    long long count, plane;         // px*ny*nz, px*ny
    Real h, lambda, mu, density;    // uniform material (used when the material arrays are null)
    Real hinv;                      // RN(1/h)
    int hinvExact;                  // h is a power of two (or FP32): x/h = x*hinv
    int rhoRecip;                   // every density lies in divBy's divisor range [2^-20, 2^20]
    const Real *metric[9];          // d(xi,eta,zeta)/d(x,y,z), row-major 3x3 per node
    const Real *jac, *damping, *source, *sg[3];
    const Real *mlambda, *mmu, *mdensity;
    const Real *normals;            // 3 per surface node (i + px*j)
    Real sdir[3];
    int src_i0, src_i1, src_j0, src_j1, src_k0, src_k1;
    int dmp_i0, dmp_i1, dmp_j0, dmp_j1, dmp_k1; // damping is zero inside this box
    // CFS-PML ADE (this library's 3D extension of the 2D ADE, src/two_d/PointKernels2D.hpp:50-64):
    // slabs of wx computational nodes on both x sides, wy on both y sides and wz at the bottom;
    // (d, kappa, alpha) per computational index along each axis; six memories per active axis of
    // a node (the axis derivative of Vx, Vy, Vz, then the axis part of the three momentum sums).
    int cpml;
    int wx, wy, wz;
    const Real *cpx, *cpy, *cpz;
    // GSLS (this library's 3D extension of the 2D relaxation, src/two_d/PointKernels2D.hpp:161-168):
    // mech mechanisms, whose memories (xx, yy, zz, xy, xz, yz) are fields 9 + 6l .. 14 + 6l
    int mech;
    Real rates[3];
    const Real *dP[3], *dS[3];
};

using k2::Clock;

template <class Real> struct StageArgs {
    Mesh<Real> m;
    const Real *in;
    Real *out;
    const Real *base;
    Real *acc;
    const Real *forcing; // 3 per step: source at t, t+dt/2, t+dt
    const Clock *clock;
    Real weight;         // stage combine weight: dt/2, dt/2, dt
    Real w6, w3;         // dt/6, dt/3
    double *surfRate;    // stage 3: |traction rate| and rate norm per surface node (2 x px*ny)
    const Real *cin;     // FP32 only: Kahan compensation of U (read) and of the new state (written)
    Real *cout;
    // CFS-PML memories, the same set scheme as the fields: stage input, stage output, U, A and the
    // FP32 compensation of U (read) and of the new memories (written)
    const Real *pin;
    Real *pout;
    const Real *pbase;
    Real *pacc;
    const Real *pcin;
    Real *pcout;
};

// Compact memory slots of padded node (i, j, k) along each axis (-1 outside that axis's slab):
// x slots 6*((kc*NY + jc)*2wx + s), then y slots 6*((kc*2wy + s)*NX + ic), then z slots
// 6*(((kc - (NZ-wz))*NY + jc)*NX + ic), over the computational indices ic, jc, kc.
template <class Real> __device__ __forceinline__ void cpmlSlots3(const Mesh<Real> &m, int i, int j, int k, long long (&slot)[3]) {
    const int ic = i - 3, jc = j - 3, kc = k - 3, NX = m.nx - 6, NY = m.ny - 6, NZ = m.nz - 6;
    const long long c0 = 6LL * 2 * m.wx * NY * NZ, c1 = 6LL * 2 * m.wy * NX * NZ;
    int s = ic < m.wx ? ic : ic >= NX - m.wx ? m.wx + ic - (NX - m.wx) : -1;
    slot[0] = s >= 0 ? 6 * (((long long)kc * NY + jc) * 2 * m.wx + s) : -1;
    s = jc < m.wy ? jc : jc >= NY - m.wy ? m.wy + jc - (NY - m.wy) : -1;
    slot[1] = s >= 0 ? c0 + 6 * (((long long)kc * 2 * m.wy + s) * NX + ic) : -1;
    slot[2] = kc >= NZ - m.wz ? c0 + c1 + 6 * (((long long)(kc - (NZ - m.wz)) * NY + jc) * NX + ic) : -1;
}

// RK combine of one value of a set (the fields' scheme, finish3): base, acc, out and the FP32
// compensation in and out.  Used for the CFS-PML memories and the GSLS memory fields.
template <class Real, int STAGE>
__device__ __forceinline__ void combineValue3(const StageArgs<Real> &p, const Real *base, Real *acc, Real *out, const Real *cin,
                                              Real *cout, long long at, Real r) {
    const Real u = (STAGE < 3 || k2::kahan<Real>()) ? k2::ld(base + at) : Real(0);
    if (STAGE == 0) {
        acc[at] = k2::kahan<Real>() ? p.w6 * r : u + p.w6 * r;
        out[at] = u + p.weight * r;
    } else if (STAGE < 3) {
        const Real a = acc[at];
        acc[at] = a + p.w3 * r;
        out[at] = u + p.weight * r;
    } else if constexpr (k2::kahan<Real>()) {
        const Real a = acc[at], c = k2::ld(cin + at);
        const Real y = (a + p.w6 * r) - c;
        const Real o = u + y;
        cout[at] = (o - u) - y;
        acc[at] = o;
    } else {
        acc[at] = acc[at] + p.w6 * r;
    }
}
template <class Real, int STAGE> __device__ __forceinline__ void combineMemory3(const StageArgs<Real> &p, long long at, Real r) {
    combineValue3<Real, STAGE>(p, p.pbase, p.pacc, p.pout, p.pcin, p.pcout, at, r);
}

using k2::ld;

// x / h as the reference forms it: the product with 1/h when that is exact, else the correctly
// rounded FMA quotient (both equal the IEEE division bit for bit).
// The three momentum quotients of a node by its density from one reciprocal: divBy forms the
// correctly rounded quotient, the same value as the division.
template <class Real> __device__ __forceinline__ void byRho3(const Mesh<Real> &m, Real rho, Real (&r)[9], Real m0, Real m1, Real m2) {
    if (m.rhoRecip) {
        const Real rinv = Real(1) / rho;
        r[0] = k2::divBy(m0, rho, rinv);
        r[1] = k2::divBy(m1, rho, rinv);
        r[2] = k2::divBy(m2, rho, rinv);
    } else {
        byRho3(m, rho, r, m0, m1, m2);
    }
}
template <class Real, bool EXACT> __device__ __forceinline__ Real overH(const Mesh<Real> &m, Real r) {
    if constexpr (EXACT) return r * m.hinv;
    else return k2::divBy(r, m.h, m.hinv);
}
// DRP derivatives over a tap source v(o) = value at offset o along the axis
// (include/SeisCommon/FiniteDifference.hpp:14-26): 5 taps, and the 2- and 3-point one-sided
// stencils of depths 1 and 2.  Sums start from the first product (the reference adds it to
// zero: the same value up to the sign of a zero).
template <class Real, int DIR, bool EXACT, class V> __device__ __forceinline__ Real d5(const Mesh<Real> &m, V v) {
    Real r;
    if (DIR == 0) {
        r = Real(-.30874) * v(-1);
        r += Real(-.6326) * v(0);
        r += Real(1.233) * v(1);
        r += Real(-.3334) * v(2);
        r += Real(.04168) * v(3);
    } else {
        r = -Real(-.30874) * v(1);
        r += -Real(-.6326) * v(0);
        r += -Real(1.233) * v(-1);
        r += -Real(-.3334) * v(-2);
        r += -Real(.04168) * v(-3);
    }
    return overH<Real, EXACT>(m, r);
}
template <class Real, int DIR, bool EXACT, class V> __device__ __forceinline__ Real d2(const Mesh<Real> &m, V v) {
    Real r;
    if (DIR == 0) {
        r = Real(-1) * v(0);
        r += Real(1) * v(1);
    } else {
        r = -Real(-1) * v(0);
        r += -Real(1) * v(-1);
    }
    return overH<Real, EXACT>(m, r);
}
template <class Real, int DIR, bool EXACT, class V> __device__ __forceinline__ Real d3(const Mesh<Real> &m, V v) {
    const Real c0 = Real(-7) / Real(6), c1 = Real(8) / Real(6), c2 = Real(-1) / Real(6);
    Real r;
    if (DIR == 0) {
        r = c0 * v(0);
        r += c1 * v(1);
        r += c2 * v(2);
    } else {
        r = -c0 * v(0);
        r += -c1 * v(-1);
        r += -c2 * v(-2);
    }
    return overH<Real, EXACT>(m, r);
}

template <class Real>
__device__ __forceinline__ Real tractionFlux(const Mesh<Real> &m, const Real *__restrict__ w, long long qq, int axis, int comp) {
    const int F[3][3] = {{3, 6, 7}, {6, 4, 8}, {7, 8, 5}};
    Real v = Real(0);
#pragma unroll
    for (int a = 0; a < 3; ++a) v += ld(m.metric[3 * axis + a] + qq) * ld(w + F[comp][a] * m.count + qq);
    return ld(m.jac + qq) * v;
}

// src/three_d/PointKernels3D.hpp:73-91 (surface rows only; reads the stage input from global memory)
// `only` >= 0: that axis's part alone (the CFS-PML split).
template <class Real, int DX, int DY, int DZ>
__device__ __noinline__ Real surfaceMomentum(const Mesh<Real> &m, const Real *__restrict__ w, long long q, int comp, int depth, Real rho,
                                             int only = -1) {
    const Real C[5] = {Real(-.30874), Real(-.6326), Real(1.233), Real(-.3334), Real(.04168)};
    Real sum = Real(0);
    for (int axis = 0; axis < 3; ++axis) {
        if (only >= 0 && axis != only) continue;
        const int dir = axis == 0 ? DX : axis == 1 ? DY : DZ;
        const long long s = axis == 0 ? 1 : axis == 1 ? m.px : m.plane;
        for (int l = 0; l < 5; ++l) {
            const int pos = l - 1;
            int off = dir ? -pos : pos;
            const Real c = dir ? -C[l] : C[l];
            Real sign = Real(1);
            if (axis == 2) {
                const int z = depth + off;
                if (z == 0) continue;
                if (z < 0) {
                    off = -z - depth;
                    sign = Real(-1);
                }
            }
            sum += sign * c * tractionFlux(m, w, q + off * s, axis, comp);
        }
    }
    return sum / (m.h * ld(m.jac + q) * rho);
}

// The same derivatives with their taps read from global memory along stride s around node q.
template <class Real, int DIR, bool EXACT>
__device__ __forceinline__ Real gd5(const Real *__restrict__ v, long long q, long long s, const Mesh<Real> &m) {
    return d5<Real, DIR, EXACT>(m, [&](int o) { return ld(v + q + o * s); });
}
template <class Real, int DIR, bool EXACT>
__device__ __forceinline__ Real gd2(const Real *__restrict__ v, long long q, long long s, const Mesh<Real> &m) {
    return d2<Real, DIR, EXACT>(m, [&](int o) { return ld(v + q + o * s); });
}
template <class Real, int DIR, bool EXACT>
__device__ __forceinline__ Real gd3(const Real *__restrict__ v, long long q, long long s, const Mesh<Real> &m) {
    return d3<Real, DIR, EXACT>(m, [&](int o) { return ld(v + q + o * s); });
}
// Four CTAs of 256 threads per SM (64 registers).  The kernel waits on its L1/L2 loads, and the
// extra resident warps hide more of that latency than the spills this bound costs: measured at
// 400x288x200, the stages run 1.3x faster with three CTAs per SM than with two, and 1.09x faster
// again with four.
template <class Real> constexpr int minBlocks3() { return 4; }

// RK combine, surface projection and stores of the nine rates of one node.  Every global load is
// issued before the first store: the stores could alias the loaded arrays as far as the compiler
// knows, and interleaving them serialised nine round trips per node (stages 1 and 2 ran 1.5x
// longer than stage 0 that way).
template <class Real, int STAGE>
__device__ __forceinline__ void finish3(const StageArgs<Real> &p, const Real (&r)[9], long long q, int depth, long long sq) {
    const Mesh<Real> &m = p.m;
    const long long n = m.count;
    // FP64: A = U + dt/6 k1, A += dt/3 k2, A += dt/3 k3, new = A + dt/6 k4 (the reference's
    // order).  FP32: A accumulates the increment alone (A = dt/6 k1, ...), and stage 3 adds
    // d = A + dt/6 k4 to U by Kahan's compensated summation (y = d - c, t = U + y,
    // c' = (t - U) - y).
    Real u[9], a[9], c[9], o[9], na[9], comp[9];
#pragma unroll
    for (int f = 0; f < 9; ++f) {
        u[f] = (STAGE < 3 || k2::kahan<Real>()) ? ld(p.base + f * n + q) : Real(0);
        a[f] = STAGE > 0 ? p.acc[f * n + q] : Real(0);
        c[f] = STAGE == 3 && k2::kahan<Real>() ? ld(p.cin + f * n + q) : Real(0);
    }
#pragma unroll
    for (int f = 0; f < 9; ++f) {
        if (STAGE == 0) {
            na[f] = k2::kahan<Real>() ? p.w6 * r[f] : u[f] + p.w6 * r[f];
            o[f] = u[f] + p.weight * r[f];
        } else if (STAGE < 3) {
            na[f] = a[f] + p.w3 * r[f];
            o[f] = u[f] + p.weight * r[f];
        } else if constexpr (k2::kahan<Real>()) {
            const Real y = (a[f] + p.w6 * r[f]) - c[f];
            o[f] = u[f] + y;
            comp[f] = (o[f] - u[f]) - y;
        } else {
            o[f] = a[f] + p.w6 * r[f];
        }
    }
    if (STAGE < 3)
#pragma unroll
        for (int f = 0; f < 9; ++f) p.acc[f * n + q] = na[f];
    if (depth == 0) { // tangential stress projection (PointKernels3D.hpp:36-51)
        const Real nn[3] = {ld(m.normals + 3 * sq), ld(m.normals + 3 * sq + 1), ld(m.normals + 3 * sq + 2)};
        const Real s[9] = {o[3], o[6], o[7], o[6], o[4], o[8], o[7], o[8], o[5]};
        Real t[3] = {0, 0, 0}, x[9];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) t[a] += s[3 * a + b] * nn[b];
        const Real nnn = t[0] * nn[0] + t[1] * nn[1] + t[2] * nn[2];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) x[3 * a + b] = s[3 * a + b] - nn[a] * t[b] - t[a] * nn[b] + nnn * nn[a] * nn[b];
        o[3] = x[0];
        o[4] = x[4];
        o[5] = x[8];
        o[6] = Real(0.5) * (x[1] + x[3]);
        o[7] = Real(0.5) * (x[2] + x[6]);
        o[8] = Real(0.5) * (x[5] + x[7]);
    }
    Real *dst = STAGE == 3 ? p.acc : p.out;
#pragma unroll
    for (int f = 0; f < 9; ++f) dst[f * n + q] = o[f];
    if (STAGE == 3 && k2::kahan<Real>())
#pragma unroll
        for (int f = 0; f < 9; ++f) p.cout[f * n + q] = comp[f];
}

// The general node: surface rows (traction-free derivative, traction-image momentum,
// projection) and the source support, with sponge damping where it applies.
template <class Real, int DX, int DY, int DZ, int STAGE, bool EXACT, bool CPML>
__device__ __forceinline__ void stageBody3(const StageArgs<Real> &p) {
    const Mesh<Real> &m = p.m;
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 3 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 3 + blockIdx.z;
    if (i >= m.nx - 3 || j >= m.ny - 3) return;
    const Clock *clk = p.clock;
    const long long n = m.count, nx = m.px, plane = m.plane;
    const long long q = i + nx * j + plane * k;
    const int depth = k - 3;
    const Real *__restrict__ w = p.in;
    const Real lam = m.mlambda ? ld(m.mlambda + q) : m.lambda;
    const Real mu = m.mmu ? ld(m.mmu + q) : m.mu;
    const Real rho = m.mdensity ? ld(m.mdensity + q) : m.density;
    Real M[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) M[c] = ld(m.metric[c] + q);

    // CFS-PML: the node's memory slots and the rates of its memories
    long long slot[3] = {-1, -1, -1};
    if constexpr (CPML)
        if (m.cpml) cpmlSlots3(m, i, j, k, slot);
    const bool split = CPML && (slot[0] >= 0 || slot[1] >= 0 || slot[2] >= 0);
    Real prate[3][6];
    auto stretchAxis = [&](int a, int f, Real d) -> Real {
        if (slot[a] < 0) return d;
        const Real *prof = (a == 0 ? m.cpx + 3 * (i - 3) : a == 1 ? m.cpy + 3 * (j - 3) : m.cpz + 3 * (k - 3));
        return k2::stretch(prof, ld(p.pin + slot[a] + f), d, prate[a][f]);
    };
    // raw xi / eta derivatives of the velocities (also used by the surface solve), stretched in a slab
    Real dv[3][2];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        dv[v][0] = gd5<Real, DX, EXACT>(w + v * n, q, 1, m);
        dv[v][1] = gd5<Real, DY, EXACT>(w + v * n, q, nx, m);
        if (split) dv[v][0] = stretchAxis(0, v, dv[v][0]), dv[v][1] = stretchAxis(1, v, dv[v][1]);
    }
    Real dzs[3] = {0, 0, 0};
    if (depth == 0) { // src/three_d/PointKernels3D.hpp:52-66
        const Real c[3] = {M[6], M[7], M[8]};
        const Real c2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2], len = sqrt(c2);
        const Real nn[3] = {c[0] / len, c[1] / len, c[2] / len};
        Real g[9], t[3] = {0, 0, 0};
#pragma unroll
        for (int v = 0; v < 3; ++v)
#pragma unroll
            for (int a = 0; a < 3; ++a) g[3 * v + a] = M[a] * dv[v][0] + M[3 + a] * dv[v][1];
        const Real trace = g[0] + g[4] + g[8];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) t[a] += ((a == b ? lam * trace : Real(0)) + mu * (g[3 * a + b] + g[3 * b + a])) * c[b];
        if constexpr (CPML) { // GSLS: the memory stresses' traction (the 2D surfaceDerivative's, PointKernels2D.hpp:84)
            const int T[3][3] = {{0, 3, 4}, {3, 1, 5}, {4, 5, 2}};
            for (int l = 0; l < m.mech; ++l) {
                const Real *mw = w + (9 + 6 * l) * n + q;
#pragma unroll
                for (int a = 0; a < 3; ++a)
                    t[a] -= (ld(mw + T[a][0] * n) * c[0] + ld(mw + T[a][1] * n) * c[1]) + ld(mw + T[a][2] * n) * c[2];
            }
        }
        const Real normal = t[0] * nn[0] + t[1] * nn[1] + t[2] * nn[2];
#pragma unroll
        for (int a = 0; a < 3; ++a) dzs[a] = -(t[a] - nn[a] * normal) / (mu * c2) - nn[a] * normal / ((lam + 2 * mu) * c2);
    }
    Real gr[9][3];
#pragma unroll
    for (int f = 0; f < 9; ++f) {
        Real dx, dy, dz;
        if (f < 3) {
            dx = dv[f][0];
            dy = dv[f][1];
            if (depth == 0) dz = dzs[f];
            else if (depth == 1) dz = gd2<Real, DZ, EXACT>(w + f * n, q, plane, m);
            else if (depth == 2) dz = gd3<Real, DZ, EXACT>(w + f * n, q, plane, m);
            else dz = gd5<Real, DZ, EXACT>(w + f * n, q, plane, m);
            if (split) dz = stretchAxis(2, f, dz);
        } else if (split) {
            continue; // a slab node takes its stress derivatives per axis, below
        } else {
            dx = gd5<Real, DX, EXACT>(w + f * n, q, 1, m);
            dy = gd5<Real, DY, EXACT>(w + f * n, q, nx, m);
            dz = gd5<Real, DZ, EXACT>(w + f * n, q, plane, m);
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) gr[f][a] = M[a] * dx + M[3 + a] * dy + M[6 + a] * dz;
    }
    Real r[9];
    const bool near = depth <= (DZ ? 3 : 1);
    if (!split) {
        if (near) {
#pragma unroll
            for (int a = 0; a < 3; ++a) r[a] = surfaceMomentum<Real, DX, DY, DZ>(m, w, q, a, depth, rho);
        } else {
            byRho3(m, rho, r, (gr[3][0] + gr[6][1]) + gr[7][2], (gr[6][0] + gr[4][1]) + gr[8][2], (gr[7][0] + gr[8][1]) + gr[5][2]);
        }
    } else {
        // the momentum of a slab node summed per axis: for axis a the part
        // (d(xi_a)/dx dS_c0 + d(xi_a)/dy dS_c1 + d(xi_a)/dz dS_c2)/rho of the a-derivatives, each part
        // stretched where the axis is active, then x + y + z
        const int F[3][3] = {{3, 6, 7}, {6, 4, 8}, {7, 8, 5}};
        const Real rinv = m.rhoRecip ? Real(1) / rho : Real(0);
        auto byRho = [&](Real x) { return m.rhoRecip ? k2::divBy(x, rho, rinv) : x / rho; };
        auto gda = [&](int a, int f) {
            return a == 0 ? gd5<Real, DX, EXACT>(w + f * n, q, 1, m) : a == 1 ? gd5<Real, DY, EXACT>(w + f * n, q, nx, m)
                                                                         : gd5<Real, DZ, EXACT>(w + f * n, q, plane, m);
        };
#pragma unroll 1
        for (int c = 0; c < 3; ++c) {
            Real part[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (near) part[a] = surfaceMomentum<Real, DX, DY, DZ>(m, w, q, c, depth, rho, a);
                else part[a] = byRho((M[3 * a] * gda(a, F[c][0]) + M[3 * a + 1] * gda(a, F[c][1])) + M[3 * a + 2] * gda(a, F[c][2]));
                part[a] = stretchAxis(a, 3 + c, part[a]);
            }
            r[c] = (part[0] + part[1]) + part[2];
        }
    }
    if (i >= m.src_i0 && i < m.src_i1 && j >= m.src_j0 && j < m.src_j1 && k >= m.src_k0 && k < m.src_k1) {
        const Real s = p.forcing[3 * (clk->step - clk->first) + (STAGE == 0 ? 0 : STAGE == 3 ? 2 : 1)];
        const Real ratio = m.density / rho;
#pragma unroll
        for (int a = 0; a < 3; ++a) r[a] += s * (m.sg[a] ? ld(m.sg[a] + q) : ld(m.source + q) * m.sdir[a]) * ratio;
    }
    const Real div = gr[0][0] + gr[1][1] + gr[2][2];
    r[3] = lam * div + 2 * mu * gr[0][0];
    r[4] = lam * div + 2 * mu * gr[1][1];
    r[5] = lam * div + 2 * mu * gr[2][2];
    r[6] = mu * (gr[0][1] + gr[1][0]);
    r[7] = mu * (gr[0][2] + gr[2][0]);
    r[8] = mu * (gr[1][2] + gr[2][1]);
    const bool damped = !(i >= m.dmp_i0 && i < m.dmp_i1 && j >= m.dmp_j0 && j < m.dmp_j1 && k < m.dmp_k1);
    if constexpr (CPML) { // GSLS: the stresses subtract the memories; memory rate = rate (drive - memory)
        for (int l = 0; l < m.mech; ++l) {
            const long long mm = (9 + 6 * l) * n + q;
            const Real dp = ld(m.dP[l] + q), ds = ld(m.dS[l] + q), dl = dp - 2 * ds;
            const Real drive[6] = {dl * div + 2 * ds * gr[0][0], dl * div + 2 * ds * gr[1][1], dl * div + 2 * ds * gr[2][2],
                                   ds * (gr[0][1] + gr[1][0]),  ds * (gr[0][2] + gr[2][0]),  ds * (gr[1][2] + gr[2][1])};
            Real wm[6];
#pragma unroll
            for (int c = 0; c < 6; ++c) wm[c] = ld(w + mm + c * n);
#pragma unroll
            for (int c = 0; c < 6; ++c) r[3 + c] -= wm[c];
            const Real d = damped ? ld(m.damping + q) : Real(0);
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                Real rm = m.rates[l] * (drive[c] - wm[c]);
                if (damped) rm -= d * wm[c];
                combineValue3<Real, STAGE>(p, p.base, p.acc, STAGE < 3 ? p.out : p.acc, p.cin, p.cout, mm + c * n, rm);
            }
        }
    }
    if (damped) {
        const Real d = ld(m.damping + q);
#pragma unroll
        for (int f = 0; f < 9; ++f) r[f] -= d * ld(w + f * n + q);
    }
    const long long sq = i + nx * j; // surface index
    if (STAGE == 3 && depth == 0 && p.surfRate) {
        // traction-rate residual of k4 (src/three_d/CurvilinearSolver.cpp:231-239)
        const double n0 = ld(m.normals + 3 * sq), n1 = ld(m.normals + 3 * sq + 1), n2 = ld(m.normals + 3 * sq + 2);
        const double t0 = double(r[3]) * n0 + double(r[6]) * n1 + double(r[7]) * n2;
        const double t1 = double(r[6]) * n0 + double(r[4]) * n1 + double(r[8]) * n2;
        const double t2 = double(r[7]) * n0 + double(r[8]) * n1 + double(r[5]) * n2;
        double norm2 = 0;
#pragma unroll
        for (int f = 3; f < 9; ++f) norm2 += (f >= 6 ? 2.0 : 1.0) * double(r[f]) * double(r[f]);
        p.surfRate[sq] = sqrt(t0 * t0 + t1 * t1 + t2 * t2);
        p.surfRate[plane + sq] = sqrt(norm2);
    }
    finish3<Real, STAGE>(p, r, q, depth, sq);
    if (split)
        for (int a = 0; a < 3; ++a)
            if (slot[a] >= 0)
#pragma unroll
                for (int f = 0; f < 6; ++f) combineMemory3<Real, STAGE>(p, slot[a] + f, prate[a][f]);
}

// The interior node (below the surface rows, outside the source support), with the sponge's
// damping term when DAMP.  The stress fields are differentiated one at a time and their physical
// gradients folded into the momentum sums as they come, in the reference's order
// r0 = (gxx,x + gxy,y) + gxz,z, r1 = (gxy,x + gyy,y) + gyz,z, r2 = (gxz,x + gyz,y) + gzz,z
// (src/three_d/PointKernels3D.hpp:92-112), so only a few gradients are live at a time.  The
// damping term is subtracted after all nine rates, as in the general form.
template <class Real, int DX, int DY, int DZ, int STAGE, bool EXACT, bool DAMP, bool GSLS>
__device__ __forceinline__ void stageInterior3(const StageArgs<Real> &p) {
    const Mesh<Real> &m = p.m;
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 3 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 3 + blockIdx.z;
    if (i >= m.nx - 3 || j >= m.ny - 3) return;
    const long long n = m.count, nx = m.px, plane = m.plane;
    const long long q = i + nx * j + plane * k;
    const Real *__restrict__ w = p.in;
    Real M[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) M[c] = ld(m.metric[c] + q);
    // physical gradient component a of field f: ((M_a dxi + M_3+a deta) + M_6+a dzeta)
    auto grad = [&](int f, Real (&g)[3], bool x, bool y, bool z) {
        const Real dx = gd5<Real, DX, EXACT>(w + f * n, q, 1, m);
        const Real dy = gd5<Real, DY, EXACT>(w + f * n, q, nx, m);
        const Real dz = gd5<Real, DZ, EXACT>(w + f * n, q, plane, m);
        if (x) g[0] = M[0] * dx + M[3] * dy + M[6] * dz;
        if (y) g[1] = M[1] * dx + M[4] * dy + M[7] * dz;
        if (z) g[2] = M[2] * dx + M[5] * dy + M[8] * dz;
    };
    Real r[9];
    {
        Real gv[3][3];
#pragma unroll
        for (int v = 0; v < 3; ++v) grad(v, gv[v], true, true, true);
        const Real lam = m.mlambda ? ld(m.mlambda + q) : m.lambda;
        const Real mu = m.mmu ? ld(m.mmu + q) : m.mu;
        const Real div = gv[0][0] + gv[1][1] + gv[2][2];
        r[3] = lam * div + 2 * mu * gv[0][0];
        r[4] = lam * div + 2 * mu * gv[1][1];
        r[5] = lam * div + 2 * mu * gv[2][2];
        r[6] = mu * (gv[0][1] + gv[1][0]);
        r[7] = mu * (gv[0][2] + gv[2][0]);
        r[8] = mu * (gv[1][2] + gv[2][1]);
        if constexpr (GSLS) { // the general form's relaxation, with the same operations in the same order
            const bool damped = DAMP && !(i >= m.dmp_i0 && i < m.dmp_i1 && j >= m.dmp_j0 && j < m.dmp_j1 && k < m.dmp_k1);
            for (int l = 0; l < m.mech; ++l) {
                const long long mm = (9 + 6 * l) * n + q;
                const Real dp = ld(m.dP[l] + q), ds = ld(m.dS[l] + q), dl = dp - 2 * ds;
                const Real drive[6] = {dl * div + 2 * ds * gv[0][0], dl * div + 2 * ds * gv[1][1], dl * div + 2 * ds * gv[2][2],
                                       ds * (gv[0][1] + gv[1][0]),  ds * (gv[0][2] + gv[2][0]),  ds * (gv[1][2] + gv[2][1])};
                Real wm[6];
#pragma unroll
                for (int c = 0; c < 6; ++c) wm[c] = ld(w + mm + c * n);
#pragma unroll
                for (int c = 0; c < 6; ++c) r[3 + c] -= wm[c];
                const Real d = damped ? ld(m.damping + q) : Real(0);
#pragma unroll
                for (int c = 0; c < 6; ++c) {
                    Real rm = m.rates[l] * (drive[c] - wm[c]);
                    if (damped) rm -= d * wm[c];
                    combineValue3<Real, STAGE>(p, p.base, p.acc, STAGE < 3 ? p.out : p.acc, p.cin, p.cout, mm + c * n, rm);
                }
            }
        }
    }
    {
        Real g[3], m0, m1, m2, t41, t52, t70;
        grad(3, g, true, false, false), m0 = g[0];
        grad(4, g, false, true, false), t41 = g[1];
        grad(5, g, false, false, true), t52 = g[2];
        grad(6, g, true, true, false), m0 = m0 + g[1], m1 = g[0] + t41;
        grad(7, g, true, false, true), m0 = m0 + g[2], t70 = g[0];
        grad(8, g, false, true, true), m1 = m1 + g[2], m2 = (t70 + g[1]) + t52;
        const Real rho = m.mdensity ? ld(m.mdensity + q) : m.density;
        byRho3(m, rho, r, m0, m1, m2);
    }
    if (DAMP && !(i >= m.dmp_i0 && i < m.dmp_i1 && j >= m.dmp_j0 && j < m.dmp_j1 && k < m.dmp_k1)) {
        const Real d = ld(m.damping + q);
#pragma unroll
        for (int f = 0; f < 9; ++f) r[f] -= d * ld(w + f * n + q);
    }
    finish3<Real, STAGE>(p, r, q, 4, i + nx * j);
}

template <class Real, int DX, int DY, int DZ, int STAGE, bool EXACT, bool CPML>
__device__ __forceinline__ void stageNode3(const StageArgs<Real> &p, bool general, bool sponge) {
    if (general) stageBody3<Real, DX, DY, DZ, STAGE, EXACT, CPML>(p);
    else if (CPML && p.m.mech > 0) { // GSLS outside the CFS-PML slabs
        if (sponge) stageInterior3<Real, DX, DY, DZ, STAGE, EXACT, true, CPML>(p);
        else stageInterior3<Real, DX, DY, DZ, STAGE, EXACT, false, CPML>(p);
    } else if (sponge) stageInterior3<Real, DX, DY, DZ, STAGE, EXACT, true, false>(p);
    else stageInterior3<Real, DX, DY, DZ, STAGE, EXACT, false, false>(p);
}

// One RK stage of a 3D shot: block 32x8 nodes of one z layer.  CTAs on the surface rows or on
// the source support run the general form; the others run the interior form, with the damping
// term when the CTA reaches into the sponge (so the sponge costs nine multiply-adds, not the
// general form).  CPML: the mesh has CFS-PML slabs or GSLS memories; CTAs that reach into a slab
// run the general form with the ADE terms, and with GSLS the interior form carries the relaxation
// too.  Plain meshes launch the CPML = false kernels, which hold none of that code.
template <class Real, int DX, int DY, int DZ, int STAGE, bool CPML>
__global__ void __launch_bounds__(256, (minBlocks3<Real>())) stage3d(const __grid_constant__ StageArgs<Real> p) {
    const Mesh<Real> &m = p.m;
    if (p.clock->faulted) return;
    const int i0 = 3 + blockIdx.x * blockDim.x, i1 = i0 + blockDim.x, j0 = 3 + blockIdx.y * blockDim.y, j1 = j0 + blockDim.y;
    const int k = 3 + blockIdx.z;
    const bool surface = k < 7;
    const bool source = i0 < m.src_i1 && i1 > m.src_i0 && j0 < m.src_j1 && j1 > m.src_j0 && k >= m.src_k0 && k < m.src_k1;
    const bool sponge = !(i0 >= m.dmp_i0 && i1 <= m.dmp_i1 && j0 >= m.dmp_j0 && j1 <= m.dmp_j1 && k < m.dmp_k1);
    // CTAs reaching into a CFS-PML slab run the general form (it holds the ADE terms)
    const bool slab = CPML && m.cpml &&
                      (i0 - 3 < m.wx || i1 - 3 > m.nx - 6 - m.wx || j0 - 3 < m.wy || j1 - 3 > m.ny - 6 - m.wy || k - 3 >= m.nz - 6 - m.wz);
    const bool general = surface || source || slab;
    if constexpr (sizeof(Real) == 4) stageNode3<Real, DX, DY, DZ, STAGE, true, CPML>(p, general, sponge);
    else if (m.hinvExact) stageNode3<Real, DX, DY, DZ, STAGE, true, CPML>(p, general, sponge);
    else stageNode3<Real, DX, DY, DZ, STAGE, false, CPML>(p, general, sponge);
}

struct Partial {
    double energy, velocity, rateTraction, rateNorm;
    double peak[5];
    int bad, pad;
};

// One partial per CTA from the per-thread diagnostics: warp shuffles, then the CTA's warps in order.
__device__ __forceinline__ void reducePartial3(Partial s, Partial *out, int slot) {
    for (int o = 16; o > 0; o >>= 1) {
        s.energy += __shfl_down_sync(0xffffffffu, s.energy, o);
        s.velocity = fmax(s.velocity, __shfl_down_sync(0xffffffffu, s.velocity, o));
        s.rateTraction = fmax(s.rateTraction, __shfl_down_sync(0xffffffffu, s.rateTraction, o));
        s.rateNorm = fmax(s.rateNorm, __shfl_down_sync(0xffffffffu, s.rateNorm, o));
#pragma unroll
        for (int c = 0; c < 5; ++c) s.peak[c] = fmax(s.peak[c], __shfl_down_sync(0xffffffffu, s.peak[c], o));
        s.bad |= __shfl_down_sync(0xffffffffu, s.bad, o);
    }
    __shared__ Partial warps[8];
    const int t = threadIdx.x + blockDim.x * threadIdx.y, lane = t & 31, wid = t >> 5, nw = (blockDim.x * blockDim.y) >> 5;
    if (lane == 0) warps[wid] = s;
    __syncthreads();
    if (t == 0) {
        Partial tot = warps[0];
        for (int w = 1; w < nw; ++w) {
            const Partial &y = warps[w];
            tot.energy += y.energy;
            tot.velocity = fmax(tot.velocity, y.velocity);
            tot.rateTraction = fmax(tot.rateTraction, y.rateTraction);
            tot.rateNorm = fmax(tot.rateNorm, y.rateNorm);
            for (int c = 0; c < 5; ++c) tot.peak[c] = fmax(tot.peak[c], y.peak[c]);
            tot.bad |= y.bad;
        }
        out[slot] = tot;
    }
}

// Energy, peaks, finiteness and the traction-rate residual of a state
// (src/three_d/CurvilinearSolver.cpp:214-250, CudaEngine3D.cu:36-55), one partial per CTA of 32 x 8
// columns over STATS_LAYERS z layers (fewer partials for the one-block verdict to read).  Each
// thread issues the thirteen loads of a node (nine fields, lambda, mu, rho, J) ahead of its
// arithmetic; the CTA reduces by warp shuffles.
constexpr int STATS_LAYERS = 8;
template <class Real>
__global__ void __launch_bounds__(256) stats3d(const Mesh<Real> m, const Real *__restrict__ w, const double *__restrict__ surfRate,
                                               const Clock *clk, Partial *out) {
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 3 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k0 = 3 + blockIdx.z * STATS_LAYERS;
    Partial s{};
    if (i < m.nx - 3 && j < m.ny - 3 && !(clk && clk->faulted)) {
        const long long n = m.count;
        const double hh = double(m.h);
        for (int k = k0; k < k0 + STATS_LAYERS && k < m.nz - 3; ++k) {
            const long long q = i + (long long)m.px * j + m.plane * k;
            double f[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) f[c] = double(ld(w + c * n + q));
            const double lam = m.mlambda ? double(ld(m.mlambda + q)) : double(m.lambda);
            const double mu = m.mmu ? double(ld(m.mmu + q)) : double(m.mu);
            const double rho = m.mdensity ? double(ld(m.mdensity + q)) : double(m.density);
            const double jac = double(ld(m.jac + q));
#pragma unroll
            for (int c = 0; c < 9; ++c)
                if (!isfinite(f[c])) s.bad = 1;
            const double v2 = f[0] * f[0] + f[1] * f[1] + f[2] * f[2], v = sqrt(v2);
            const double mean = (f[3] + f[4] + f[5]) / 3;
            s.velocity = fmax(s.velocity, v);
            s.peak[0] = fmax(s.peak[0], fabs(f[2])), s.peak[1] = fmax(s.peak[1], fabs(f[0]));
            s.peak[2] = fmax(s.peak[2], fabs(f[1])), s.peak[3] = fmax(s.peak[3], v);
            s.peak[4] = fmax(s.peak[4], fabs((f[3] + f[4] + f[5]) / 3.0));
            double dev = 0;
#pragma unroll
            for (int c = 0; c < 3; ++c) dev += (f[c + 3] - mean) * (f[c + 3] - mean);
#pragma unroll
            for (int c = 6; c < 9; ++c) dev += 2 * f[c] * f[c];
            const double e = (0.5 * rho * v2 + dev / (4 * mu) + mean * mean / (2 * (lam + 2 * mu / 3))) * jac * hh * hh * hh;
            if (!isfinite(e)) s.bad = 1;
            s.energy += e;
        }
        if (k0 == 3 && surfRate) {
            const long long sq = i + (long long)m.px * j;
            s.rateTraction = surfRate[sq];
            s.rateNorm = surfRate[m.plane + sq];
        }
    }
    reducePartial3(s, out, blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z));
}

struct Clock3 {
    double sourcePeak;
};

// Acceptance rule of CpuSimulation3D::advance (src/three_d/CurvilinearSolver.cpp:475-488):
// non-finite fields, or energy above 1e4 x the peak of the source window (t <= 3/f).
template <class Real>
__global__ void __launch_bounds__(512) verdict3d(const Partial *__restrict__ parts, int nparts, const Real *__restrict__ w,
                                                  long long count, const long long *__restrict__ receivers, int nrec,
                                                  double *__restrict__ traces, Clock *clk) {
    __shared__ Partial sh[512];
    __shared__ int accept;
    const int t = threadIdx.x;
    if (clk->faulted) return;
    Partial s{};
    for (int b = t; b < nparts; b += blockDim.x) {
        const Partial y = parts[b];
        s.energy += y.energy;
        s.velocity = fmax(s.velocity, y.velocity);
        s.rateTraction = fmax(s.rateTraction, y.rateTraction);
        s.rateNorm = fmax(s.rateNorm, y.rateNorm);
        for (int c = 0; c < 5; ++c) s.peak[c] = fmax(s.peak[c], y.peak[c]);
        s.bad |= y.bad;
    }
    sh[t] = s;
    __syncthreads();
    for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
        if (t < stride) {
            Partial &x = sh[t];
            const Partial y = sh[t + stride];
            x.energy += y.energy;
            x.velocity = fmax(x.velocity, y.velocity);
            x.rateTraction = fmax(x.rateTraction, y.rateTraction);
            x.rateNorm = fmax(x.rateNorm, y.rateNorm);
            for (int c = 0; c < 5; ++c) x.peak[c] = fmax(x.peak[c], y.peak[c]);
            x.bad |= y.bad;
        }
        __syncthreads();
    }
    if (t == 0) {
        const Partial tot = sh[0];
        const double ratio = tot.rateTraction / fmax(tot.rateNorm, 1.0e-30);
        const bool finite = !tot.bad && isfinite(tot.energy) && isfinite(ratio);
        const double tnext = (clk->step + 1) * clk->dt;
        // the source-window peak lives in peak_energy
        double peak = clk->peak_energy;
        if (tnext <= clk->growth_after) peak = fmax(peak, tot.energy);
        const bool growth = tnext > clk->growth_after && peak > 0 && tot.energy > 1e4 * peak;
        const int ok = finite && !growth;
        clk->finite = finite;
        if (ok) {
            clk->peak_energy = peak;
            clk->energy = tot.energy;
            clk->max_velocity = tot.velocity;
            clk->traction = ratio;
            for (int c = 0; c < 5; ++c) clk->peaks[c] = tot.peak[c];
        }
        accept = ok;
    }
    __syncthreads();
    if (!accept) {
        if (t == 0) clk->faulted = 1, clk->fault_step = clk->step;
        return;
    }
    const int row = clk->step - clk->first;
    if (row < clk->trace_steps)
        for (int r = t; r < nrec; r += blockDim.x) {
            const long long qq = receivers[r];
            for (int c = 0; c < 3; ++c) traces[((long long)row * nrec + r) * 3 + c] = double(w[c * count + qq]);
        }
    __syncthreads();
    if (t == 0) clk->step += 1, clk->accepted += 1;
}

} // namespace swl::k3
