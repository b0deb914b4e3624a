// 2D P-SV / GSLS device code: one fused kernel per classic-RK4 stage.
//
// Each stage kernel evaluates, per node, the MacCormack-DRP derivatives of the five stencil
// fields (Vx, Vz, Sxx, Szz, Sxz), the metric-transformed right-hand side
// (src/two_d/PointKernels2D.hpp:121-172) with the traction-image surface rows, CFS-PML ADE
// memories and GSLS relaxation, and immediately its part of the RK combine and the
// free-surface projection -- the rates never touch HBM.  A CTA walks a 32-column strip down 64
// rows, 8 rows at a time, with the five stencil fields (a ring of rows), U, A and the model words
// staged in shared memory by tensor copies one row block ahead of the arithmetic; the GSLS
// fields (Syy and the memories, index >= 5) and strengths are read from global memory per node.
// Three state sets stay resident beside the stage outputs:
//   U (state at the start of the step), A (running RK accumulator), S (stage state).
// Stage 0 writes A = k1 and S = U + dt/2 k1; stages 1-2 add 2k to A and write
// S = U + w k; stage 3 writes U + dt (A + k4) / 6 over A and (optionally) reduces the
// diagnostics of the new state per CTA.  Sums are formed in the reference's order
// (src/two_d/CurvilinearSolver2D.cpp:80-97), so with FMA contraction off the FP64 results equal
// the reference CPU build's.
#pragma once
#include "runtime.cuh"
#include <cstdint>
#include <cuda.h>

namespace swl::k2 {

// Device view of the model (Point::MeshT, src/two_d/PointKernels2D.hpp:14-27), plus the
// boxes outside which the sparse source and sponge arrays are exactly zero.
// Arrays are stored with a row pitch: node (i, k) of the padded nx x nz grid lives at
// i + xoff + pitch * k, with pitch a multiple of 8 >= nx + 1 and xoff = 1, so that every row
// and every 32-column strip starts on a 16-byte boundary (the alignment tensor copies need).
template <class Real> struct Mesh {
    int nx, nz; // padded
    int pitch, xoff;
    long long count; // pitch * nz: the stride between fields
    int seg;         // row blocks per streaming segment (chosen per grid by the engine's tuner)
    Real h, hinv;   // hinv = RN(1/h); x/h is x*hinv when h is a power of two (or in FP32),
    int hinvExact;  // else the correctly rounded divBy(x, h, hinv)
    int rhoRecip;   // every density lies in divBy's divisor range: x/rho = divBy(x, rho, RN(1/rho))
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
    int stalled;     // set by a stage kernel whose copy wait ran out (the host reports an error)
    double peak_energy;
    double energy, max_velocity, traction;
    double peaks[5]; // 3D: |Vz|, |Vx|, |Vy|, |V|, |mean stress| of the last accepted step
    int finite;
    int accepted;    // steps accepted in this batch
    double dt, growth_after; // energy-growth rule applies when (step+1)*dt > growth_after
};

// Per-CTA diagnostics of a state (src/two_d/CudaEngine2D.cu:43-78 semantics).
struct Partial {
    double energy, velocity, traction;
    int bad, pad;
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
    // FP32 only: Kahan compensation of U (read) and of the new state (written by stage 3),
    // for the fields and for the CFS-PML memories
    const Real *cin;
    Real *cout;
    const Real *pcin;
    Real *pcout;
    const Real *forcing; // 3 values per step of the batch: t, t+dt/2, t+dt
    const Clock *clock;
    Real weight;         // dt/2, dt/2, dt for stages 0..2
    Real delta;          // dt
    Partial *partials;   // stage 3: per-CTA diagnostics of the new state (null: none)
    // Tensor maps of the streaming kernel (elastic only): the stage input as 40x8x5 boxes,
    // U, A and the compensation terms as 32x8x5 boxes, the model words as 32x8x5 (stages 0-2) or
    // 32x8x6 (stage 3, with J) boxes.
    CUtensorMap ringMap, uMap, aMap, modelMap, compMap;
    // GSLS only: the per-node words the node arithmetic reads from global memory -- Syy and the
    // 4L memories of the stage input, of U and of A (and their FP32 compensation), and the 2L
    // relaxation strengths -- as 32x8x(4L+1) and 32x8x2L boxes.  The CTA's copy thread prefetches a
    // row block's boxes into L2, so the per-node loads hit L2 instead of waiting on DRAM:
    // gslsPrefetch = 2 with the block's tensor copies (two blocks ahead of its arithmetic), 3 with the
    // copies of the block before it (three ahead), 1 when the block before it starts (one ahead), 0 off.
    CUtensorMap gslsInMap, gslsUMap, gslsAMap, gslsCompMap, strengthMap;
    int gslsPrefetch;
};

// The FP32 form adds each step's increment to the state with compensated (Kahan) summation;
// the FP64 form keeps the reference's plain sum.
template <class Real> constexpr bool kahan() { return sizeof(Real) == 4; }

template <class Real> __device__ __forceinline__ Real ld(const Real *p) { return __ldg(p); }
// Loads of state that the step itself writes (stage inputs, U, the ADE memories, the Kahan
// terms).  A stage kernel only reads arrays that the previous launches wrote, so they may take
// the read-only path; the persistent multi-shot kernel (queue2d.cuh) reads state that other CTAs
// wrote in the same launch, which the non-coherent read-only path may serve stale, so it is
// compiled with SWL_STAGE_COHERENT and uses ordinary cached loads (ld.global.ca), which see those
// writes after the acquire fence each work item starts with.
#ifdef SWL_STAGE_COHERENT
template <class Real> __device__ __forceinline__ Real lds(const Real *p) { return __ldca(p); }
#else
template <class Real> __device__ __forceinline__ Real lds(const Real *p) { return __ldg(p); }
#endif

// Correctly rounded y / 6 without a division instruction sequence.  y/6 = (y/2)/3 with y/2 exact,
// and x/3 by Markstein's correction (P. W. Markstein, "Computation of elementary functions on the
// IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990): with c = RN(1/3) -- here
// 3c = 1 - 2^-54 (FP32: 1 + 2^-25), so q0 = RN(x c) is within one ulp of x/3 -- the remainder
// r = x - 3 q0 is exact under an FMA and RN(q0 + r c) = RN(x/3).  The theorem excludes
// underflow, so tiny (but nonzero), huge and non-finite x take the plain division -- out of line,
// so that the compiler cannot evaluate that division speculatively on the common path.  A zero
// passes through the FMA form exactly.
template <class Real> __device__ __noinline__ Real plainDiv6(Real y) { return y / Real(6); }
template <class Real> __device__ __forceinline__ Real div6(Real y) {
    constexpr Real c = Real(1) / Real(3);
    constexpr Real tiny = sizeof(Real) == 8 ? Real(0x1p-960) : Real(0x1p-100f);
    constexpr Real huge = sizeof(Real) == 8 ? Real(0x1p+1000) : Real(0x1p+120f);
    const Real x = y * Real(0.5);
    const Real ax = fabs(x);
    if (!(ax <= huge) || (ax < tiny && ax != Real(0))) return plainDiv6(y);
    const Real q0 = x * c;
    const Real r = fma(-q0, Real(3), x);
    return fma(r, c, q0);
}

// Correctly rounded x / d from dinv = RN(1/d) without a division instruction sequence, by two
// Markstein corrections: q0 = RN(x dinv) is within 1.5 ulp of x/d, q1 = RN(q0 + (x - d q0) dinv)
// is within one ulp, and then RN(q1 + (x - d q1) dinv) = RN(x/d) (P. W. Markstein, IBM J. Res.
// Dev. 34(1), 1990; each remainder is exact under an FMA).  The divisor must lie in
// [2^-20, 2^20]; tiny (nonzero), huge and non-finite x take the plain division out of line.  FP64
// tests that window on the high word with integer instructions, which keeps the FP64 pipe for the
// arithmetic (3D FP64 steps 0.4 % faster than with three FP64 compares).
template <class Real> __device__ __noinline__ Real plainDiv(Real x, Real d) { return x / d; }
template <class Real> __device__ __forceinline__ Real divBy(Real x, Real d, Real dinv) {
    constexpr Real tiny = sizeof(Real) == 8 ? Real(0x1p-960) : Real(0x1p-100f);
    constexpr Real huge = sizeof(Real) == 8 ? Real(0x1p+1000) : Real(0x1p+100f);
    if constexpr (sizeof(Real) == 8) {
        // the same window from the high word on the integer pipe: 2^-960 <= |x| < 2^1000 (high words
        // 0x03f00000 .. 0x7e6fffff), or a zero
        const unsigned hi = unsigned(__double2hiint(double(x))) & 0x7fffffffu;
        if (hi - 0x03f00000u >= 0x7e700000u - 0x03f00000u && (hi | unsigned(__double2loint(double(x)))) != 0u) return plainDiv(x, d);
    } else {
        const Real ax = fabs(x);
        if (!(ax <= huge) || (ax < tiny && ax != Real(0))) return plainDiv(x, d);
    }
    const Real q0 = x * dinv;
    const Real q1 = fma(fma(-q0, d, x), dinv, q0);
    return fma(fma(-q1, d, x), dinv, q1);
}

// ------------------------------------------------------------- node sources
// The node arithmetic reads its operands through a source: the five stencil fields of the
// stage input at (dx, dz) from the node, the start-of-step state U and the RK accumulator A of
// the node, and its model words.  StreamNode serves the streaming kernel (every word staged in
// shared memory one row block ahead of use).  `exact`: h is a power of two, so x/h is formed as
// x*(1/h) -- the same value; otherwise the correctly rounded divBy.
// Streaming geometry: a CTA owns a strip of SW node columns and a segment of SB*seg node rows
// (seg <= MAX_SEG row blocks, picked per grid), and walks down the segment one block of SB rows
// (one row per warp) at a time.
// Shared memory holds a ring of three chunks of SB stencil rows (five fields, SW + 8 columns:
// the strip and four columns either side) and two buffers of the per-node words of a row block.
// Both are filled by tensor copies, so their layout is the copy box: [chunk][field][row][column]
// and [word][row][column].
constexpr int SW = 32, SB = 8, MAX_SEG = 8, CHUNKS = 3, RC = SW + 8, RF = SB * RC, CH = 5 * RF;
constexpr int RING = CHUNKS * SB, STREAM_THREADS = SW * SB;
enum : int { PW_U = 0, PW_A = 5, PW_a = 10, PW_b = 11, PW_lam = 12, PW_mu = 13, PW_rho = 14, PW_jac = 15, PW_C = 16 };
// per-node words: U, A, five model words and J, plus the five compensation terms of the last FP32
// stage (the only one that reads them)
// Stage 0 takes U from the ring and J from global memory, so it stages only the five model words
// a, b, lambda, mu, rho: its buffers start at word PW_a.
template <int STAGE> constexpr int firstWord() { return STAGE == 0 ? PW_a : 0; }
template <class Real, int STAGE = 3> constexpr int pwWords() {
    return STAGE == 0 ? PW_rho + 1 - PW_a : kahan<Real>() && STAGE == 3 ? PW_C + 5 : PW_C;
}
// two mbarriers, then the ring and the two word buffers (128-byte aligned), plus alignment slack
template <class Real, int STAGE = 3> constexpr std::size_t streamBytes() {
    return 128 + sizeof(Real) * (CHUNKS * CH + 2 * pwWords<Real, STAGE>() * STREAM_THREADS) + 128;
}

template <class Real, bool EXACT, int STAGE> struct StreamNode {
    static constexpr bool exact = EXACT;
    const Real *col; // ring chunk 0, field 0, row 0, this node's column
    const Real *pw;  // this node's per-node words (stride STREAM_THREADS)
    long long q;
    // Offset in the ring of the row dz = -3..3 away from this node's (chunk and row within the
    // chunk, wrapped): set once per row block (it is the same for a whole warp), so that every tap
    // is one shared-memory load at a constant offset from one of seven bases.
    int row[7];
    int centre; // ring row (0..RING-1) of this node
    __device__ __forceinline__ void setCentre(int c) {
        centre = c;
#pragma unroll
        for (int d = -3; d <= 3; ++d) {
            int s = c + d; // one wrap at most
            s = s < 0 ? s + RING : s >= RING ? s - RING : s;
            const unsigned u = unsigned(s);
            row[d + 3] = int((u / unsigned(SB)) * CH + (u % unsigned(SB)) * RC);
        }
    }
    // dz a compile-time constant (the stencil taps): a load from one of the seven row bases
    __device__ __forceinline__ Real at(int f, int dx, int dz) const { return col[row[dz + 3] + f * RF + dx]; }
    // dz known only at run time (the traction-image taps near the surface): the row is computed
    __device__ __forceinline__ Real atRow(int f, int dx, int dz) const {
        int s = centre + dz; // dz in [-3, 3]: one wrap at most
        s = s < 0 ? s + RING : s >= RING ? s - RING : s;
        const unsigned u = unsigned(s);
        return col[(u / unsigned(SB)) * CH + f * RF + (u % unsigned(SB)) * RC + dx];
    }
    __device__ __forceinline__ Real word(int w) const { return pw[(w - firstWord<STAGE>()) * STREAM_THREADS]; }
    __device__ __forceinline__ Real u(const StageArgs<Real> &, int f) const { return STAGE == 0 ? at(f, 0, 0) : word(PW_U + f); }
    __device__ __forceinline__ Real acc(const StageArgs<Real> &, int f) const { return word(PW_A + f); }
    __device__ __forceinline__ Real comp(const StageArgs<Real> &, int f) const { return word(PW_C + f); }
    __device__ __forceinline__ Real a(const Mesh<Real> &) const { return word(PW_a); }
    __device__ __forceinline__ Real b(const Mesh<Real> &) const { return word(PW_b); }
    __device__ __forceinline__ Real lam(const Mesh<Real> &) const { return word(PW_lam); }
    __device__ __forceinline__ Real mu(const Mesh<Real> &) const { return word(PW_mu); }
    __device__ __forceinline__ Real rho(const Mesh<Real> &) const { return word(PW_rho); }
    __device__ __forceinline__ Real jac(const Mesh<Real> &m) const { return STAGE == 3 ? word(PW_jac) : ld(m.jac + q); }
};

// ------------------------------------------------------------- stencils on a node source
// The reference accumulates each derivative from zero (PointKernels2D.hpp:38-47); starting
// from the first product gives the same value (0 + x == x, up to the sign of a zero result).
template <class Real, class S> __device__ __forceinline__ Real scaled(const Mesh<Real> &m, Real r) {
    if constexpr (S::exact) return r * m.hinv;
    else return divBy(r, m.h, m.hinv);
}
template <class Real, int DIR, class S> __device__ __forceinline__ Real tdrp(const S &t, const Mesh<Real> &m, int f, int axis) {
    const int sx = axis ? 0 : 1, sz = axis ? 1 : 0;
    Real r;
    if (DIR == 0) {
        r = Real(-.30874) * t.at(f, -sx, -sz);
        r += Real(-.6326) * t.at(f, 0, 0);
        r += Real(1.233) * t.at(f, sx, sz);
        r += Real(-.3334) * t.at(f, 2 * sx, 2 * sz);
        r += Real(.04168) * t.at(f, 3 * sx, 3 * sz);
    } else {
        r = -Real(-.30874) * t.at(f, sx, sz);
        r += -Real(-.6326) * t.at(f, 0, 0);
        r += -Real(1.233) * t.at(f, -sx, -sz);
        r += -Real(-.3334) * t.at(f, -2 * sx, -2 * sz);
        r += -Real(.04168) * t.at(f, -3 * sx, -3 * sz);
    }
    return scaled<Real, S>(m, r);
}
template <class Real, int DIR, class S> __device__ __forceinline__ Real tnear2(const S &t, const Mesh<Real> &m, int f) {
    Real r;
    if (DIR == 0) {
        r = Real(-1) * t.at(f, 0, 0);
        r += Real(1) * t.at(f, 0, 1);
    } else {
        r = -Real(-1) * t.at(f, 0, 0);
        r += -Real(1) * t.at(f, 0, -1);
    }
    return scaled<Real, S>(m, r);
}
template <class Real, int DIR, class S> __device__ __forceinline__ Real tnear3(const S &t, const Mesh<Real> &m, int f) {
    const Real c0 = Real(-7) / Real(6), c1 = Real(8) / Real(6), c2 = Real(-1) / Real(6);
    Real r;
    if (DIR == 0) {
        r = c0 * t.at(f, 0, 0);
        r += c1 * t.at(f, 0, 1);
        r += c2 * t.at(f, 0, 2);
    } else {
        r = -c0 * t.at(f, 0, 0);
        r += -c1 * t.at(f, 0, -1);
        r += -c2 * t.at(f, 0, -2);
    }
    return scaled<Real, S>(m, r);
}

// Traction flux J (x sigma_a + z sigma_b) at the tap (dx, dz) (PointKernels2D.hpp:90-93).
template <class Real, class S>
__device__ __forceinline__ Real flux(const Mesh<Real> &m, const S &t, int dx, int dz, int axis, int comp) {
    const long long qq = t.q + dx + (long long)dz * m.pitch;
    const Real x = axis ? ld(m.a + qq) : Real(1), z = axis ? ld(m.b + qq) : Real(0);
    return ld(m.jac + qq) * (x * t.atRow(comp ? 4 : 2, dx, dz) + z * t.atRow(comp ? 3 : 4, dx, dz));
}

// Conservative traction-image momentum near the surface (PointKernels2D.hpp:94-120):
// the surface tap is dropped and taps above it mirror with a sign flip.  only = -1: both axes.
template <class Real, int DX, int DZ, class S>
__device__ __forceinline__ Real momentum(const Mesh<Real> &m, const S &t, Real jac, Real rho, int comp, int depth, int only) {
    const Real C[5] = {Real(-.30874), Real(-.6326), Real(1.233), Real(-.3334), Real(.04168)};
    Real r = Real(0);
#pragma unroll
    for (int axis = 0; axis < 2; ++axis) {
        if (only >= 0 && axis != only) continue;
        const int dir = axis ? DZ : DX;
#pragma unroll
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
            r += sign * c * flux(m, t, axis ? 0 : off, axis ? off : 0, axis, comp);
        }
    }
    return r / (m.h * jac * rho);
}

// CFS-PML ADE (PointKernels2D.hpp:57-64): returns d/kappa + psi, rate -(d/k+a) psi - d/k^2 d.
template <class Real>
__device__ __forceinline__ Real stretch(const Real *prof, Real psi, Real d, Real &rate) {
    const Real dd = prof[0], kappa = prof[1], alpha = prof[2];
    rate = -(dd / kappa + alpha) * psi - dd / (kappa * kappa) * d;
    return d / kappa + psi;
}

// RK combine of one value (reference order, src/two_d/CurvilinearSolver2D.cpp:89):
// stage 0: A = k, out = U + w k;  stages 1-2: A = A + 2k, out = U + w k;  stage 3: U + dt (A + k) / 6.
// `acc` is the node's A (unused in stage 0); `accOut` receives the new A (stages 0-2).
// FP32 stage 3 adds the increment d = dt (A + k) / 6 to U by Kahan's compensated summation
// (y = d - c, t = U + y, c' = (t - U) - y): `cin` is c and `accOut` receives c'.
template <class Real, int STAGE>
__device__ __forceinline__ Real combine(const StageArgs<Real> &p, Real acc, Real u, Real r, Real cin, Real &accOut) {
    if (STAGE == 0) {
        accOut = r;
        return u + p.weight * r;
    } else if (STAGE < 3) {
        accOut = acc + 2 * r;
        return u + p.weight * r;
    }
    if constexpr (kahan<Real>()) {
        const Real y = div6(p.delta * (acc + r)) - cin;
        const Real t = u + y;
        accOut = (t - u) - y;
        return t;
    }
    accOut = Real(0);
    return u + div6(p.delta * (acc + r));
}
// Stages 0-2 write A and the stage output; stage 3 writes the new state over A (and, in FP32,
// its compensation term).
template <class Real, int STAGE>
__device__ __forceinline__ void store(const StageArgs<Real> &p, long long at, Real out, Real accOut) {
    if (STAGE < 3) {
        p.acc[at] = accOut;
        p.out[at] = out;
    } else {
        p.acc[at] = out;
        if constexpr (kahan<Real>()) p.cout[at] = accOut;
    }
}
// ADE memory update of one slot value (same scheme as the fields).
template <class Real, int STAGE>
__device__ __forceinline__ void combineMemory(const StageArgs<Real> &p, long long at, Real rate, Partial &diag, bool withDiag) {
    const Real u = lds(p.pbase + at);
    if (STAGE == 0) {
        p.pacc[at] = rate;
        p.pout[at] = u + p.weight * rate;
    } else if (STAGE < 3) {
        p.pacc[at] = p.pacc[at] + 2 * rate;
        p.pout[at] = u + p.weight * rate;
    } else {
        Real v;
        if constexpr (kahan<Real>()) {
            const Real y = div6(p.delta * (p.pacc[at] + rate)) - lds(p.pcin + at);
            v = u + y;
            p.pcout[at] = (v - u) - y;
        } else {
            v = u + div6(p.delta * (p.pacc[at] + rate));
        }
        p.pacc[at] = v;
        if (withDiag && !isfinite(v)) diag.bad = 1;
    }
}

// One node of one stage, in two phases that keep few values live: (1) velocity derivatives ->
// stress (and GSLS) rates -> combine/store of the stresses; (2) stress derivatives -> velocity
// rates -> combine/store of the velocities.  Every expression keeps the reference's operation
// order (src/two_d/PointKernels2D.hpp:121-172); only independent computations are reordered.
// GSLS memory fields (index >= 5) are read and written in global memory directly.
// FULL = false compiles the interior form: the caller guarantees that the node lies outside the
// CFS-PML strips, the sponge, the source support and the four surface rows.
template <class Real, int DX, int DZ, int MECH, int STAGE, bool FULL, class S>
__device__ __forceinline__ void stageNode(const StageArgs<Real> &p, const S &t, int i, int k, Partial &diag, bool withDiag) {
    const Mesh<Real> &m = p.m;
    constexpr bool KAHAN3 = STAGE == 3 && kahan<Real>();
    // A mesh with CFS-PML sums every node's momentum per axis, x/rho + z/rho, and stretches the
    // terms of the nodes that own memory slots (PointKernels2D.hpp:148-153); without CFS-PML the
    // momentum is one quotient, (x + z)/rho.  SPLIT follows the mesh; CPML (slot handling) is
    // compiled out of the interior form, whose nodes own no slots.
    const bool SPLIT = m.wz > 0;
    const bool CPML = FULL && SPLIT;
    const long long n = m.count, q = t.q;
    const int depth = FULL ? k - 3 : 4; // any depth past the near-surface rows
    const Real *__restrict__ w = p.in;
    const bool damped = FULL && !(i >= m.dmp_i0 && i < m.dmp_i1 && k < m.dmp_k1);
    const Real damp = damped ? ld(m.damping + q) : Real(0);

    // CFS-PML slots of this node (src/two_d/PointKernels2D.hpp:50-56)
    long long slot0 = -1, slot1 = -1;
    const Real *prof0 = nullptr, *prof1 = nullptr;
    if (CPML) {
        const int ic = i - 3, kc = k - 3, nxc = m.nx - 6, nzc = m.nz - 6;
        const int j = ic < m.wx ? ic : ic >= nxc - m.wx ? m.wx + ic - (nxc - m.wx) : -1;
        if (j >= 0) slot0 = 4 * ((long long)kc * 2 * m.wx + j), prof0 = m.cpx + 3 * ic;
        if (kc >= nzc - m.wz)
            slot1 = 4 * ((long long)(2 * m.wx) * nzc + (long long)(kc - (nzc - m.wz)) * nxc + ic), prof1 = m.cpz + 3 * kc;
    }
    const Real a = t.a(m), b = t.b(m);

    // ---- phase 1: velocity derivatives -> stress and GSLS rates
    Real xv[2], vxs[2], ev[2];
    xv[0] = tdrp<Real, DX>(t, m, 0, 0);
    xv[1] = tdrp<Real, DX>(t, m, 1, 0);
    vxs[0] = xv[0], vxs[1] = xv[1];
    Real prate[4] = {0, 0, 0, 0}; // ADE rates of the velocity-derivative memories: slot0 f0,f1, slot1 f0,f1
    if (CPML && slot0 >= 0)
        for (int v = 0; v < 2; ++v) vxs[v] = stretch(prof0, lds(p.pin + slot0 + v), xv[v], prate[v]);
    const Real lam = t.lam(m), mu = t.mu(m);
    if (depth == 0) { // surface eta-derivative from the traction-free condition (PointKernels2D.hpp:79-89)
        const Real c0 = a, c1 = b, c2 = c0 * c0 + c1 * c1, len = sqrt(c2);
        const Real nn[2] = {c0 / len, c1 / len};
        const Real dx = vxs[0], dz = vxs[1];
        Real tt[2] = {(lam + 2 * mu) * dx * c0 + mu * dz * c1, mu * dz * c0 + lam * dx * c1};
#pragma unroll
        for (int l = 0; l < MECH; ++l) {
            const int mm = 6 + 4 * l;
            tt[0] -= lds(w + mm * n + q) * c0 + lds(w + (mm + 2) * n + q) * c1;
            tt[1] -= lds(w + (mm + 2) * n + q) * c0 + lds(w + (mm + 1) * n + q) * c1;
        }
        const Real normal = tt[0] * nn[0] + tt[1] * nn[1];
        for (int v = 0; v < 2; ++v)
            ev[v] = -(tt[v] - nn[v] * normal) / (mu * c2) - nn[v] * normal / ((lam + 2 * mu) * c2);
    } else if (depth == 1) {
        ev[0] = tnear2<Real, DZ>(t, m, 0);
        ev[1] = tnear2<Real, DZ>(t, m, 1);
    } else if (depth == 2) {
        ev[0] = tnear3<Real, DZ>(t, m, 0);
        ev[1] = tnear3<Real, DZ>(t, m, 1);
    } else {
        ev[0] = tdrp<Real, DZ>(t, m, 0, 1);
        ev[1] = tdrp<Real, DZ>(t, m, 1, 1);
    }
    Real dxv[2], dzv[2];
#pragma unroll
    for (int f = 0; f < 2; ++f) {
        Real vz = ev[f];
        if (CPML && slot1 >= 0) vz = stretch(prof1, lds(p.pin + slot1 + f), ev[f], prate[2 + f]);
        dxv[f] = vxs[f] + a * vz;
        dzv[f] = b * vz;
    }
    const Real div = dxv[0] + dzv[1];
    Real r2 = lam * div + 2 * mu * dxv[0];
    Real r3 = lam * div + 2 * mu * dzv[1];
    Real r4 = mu * (dzv[0] + dxv[1]);
    if (MECH) {
        // The accumulator words of the 4L memory fields and of Syy are loaded before the first
        // store: a store could alias them as far as the compiler knows, so loading each after the
        // previous field's store would serialise 4L+1 round trips per node.  (The other words are
        // read-only loads, which the compiler may move.)
        constexpr int NM = 4 * MECH + 1; // memory fields 6 .. 6+4L-1, then Syy (field 5)
        Real am[NM];
#pragma unroll
        for (int j = 0; j < NM; ++j) am[j] = STAGE ? p.acc[(j < 4 * MECH ? 6 + j : 5) * n + q] : Real(0);
        const Real w5 = damped ? lds(w + 5 * n + q) : Real(0);
        Real r5 = lam * div;
#pragma unroll
        for (int l = 0; l < MECH; ++l) {
            const int mm = 6 + 4 * l;
            const Real dp = ld(m.dP[l] + q), ds = ld(m.dS[l] + q), dl = dp - 2 * ds;
            const Real drive[4] = {dl * div + 2 * ds * dxv[0], dl * div + 2 * ds * dzv[1], ds * (dzv[0] + dxv[1]), dl * div};
            Real wm[4];
#pragma unroll
            for (int f = 0; f < 4; ++f) wm[f] = lds(w + (mm + f) * n + q);
            r2 -= wm[0];
            r3 -= wm[1];
            r4 -= wm[2];
            r5 -= wm[3];
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                Real rm = m.rates[l] * (drive[f] - wm[f]);
                if (damped) rm -= damp * wm[f];
                const long long at = (mm + f) * n + q;
                Real an;
                const Real o = combine<Real, STAGE>(p, am[4 * l + f], lds(p.base + at), rm, KAHAN3 ? lds(p.cin + at) : Real(0), an);
                store<Real, STAGE>(p, at, o, an);
                if (withDiag && !isfinite(o)) diag.bad = 1;
            }
        }
        if (damped) r5 -= damp * w5;
        const long long at = 5 * n + q;
        Real an;
        const Real o = combine<Real, STAGE>(p, am[NM - 1], lds(p.base + at), r5, KAHAN3 ? lds(p.cin + at) : Real(0), an);
        store<Real, STAGE>(p, at, o, an);
        if (withDiag && !isfinite(o)) diag.bad = 1;
    }
    if (damped) {
        r2 -= damp * t.at(2, 0, 0);
        r3 -= damp * t.at(3, 0, 0);
        r4 -= damp * t.at(4, 0, 0);
    }
    Real a2, a3, a4;
    Real o2 = combine<Real, STAGE>(p, STAGE ? t.acc(p, 2) : Real(0), t.u(p, 2), r2, KAHAN3 ? t.comp(p, 2) : Real(0), a2);
    Real o3 = combine<Real, STAGE>(p, STAGE ? t.acc(p, 3) : Real(0), t.u(p, 3), r3, KAHAN3 ? t.comp(p, 3) : Real(0), a3);
    Real o4 = combine<Real, STAGE>(p, STAGE ? t.acc(p, 4) : Real(0), t.u(p, 4), r4, KAHAN3 ? t.comp(p, 4) : Real(0), a4);
    Real nx_ = 0, nz_ = 0;
    if (depth == 0) { // free-surface projection, PointKernels2D.hpp:70-78
        nx_ = ld(m.normals + 2 * q), nz_ = ld(m.normals + 2 * q + 1);
        const Real tx = o2 * nx_ + o4 * nz_, tz = o4 * nx_ + o3 * nz_, nn = nx_ * tx + nz_ * tz;
        o2 += -2 * nx_ * tx + nn * nx_ * nx_;
        o3 += -2 * nz_ * tz + nn * nz_ * nz_;
        o4 += -nx_ * tz - tx * nz_ + nn * nx_ * nz_;
    }
    store<Real, STAGE>(p, 2 * n + q, o2, a2);
    store<Real, STAGE>(p, 3 * n + q, o3, a3);
    store<Real, STAGE>(p, 4 * n + q, o4, a4);
    if (CPML) {
        if (slot0 >= 0)
            for (int f = 0; f < 2; ++f) combineMemory<Real, STAGE>(p, slot0 + f, prate[f], diag, withDiag);
        if (slot1 >= 0)
            for (int f = 0; f < 2; ++f) combineMemory<Real, STAGE>(p, slot1 + f, prate[2 + f], diag, withDiag);
    }

    // ---- phase 2: stress derivatives -> velocity rates
    const Real rho = t.rho(m);
    // The node's quotients by rho (two to four of them) from one reciprocal: divBy forms the
    // correctly rounded quotient, the same value as the division.
    const Real rinv = m.rhoRecip ? Real(1) / rho : Real(0);
    auto byRho = [&](Real x) { return m.rhoRecip ? divBy(x, rho, rinv) : x / rho; };
    Real r0, r1;
    const bool near = depth <= (DZ ? 3 : 1);
    if (!SPLIT) {
        if (near) {
            const Real jac = t.jac(m);
            r0 = momentum<Real, DX, DZ>(m, t, jac, rho, 0, depth, -1);
            r1 = momentum<Real, DX, DZ>(m, t, jac, rho, 1, depth, -1);
        } else {
            const Real x2 = tdrp<Real, DX>(t, m, 2, 0), x4 = tdrp<Real, DX>(t, m, 4, 0);
            const Real e2 = tdrp<Real, DZ>(t, m, 2, 1), e3 = tdrp<Real, DZ>(t, m, 3, 1), e4 = tdrp<Real, DZ>(t, m, 4, 1);
            r0 = byRho((x2 + a * e2) + b * e4);
            r1 = byRho((x4 + a * e4) + b * e3);
        }
    } else {
        Real mrate[4] = {0, 0, 0, 0}; // ADE rates of the momentum memories: slot0 f2,f3, slot1 f2,f3
        Real rv[2];
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            const int f = v ? 4 : 2, o = v ? 3 : 4;
            Real X, Z;
            if (near) {
                const Real jac = t.jac(m);
                X = momentum<Real, DX, DZ>(m, t, jac, rho, v, depth, 0);
                Z = momentum<Real, DX, DZ>(m, t, jac, rho, v, depth, 1);
            } else {
                X = byRho(tdrp<Real, DX>(t, m, f, 0));
                Z = byRho(a * tdrp<Real, DZ>(t, m, f, 1) + b * tdrp<Real, DZ>(t, m, o, 1));
            }
            if (CPML && slot0 >= 0) X = stretch(prof0, lds(p.pin + slot0 + 2 + v), X, mrate[v]);
            if (CPML && slot1 >= 0) Z = stretch(prof1, lds(p.pin + slot1 + 2 + v), Z, mrate[2 + v]);
            rv[v] = X + Z;
        }
        r0 = rv[0], r1 = rv[1];
        if (CPML && slot0 >= 0)
            for (int v = 0; v < 2; ++v) combineMemory<Real, STAGE>(p, slot0 + 2 + v, mrate[v], diag, withDiag);
        if (CPML && slot1 >= 0)
            for (int v = 0; v < 2; ++v) combineMemory<Real, STAGE>(p, slot1 + 2 + v, mrate[2 + v], diag, withDiag);
    }
    if (FULL && i >= m.src_i0 && i < m.src_i1 && k >= m.src_k0 && k < m.src_k1) {
        const Clock *clk = p.clock;
        const Real forcing = p.forcing[3 * (clk->step - clk->first) + (STAGE == 0 ? 0 : STAGE == 3 ? 2 : 1)];
        if (m.sgx) {
            r0 += byRho(forcing * ld(m.sgx + q));
            r1 += byRho(forcing * ld(m.sgz + q));
        } else {
            const Real s = ld(m.source + q);
            r0 += byRho(forcing * (s * m.sdx));
            r1 += byRho(forcing * (s * m.sdz));
        }
    }
    if (damped) {
        r0 -= damp * t.at(0, 0, 0);
        r1 -= damp * t.at(1, 0, 0);
    }
    Real a0, a1;
    const Real o0 = combine<Real, STAGE>(p, STAGE ? t.acc(p, 0) : Real(0), t.u(p, 0), r0, KAHAN3 ? t.comp(p, 0) : Real(0), a0);
    const Real o1 = combine<Real, STAGE>(p, STAGE ? t.acc(p, 1) : Real(0), t.u(p, 1), r1, KAHAN3 ? t.comp(p, 1) : Real(0), a1);
    store<Real, STAGE>(p, q, o0, a0);
    store<Real, STAGE>(p, n + q, o1, a1);

    if (STAGE == 3 && withDiag) { // energy, |v|^2, surface traction, finiteness (PointKernels2D.hpp:173-184)
        diag.bad |= int(!isfinite(o0)) | int(!isfinite(o1)) | int(!isfinite(o2)) | int(!isfinite(o3)) | int(!isfinite(o4));
        const double l = lam, mu_ = mu, xx = o2, zz = o3, xz = o4, vx = o0, vz = o1;
        // (l+2m)(xx^2+zz^2) - 2 l xx zz over 8m(l+m), plus xz^2/(2m), over one division
        const double e = (.5 * double(rho) * (vx * vx + vz * vz) +
                          (((l + 2 * mu_) * (xx * xx + zz * zz) - 2 * l * xx * zz) + 4 * (l + mu_) * xz * xz) / (8 * mu_ * (l + mu_))) *
                         double(t.jac(m)) * double(m.h) * double(m.h);
        const double v2 = vx * vx + vz * vz;
        diag.bad |= int(!isfinite(e));
        diag.energy += e;
        diag.velocity = fmax(diag.velocity, v2); // squared; the root is taken once per CTA
        if (depth == 0) {
            const double tx = xx * double(nx_) + xz * double(nz_), tz = xz * double(nx_) + zz * double(nz_);
            const double norm = sqrt(xx * xx + zz * zz + 2 * xz * xz);
            diag.traction = fmax(diag.traction, sqrt(tx * tx + tz * tz) / fmax(norm, 1e-25));
        }
    }
}

constexpr int TILE_THREADS = 256; // threads of a stage CTA (8 warps)

// Block reduction of the per-thread diagnostics into one partial per CTA (256 threads).
__device__ __forceinline__ void reducePartial(Partial s, Partial *out, int slot) {
    for (int o = 16; o > 0; o >>= 1) {
        s.energy += __shfl_down_sync(0xffffffffu, s.energy, o);
        s.velocity = fmax(s.velocity, __shfl_down_sync(0xffffffffu, s.velocity, o));
        s.traction = fmax(s.traction, __shfl_down_sync(0xffffffffu, s.traction, o));
        s.bad |= __shfl_down_sync(0xffffffffu, s.bad, o);
    }
    __shared__ Partial warps[TILE_THREADS / 32];
    const int t = threadIdx.x + blockDim.x * threadIdx.y, lane = t & 31, wid = t >> 5;
    if (lane == 0) warps[wid] = s;
    __syncthreads();
    if (t == 0) {
        Partial tot = warps[0];
        for (int w = 1; w < TILE_THREADS / 32; ++w) {
            tot.energy += warps[w].energy;
            tot.velocity = fmax(tot.velocity, warps[w].velocity);
            tot.traction = fmax(tot.traction, warps[w].traction);
            tot.bad |= warps[w].bad;
        }
        tot.velocity = sqrt(tot.velocity); // the nodes accumulated |v|^2
        out[slot] = tot;
    }
}

// ------------------------------------------------------------- streaming stage
// A CTA walks its strip down one block of 8 rows at a time.  One thread issues tensor copies;
// group g (ring chunk g + 1 -- chunks 0 and 1 for g = 0 -- and the U, A and model words of block
// g) completes on mbarrier g & 1.  While the CTA evaluates block b from shared memory, group b+1
// is in flight; after block b, group b+2 reuses the ring chunk and word buffer block b released.
// Waits are bounded: a wait that runs out flags the clock (`stalled`) and the CTA stops.
__device__ __forceinline__ unsigned smemAddr(const void *p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ void mbarInit(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smemAddr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbarExpectTx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smemAddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbarTryWait(uint64_t *bar, unsigned parity) {
    unsigned done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done)
                 : "r"(smemAddr(bar)), "r"(parity)
                 : "memory");
    return done != 0;
}
// Bounded wait for the phase of `parity`; false when the limit ran out.
__device__ __forceinline__ bool mbarWait(uint64_t *bar, unsigned parity) {
    for (int it = 0; it < (1 << 22); ++it)
        if (mbarTryWait(bar, parity)) return true;
    return false;
}
// L2 prefetch of a 3D tensor box (no shared memory, no completion to wait for).
__device__ __forceinline__ void tmaPrefetch3(const CUtensorMap *map, int x, int y, int z) {
    asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];\n" ::"l"(reinterpret_cast<uint64_t>(map)), "r"(x),
                 "r"(y), "r"(z)
                 : "memory");
}
// 3D tiled tensor copy global -> shared (no multicast), completing on `bar`.
__device__ __forceinline__ void tmaLoad3(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(
                     smemAddr(dst)),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smemAddr(bar))
                 : "memory");
}

// Resident CTAs per SM.  FP64: 2 x 101.8 KB of shared memory; stage 0 (five model words staged)
// 3 x 59 KB at 80 registers.  FP32: 3 x 61 KB in the last stage (it also stages the compensation
// terms); 4 x 51 KB in the others, which then hold 64 registers (elastic: GSLS stages keep three
// CTAs and their 80 registers).
template <class Real, int STAGE = 3, int MECH = 0> constexpr int streamBlocks() {
    return sizeof(Real) == 8 ? (STAGE == 0 ? 3 : 2) : STAGE < 3 && MECH == 0 ? 4 : 3;
}

// Whether every node of the CTA's strip and segment is an interior node (outside the CFS-PML
// strips, the sponge, the source support and the surface rows 3..6).  The host evaluates the
// same predicate to report how many CTAs take the interior form (swl2d_layout).
template <class Real> __host__ __device__ __forceinline__ bool interiorBlock(const Mesh<Real> &m, int i0, int z0) {
    const int i1 = i0 + SW, z1 = z0 + SB * m.seg; // exclusive ends
    const bool pml = i0 - 3 < m.wx || i1 - 3 > m.nx - 6 - m.wx || z1 - 3 > m.nz - 6 - m.wz;
    const bool surface = z0 < 7;
    const bool source = i0 < m.src_i1 && i1 > m.src_i0 && z0 < m.src_k1 && z1 > m.src_k0;
    const bool sponge = !(i0 >= m.dmp_i0 && i1 <= m.dmp_i1 && z1 <= m.dmp_k1);
    return !(pml || surface || source || sponge);
}

// Tile (bx, by) of the stage grid; its diagnostics go to partial `slot`.  `reinit`: the
// mbarriers were used by an earlier tile of this CTA (every copy of which has landed) and are
// invalidated before they are initialised again.  Returns false when a copy wait ran out.
__device__ __forceinline__ void mbarInval(uint64_t *bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smemAddr(bar)) : "memory");
}
template <class Real, int DX, int DZ, int MECH, int STAGE, bool EXACT, bool FULL>
__device__ __forceinline__ bool streamBody(const StageArgs<Real> &p, uint64_t *bar, Real *ring, Real *pw, int bx, int by, int slot,
                                           bool reinit) {
    constexpr int T = STREAM_THREADS, PW = pwWords<Real, STAGE>();
    constexpr unsigned S = sizeof(Real);
    constexpr unsigned chunkBytes = S * CH, fiveBytes = S * 5 * T, modelBytes = S * (STAGE == 3 ? 6 : 5) * T;
    constexpr unsigned wordBytes = (STAGE > 0 ? 2 * fiveBytes : 0) + modelBytes + (STAGE == 3 && kahan<Real>() ? fiveBytes : 0);
    const Mesh<Real> &m = p.m;
    const int lane = threadIdx.x, wy = threadIdx.y, tid = lane + SW * wy;
    const int i0 = 3 + bx * SW, z0 = 3 + by * (SB * m.seg), zb = z0 - 3;
    const int iEnd = m.nx - 3, kEnd = m.nz - 3;
    const int blocks = min(m.seg, (kEnd - z0 + SB - 1) / SB);
    __shared__ int stop;
    // thread 0: L2 prefetch of row block g's GSLS words (x of the word boxes: node i0)
    auto prefetchGsls = [&](int g) {
        const int x = i0 + m.xoff, y = z0 + SB * g;
        tmaPrefetch3(&p.gslsInMap, x, y, 0);
        if (STAGE > 0) tmaPrefetch3(&p.gslsUMap, x, y, 0), tmaPrefetch3(&p.gslsAMap, x, y, 0);
        if (STAGE == 3 && kahan<Real>()) tmaPrefetch3(&p.gslsCompMap, x, y, 0);
        tmaPrefetch3(&p.strengthMap, x, y, 0);
    };
    // thread 0: issue copy group g (x of the ring box: node i0 - 4; of the word boxes: node i0)
    auto issue = [&](int g) {
        uint64_t *b = bar + (g & 1);
        const int c0 = g == 0 ? 0 : g + 1, c1 = g + 1;
        mbarExpectTx(b, (c1 - c0 + 1) * chunkBytes + wordBytes);
        for (int c = c0; c <= c1; ++c) tmaLoad3(ring + (c % CHUNKS) * CH, &p.ringMap, i0 - 4 + m.xoff, zb + SB * c, 0, b);
        Real *dst = pw + (g & 1) * (PW * T);
        const int x = i0 + m.xoff, y = z0 + SB * g;
        if (STAGE > 0) {
            tmaLoad3(dst + PW_U * T, &p.uMap, x, y, 0, b);
            tmaLoad3(dst + PW_A * T, &p.aMap, x, y, 0, b);
        }
        tmaLoad3(dst + (PW_a - firstWord<STAGE>()) * T, &p.modelMap, x, y, 0, b);
        if (STAGE == 3 && kahan<Real>()) tmaLoad3(dst + PW_C * T, &p.compMap, x, y, 0, b);
        if (MECH > 0 && p.gslsPrefetch == 2) prefetchGsls(g);
        if (MECH > 0 && p.gslsPrefetch == 3 && g + 1 < blocks) prefetchGsls(g + 1);
    };
    if (tid == 0) {
        stop = 0;
        if (reinit) mbarInval(bar), mbarInval(bar + 1);
        mbarInit(bar, 1);
        mbarInit(bar + 1, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        issue(0);
        if (blocks > 1) issue(1);
    }
    Partial diag{0, 0, 0, 0, 0};
    const bool withDiag = STAGE == 3 && p.partials != nullptr;
    int waited = 0; // groups this CTA has seen complete
#pragma unroll 1
    for (int blk = 0; blk < blocks; ++blk) {
        if (!mbarWait(bar + (blk & 1), (blk >> 1) & 1)) stop = 1;
        __syncthreads();
        if (stop) break;
        waited = blk + 1;
        if (MECH > 0 && p.gslsPrefetch == 1 && tid == 0 && blk + 1 < blocks) prefetchGsls(blk + 1); // one block ahead
        const int k = z0 + blk * SB + wy, i = i0 + lane;
        if (k < kEnd && i < iEnd) {
            StreamNode<Real, EXACT, STAGE> s;
            s.col = ring + lane + 4;
            s.pw = pw + (blk & 1) * (PW * T) + tid;
            s.q = i + m.xoff + (long long)m.pitch * k;
            const int c = SB * (blk % 3) + wy + 3; // ring row of row k (rows counted from zb)
            s.setCentre(c >= RING ? c - RING : c);
            stageNode<Real, DX, DZ, MECH, STAGE, FULL>(p, s, i, k, diag, withDiag);
        }
        __syncthreads(); // block blk's ring chunk and word buffer are free
        if (tid == 0 && blk + 2 < blocks) issue(blk + 2);
    }
    if (stop) { // a copy wait ran out: flag it, let the copies still in flight land, and stop
        if (tid == 0) {
            atomicExch(const_cast<int *>(&p.clock->stalled), 1);
            const int issued = min(blocks, waited + 2);
            for (int g = waited; g < issued; ++g) mbarWait(bar + (g & 1), (g >> 1) & 1);
        }
        return false;
    }
    if (withDiag) reducePartial(diag, p.partials, slot);
    return true;
}

// One tile of one stage in the form its position calls for: the interior form away from the
// boundaries, the general form elsewhere; x/h by a product or the correctly rounded quotient.
template <class Real, int DX, int DZ, int MECH, int STAGE>
__device__ __forceinline__ bool streamTile(const StageArgs<Real> &p, uint64_t *bar, Real *ring, Real *pw, int bx, int by, int slot,
                                           bool reinit) {
    const bool interior = interiorBlock(p.m, 3 + bx * SW, 3 + by * (SB * p.m.seg));
    if constexpr (sizeof(Real) == 4) {
        if (interior) return streamBody<Real, DX, DZ, MECH, STAGE, true, false>(p, bar, ring, pw, bx, by, slot, reinit);
        return streamBody<Real, DX, DZ, MECH, STAGE, true, true>(p, bar, ring, pw, bx, by, slot, reinit);
    } else if (p.m.hinvExact) {
        if (interior) return streamBody<Real, DX, DZ, MECH, STAGE, true, false>(p, bar, ring, pw, bx, by, slot, reinit);
        return streamBody<Real, DX, DZ, MECH, STAGE, true, true>(p, bar, ring, pw, bx, by, slot, reinit);
    } else {
        if (interior) return streamBody<Real, DX, DZ, MECH, STAGE, false, false>(p, bar, ring, pw, bx, by, slot, reinit);
        return streamBody<Real, DX, DZ, MECH, STAGE, false, true>(p, bar, ring, pw, bx, by, slot, reinit);
    }
}

// The streaming stage: grid (strips of 32 columns, segments of 64 rows), block 32x8.  DX/DZ:
// MacCormack directions of this (step, stage); MECH: GSLS mechanisms (0: elastic); STAGE: 0..3.
template <class Real, int DX, int DZ, int MECH, int STAGE>
__global__ void __launch_bounds__(STREAM_THREADS, (streamBlocks<Real, STAGE, MECH>())) stream2d(const __grid_constant__ StageArgs<Real> p) {
    extern __shared__ __align__(16) unsigned char smemRaw[];
    if (p.clock->faulted) return; // uniform across the grid
    unsigned char *base = smemRaw + ((128 - (smemAddr(smemRaw) & 127)) & 127);
    uint64_t *bar = reinterpret_cast<uint64_t *>(base);
    Real *ring = reinterpret_cast<Real *>(base + 128);
    Real *pw = ring + CHUNKS * CH;
    streamTile<Real, DX, DZ, MECH, STAGE>(p, bar, ring, pw, blockIdx.x, blockIdx.y, blockIdx.x + gridDim.x * blockIdx.y, false);
}

// ---------------------------------------------------------------- diagnostics ------------
// Per-block energy / peak velocity / surface traction / finiteness of a state
// (src/two_d/CudaEngine2D.cu:43-78 semantics, PointKernels2D.hpp:181-184 energy); used by
// swl2d_diagnostics outside the step batches.
template <class Real>
__global__ void __launch_bounds__(256) stats2d(const Mesh<Real> m, const Real *__restrict__ w, const Real *__restrict__ pml,
                                               const Clock *clk, Partial *out) {
    __shared__ Partial sh[256];
    const int t = threadIdx.x + blockDim.x * threadIdx.y;
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = 3 + blockIdx.y * blockDim.y + threadIdx.y;
    Partial s{0, 0, 0, 0, 0};
    if (i < m.nx - 3 && k < m.nz - 3 && !(clk && clk->faulted)) {
        const long long n = m.count, q = i + m.xoff + (long long)m.pitch * k;
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
    // The clock's words are read once, in parallel, by the first warp: the rule and the record
    // below then read shared memory instead of a chain of dependent global loads.
    __shared__ union {
        Clock c;
        int w[sizeof(Clock) / sizeof(int)];
    } snap;
    static_assert(sizeof(Clock) % sizeof(int) == 0 && sizeof(Clock) / sizeof(int) <= 32, "Clock must fit one warp's loads");
    const int t = threadIdx.x;
    if (t < int(sizeof(Clock) / sizeof(int))) snap.w[t] = reinterpret_cast<const int *>(clk)[t];
    __syncthreads();
    const Clock &c0 = snap.c;
    if (c0.faulted) return;
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
            const bool growth = (c0.step + 1) * c0.dt > c0.growth_after && c0.peak_energy > 0 &&
                                tot.energy > c0.peak_energy * 10000;
            ok = finite && !growth;
            clk->finite = finite;
            if (ok) {
                clk->energy = tot.energy;
                clk->max_velocity = tot.velocity;
                clk->traction = tot.traction;
                clk->peak_energy = fmax(c0.peak_energy, tot.energy);
            }
        }
        accept = ok;
    }
    __syncthreads();
    if (!accept) {
        if (t == 0) {
            clk->faulted = 1;
            clk->fault_step = c0.step;
        }
        return;
    }
    const int row = c0.step - c0.first;
    if (row < c0.trace_steps)
        for (int r = t; r < nrec; r += blockDim.x) {
            const long long qq = receivers[r];
            traces[((long long)row * nrec + r) * 2] = double(w[qq]);
            traces[((long long)row * nrec + r) * 2 + 1] = double(w[count + qq]);
        }
    __syncthreads();
    if (t == 0) {
        clk->step = c0.step + 1;
        clk->accepted = c0.accepted + 1;
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
