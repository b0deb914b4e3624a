// swl2d_stats_noalloc: the 2D diagnostics reduction for callers that cannot allocate device
// memory.  It computes what swl2d_diagnostics computes (energy, peak |v|, peak surface traction
// ratio, finiteness; src/two_d/CudaEngine2D.cu:43-78 semantics) from device arrays the caller
// owns, and keeps its per-block partial sums in a fixed array defined in this file instead of an
// allocated buffer.  Nothing here calls cudaMalloc, cudaFree or an allocating library routine.
#include "../../include/swl_b200.h"
#include "runtime.cuh"
#include <mutex>

namespace {

struct Part {
    double energy, velocity, traction;
    int bad, pad;
};

constexpr int kBlockX = 32, kBlockY = 8;
constexpr int kMaxBlocks = 65536; // 16.7 M physical nodes at 256 nodes per block

// Scratch for the per-block partials (2 MiB).  Every device that loads the library holds it.
// Host code must not pass this symbol to a kernel: on the host it is only a stand-in for the
// device array; its device address comes from cudaGetSymbolAddress (scratchAddress below).
static __device__ __align__(256) Part stats2dScratch[kMaxBlocks];

// The array's device address belongs to the CUDA context the module was loaded into.  A device
// reset (cudaDeviceReset) or another context on the same device gives the array a new address, so
// the address is looked up again on every call that is not being captured into a graph, and the
// last address seen per context is kept only for calls made during a capture (where the lookup,
// which may load the module, is not made).
using CtxGetCurrent = CUresult (*)(CUcontext *);
constexpr int kMaxContexts = 64;
struct CachedAddress {
    CUcontext context;
    Part *address;
};
CachedAddress scratchCache[kMaxContexts] = {};
std::mutex scratchMutex;

CUcontext currentContext() {
    static CtxGetCurrent fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        swl::check(cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q), "find cuCtxGetCurrent");
        if (!f || q != cudaDriverEntryPointSuccess) throw swl::Error(SWL_ERR_CUDA, "the driver has no cuCtxGetCurrent");
        return reinterpret_cast<CtxGetCurrent>(f);
    }();
    CUcontext c = nullptr;
    if (fn(&c) != CUDA_SUCCESS || !c) throw swl::Error(SWL_ERR_CUDA, "no current CUDA context");
    return c;
}

// Device address of the scratch array in the current context.  Outside a capture the lookup
// comes first: it also makes the device's primary context current if nothing has yet.
Part *scratchAddress(cudaStream_t stream) {
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    swl::check(cudaStreamIsCapturing(stream, &capture), "query stream capture");
    void *p = nullptr;
    if (capture == cudaStreamCaptureStatusNone)
        swl::check(cudaGetSymbolAddress(&p, stats2dScratch), "look up the diagnostics scratch array");
    const CUcontext ctx = currentContext();
    std::lock_guard<std::mutex> lock(scratchMutex);
    int slot = -1, empty = -1;
    for (int c = 0; c < kMaxContexts; ++c) {
        if (scratchCache[c].context == ctx) slot = c;
        if (!scratchCache[c].context && empty < 0) empty = c;
    }
    if (capture != cudaStreamCaptureStatusNone) {
        if (slot < 0 || !scratchCache[slot].address)
            throw swl::Error(SWL_ERR_INVALID, "swl2d_stats_noalloc: make the first call in this context before stream capture");
        return scratchCache[slot].address;
    }
    if (slot < 0) slot = empty >= 0 ? empty : 0; // more contexts than slots: reuse the first
    scratchCache[slot] = {ctx, static_cast<Part *>(p)};
    return static_cast<Part *>(p);
}

__global__ void __launch_bounds__(kBlockX *kBlockY) partials(const swl_state2d_view v, Part *scratch) {
    __shared__ Part sh[kBlockX * kBlockY];
    const int t = threadIdx.x + kBlockX * threadIdx.y;
    const int i = 3 + blockIdx.x * kBlockX + threadIdx.x;
    const int k = 3 + blockIdx.y * kBlockY + threadIdx.y;
    Part s{0, 0, 0, 0, 0};
    if (i < v.nx - 3 && k < v.nz - 3) {
        const long long q = i + (long long)v.nx * k;
        const double vx = v.vx[q], vz = v.vz[q], xx = v.sxx[q], zz = v.szz[q], xz = v.sxz[q];
        if (!isfinite(vx) || !isfinite(vz) || !isfinite(xx) || !isfinite(zz) || !isfinite(xz)) s.bad = 1;
        if (v.pml) { // the node's compact CFS-PML slots (src/two_d/PointKernels2D.hpp:50-56)
            const int ic = i - 3, kc = k - 3, nxc = v.nx - 6, nzc = v.nz - 6, wx = v.cpml_width_x, wz = v.cpml_width_z;
            const int j = ic < wx ? ic : ic >= nxc - wx ? wx + ic - (nxc - wx) : -1;
            const long long slots[2] = {j >= 0 ? 4 * ((long long)kc * 2 * wx + j) : -1,
                                        kc >= nzc - wz ? 4 * ((long long)(2 * wx) * nzc + (long long)(kc - (nzc - wz)) * nxc + ic) : -1};
            for (int a = 0; a < 2; ++a)
                if (slots[a] >= 0)
                    for (int f = 0; f < 4; ++f)
                        if (!isfinite(v.pml[slots[a] + f])) s.bad = 1;
        }
        const double l = v.lambda[q], mu = v.mu[q];
        s.energy = (.5 * v.rho[q] * (vx * vx + vz * vz) + ((l + 2 * mu) * (xx * xx + zz * zz) - 2 * l * xx * zz) / (8 * mu * (l + mu)) +
                    xz * xz / (2 * mu)) *
                   v.jac[q] * v.h * v.h;
        s.velocity = sqrt(vx * vx + vz * vz);
        if (!isfinite(s.energy) || !isfinite(s.velocity)) s.bad = 1;
        if (k == 3) {
            const double nx_ = v.normals[2 * q], nz_ = v.normals[2 * q + 1];
            const double tx = xx * nx_ + xz * nz_, tz = xz * nx_ + zz * nz_, norm = sqrt(xx * xx + zz * zz + 2 * xz * xz);
            s.traction = sqrt(tx * tx + tz * tz) / fmax(norm, 1e-25);
        }
    }
    sh[t] = s;
    __syncthreads();
    for (int stride = kBlockX * kBlockY / 2; stride > 0; stride >>= 1) {
        if (t < stride) {
            Part &x = sh[t];
            const Part y = sh[t + stride];
            x.energy += y.energy;
            x.velocity = fmax(x.velocity, y.velocity);
            x.traction = fmax(x.traction, y.traction);
            x.bad |= y.bad;
        }
        __syncthreads();
    }
    if (t == 0) scratch[blockIdx.x + gridDim.x * blockIdx.y] = sh[0]; // every used slot is rewritten by each call
}

__global__ void __launch_bounds__(1024) finish(const Part *scratch, int nparts, double *out) {
    __shared__ Part sh[1024];
    const int t = threadIdx.x;
    Part s{0, 0, 0, 0, 0};
    for (int b = t; b < nparts; b += blockDim.x) {
        const Part y = scratch[b];
        s.energy += y.energy;
        s.velocity = fmax(s.velocity, y.velocity);
        s.traction = fmax(s.traction, y.traction);
        s.bad |= y.bad;
    }
    sh[t] = s;
    __syncthreads();
    for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
        if (t < stride) {
            Part &x = sh[t];
            const Part y = sh[t + stride];
            x.energy += y.energy;
            x.velocity = fmax(x.velocity, y.velocity);
            x.traction = fmax(x.traction, y.traction);
            x.bad |= y.bad;
        }
        __syncthreads();
    }
    if (t == 0) {
        out[0] = sh[0].energy;
        out[1] = sh[0].velocity;
        out[2] = sh[0].traction;
        out[3] = (!sh[0].bad && isfinite(sh[0].energy)) ? 1.0 : 0.0;
    }
}

} // namespace

extern "C" swl_status swl2d_stats_noalloc(const swl_state2d_view *v, double *out, void *stream) {
    try {
        swl::lastErrorRef().clear();
        if (!v || !out) throw swl::Error(SWL_ERR_INVALID, "state and out are required");
        if (v->nx < 7 || v->nz < 7) throw swl::Error(SWL_ERR_INVALID, "state needs at least 7x7 padded nodes");
        if (!v->vx || !v->vz || !v->sxx || !v->szz || !v->sxz || !v->lambda || !v->mu || !v->rho || !v->jac || !v->normals)
            throw swl::Error(SWL_ERR_INVALID, "every field and model pointer of the state is required");
        if (v->pml && (v->cpml_width_x < 0 || v->cpml_width_z < 1))
            throw swl::Error(SWL_ERR_INVALID, "CFS-PML widths are required with the memories");
        // The memory slots of a node are computed from the widths; widths wider than the grid
        // would index past the caller's memories (the reference caps them at a third of the grid,
        // src/two_d/CurvilinearSolver2D.cpp:507).
        if (v->pml && (2 * int64_t(v->cpml_width_x) > v->nx - 6 || v->cpml_width_z > v->nz - 6))
            throw swl::Error(SWL_ERR_INVALID, "CFS-PML widths exceed the grid: need 2*wx <= nx-6 and wz <= nz-6");
        const dim3 block(kBlockX, kBlockY), grid((v->nx - 6 + kBlockX - 1) / kBlockX, (v->nz - 6 + kBlockY - 1) / kBlockY);
        const long long blocks = (long long)grid.x * grid.y;
        if (blocks > kMaxBlocks)
            throw swl::Error(SWL_ERR_INVALID, "state too large for swl2d_stats_noalloc: " + std::to_string(blocks) +
                                                  " blocks of 32x8 nodes, at most " + std::to_string(kMaxBlocks));
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        Part *scratch = scratchAddress(s);
        partials<<<grid, block, 0, s>>>(*v, scratch);
        swl::check(cudaGetLastError(), "no-allocation diagnostics launch");
        finish<<<1, 1024, 0, s>>>(scratch, int(blocks), out);
        swl::check(cudaGetLastError(), "no-allocation diagnostics reduction");
        return SWL_OK;
    } catch (const swl::Error &e) {
        swl::lastErrorRef() = e.what();
        return e.status;
    } catch (const std::exception &e) {
        swl::lastErrorRef() = e.what();
        return SWL_ERR_INVALID;
    }
}
