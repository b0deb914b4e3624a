// Device inventory and shared host math.
#include "runtime.cuh"
#include <algorithm>
#include <map>
#include <mutex>
#include <cmath>

namespace swl {

// Device selection in the manner of selectCudaDevice3D (src/common/ComputeDevices.cpp:16-40):
// an explicit index must be a usable sm_100 device; -1 picks the one with the most memory.
namespace {
constexpr std::size_t kPinnedCacheBytes = std::size_t(1) << 30;
std::mutex pinnedMutex;
std::multimap<std::size_t, void *> pinnedIdle; // size -> block
std::size_t pinnedIdleBytes = 0;
} // namespace

void *pinnedTake(std::size_t n, std::size_t &got) {
    {
        std::lock_guard<std::mutex> g(pinnedMutex);
        const auto it = pinnedIdle.lower_bound(n);
        if (it != pinnedIdle.end() && it->first <= 4 * n + 4096) { // first fit, not far larger
            void *p = it->second;
            got = it->first;
            pinnedIdleBytes -= it->first;
            pinnedIdle.erase(it);
            return p;
        }
    }
    const std::size_t size = std::max<std::size_t>(n, 4096);
    void *p = nullptr;
    check(cudaMallocHost(&p, size), "allocate pinned host buffer");
    got = size;
    return p;
}

void pinnedGive(void *p, std::size_t n) {
    {
        std::lock_guard<std::mutex> g(pinnedMutex);
        if (pinnedIdleBytes + n <= kPinnedCacheBytes) {
            pinnedIdle.emplace(n, p);
            pinnedIdleBytes += n;
            return;
        }
    }
    cudaFreeHost(p);
}

int selectDevice(int requested) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    int best = -1;
    std::size_t bestMem = 0;
    for (int d = 0; d < n; ++d) {
        cudaDeviceProp p{};
        if (cudaGetDeviceProperties(&p, d) != cudaSuccess) continue;
        if (p.major != 10) continue; // the kernels are built for sm_100a only
        if (requested >= 0) {
            if (d == requested) return d;
            continue;
        }
        if (p.totalGlobalMem > bestMem) best = d, bestMem = p.totalGlobalMem;
    }
    return requested >= 0 ? -1 : best;
}

void encodeTensorMap3D(CUtensorMap *map, bool fp64, const void *base, const uint64_t dims[3], const uint64_t strides[2],
                       const uint32_t box[3]) {
    using Encode = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *, const cuuint64_t *,
                                const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static Encode encode = [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        check(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q), "find the tensor-map encoder");
        if (!fn || q != cudaDriverEntryPointSuccess) throw Error(-5, "the driver has no tensor-map encoder");
        return reinterpret_cast<Encode>(fn);
    }();
    const cuuint64_t gdim[3] = {dims[0], dims[1], dims[2]}, gstride[2] = {strides[0], strides[1]};
    const cuuint32_t bdim[3] = {box[0], box[1], box[2]}, estride[3] = {1, 1, 1};
    const CUresult r = encode(map, fp64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void *>(base),
                              gdim, gstride, bdim, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(-2, "CUDA encode tensor map: error " + std::to_string(int(r)));
}

// src/two_d/CurvilinearSolver2D.cpp:31-34
double ricker(double t, double f) {
    const double a = 3.14159265358979323846 * f * (t - 1.5 / f);
    return (1 - 2 * a * a) * std::exp(-a * a);
}

} // namespace swl
