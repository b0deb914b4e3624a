// Device inventory and shared host math.
#include "runtime.cuh"
#include <cmath>

namespace swl {

// Device selection in the manner of selectCudaDevice3D (src/common/ComputeDevices.cpp:16-40):
// an explicit index must be a usable sm_100 device; -1 picks the one with the most memory.
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

// src/two_d/CurvilinearSolver2D.cpp:31-34
double ricker(double t, double f) {
    const double a = 3.14159265358979323846 * f * (t - 1.5 / f);
    return (1 - 2 * a * a) * std::exp(-a * a);
}

} // namespace swl
