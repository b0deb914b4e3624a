// FP64 instantiation of the 2D engine.  Built with --fmad=false: the reference builds its
// kernels without FMA contraction (cmake/Targets.cmake:99) and its CPU oracle has none, so
// the plain FP64 path reproduces the reference arithmetic operation for operation.
#include "engine2d.cuh"

namespace swl {
std::unique_ptr<Engine2D> makeEngine2D64(const swl_mesh2d &m, const int64_t *rec, int n, int device) {
    return std::make_unique<TypedEngine2D<double>>(m, rec, n, device);
}
std::unique_ptr<Queue2D> makeQueue2D64(int device) { return std::make_unique<TypedQueue2D<double>>(device); }
} // namespace swl
