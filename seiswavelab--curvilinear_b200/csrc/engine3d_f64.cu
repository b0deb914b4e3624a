// FP64 instantiation of the 3D engine, built with --fmad=false like the reference kernels
// (cmake/Targets.cmake:99) so the plain path reproduces the reference arithmetic.
#include "engine3d.cuh"

namespace swl {
std::unique_ptr<Engine3D> makeEngine3D64(const swl_mesh3d &m, const int64_t *rec, int n, int device) {
    return std::make_unique<TypedEngine3D<double>>(m, rec, n, device);
}
} // namespace swl
