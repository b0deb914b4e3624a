// FP32 instantiation of the 3D engine (serving form; the reference 3D path is FP64 only).
#include "engine3d.cuh"

namespace swl {
std::unique_ptr<Engine3D> makeEngine3D32(const swl_mesh3d &m, const int64_t *rec, int n, int device) {
    return std::make_unique<TypedEngine3D<float>>(m, rec, n, device);
}
} // namespace swl
