// FP32 instantiation of the 2D engine (the batched serving form): FP32 state, coefficients
// and accumulation, FMA contraction allowed.
#include "engine2d.cuh"

namespace swl {
std::unique_ptr<Engine2D> makeEngine2D32(const swl_mesh2d &m, const int64_t *rec, int n, int device) {
    return std::make_unique<TypedEngine2D<float>>(m, rec, n, device);
}
std::unique_ptr<Queue2D> makeQueue2D32(int device) { return std::make_unique<TypedQueue2D<float>>(device); }
} // namespace swl
