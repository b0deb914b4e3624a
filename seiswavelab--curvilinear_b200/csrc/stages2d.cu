// Instantiations of the 2D stage kernels for one precision (SWL_STAGE_REAL) and one GSLS
// mechanism count (SWL_STAGE_MECH); build.py compiles this unit once per pair.
#include "launch2d.cuh"

#ifndef SWL_STAGE_REAL
#error "SWL_STAGE_REAL (float or double) must be defined"
#endif
#ifndef SWL_STAGE_MECH
#error "SWL_STAGE_MECH (0..3) must be defined"
#endif

namespace swl::detail2 {
namespace {
template <class Real, int MECH, int DX, int DZ, int ST> void go(dim3 g, dim3 b, cudaStream_t s, const k2::StageArgs<Real> &a) {
    k2::stream2d<Real, DX, DZ, MECH, ST><<<g, b, k2::streamBytes<Real, ST>(), s>>>(a);
}
template <class Real, int MECH, int DX, int DZ> void stages(int stage, dim3 g, dim3 b, cudaStream_t s, const k2::StageArgs<Real> &a) {
    switch (stage) {
    case 0: go<Real, MECH, DX, DZ, 0>(g, b, s, a); break;
    case 1: go<Real, MECH, DX, DZ, 1>(g, b, s, a); break;
    case 2: go<Real, MECH, DX, DZ, 2>(g, b, s, a); break;
    default: go<Real, MECH, DX, DZ, 3>(g, b, s, a); break;
    }
}
template <class Real, int ST, class K> void allow(K kernel) {
    check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(k2::streamBytes<Real, ST>())),
          "2D stage shared memory");
    check(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, int(cudaSharedmemCarveoutMaxShared)),
          "2D stage shared-memory carveout");
}
template <class Real, int MECH, int DX, int DZ> void allowStages() {
    allow<Real, 0>(k2::stream2d<Real, DX, DZ, MECH, 0>), allow<Real, 1>(k2::stream2d<Real, DX, DZ, MECH, 1>);
    allow<Real, 2>(k2::stream2d<Real, DX, DZ, MECH, 2>), allow<Real, 3>(k2::stream2d<Real, DX, DZ, MECH, 3>);
}
} // namespace

template <class Real, int MECH>
void launchStage2D(int dx, int dz, int stage, dim3 g, dim3 b, cudaStream_t s, const k2::StageArgs<Real> &a) {
    if (dx == 0 && dz == 0) stages<Real, MECH, 0, 0>(stage, g, b, s, a);
    else if (dx == 0) stages<Real, MECH, 0, 1>(stage, g, b, s, a);
    else if (dz == 0) stages<Real, MECH, 1, 0>(stage, g, b, s, a);
    else stages<Real, MECH, 1, 1>(stage, g, b, s, a);
}
template <class Real, int MECH> void prepareStages2D() {
    allowStages<Real, MECH, 0, 0>(), allowStages<Real, MECH, 0, 1>(), allowStages<Real, MECH, 1, 0>(), allowStages<Real, MECH, 1, 1>();
}
template <class Real, int MECH> cudaFuncAttributes stageAttributes2D() {
    cudaFuncAttributes attr{};
    check(cudaFuncGetAttributes(&attr, k2::stream2d<Real, 0, 0, MECH, 1>), "2D kernel compatibility");
    return attr;
}

template void launchStage2D<SWL_STAGE_REAL, SWL_STAGE_MECH>(int, int, int, dim3, dim3, cudaStream_t,
                                                             const k2::StageArgs<SWL_STAGE_REAL> &);
template void prepareStages2D<SWL_STAGE_REAL, SWL_STAGE_MECH>();
template cudaFuncAttributes stageAttributes2D<SWL_STAGE_REAL, SWL_STAGE_MECH>();

} // namespace swl::detail2
