// Instantiations of the persistent multi-shot 2D kernel for one precision (SWL_STAGE_REAL) and
// one GSLS mechanism count (SWL_STAGE_MECH); build.py compiles this unit once per pair, with
// SWL_STAGE_COHERENT (state written within the launch is read by coherent loads, not the read-only path).
#include "launchq2d.cuh"

#ifndef SWL_STAGE_REAL
#error "SWL_STAGE_REAL (float or double) must be defined"
#endif
#ifndef SWL_STAGE_MECH
#error "SWL_STAGE_MECH (0..3) must be defined"
#endif
#ifndef SWL_STAGE_COHERENT
#error "SWL_STAGE_COHERENT must be defined for the persistent kernel"
#endif

namespace swl::detail2 {

template <class Real, int MECH> int queueOccupancy2D() {
    static const int blocks = [] {
        auto kernel = k2::queue2d<Real, MECH>;
        check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(k2::streamBytes<Real>())),
              "2D queue shared memory");
        check(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, int(cudaSharedmemCarveoutMaxShared)),
              "2D queue shared-memory carveout");
        int n = 0;
        check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, k2::STREAM_THREADS, k2::streamBytes<Real>()),
              "2D queue occupancy");
        return n;
    }();
    return blocks;
}

template <class Real, int MECH>
void launchQueue2D(int blocks, cudaStream_t stream, k2::QueueHeader *header, const k2::QueueShot<Real> *shots) {
    queueOccupancy2D<Real, MECH>(); // opts the kernel into its shared memory once
    k2::queue2d<Real, MECH><<<blocks, dim3(k2::SW, k2::SB), k2::streamBytes<Real>(), stream>>>(header, shots);
    check(cudaGetLastError(), "2D queue launch");
}

template void launchQueue2D<SWL_STAGE_REAL, SWL_STAGE_MECH>(int, cudaStream_t, k2::QueueHeader *, const k2::QueueShot<SWL_STAGE_REAL> *);
template int queueOccupancy2D<SWL_STAGE_REAL, SWL_STAGE_MECH>();

} // namespace swl::detail2
