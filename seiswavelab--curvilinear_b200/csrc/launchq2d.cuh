// Launch interface of the persistent multi-shot 2D kernel (queue2d.cuh).  It is instantiated in
// queue2d.cu, once per (precision, GSLS mechanism count), with the coherent state loads.
#pragma once
#include "queue2d.cuh"

namespace swl::detail2 {

template <class Real, int MECH>
void launchQueue2D(int blocks, cudaStream_t stream, k2::QueueHeader *header, const k2::QueueShot<Real> *shots);
// Resident CTAs per SM of the instantiation (after opting it into its shared memory).
template <class Real, int MECH> int queueOccupancy2D();

} // namespace swl::detail2
