// Launch interface of the 2D stage kernels.  The kernels are instantiated in stages2d.cu, once
// per (precision, GSLS mechanism count), as separate compilation units built in parallel; the
// engine only calls these functions.
#pragma once
#include "stage2d.cuh"

namespace swl::detail2 {

// One RK stage: MacCormack directions (dx, dz) of this (step, stage), on `stream`.
template <class Real, int MECH>
void launchStage2D(int dx, int dz, int stage, dim3 grid, dim3 block, cudaStream_t stream, const k2::StageArgs<Real> &args);
// Opt every stage instantiation into its dynamic shared memory and the largest carveout.
template <class Real, int MECH> void prepareStages2D();
// Attributes (registers, local memory) of one stage instantiation.
template <class Real, int MECH> cudaFuncAttributes stageAttributes2D();

} // namespace swl::detail2
