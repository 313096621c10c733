// simple.cuh -- batched SIMPLE stages (stages.cu), used by the single-case API and the service.
#pragma once
#include "case.cuh"

namespace ufvm {

int stage_init(const BatchLaunch& b, bool compute_mdot);          // BCs, gradients, mdot_f
int stage_update_fields(const BatchLaunch& b);                    // cfdUpdateFields
// cfdAssembleEquation('U', comp); interior_ready: stage_uface_interior has formed the interior
// faces' terms of all three components in this iteration
int stage_assemble_u(const BatchLaunch& b, int comp, bool interior_ready = false);
int stage_uface_interior(const BatchLaunch& b);  // interior face terms of U, all three components
int stage_assemble_p(const BatchLaunch& b);                       // cfdAssembleEquation('p')
int stage_correct_u(const BatchLaunch& b, int comp);              // cfdCorrectEquation('U', comp)
int stage_correct_p(const BatchLaunch& b, int max_patches, double* unused);  // cfdCorrectEquation('p')

}  // namespace ufvm
