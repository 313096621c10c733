// simple.cuh -- batched SIMPLE stages (stages.cu), used by the single-case API and the service.
#pragma once
#include "case.cuh"

namespace ufvm {

int stage_init(const BatchLaunch& b, bool compute_mdot);          // BCs, gradients, mdot_f
int stage_update_fields(const BatchLaunch& b);                    // cfdUpdateFields
int stage_assemble_u(const BatchLaunch& b, int comp);             // cfdAssembleEquation('U', comp)
int stage_assemble_p(const BatchLaunch& b);                       // cfdAssembleEquation('p')
int stage_correct_u(const BatchLaunch& b, int comp);              // cfdCorrectEquation('U', comp)
int stage_correct_p(const BatchLaunch& b, int max_patches, double* unused);  // cfdCorrectEquation('p')

}  // namespace ufvm
