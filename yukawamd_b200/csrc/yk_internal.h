// yk_internal.h -- helpers shared by the engine's translation units
// (not part of the C-ABI; hidden symbols).
#pragma once

#include "../../include/yukawa_engine.h"
#include "yk_force.cuh"
#include "yk_verlet.cuh"

namespace yk {

// Kernel argument blocks of one box (same builder for single boxes,
// batches and the allocation-free call).
void make_args(const yk_params& p, int n, ForceArgs* fa, StepArgs* sa, FinishArgs* fz);

// Add k to the process-wide count of kernels launched by this library.
void count_launches(int k);

}  // namespace yk
