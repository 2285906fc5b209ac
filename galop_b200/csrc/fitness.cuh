// fitness.cuh -- fitness of a program from its sum of squared errors.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace galop {

enum ObjectiveKind : int32_t { kObjectiveMse = 0, kObjectiveR2 = 1 };

// What "fitness" means for a dataset: the objective, and for R^2 the total
// sum of squares of its targets (computed on the host, in case order).
struct Objective {
    int32_t kind;
    int32_t reserved;
    double ss_tot;
};

// MSE: Fitness::mse_to_fitness(float(sse / N)) (src/Evaluator.cpp:44,
// :88-91).  R^2: Evaluator::evaluate_sr_r2 (src/Evaluator.cpp:49-85; 0 for a
// degenerate target or a non-finite sse, else float(1 - sse / ss_tot)) and
// Fitness::r2_to_fitness (:93-97; non-finite -> 0, negative -> 0).
__device__ __forceinline__ float fitness_of(double sse, int64_t n_cases, const Objective& obj) {
    if (obj.kind == kObjectiveR2) {
        if (!(obj.ss_tot > 0.0) || !isfinite(sse)) return 0.0f;
        const float r2 = (float)__dsub_rn(1.0, __ddiv_rn(sse, obj.ss_tot));
        if (!isfinite(r2)) return 0.0f;
        return r2 < 0.0f ? 0.0f : r2;
    }
    const float mse = (float)(sse / (double)n_cases);
    if (!isfinite(mse)) return 0.0f;
    return __fdiv_rn(1.0f, __fadd_rn(1.0f, mse));
}

}  // namespace galop
