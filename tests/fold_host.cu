// Host build of the folding pass (galop_b200/csrc/fold.cuh) for the CPU
// tests: fold_one is the function fold_kernel runs for each program, here
// called on the CPU on one program's wide micro-ops (four uint32 each).
#include "fold.cuh"

extern "C" int64_t fold_host(uint32_t* u, int64_t L, int profile, int num_registers, int output_reg,
                             uint32_t stride_shift, int k_in, int fold, int rename, uint32_t* livein) {
    galop::FoldParams fp{profile, num_registers, output_reg, stride_shift, k_in, nullptr, nullptr, fold, rename};
    uint32_t lv = 0;
    const int64_t kept = galop::fold_one(reinterpret_cast<uint4*>(u), L, fp, k_in, lv);
    *livein = lv;
    return kept;
}
