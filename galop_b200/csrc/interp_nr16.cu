// Instantiations of the interpreter for 16-register ISAs.
#include "interp.cuh"
#include "interp_wide.cuh"

namespace galop {

template <int K, int P>
static const void* pick_wide_mode(int reduce, int mode) {
    if (mode == kModeOutputs) return (const void*)&interp_wide_kernel<16, K, P, kReduceFp64, kModeOutputs>;
    if (mode == kModeTrace) return (const void*)&interp_wide_kernel<16, K, P, kReduceFp64, kModeTrace>;
    switch (reduce) {
        case kReduceKahan32: return (const void*)&interp_wide_kernel<16, K, P, kReduceKahan32, kModeFitness>;
        case kReduceFp64: return (const void*)&interp_wide_kernel<16, K, P, kReduceFp64, kModeFitness>;
        case kReduceOrdered: return (const void*)&interp_wide_kernel<16, K, P, kReduceOrdered, kModeFitness>;
        default: return nullptr;
    }
}

template <int K, int P>
static const void* pick_smem_mode(int reduce, int mode) {
    if (mode == kModeOutputs) return (const void*)&interp_smem_kernel<16, K, P, kReduceFp64, kModeOutputs>;
    if (mode == kModeTrace) return (const void*)&interp_smem_kernel<16, K, P, kReduceFp64, kModeTrace>;
    switch (reduce) {
        case kReduceKahan32: return (const void*)&interp_smem_kernel<16, K, P, kReduceKahan32, kModeFitness>;
        case kReduceFp64: return (const void*)&interp_smem_kernel<16, K, P, kReduceFp64, kModeFitness>;
        case kReduceOrdered: return (const void*)&interp_smem_kernel<16, K, P, kReduceOrdered, kModeFitness>;
        default: return nullptr;
    }
}

template <int K>
static const void* pick_dispatch(int dispatch, int profile, int reduce, int mode) {
    if (dispatch == 3) {
        if (profile == kProfileRef) return pick_wide_mode<K, kProfileRef>(reduce, mode);
        if (profile == kProfileBj) return pick_wide_mode<K, kProfileBj>(reduce, mode);
        return nullptr;
    }
    if (dispatch == 2) {
        if (profile == kProfileRef) return pick_smem_mode<K, kProfileRef>(reduce, mode);
        if (profile == kProfileBj) return pick_smem_mode<K, kProfileBj>(reduce, mode);
        return nullptr;
    }
    return nullptr;
}

const void* interp_kernel_nr16(int k, int dispatch, int profile, int reduce, int mode) {
    switch (k) {
        case 1: return pick_dispatch<1>(dispatch, profile, reduce, mode);
        case 2: return pick_dispatch<2>(dispatch, profile, reduce, mode);
        case 4: return pick_dispatch<4>(dispatch, profile, reduce, mode);
        case 8: return pick_dispatch<8>(dispatch, profile, reduce, mode);
        default: return nullptr;
    }
}

}  // namespace galop
