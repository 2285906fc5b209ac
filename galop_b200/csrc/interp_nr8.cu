// Instantiations of the interpreter for 8-register ISAs.
#include "interp.cuh"

namespace galop {

template <int K, int P>
static const void* pick_mode(int reduce, int mode) {
    if (mode == kModeOutputs) return (const void*)&interp_kernel<8, K, P, kReduceFp64, kModeOutputs>;
    if (mode == kModeTrace) return (const void*)&interp_kernel<8, K, P, kReduceFp64, kModeTrace>;
    switch (reduce) {
        case kReduceKahan32: return (const void*)&interp_kernel<8, K, P, kReduceKahan32, kModeFitness>;
        case kReduceFp64: return (const void*)&interp_kernel<8, K, P, kReduceFp64, kModeFitness>;
        case kReduceOrdered: return (const void*)&interp_kernel<8, K, P, kReduceOrdered, kModeFitness>;
        default: return nullptr;
    }
}

template <int K>
static const void* pick_profile(int profile, int reduce, int mode) {
    if (profile == kProfileRef) return pick_mode<K, kProfileRef>(reduce, mode);
    if (profile == kProfileBj) return pick_mode<K, kProfileBj>(reduce, mode);
    return nullptr;
}

const void* interp_kernel_nr8(int k, int profile, int reduce, int mode) {
    switch (k) {
        case 1: return pick_profile<1>(profile, reduce, mode);
        case 2: return pick_profile<2>(profile, reduce, mode);
        case 4: return pick_profile<4>(profile, reduce, mode);
        case 8: return pick_profile<8>(profile, reduce, mode);
        default: return nullptr;
    }
}

}  // namespace galop
