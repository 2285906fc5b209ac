// dedup.cuh -- programs whose interpreted micro-ops are identical get the
// same fitness, so only one of each is interpreted.
//
// Evolved populations are mostly copies of each other once introns are
// stripped (neutral mutations land in non-effective code): after 100
// generations of the reference engine's standard settings, 82-85% of the
// programs have an effective program another one already has.  Each
// program's interpreted micro-ops are hashed, the (hash, program) pairs are
// radix-sorted, a max-scan gives every sorted position the first position
// of its run of equal hashes, and every member whose micro-ops equal the
// run head's word for word takes the head as its representative (a member
// that only collides in the hash keeps itself).
// Representatives are ordered and interpreted as usual; the others are
// left out of the work queue and receive their representative's fitness
// afterwards.  The fitness of a copy is the representative's, computed by
// the same kernel on the same micro-ops with the same case chunking, so it
// is the value the copy itself would have received.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace galop {

// 64-bit FNV-1a over the length and the micro-op words.
// group (may be null): programs of different groups (populations of a
// batch, each on its own dataset) are never merged.
// livein (may be null): the per-program live-in words of the folding pass,
// part of what makes two programs equal (renamed micro-ops do not say which
// registers their slots start from).
static __global__ void dedup_hash_kernel(const uint4* __restrict__ uops, const int64_t* __restrict__ eff_off,
                                         const int32_t* __restrict__ len, int64_t n,
                                         unsigned long long* __restrict__ keys, int32_t* __restrict__ vals,
                                         int32_t* __restrict__ rep, const int32_t* __restrict__ group,
                                         const uint32_t* __restrict__ livein) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t L = len[i];
    const uint4* p = uops + eff_off[i + 1] - L;   // packed against the slot's end (fold.cuh)
    unsigned long long h = 0xcbf29ce484222325ull;
    auto mix = [&](uint32_t w) {
        h ^= w;
        h *= 0x100000001b3ull;
    };
    mix((uint32_t)L);
    if (group) mix((uint32_t)group[i]);
    if (livein) mix(livein[i]);
    for (int32_t j = 0; j < L; ++j) {
        const uint4 u = p[j];
        mix(u.x);
        mix(u.y);
        mix(u.z);
        mix(u.w);
    }
    keys[i] = h;
    vals[i] = (int32_t)i;
    rep[i] = (int32_t)i;
}

// Position of the first element of each run of equal hashes: j where the
// hash changes, 0 elsewhere (an inclusive max-scan then gives every
// position its run's first position).
static __global__ void dedup_run_start_kernel(const unsigned long long* __restrict__ keys, int64_t n,
                                              int32_t* __restrict__ start) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    start[j] = (j > 0 && keys[j] == keys[j - 1]) ? 0 : (int32_t)j;
}

// Every member of a run compares its micro-ops with the run head's; an
// equal one points at the head and leaves the work order.  dup_count[0]
// counts the copies, dup_count[1] their interpreted instructions.
static __global__ void dedup_rep_kernel(const int32_t* __restrict__ head_pos, const int32_t* __restrict__ vals,
                                        int64_t n, const uint4* __restrict__ uops,
                                        const int64_t* __restrict__ eff_off, int32_t* __restrict__ len,
                                        int32_t* __restrict__ rep, unsigned long long* __restrict__ dup_count,
                                        const int32_t* __restrict__ group, const uint32_t* __restrict__ livein) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool copy = false;
    int32_t L = 0;
    if (j < n) {
        const int64_t h = head_pos[j];
        if (h != j) {
            const int32_t head = vals[h], i = vals[j];
            L = len[head];
            if (len[i] == L && (!group || group[i] == group[head]) && (!livein || livein[i] == livein[head])) {
                const uint4* hp = uops + eff_off[head + 1] - L;
                const uint4* ip = uops + eff_off[i + 1] - L;
                copy = true;
                for (int32_t k = 0; k < L && copy; ++k) {
                    const uint4 a = hp[k], b = ip[k];
                    copy = a.x == b.x && a.y == b.y && a.z == b.z && a.w == b.w;
                }
                if (copy) rep[i] = head;
            }
        }
    }
    // A copy's length marks it as left out; only this thread reads it, and
    // the head, whose length the others read, is never a copy.
    if (copy) len[vals[j]] = -1;
    __shared__ unsigned long long sc, si;
    if (threadIdx.x == 0) { sc = 0; si = 0; }
    __syncthreads();
    if (copy) {
        atomicAdd(&sc, 1ull);
        atomicAdd(&si, (unsigned long long)L);
    }
    __syncthreads();
    if (threadIdx.x == 0 && sc) {
        atomicAdd(&dup_count[0], sc);
        atomicAdd(&dup_count[1], si);
    }
}

// Copies take their representative's results.
static __global__ void dedup_scatter_kernel(const int32_t* __restrict__ rep, int64_t n, float* __restrict__ fitness,
                                            double* __restrict__ sse) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t r = rep[i];
    if (r == (int32_t)i) return;
    fitness[i] = fitness[r];
    if (sse) sse[i] = sse[r];
}

}  // namespace galop
