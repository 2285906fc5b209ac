// ref_cuda_shim.cu -- launches the reference's own GPU kernel for timing.
//
// TEST / BASELINE INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file
// together with the reference's src/EvaluatorCuda.cu (read where it lies)
// for sm_100a with the reference's nvcc flags (its Makefile:43, -arch=native
// replaced by the B200's sm_100a), 16-register configuration, into
// oracle/_ref/libref_cuda_nr16.so.  The launch mirrors how the reference's
// capacity probe drives evaluate_kernel_packed (tests/cuda_capacity.cu:119-132):
// grid ceil(n/8) x 256 threads, CSR int64 offsets, case-major inputs padded
// to a multiple of 32 cases.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstring>
#include <vector>

#include "LGPConfig.h"
#include "eval_kernels.cuh"

extern "C" {

// Uploads one CSR population and a case-major dataset, runs the reference
// kernel `reps` times, returns the fitness of the last run and the mean
// kernel time (CUDA events).  Returns 0 on success, else a cudaError_t.
int refcuda_evaluate_packed(const uint32_t* words, const int64_t* offsets, int n, const float* inputs,
                            const float* targets, int n_cases, int num_inputs, int reps, float* fitness,
                            float* mean_kernel_ms) {
    const int padded = ((n_cases + LGPConfig::NUM_CONTEXTS - 1) / LGPConfig::NUM_CONTEXTS) *
                       LGPConfig::NUM_CONTEXTS;
    std::vector<float> xin((size_t)padded * num_inputs, 0.0f), yin((size_t)padded, 0.0f);
    std::memcpy(xin.data(), inputs, (size_t)n_cases * num_inputs * sizeof(float));
    std::memcpy(yin.data(), targets, (size_t)n_cases * sizeof(float));
    uint32_t* d_words = nullptr;
    long long* d_off = nullptr;
    float *d_x = nullptr, *d_y = nullptr, *d_fit = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t err = cudaSuccess;
    const size_t nw = (size_t)offsets[n];
#define REF_TRY(x) do { err = (x); if (err != cudaSuccess) goto done; } while (0)
    REF_TRY(cudaMalloc(&d_words, nw * sizeof(uint32_t) + 4));
    REF_TRY(cudaMalloc(&d_off, (size_t)(n + 1) * sizeof(long long)));
    REF_TRY(cudaMalloc(&d_x, xin.size() * sizeof(float) + 4));
    REF_TRY(cudaMalloc(&d_y, yin.size() * sizeof(float) + 4));
    REF_TRY(cudaMalloc(&d_fit, (size_t)n * sizeof(float) + 4));
    REF_TRY(cudaMemcpy(d_words, words, nw * sizeof(uint32_t), cudaMemcpyHostToDevice));
    REF_TRY(cudaMemcpy(d_off, offsets, (size_t)(n + 1) * sizeof(long long), cudaMemcpyHostToDevice));
    REF_TRY(cudaMemcpy(d_x, xin.data(), xin.size() * sizeof(float), cudaMemcpyHostToDevice));
    REF_TRY(cudaMemcpy(d_y, yin.data(), yin.size() * sizeof(float), cudaMemcpyHostToDevice));
    cuda_upload_constants();
    REF_TRY(cudaEventCreate(&e0));
    REF_TRY(cudaEventCreate(&e1));
    {
        const int threads = 256, wpb = threads / 32;
        const int blocks = (int)(((long long)n + wpb - 1) / wpb);
        evaluate_kernel_packed<<<blocks, threads>>>(d_words, d_off, d_fit, d_x, d_y, n, n_cases, num_inputs);
        REF_TRY(cudaGetLastError());
        REF_TRY(cudaDeviceSynchronize());
        REF_TRY(cudaEventRecord(e0));
        for (int r = 0; r < reps; ++r)
            evaluate_kernel_packed<<<blocks, threads>>>(d_words, d_off, d_fit, d_x, d_y, n, n_cases, num_inputs);
        REF_TRY(cudaEventRecord(e1));
        REF_TRY(cudaEventSynchronize(e1));
        REF_TRY(cudaGetLastError());
        float ms = 0.0f;
        REF_TRY(cudaEventElapsedTime(&ms, e0, e1));
        *mean_kernel_ms = ms / (reps > 0 ? reps : 1);
        REF_TRY(cudaMemcpy(fitness, d_fit, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost));
    }
done:
#undef REF_TRY
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(d_words);
    cudaFree(d_off);
    cudaFree(d_x);
    cudaFree(d_y);
    cudaFree(d_fit);
    return (int)err;
}

}  // extern "C"
