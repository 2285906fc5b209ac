// ref_shim.cpp -- C entry points over the reference's own evaluation code.
//
// TEST INFRASTRUCTURE ONLY: compiled by oracle/Makefile together with the
// reference's src/{Interpreter,Evaluator,EvaluatorCpu,Dataset}.cpp (read where
// they lie, never copied) into oracle/_ref/libref_*.so, one library per
// compile-time configuration (NUM_REGISTERS 8/16, INPUT_PROTECT).  Used to
// pin the CPU restatement in oracle.c and to generate golden vectors; also the
// "reference" CPU baseline of bench.py.
#include <cstdint>
#include <cstring>
#include <vector>

#include "Dataset.h"
#include "EvaluatorCpu.h"
#include "Evaluator.h"
#include "ISA.h"
#include "Interpreter.h"
#include "Introns.h"
#include "LGPConfig.h"
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// A reference Dataset (src/Dataset.h:22-38) built from raw case-major arrays,
// padded to a multiple of NUM_CONTEXTS with zero rows as the loaders do.
Dataset make_dataset(const float* inputs, const float* targets, int n, int k) {
    Dataset d;
    d.N = n;
    d.num_inputs = k;
    const int padded = d.padded_N();
    d.inputs.assign((size_t)padded * k, 0.0f);
    d.targets.assign(padded, 0.0f);
    if (n > 0) {
        std::memcpy(d.inputs.data(), inputs, (size_t)n * k * sizeof(float));
        std::memcpy(d.targets.data(), targets, (size_t)n * sizeof(float));
    }
    return d;
}

}  // namespace

extern "C" {

int ref_num_registers() { return LGPConfig::NUM_REGISTERS; }
int ref_output_reg() { return LGPConfig::OUTPUT_REG; }
int ref_input_protect() { return LGPConfig::INPUT_PROTECT ? 1 : 0; }
int ref_max_program_size() { return LGPConfig::MAX_PROGRAM_SIZE; }
int ref_num_contexts() { return LGPConfig::NUM_CONTEXTS; }
void ref_constants(float* out) {
    for (int i = 0; i < LGPConfig::NUM_CONSTANTS; ++i) out[i] = LGPConfig::CONSTANTS[i];
}

uint32_t ref_encode_manual(int op, int dest, int src1, int src2, int is_const) {
    return ISA::encode_manual((uint8_t)op, (uint8_t)dest, (uint8_t)src1, (uint8_t)src2, is_const != 0);
}
uint32_t ref_encode_from_random(uint32_t raw) { return ISA::encode_from_random(raw); }
void ref_decode(uint32_t w, int* out5) {
    out5[0] = ISA::get_op(w);
    out5[1] = ISA::get_dest_index(w);
    out5[2] = ISA::get_src1_index(w);
    out5[3] = ISA::get_src2_index(w);
    out5[4] = ISA::is_src2_constant(w) ? 1 : 0;
}
float ref_apply_op(int op, float a, float b) { return ISA::apply_op((uint8_t)op, a, b); }

// Interpreter::run_stateless over NUM_CONTEXTS contexts (src/Interpreter.cpp:36-59).
void ref_run_stateless(const uint32_t* prog, int len, const float* inputs, int num_inputs, float* outputs) {
    Interpreter::run_stateless(prog, len, inputs, num_inputs, outputs);
}

// Per-case outputs for n cases, chunked by NUM_CONTEXTS exactly as
// Evaluator::evaluate_sr_mse drives the interpreter (src/Evaluator.cpp:23-33).
void ref_case_outputs(const uint32_t* prog, int len, const float* inputs, int num_inputs, int n,
                      float* out) {
    constexpr int C = LGPConfig::NUM_CONTEXTS;
    const int padded = ((n + C - 1) / C) * C;
    std::vector<float> pad((size_t)padded * num_inputs, 0.0f);
    if (n > 0) std::memcpy(pad.data(), inputs, (size_t)n * num_inputs * sizeof(float));
    float chunk[C];
    for (int base = 0; base < n; base += C) {
        Interpreter::run_stateless(prog, len, pad.data() + (size_t)base * num_inputs, num_inputs, chunk);
        const int valid = (n - base) < C ? (n - base) : C;
        for (int c = 0; c < valid; ++c) out[base + c] = chunk[c];
    }
}

// CpuEvaluator::evaluate_population (src/EvaluatorCpu.cpp:7-15): dense
// programs, stride MAX_PROGRAM_SIZE, uint8 lengths.
void ref_evaluate_population(const uint32_t* instr, const uint8_t* lengths, float* fitness, int n,
                             const float* inputs, const float* targets, int n_cases, int num_inputs) {
    Dataset d = make_dataset(inputs, targets, n_cases, num_inputs);
    CpuEvaluator{}.evaluate_population(instr, lengths, fitness, n, d);
}

// Evaluator::evaluate_sr_mse + Fitness::mse_to_fitness per CSR program
// (src/Evaluator.cpp:11-45, :88-91).  ProgramView takes an int length, so
// programs longer than the uint8 engine limit run unchanged.  threads > 1:
// OpenMP parallel for over programs, each program still evaluated serially.
void ref_evaluate_csr(const uint32_t* words, const int64_t* offsets, int64_t n, const float* inputs,
                      const float* targets, int n_cases, int num_inputs, float* fitness, float* mse_out,
                      int threads) {
    Dataset d = make_dataset(inputs, targets, n_cases, num_inputs);
#ifdef _OPENMP
    if (threads < 1) threads = omp_get_max_threads();
    #pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
#endif
    for (int64_t i = 0; i < n; ++i) {
        ProgramView pv{words + offsets[i], (int)(offsets[i + 1] - offsets[i])};
        const float mse = Evaluator::evaluate_sr_mse(pv, d);
        if (mse_out) mse_out[i] = mse;
        fitness[i] = Fitness::mse_to_fitness(mse);
    }
    (void)threads;
}

// Evaluator::evaluate_sr_r2 + Fitness::r2_to_fitness (src/Evaluator.cpp:49-97)
// with the dataset's ss_tot given (as the reference's loaders compute it).
void ref_evaluate_csr_r2(const uint32_t* words, const int64_t* offsets, int64_t n, const float* inputs,
                         const float* targets, int n_cases, int num_inputs, double ss_tot, float* fitness,
                         float* r2_out) {
    Dataset d = make_dataset(inputs, targets, n_cases, num_inputs);
    d.ss_tot = ss_tot;
    for (int64_t i = 0; i < n; ++i) {
        ProgramView pv{words + offsets[i], (int)(offsets[i + 1] - offsets[i])};
        const float r2 = Evaluator::evaluate_sr_r2(pv, d);
        if (r2_out) r2_out[i] = r2;
        fitness[i] = Fitness::r2_to_fitness(r2);
    }
}

// load_csv_1d / load_csv_multi (src/Dataset.cpp:83-151).  With inputs ==
// NULL only the sizes and ss_tot are returned; call again with buffers of
// n*k and n floats.  -1 when the reference's loader throws.
int ref_load_csv(const char* path, int multi, int64_t* n, int* k, float* inputs, float* targets,
                 double* ss_tot) {
    try {
        const Dataset d = multi ? load_csv_multi(path) : load_csv_1d(path);
        *n = d.N;
        *k = d.num_inputs;
        *ss_tot = d.ss_tot;
        if (inputs)
            for (int64_t i = 0; i < (int64_t)d.N * d.num_inputs; ++i) inputs[i] = d.inputs[i];
        if (targets)
            for (int64_t i = 0; i < d.N; ++i) targets[i] = d.targets[i];
        return 0;
    } catch (...) {
        return -1;
    }
}

// Introns::effective_mask (src/Introns.h:28-46).
int ref_effective_mask(const uint32_t* prog, int len, char* mask) {
    return Introns::effective_mask(prog, len, mask);
}

// make_sr_dataset_1d + write_csv (src/Dataset.cpp:49-81) for Nguyen target
// `which` (1..6), as tools/gen_datasets.cpp:15-27 drives them.
int ref_write_nguyen_csv(int which, int n, float lo, float hi, uint32_t seed, const char* path) {
    float (*fns[6])(float) = {Nguyen::Nguyen_1, Nguyen::Nguyen_2, Nguyen::Nguyen_3,
                              Nguyen::Nguyen_4, Nguyen::Nguyen_5, Nguyen::Nguyen_6};
    if (which < 1 || which > 6) return -1;
    write_csv(make_sr_dataset_1d(n, lo, hi, fns[which - 1], seed), path);
    return 0;
}

int ref_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
