/*
 * oracle.c -- CPU restatement of Galop's linear-GP fitness evaluation.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
 * compared against; it is never linked into, loaded by, or called from the
 * product library (galop_b200/csrc).  Only tests/, the smoke check in
 * __graft_entry__.py and the cpu_baseline / --impl reference legs of bench.py
 * load it.
 *
 * It restates, with runtime parameters instead of compile-time ones, the
 * reference's evaluation path:
 *
 *   decode           src/ISA.h:176-206   (get_op, get_dest_index incl. the
 *                                         INPUT_PROTECT fold :183-185,
 *                                         get_src1_index, get_src2_index,
 *                                         is_src2_constant)
 *   apply_op         src/ISA.h:219-231
 *   run_stateless    src/Interpreter.cpp:36-59 (inputs -> r0..k-1, the rest
 *                                         0, output register OUTPUT_REG)
 *   execute          src/Interpreter.cpp:11-34
 *   evaluate_sr_mse  src/Evaluator.cpp:11-45 (double SSE summed in case
 *                                         order, float(sse/N))
 *   mse_to_fitness   src/Evaluator.cpp:88-91
 *   evaluate_pop.    src/EvaluatorCpu.cpp:7-15
 *   effective_mask   src/Introns.h:28-46
 *   extract_effect.  src/Introns.h:50-57
 *
 * Two ISA profiles share the reference's 32-bit encoding (src/ISA.h:20-41):
 *   REF: ops ADD SUB MUL DIV SIN COS LT GT  (src/ISA.h:69-72), bit-compatible
 *        with the reference; parity pinned by its tests and golden files.
 *   BJ : ops ADD SUB MUL DIV SIN COS EXP LOG, runtime constant pool.  EXP and
 *        LOG are unary like SIN/COS (they read src2 only).  Protected log is
 *        LOG(b) = (b != 0) ? logf(|b|) : 0.  No reference test covers EXP/LOG:
 *        parity for those two opcodes is unpinned.
 *
 * Transcendentals: SIN and COS use the C library's sinf/cosf, as the
 * reference does (orc_isa_t.trig = ORC_TRIG_LIBM).  With ORC_TRIG_DEVICE
 * they use the device's own functions instead.  Those come from
 * galop_b200/csrc/trig.cuh, compiled here for the host, where it gives the
 * same bits as on the GPU.  Every other op is unchanged, so GPU outputs can
 * be checked bit for bit on programs that use SIN/COS.  How far those
 * functions are from the exact values is pinned separately, against
 * correctly rounded results and glibc.
 *
 * Build: see oracle/Makefile.  Compiled with -O2 -ffp-contract=off and no
 * fast-math so that float arithmetic rounds exactly like the reference's
 * g++ -std=c++20 -O2 build (ISO mode, no FMA contraction, SSE2 arithmetic).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../galop_b200/csrc/trig.cuh"

enum { ORC_PROFILE_REF = 0, ORC_PROFILE_BJ = 1 };
enum { ORC_TRIG_LIBM = 0, ORC_TRIG_DEVICE = 1 };
/* orc_apply_op's `profile` argument: the profile, plus this flag for the
 * device's sine and cosine. */
#define ORC_OP_DEVICE_TRIG 0x100
enum { OP_ADD = 0, OP_SUB, OP_MUL, OP_DIV, OP_SIN, OP_COS, OP_6, OP_7 };

typedef struct {
    int32_t profile;        /* ORC_PROFILE_REF or ORC_PROFILE_BJ             */
    int32_t num_registers;  /* power of two, 2..128                          */
    int32_t input_protect;  /* 1: dest folded into the upper register half   */
    int32_t trig;           /* ORC_TRIG_LIBM or ORC_TRIG_DEVICE (SIN/COS)     */
    const float* constants; /* num_registers entries (pool size == NR)       */
} orc_isa_t;

typedef struct {
    uint8_t op, dest, src1, src2, is_const, unary;
} orc_ins_t;

int64_t orc_extract_effective(const orc_isa_t* isa, const uint32_t* prog, int64_t len, uint32_t* out);

/* Output register: r0, or the first scratch register NR/2 under
 * INPUT_PROTECT (src/LGPConfig.h:294-300). */
/* orc_apply_op's mode word for this configuration. */
static inline int orc_op_mode(const orc_isa_t* isa) {
    return isa->profile | (isa->trig == ORC_TRIG_DEVICE ? ORC_OP_DEVICE_TRIG : 0);
}

int orc_output_reg(const orc_isa_t* isa) {
    return isa->input_protect ? isa->num_registers / 2 : 0;
}

/* Field extraction, src/ISA.h:176-206.  The opcode field is 3 bits wide
 * (OPERATION_MASK = 7, src/LGPConfig.h:189-191); register fields are masked
 * with NR-1; src2's index uses the same mask, its bit 7 is the mode flag. */
static inline orc_ins_t orc_decode_word(const orc_isa_t* isa, uint32_t w) {
    const uint32_t rmask = (uint32_t)isa->num_registers - 1u;
    orc_ins_t d;
    d.op = (uint8_t)(w & 7u);
    if (isa->input_protect)
        d.dest = (uint8_t)(orc_output_reg(isa) + ((w >> 8) & (rmask >> 1)));
    else
        d.dest = (uint8_t)((w >> 8) & rmask);
    d.src1 = (uint8_t)((w >> 16) & rmask);
    d.src2 = (uint8_t)((w >> 24) & rmask);
    d.is_const = (uint8_t)(((w >> 24) & 0x80u) != 0);
    d.unary = (uint8_t)(d.op == OP_SIN || d.op == OP_COS ||
                        (isa->profile == ORC_PROFILE_BJ && (d.op == OP_6 || d.op == OP_7)));
    return d;
}

int orc_decode(const orc_isa_t* isa, uint32_t w, int32_t* out5) {
    orc_ins_t d = orc_decode_word(isa, w);
    out5[0] = d.op; out5[1] = d.dest; out5[2] = d.src1; out5[3] = d.src2; out5[4] = d.is_const;
    return d.unary;
}

/* Op semantics, src/ISA.h:219-231 for REF; BJ swaps LT/GT for EXP/LOG.
 * `profile` may carry ORC_OP_DEVICE_TRIG (SIN/COS as on the device). */
float orc_apply_op(int profile, int op, float a, float b) {
    const int device_trig = (profile & ORC_OP_DEVICE_TRIG) != 0;
    profile &= 0xff;
    switch (op) {
        case OP_ADD: return a + b;
        case OP_SUB: return a - b;
        case OP_MUL: return a * b;
        case OP_DIV: return (b != 0.0f) ? a / b : 1.0f;
        case OP_SIN: return device_trig ? galop_sinf(b) : sinf(b);
        case OP_COS: return device_trig ? galop_cosf(b) : cosf(b);
        case OP_6:
            if (profile == ORC_PROFILE_BJ) return expf(b);
            return (a < b) ? 1.0f : 0.0f;
        default:
            if (profile == ORC_PROFILE_BJ) return (b != 0.0f) ? logf(fabsf(b)) : 0.0f;
            return (a > b) ? 1.0f : 0.0f;
    }
}

/* apply_op over n operand pairs (replaying long register traces). */
void orc_apply_op_n(int profile, int op, const float* a, const float* b, int64_t n, float* out) {
    for (int64_t i = 0; i < n; ++i) out[i] = orc_apply_op(profile, op, a[i], b[i]);
}

/* The same op semantics in double precision: the precision-stability probe
 * the reference's differential test uses (tests/cuda_diff.cu:92-144). */
static inline double orc_apply_op_f64(int profile, int op, double a, double b) {
    switch (op) {
        case OP_ADD: return a + b;
        case OP_SUB: return a - b;
        case OP_MUL: return a * b;
        case OP_DIV: return (b != 0.0) ? a / b : 1.0;
        case OP_SIN: return sin(b);
        case OP_COS: return cos(b);
        case OP_6:
            if (profile == ORC_PROFILE_BJ) return exp(b);
            return (a < b) ? 1.0 : 0.0;
        default:
            if (profile == ORC_PROFILE_BJ) return (b != 0.0) ? log(fabs(b)) : 0.0;
            return (a > b) ? 1.0 : 0.0;
    }
}

static orc_ins_t* orc_decode_program(const orc_isa_t* isa, const uint32_t* prog, int64_t len) {
    orc_ins_t* p = (orc_ins_t*)malloc(sizeof(orc_ins_t) * (size_t)(len > 0 ? len : 1));
    for (int64_t i = 0; i < len; ++i) p[i] = orc_decode_word(isa, prog[i]);
    return p;
}

/* One fitness case: registers r0..k-1 = inputs, the rest 0
 * (src/Interpreter.cpp:47-56), run every instruction (execute,
 * src/Interpreter.cpp:11-34), return r[OUTPUT_REG]. */
static inline float orc_run_case(const orc_isa_t* isa, const orc_ins_t* p, int64_t len,
                                 const float* x, int num_inputs) {
    float r[128];
    const int nr = isa->num_registers;
    for (int i = 0; i < num_inputs; ++i) r[i] = x[i];
    for (int i = num_inputs; i < nr; ++i) r[i] = 0.0f;
    for (int64_t pc = 0; pc < len; ++pc) {
        const orc_ins_t in = p[pc];
        const float a = r[in.src1];
        const float b = in.is_const ? isa->constants[in.src2] : r[in.src2];
        r[in.dest] = orc_apply_op(orc_op_mode(isa), in.op, a, b);
    }
    return r[orc_output_reg(isa)];
}

static inline double orc_run_case_f64(const orc_isa_t* isa, const orc_ins_t* p, int64_t len,
                                      const float* x, int num_inputs) {
    double r[128];
    const int nr = isa->num_registers;
    for (int i = 0; i < num_inputs; ++i) r[i] = (double)x[i];
    for (int i = num_inputs; i < nr; ++i) r[i] = 0.0;
    for (int64_t pc = 0; pc < len; ++pc) {
        const orc_ins_t in = p[pc];
        const double a = r[in.src1];
        const double b = in.is_const ? (double)isa->constants[in.src2] : r[in.src2];
        r[in.dest] = orc_apply_op_f64(isa->profile, in.op, a, b);
    }
    return r[orc_output_reg(isa)];
}

/* Per-case outputs of one program; inputs are case-major (AoS),
 * inputs[c*num_inputs + i] as in src/Dataset.h:22-24. */
void orc_case_outputs(const orc_isa_t* isa, const uint32_t* prog, int64_t len,
                      const float* inputs, int num_inputs, int64_t n_cases, float* out) {
    orc_ins_t* p = orc_decode_program(isa, prog, len);
    for (int64_t c = 0; c < n_cases; ++c)
        out[c] = orc_run_case(isa, p, len, inputs + c * num_inputs, num_inputs);
    free(p);
}

void orc_case_outputs_f64(const orc_isa_t* isa, const uint32_t* prog, int64_t len,
                          const float* inputs, int num_inputs, int64_t n_cases, double* out) {
    orc_ins_t* p = orc_decode_program(isa, prog, len);
    for (int64_t c = 0; c < n_cases; ++c)
        out[c] = orc_run_case_f64(isa, p, len, inputs + c * num_inputs, num_inputs);
    free(p);
}

/* Register-file trace: state[(pc+1)*nr + j] = r_j after instruction pc, with
 * state[0..nr) the initial file.  One case.  Used to replay each instruction
 * of a GPU trace in isolation. */
void orc_trace_case(const orc_isa_t* isa, const uint32_t* prog, int64_t len,
                    const float* x, int num_inputs, float* state) {
    const int nr = isa->num_registers;
    float r[128];
    for (int i = 0; i < num_inputs; ++i) r[i] = x[i];
    for (int i = num_inputs; i < nr; ++i) r[i] = 0.0f;
    memcpy(state, r, sizeof(float) * (size_t)nr);
    for (int64_t pc = 0; pc < len; ++pc) {
        const orc_ins_t in = orc_decode_word(isa, prog[pc]);
        const float a = r[in.src1];
        const float b = in.is_const ? isa->constants[in.src2] : r[in.src2];
        r[in.dest] = orc_apply_op(orc_op_mode(isa), in.op, a, b);
        memcpy(state + (size_t)(pc + 1) * nr, r, sizeof(float) * (size_t)nr);
    }
}

/* SSE in double, accumulated in case order 0..N-1 (src/Evaluator.cpp:20-42):
 * err = double(out) - double(target); sse += err*err. */
double orc_sse(const orc_isa_t* isa, const uint32_t* prog, int64_t len,
               const float* inputs, const float* targets, int num_inputs, int64_t n_cases) {
    orc_ins_t* p = orc_decode_program(isa, prog, len);
    double sse = 0.0;
    for (int64_t c = 0; c < n_cases; ++c) {
        const float o = orc_run_case(isa, p, len, inputs + c * num_inputs, num_inputs);
        const double err = (double)o - (double)targets[c];
        sse += err * err;
    }
    free(p);
    return sse;
}

/* src/Evaluator.cpp:44: float(sse / double(N)). */
float orc_evaluate_sr_mse(const orc_isa_t* isa, const uint32_t* prog, int64_t len,
                          const float* inputs, const float* targets, int num_inputs,
                          int64_t n_cases) {
    const double sse = orc_sse(isa, prog, len, inputs, targets, num_inputs, n_cases);
    return (float)(sse / (double)n_cases);
}

/* src/Evaluator.cpp:88-91. */
float orc_mse_to_fitness(float mse) {
    if (!isfinite(mse)) return 0.0f;
    return 1.0f / (1.0f + mse);
}

/* Two-pass total sum of squares of the targets, each pass a double sum in
 * case order (compute_ss_tot, src/Dataset.cpp:35-47). */
double orc_ss_tot(const float* targets, int64_t n) {
    if (n <= 0) return 0.0;
    double mean = 0.0;
    for (int64_t i = 0; i < n; ++i) mean += (double)targets[i];
    mean /= (double)n;
    double ss = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double d = (double)targets[i] - mean;
        ss += d * d;
    }
    return ss;
}

/* R^2 of one program (Evaluator::evaluate_sr_r2, src/Evaluator.cpp:49-85):
 * 0 for a degenerate target (ss_tot <= 0) or a non-finite SSE, else
 * float(1 - sse/ss_tot); the SSE is the same case-order sum as the MSE's. */
float orc_evaluate_sr_r2(const orc_isa_t* isa, const uint32_t* prog, int64_t len,
                         const float* inputs, const float* targets, int num_inputs,
                         int64_t n_cases, double ss_tot) {
    if (ss_tot <= 0.0) return 0.0f;
    const double sse = orc_sse(isa, prog, len, inputs, targets, num_inputs, n_cases);
    if (!isfinite(sse)) return 0.0f;
    return (float)(1.0 - sse / ss_tot);
}

/* src/Evaluator.cpp:93-97. */
float orc_r2_to_fitness(float r2) {
    if (!isfinite(r2)) return 0.0f;
    return r2 < 0.0f ? 0.0f : r2;
}

/* R^2 fitness of CSR programs, as orc_evaluate_population_csr. */
void orc_evaluate_population_csr_r2(const orc_isa_t* isa, const uint32_t* words,
                                    const int64_t* offsets, int64_t n_programs,
                                    const float* inputs, const float* targets, int num_inputs,
                                    int64_t n_cases, float* fitness_out, int threads) {
    const double ss_tot = orc_ss_tot(targets, n_cases);
#ifdef _OPENMP
    if (threads < 1) threads = omp_get_max_threads();
    #pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
#endif
    for (int64_t i = 0; i < n_programs; ++i)
        fitness_out[i] = orc_r2_to_fitness(orc_evaluate_sr_r2(isa, words + offsets[i], offsets[i + 1] - offsets[i],
                                                              inputs, targets, num_inputs, n_cases, ss_tot));
    (void)threads;
}

/* Population evaluation over CSR programs: program i is
 * words[offsets[i] : offsets[i+1]].  The loop over programs follows
 * src/EvaluatorCpu.cpp:7-15; `threads` > 1 runs it as an OpenMP parallel for
 * (each program is still evaluated serially, so results do not depend on the
 * thread count).  sse_out may be NULL. */
void orc_evaluate_population_csr(const orc_isa_t* isa, const uint32_t* words,
                                 const int64_t* offsets, int64_t n_programs,
                                 const float* inputs, const float* targets, int num_inputs,
                                 int64_t n_cases, float* fitness_out, double* sse_out,
                                 int threads) {
#ifdef _OPENMP
    if (threads < 1) threads = omp_get_max_threads();
    #pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
#endif
    for (int64_t i = 0; i < n_programs; ++i) {
        const double sse = orc_sse(isa, words + offsets[i], offsets[i + 1] - offsets[i],
                                   inputs, targets, num_inputs, n_cases);
        if (sse_out) sse_out[i] = sse;
        fitness_out[i] = orc_mse_to_fitness((float)(sse / (double)n_cases));
    }
    (void)threads;
}

/* Per-case outputs of CSR programs: out[i*n_cases + c] = r[OUTPUT_REG] of
 * program i on case c (src/Interpreter.cpp:36-59, one program after the
 * other as src/EvaluatorCpu.cpp:7-15 walks them; OpenMP over programs, so
 * results do not depend on the thread count).  effective_only != 0 runs
 * each program's effective instructions only (src/Introns.h:50-57), whose
 * outputs the reference's own intron test proves bit-identical to the full
 * program's (tests/test_bed.cpp:1355-1381); it makes large case counts
 * affordable. */
void orc_case_outputs_csr(const orc_isa_t* isa, const uint32_t* words, const int64_t* offsets,
                          int64_t n_programs, const float* inputs, int num_inputs, int64_t n_cases,
                          float* out, int threads, int effective_only) {
#ifdef _OPENMP
    if (threads < 1) threads = omp_get_max_threads();
    #pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
#endif
    for (int64_t i = 0; i < n_programs; ++i) {
        const uint32_t* prog = words + offsets[i];
        int64_t len = offsets[i + 1] - offsets[i];
        uint32_t* eff = NULL;
        if (effective_only) {
            eff = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(len > 0 ? len : 1));
            len = orc_extract_effective(isa, prog, len, eff);
            prog = eff;
        }
        orc_ins_t* p = orc_decode_program(isa, prog, len);
        float* o = out + i * n_cases;
        for (int64_t c = 0; c < n_cases; ++c)
            o[c] = orc_run_case(isa, p, len, inputs + c * num_inputs, num_inputs);
        free(p);
        free(eff);
    }
    (void)threads;
}

/* Fitness and double SSE of CSR programs as orc_evaluate_population_csr,
 * with the effective-instructions-only option of orc_case_outputs_csr. */
void orc_evaluate_population_csr_opt(const orc_isa_t* isa, const uint32_t* words,
                                     const int64_t* offsets, int64_t n_programs,
                                     const float* inputs, const float* targets, int num_inputs,
                                     int64_t n_cases, float* fitness_out, double* sse_out,
                                     int threads, int effective_only) {
#ifdef _OPENMP
    if (threads < 1) threads = omp_get_max_threads();
    #pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
#endif
    for (int64_t i = 0; i < n_programs; ++i) {
        const uint32_t* prog = words + offsets[i];
        int64_t len = offsets[i + 1] - offsets[i];
        uint32_t* eff = NULL;
        if (effective_only) {
            eff = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(len > 0 ? len : 1));
            len = orc_extract_effective(isa, prog, len, eff);
            prog = eff;
        }
        const double sse = orc_sse(isa, prog, len, inputs, targets, num_inputs, n_cases);
        if (sse_out) sse_out[i] = sse;
        fitness_out[i] = orc_mse_to_fitness((float)(sse / (double)n_cases));
        free(eff);
    }
    (void)threads;
}

/* Dense layout of the EvalBackend boundary (src/EvalBackend.h:11-17):
 * program i at instructions + i*stride, lengths[i] instructions. */
void orc_evaluate_population_dense(const orc_isa_t* isa, const uint32_t* instructions,
                                   const uint8_t* lengths, int64_t stride, int64_t n_programs,
                                   const float* inputs, const float* targets, int num_inputs,
                                   int64_t n_cases, float* fitness_out) {
    for (int64_t i = 0; i < n_programs; ++i) {
        const float mse = orc_evaluate_sr_mse(isa, instructions + i * stride, lengths[i],
                                              inputs, targets, num_inputs, n_cases);
        fitness_out[i] = orc_mse_to_fitness(mse);
    }
}

/* Backward liveness, src/Introns.h:28-46.  live = {OUTPUT_REG}; an
 * instruction is effective iff its dest is live; then dest is killed and the
 * registers it reads become live (unary ops read only src2; a constant src2
 * reads no register). */
int64_t orc_effective_mask(const orc_isa_t* isa, const uint32_t* prog, int64_t len,
                           uint8_t* mask) {
    uint8_t live[128];
    memset(live, 0, sizeof(live));
    live[orc_output_reg(isa)] = 1;
    int64_t cnt = 0;
    for (int64_t i = len - 1; i >= 0; --i) {
        const orc_ins_t in = orc_decode_word(isa, prog[i]);
        if (!live[in.dest]) { mask[i] = 0; continue; }
        mask[i] = 1; ++cnt;
        live[in.dest] = 0;
        if (!in.unary) live[in.src1] = 1;
        if (!in.is_const) live[in.src2] = 1;
    }
    return cnt;
}

/* src/Introns.h:50-57: effective instructions in program order. */
int64_t orc_extract_effective(const orc_isa_t* isa, const uint32_t* prog, int64_t len,
                              uint32_t* out) {
    uint8_t* mask = (uint8_t*)malloc((size_t)(len > 0 ? len : 1));
    const int64_t cnt = orc_effective_mask(isa, prog, len, mask);
    int64_t k = 0;
    for (int64_t i = 0; i < len; ++i)
        if (mask[i]) out[k++] = prog[i];
    free(mask);
    return cnt;
}

/* Effective lengths of a CSR population (OpenMP over programs). */
void orc_effective_lengths_csr(const orc_isa_t* isa, const uint32_t* words,
                               const int64_t* offsets, int64_t n_programs, int64_t* eff_len) {
    #pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n_programs; ++i) {
        const int64_t len = offsets[i + 1] - offsets[i];
        uint8_t* mask = (uint8_t*)malloc((size_t)(len > 0 ? len : 1));
        eff_len[i] = orc_effective_mask(isa, words + offsets[i], len, mask);
        free(mask);
    }
}

/* Host intron strip of a CSR population into CSR effective code (the
 * reference's PackedEffective layout, src/EvaluatorCuda.cu:374-422):
 * eff_offsets[n+1] must hold the exclusive scan of the effective lengths
 * (orc_effective_lengths_csr); out_words receives each program's effective
 * instructions in program order (src/Introns.h:50-57).  OpenMP over
 * programs. */
void orc_extract_effective_csr(const orc_isa_t* isa, const uint32_t* words, const int64_t* offsets,
                               int64_t n_programs, const int64_t* eff_offsets, uint32_t* out_words,
                               int threads) {
#ifdef _OPENMP
    if (threads < 1) threads = omp_get_max_threads();
    #pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
#endif
    for (int64_t i = 0; i < n_programs; ++i)
        orc_extract_effective(isa, words + offsets[i], offsets[i + 1] - offsets[i], out_words + eff_offsets[i]);
    (void)threads;
}

/* Accuracy of the device's sine (cosine = 0) or cosine (trig.cuh) over the
 * floats with bit patterns lo, lo + stride, ... <= hi, against sinl/cosl
 * rounded to float (the correctly rounded value, up to rare double roundings
 * in long double) and against the C library's sinf/cosf.  Also checks
 * sin(-x) = -sin(x) and cos(-x) = cos(x) bit for bit.  out[0..6]: values
 * checked, largest error in ulps of the exact value, the argument where it
 * occurs, correctly rounded count, count equal to the C library's, count
 * above 1 ulp, symmetry violations. */
static double orc_ulp_error(float y, long double t) {
    if (isnan(y) || isnan((double)t)) return (isnan(y) && isnan((double)t)) ? 0.0 : 1e30;
    int e;
    frexpl(fabsl(t), &e);
    int ue = e - 24;
    if (ue < -149) ue = -149;
    return (double)(fabsl((long double)y - t) / ldexpl(1.0L, ue));
}

void orc_trig_accuracy(int cosine, uint32_t lo, uint32_t hi, uint32_t stride, double* out) {
    if (stride == 0) stride = 1;
    const int64_t n = ((int64_t)hi - (int64_t)lo) / stride + 1;
    double maxe = 0.0, arg = 0.0;
    int64_t cr = 0, libm = 0, over1 = 0, asym = 0;
#pragma omp parallel
    {
        double lmax = 0.0, larg = 0.0;
#pragma omp for schedule(dynamic, 4096) reduction(+ : cr, libm, over1, asym)
        for (int64_t i = 0; i < n; ++i) {
            const float x = gt_float((uint32_t)((int64_t)lo + i * (int64_t)stride));
            const float y = cosine ? galop_cosf(x) : galop_sinf(x);
            const float yn = cosine ? galop_cosf(-x) : galop_sinf(-x);
            const long double t = cosine ? cosl((long double)x) : sinl((long double)x);
            const float g = cosine ? cosf(x) : sinf(x);
            const double e = orc_ulp_error(y, t);
            if (!isnan(y)) asym += gt_bits(yn) != (cosine ? gt_bits(y) : (gt_bits(y) ^ 0x80000000u));
            cr += gt_bits(y) == gt_bits((float)t) || (isnan(y) && isnan((double)t));
            libm += gt_bits(y) == gt_bits(g) || (isnan(y) && isnan(g));
            over1 += e > 1.0;
            if (e > lmax) { lmax = e; larg = x; }
        }
#pragma omp critical
        if (lmax > maxe) { maxe = lmax; arg = larg; }
    }
    out[0] = (double)n; out[1] = maxe; out[2] = arg; out[3] = (double)cr; out[4] = (double)libm;
    out[5] = (double)over1; out[6] = (double)asym;
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
