/*
 * galop_b200.h -- C ABI of the B200 fitness evaluator for Galop's linear-GP
 * symbolic regression.
 *
 * Plain C: pointers, sizes and status codes only.  Every call returns a
 * galop_status (0 = success, negative = error; the message is in
 * galop_last_error()).  No call terminates the process; the reference's
 * ERR()/exit() convention (src/cuda_errors.h:3-15) is replaced by these codes.
 *
 * Semantics follow the reference exactly:
 *   - instruction word layout  src/ISA.h:20-41 ([SRC2 mode|idx][SRC1][DEST][OP])
 *   - op semantics             src/ISA.h:219-231 (REF profile)
 *   - register init / output   src/Interpreter.cpp:36-59
 *   - fitness                  src/Evaluator.cpp:11-45 + :88-91
 *                              fitness = non-finite(mse) ? 0 : 1/(1+mse),
 *                              mse = float(sse / N)
 * Per-case outputs are bit-identical to the CPU interpreter for ADD, SUB,
 * MUL, protected DIV, LT and GT; SIN, COS, EXP and LOG use CUDA's sinf,
 * cosf, expf, logf (at most 2 ulp from the CPU's libm).
 */
#ifndef GALOP_B200_H
#define GALOP_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define GALOP_API __attribute__((visibility("default")))
#else
#define GALOP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define GALOP_ABI_VERSION 2

typedef enum {
    GALOP_OK            = 0,
    GALOP_E_INVALID     = -1,  /* bad argument (sizes, nulls, options)          */
    GALOP_E_CUDA        = -2,  /* CUDA runtime error; see galop_last_error()    */
    GALOP_E_NOMEM       = -3,  /* device or pinned allocation failed            */
    GALOP_E_NO_DATASET  = -4,  /* evaluate called before galop_set_dataset()    */
    GALOP_E_TIMEOUT     = -5,  /* a bounded device-side wait gave up            */
    GALOP_E_CAPACITY    = -6,  /* request exceeds an admission or size limit    */
    GALOP_E_NO_DEVICE   = -7,  /* no CUDA device / wrong architecture           */
    GALOP_E_STATE       = -8   /* call not valid in the object's current state  */
} galop_status;

/* ISA profiles.  Both use the reference's 32-bit encoding and 3-bit opcode.
 *   REF: ADD SUB MUL DIV SIN COS LT GT      (src/ISA.h:69-72)
 *   BJ : ADD SUB MUL DIV SIN COS EXP LOG    (EXP, LOG unary on src2;
 *        LOG(b) = b != 0 ? logf(|b|) : 0)                                    */
typedef enum { GALOP_PROFILE_REF = 0, GALOP_PROFILE_BJ = 1 } galop_profile;

/* SSE accumulation.
 *   KAHAN32 : per-lane compensated FP32 sum of FP32 squared errors, FP64
 *             across lanes, warps and case chunks.
 *   FP64    : per-case error and square in FP64 (as src/Evaluator.cpp:38-39),
 *             FP64 sums; only the summation order differs from the CPU.
 *   ORDERED : FP64 terms summed strictly in case order 0..N-1, exactly as
 *             src/Evaluator.cpp:23-42: fitness is bit-identical to the CPU
 *             whenever the per-case outputs are.                             */
typedef enum {
    GALOP_REDUCE_KAHAN32 = 0,
    GALOP_REDUCE_FP64    = 1,
    GALOP_REDUCE_ORDERED = 2
} galop_reduce;

/* Fitness of a program from its SSE over the N cases.
 *   MSE : 1/(1 + mse), mse = float(sse/N), 0 if not finite
 *         (src/Evaluator.cpp:44, Fitness::mse_to_fitness :88-91)
 *   R2  : r2 = float(1 - sse/ss_tot), ss_tot = sum of (y - mean y)^2 over
 *         the N cases in double, two passes in case order; 0 when
 *         ss_tot <= 0 or sse is not finite (Evaluator::evaluate_sr_r2
 *         src/Evaluator.cpp:49-85), then max(r2, 0), 0 if not finite
 *         (Fitness::r2_to_fitness :93-97).                                  */
typedef enum { GALOP_OBJECTIVE_MSE = 0, GALOP_OBJECTIVE_R2 = 1 } galop_objective;

/* How the interpreter's work is scheduled on the GPU.
 *   PERSISTENT : one grid of resident warps pulls (program, case chunk)
 *                items from a device queue, longest interpreted program
 *                first; long case ranges are split into chunks (default).
 *   PLAIN      : the reference's launch shape (src/EvaluatorCuda.cu:433-441):
 *                one warp per program over all its cases, programs in
 *                population order, no queue and no case chunking.  Same
 *                pre-pass, folding and dedup; results equal PERSISTENT's
 *                within the reduction mode's tolerance (bit for bit in
 *                ORDERED mode).                                             */
typedef enum { GALOP_SCHEDULE_PERSISTENT = 0, GALOP_SCHEDULE_PLAIN = 1 } galop_schedule;

typedef struct {
    int32_t profile;          /* galop_profile                                  */
    int32_t num_registers;    /* 8 or 16 (src/LGPConfig.h:132-140)              */
    int32_t input_protect;    /* 1: dest folded to the upper half, output
                                 register NR/2 (src/LGPConfig.h:289-300)        */
    int32_t reduce;           /* galop_reduce                                   */
    const float* constants;   /* num_registers floats; NULL selects the
                                 reference pool (src/LGPConfig.h:159-168)       */
    int32_t device;           /* CUDA device ordinal                            */
    int32_t intron_prepass;   /* 1: interpret only effective instructions
                                 (src/Introns.h:28-57); outputs unchanged       */
    int32_t cases_per_lane;   /* 0 = default (8; 4 for dispatch 2); else 1, 2,
                                 4 or 8                                         */
    int32_t warps_per_block;  /* 0 = tuned default; else 1..8                  */
    int32_t dispatch;         /* interpreter: 3 = shared-memory register file,
                                 16-byte pre-decoded micro-ops, constant
                                 folding, operand forwarding (default);
                                 2 = shared-memory register file, 32-bit
                                 micro-ops, one instruction at a time.
                                 Both give identical results; any other
                                 value is GALOP_E_INVALID.                  */
    int32_t objective;        /* galop_objective (default MSE)                  */
    int32_t dedup;            /* 1: programs whose interpreted code is identical
                                 are interpreted once and share the fitness
                                 (dispatch 3, intron pass on; default 1)     */
    int32_t schedule;         /* galop_schedule (default PERSISTENT)            */
} galop_options;

typedef struct galop_ctx galop_ctx;

/* Timings (CUDA events on the context's stream) and counts of the most
 * recent evaluate call. */
typedef struct {
    int64_t n_programs;
    int64_t n_cases;
    int64_t raw_instructions;      /* sum of program lengths                    */
    int64_t eff_instructions;      /* sum of interpreted (effective) lengths    */
    double  h2d_ms;                /* host->device copies of the call           */
    double  prepass_ms;            /* intron pass, compaction, scheduling       */
    double  interp_ms;             /* interpreter kernel(s)                     */
    double  finalize_ms;           /* cross-chunk reduction + fitness           */
    double  d2h_ms;                /* device->host copies of the call           */
    double  total_ms;              /* first to last event of the call           */
    int32_t cases_per_lane;        /* configuration that ran                    */
    int32_t warps_per_block;
    int32_t blocks;
    int32_t case_chunks;           /* work items per program                    */
    int32_t kernels_launched;      /* this library's kernel launches            */
    int32_t reserved0;
    int64_t interp_instructions;   /* instructions interpreted per case
                                      (dispatch 3 with the intron pass): the
                                      effective ones minus those whose result
                                      is known before any case is read (done
                                      once per program) and minus the copies
                                      of programs interpreted once (dedup)  */
} galop_stats;

/* ---- lifetime ------------------------------------------------------------ */

/* Fill *opt with defaults: REF profile, 8 registers, no input protection,
 * KAHAN32, reference constant pool, device 0, intron pre-pass on, tuned tile. */
GALOP_API int galop_options_init(galop_options* opt);

/* Replaces `new CudaEvaluator(...)` (src/EvaluatorCuda.cu:21-62): binds the
 * device, creates a stream and events, uploads the constant pool. */
GALOP_API int galop_create(const galop_options* opt, galop_ctx** out);
GALOP_API void galop_destroy(galop_ctx* ctx);
GALOP_API const char* galop_last_error(const galop_ctx* ctx);
GALOP_API const char* galop_status_string(int status);
GALOP_API int galop_abi_version(void);

/* ---- the evolution loop on the device ------------------------------------ */

/* Replaces LGPEngine::evolve_sr (src/LGPEngine.cpp:519-557) with the whole
 * generation on the GPU: the population stays in device memory; elites
 * (top_k_indices + copy_elite_to_next, :381-425), tournament selection
 * (tournament_t, :148-171), crossover (crossover_t, :175-207) and mutation
 * (mutate_t, micro_mutate_instruction_t, :213-341) run as device kernels with
 * the engine's own random streams (one PCG32 per pair seeded from two draws
 * of the engine's mt19937 per generation, :427-456), and evaluation of the
 * non-elites uses this evaluator on the context's resident dataset.  Given
 * the same options and seed, the populations, fitness values and history
 * equal the reference engine's with this evaluator as its backend.
 * Initialization is the engine's serial one (:49-81): one mt19937 draw per
 * instruction slot, on the host, uploaded once. */
typedef struct {
    int64_t population;            /* POPULATION_SIZE (even non-elite count)  */
    int32_t max_program_size;      /* MAX_PROGRAM_SIZE (<= 254)                */
    int32_t starting_program_size; /* STARTING_PROGRAM_SIZE                    */
    int32_t max_generations;       /* MAX_GENERATIONS (generation 0 included)  */
    int32_t elite_count;           /* ELITE_COUNT = int(P * ELITES)            */
    int32_t tournament_size;       /* TOURNAMENT_SIZE                          */
    int32_t macro_inserts;         /* MACRO_INSERTS                            */
    int32_t effmut;                /* EFFMUT (effective mutation)              */
    int32_t macro_random_pos;      /* MACRO_RANDOM_POS                         */
    float crossover_rate;          /* CROSSOVER_RATE                           */
    float micro_rate;              /* MICRO_RATE                               */
    float micro_per_instr;         /* MICRO_PER_INSTR                          */
    float effmut_rate;             /* EFFMUT_RATE                              */
    float insert_tail_rate;        /* INSERT_TAIL_RATE                         */
    float delete_tail_rate;        /* DELETE_TAIL_RATE                         */
    uint32_t seed;                 /* the engine's seed                        */
    int32_t reserved[3];
} galop_engine_options;

/* One row of the run's history (GenerationStats, src/GenerationStats.h). */
typedef struct {
    int32_t generation;
    float best_fitness;
    float mean_fitness;
    int32_t best_length;
    float mean_length;
    int32_t best_index;
} galop_generation_stats;

/* Seconds spent per phase over the last run (CUDA events and host clock). */
typedef struct {
    double total_s, init_s, evaluate_s, select_vary_s, stats_s;
    int64_t eff_instructions;      /* interpreted instructions over the run   */
} galop_engine_times;

typedef struct galop_engine galop_engine;

/* Defaults: the reference's default LGPConfig (P 1000, MAX_PROGRAM_SIZE 50,
 * start 8, 1000 generations, elites int(P*0.1f), tournament 3, 1 macro
 * insert, no EFFMUT, random positions, crossover 1.0, micro 0.8, per-instr
 * 0, EFFMUT rate 1.0, insert 0.8, delete 0.75, seed 42). */
GALOP_API int galop_engine_options_init(galop_engine_options* o);
/* Device buffers for two generations, sized once.  The ISA (registers,
 * input protection, profile, constants) and the reduction are ctx's. */
GALOP_API int galop_engine_create(galop_ctx* ctx, const galop_engine_options* o, galop_engine** out);
GALOP_API int galop_engine_destroy(galop_engine* e);
/* init + max_generations generations on ctx's resident dataset; history gets
 * max_generations rows (capacity must be at least that). */
GALOP_API int galop_engine_evolve(galop_engine* e, galop_generation_stats* history, int32_t capacity);
/* The current generation: dense words (population x max_program_size),
 * lengths and fitness, copied to host memory (any pointer may be NULL). */
GALOP_API int galop_engine_population(galop_engine* e, uint32_t* words, uint8_t* lengths, float* fitness);
GALOP_API int galop_engine_times_get(const galop_engine* e, galop_engine_times* out);

/* ---- CSV datasets ---------------------------------------------------------- */

/* Replaces load_csv_1d (multi = 0) and load_csv_multi (multi = 1)
 * (src/Dataset.cpp:83-151): reads a header line, then one case per
 * non-empty line, into case-major inputs[c*num_inputs + i] and targets[c]
 * (malloc'd; release with galop_csv_free), and the targets' total sum of
 * squares (src/Dataset.cpp:35-47).  Numbers are read as std::stof reads
 * them.  Returns GALOP_E_INVALID with a message in err (err_len bytes, may
 * be NULL) for a missing file, a field that is not a float or is out of
 * float range, or a ragged row.  Host only: no device is touched. */
typedef struct {
    float* inputs;
    float* targets;
    int64_t n_cases;
    int32_t num_inputs;
    int32_t reserved;
    double ss_tot;
} galop_csv_dataset;

GALOP_API int galop_csv_read(const char* path, int32_t multi, galop_csv_dataset* out, char* err, int32_t err_len);
GALOP_API void galop_csv_free(galop_csv_dataset* d);

/* ---- autotuner ----------------------------------------------------------- */

/* No counterpart in the reference, whose kernel shape is fixed at compile
 * time (src/EvaluatorCuda.cu:28-31).  Chooses the interpreter tile for this
 * context and a population like `words`/`offsets` (CSR, host memory) on the
 * resident dataset: every candidate of dispatch {3, 2} x cases per lane
 * {1, 2, 4, 8} x warps per block {2, 4, 8} evaluates a sample of the
 * population (every s-th program, at most sample_programs; 0 = 16,384), one
 * warm-up and `reps` timed calls (0 = 2), and the shortest interpreter time
 * wins.  The choice is written into the context's options, so later calls,
 * and batches and servers created afterwards, use it.
 *
 * With cache_path non-NULL the choice is appended to that file as one JSON
 * object per line under `key` = device name and SM count, ISA (registers,
 * profile, input protection), reduction, intron pass, and the workload's
 * size class (case count, mean raw program length and program count, each
 * rounded to a power of two).  A later call whose key is in the file applies
 * the file's last entry for it without measuring (from_cache = 1).
 * Candidates run as ordinary evaluate calls on the context's stream. */
typedef struct {
    int32_t dispatch;
    int32_t cases_per_lane;
    int32_t warps_per_block;
    int32_t from_cache;            /* 1: taken from the cache file            */
    int32_t candidates;            /* tiles measured (0 when from the cache)  */
    int32_t reserved0;
    int64_t sample_programs;       /* programs in the timed sample            */
    double gpops;                  /* effective GPop/s of the choice (sample) */
    double default_gpops;          /* the default tile (3, 8, 4) on the sample */
    char key[320];
} galop_tune_result;

GALOP_API int galop_autotune(galop_ctx* ctx, const uint32_t* words, const int64_t* offsets,
                             int64_t n_programs, int64_t sample_programs, int32_t reps,
                             const char* cache_path, galop_tune_result* out);

/* ---- dataset ------------------------------------------------------------- */

/* Replaces CudaEvaluator::upload_dataset (src/EvaluatorCuda.cu:96-110).
 * inputs: case-major, inputs[c*num_inputs + i] (src/Dataset.h:22-24);
 * targets[c]; n_cases >= 0; 0 <= num_inputs <= num_registers.  The data are
 * transposed on the device to feature-major and stay resident until the next
 * call.  Host buffers are not retained. */
GALOP_API int galop_set_dataset(galop_ctx* ctx, const float* inputs, const float* targets,
                      int64_t n_cases, int32_t num_inputs);

/* Same, with device pointers already holding the case-major data. */
GALOP_API int galop_set_dataset_device(galop_ctx* ctx, const float* d_inputs, const float* d_targets,
                             int64_t n_cases, int32_t num_inputs);

/* ---- evaluation ---------------------------------------------------------- */

/* The EvalBackend::evaluate_population boundary (src/EvalBackend.h:11-17,
 * src/EvaluatorCuda.cu:298-469).  Program i is instructions[i*stride ..
 * i*stride + lengths[i]).  Host pointers; returns with fitness_out filled. */
GALOP_API int galop_evaluate_population(galop_ctx* ctx, const uint32_t* instructions,
                              const uint8_t* lengths, int64_t stride, int64_t n_programs,
                              float* fitness_out);

/* Packed (CSR) layout of the reference (src/eval_kernels.cuh:292-303):
 * program i is words[offsets[i] .. offsets[i+1]), int64 offsets, any length.
 * Host pointers.  sse_out (may be NULL) receives the per-program SSE. */
GALOP_API int galop_evaluate_csr(galop_ctx* ctx, const uint32_t* words, const int64_t* offsets,
                       int64_t n_programs, float* fitness_out, double* sse_out);

/* Device-resident form of galop_evaluate_csr: all pointers are device memory
 * on the context's device, total_words = d_offsets[n_programs] as the caller
 * knows it (the size of d_words).  Work is ordered on `stream` (a
 * cudaStream_t, or NULL for the context's own stream, which is a
 * non-blocking stream: with NULL the call does not wait for work the caller
 * queued on other streams, so pass the stream that wrote the inputs, or
 * synchronize it first; the legacy default stream, whose handle is also
 * NULL, cannot be named here) and the call returns
 * without waiting for the device; it only blocks when a working buffer must
 * grow (the first call, or a larger population), and waits once for the
 * effective instruction count when a buffer sized for total_words would take
 * more than half the free device memory.  The offsets are checked on
 * the device before any word is read: if d_offsets[0] != 0, an offset
 * decreases, a program is longer than 2^30 words, or d_offsets[n_programs]
 * != total_words, no word is read, every d_fitness (and d_sse) is NaN, and
 * galop_last_stats returns GALOP_E_INVALID for the call.  Its result is read
 * once the stream has reached it (galop_last_stats waits for that). */
GALOP_API int galop_evaluate_csr_device(galop_ctx* ctx, const uint32_t* d_words, const int64_t* d_offsets,
                              int64_t n_programs, int64_t total_words, float* d_fitness, double* d_sse,
                              void* stream);

/* Per-case outputs r[OUTPUT_REG] (src/Interpreter.cpp:54-57), host pointers:
 * outputs[i*n_cases + c] for program i, case c. */
GALOP_API int galop_case_outputs_csr(galop_ctx* ctx, const uint32_t* words, const int64_t* offsets,
                           int64_t n_programs, float* outputs);

/* Register-file trace of one program over the first min(32*cases_per_lane,
 * n_cases) cases: state[(pc*num_registers + j)*n + c] = r_j of case c after
 * pc instructions (pc = 0 is the initial file), n = number of traced cases.
 * Runs the raw program (no intron pass).  For instruction-level parity. */
GALOP_API int galop_trace_program(galop_ctx* ctx, const uint32_t* words, int64_t len,
                        float* state, int64_t* n_traced);

/* Intron pass only (src/Introns.h:28-57): eff_len[i] and the effective
 * instructions of every program, packed program after program, in program
 * order (raw encoding).  eff_words may be NULL. */
GALOP_API int galop_effective_csr(galop_ctx* ctx, const uint32_t* words, const int64_t* offsets,
                        int64_t n_programs, int64_t* eff_len, uint32_t* eff_words);

/* Stats of the most recent evaluate call; after galop_evaluate_csr_device
 * this waits for that call's work to finish, and returns GALOP_E_INVALID if
 * the device found its offsets inconsistent. */
GALOP_API int galop_last_stats(galop_ctx* ctx, galop_stats* out);

/* Blocks until the context's stream is idle. */
GALOP_API int galop_synchronize(galop_ctx* ctx);

/* CUDA-event timers on the context's stream: record marker `slot` (0..7);
 * elapsed milliseconds between two recorded markers (waits for `slot_b`). */
GALOP_API int galop_timer_record(galop_ctx* ctx, int32_t slot);
GALOP_API int galop_timer_elapsed(galop_ctx* ctx, int32_t slot_a, int32_t slot_b, double* ms);

/* Page-locked host memory for staging populations and fitness (the
 * reference's cudaMallocHost staging, src/EvaluatorCuda.cu:40-51): copies
 * from it run at full link speed and overlap with device work. */
GALOP_API int galop_host_alloc(int64_t bytes, void** out);
GALOP_API int galop_host_free(void* p);

/* Device memory on the context's device (for callers that keep populations
 * resident and use galop_evaluate_csr_device). */
GALOP_API int galop_device_alloc(galop_ctx* ctx, int64_t bytes, void** out);
GALOP_API int galop_device_free(galop_ctx* ctx, void* p);
GALOP_API int galop_memcpy_h2d(galop_ctx* ctx, void* dst, const void* src, int64_t bytes);
GALOP_API int galop_memcpy_d2h(galop_ctx* ctx, void* dst, const void* src, int64_t bytes);

/* ---- resident datasets and batched populations ---------------------------- */

/* A dataset uploaded once and kept on the device (feature-major, padded).
 * Destroy datasets, batches and servers before the context they came from,
 * and a dataset only when no evaluation using it is still running. */
typedef struct galop_dataset galop_dataset;
GALOP_API int galop_dataset_create(galop_ctx* ctx, const float* inputs, const float* targets,
                                   int64_t n_cases, int32_t num_inputs, galop_dataset** out);
GALOP_API int galop_dataset_destroy(galop_dataset* ds);
GALOP_API int64_t galop_dataset_device_bytes(const galop_dataset* ds);

/* A fixed set of populations evaluated together, one generation per
 * galop_batch_evaluate: one persistent interpreter launch pulls (program,
 * case chunk) items of every population from a device queue, largest work
 * (effective length x cases) first.  Each population has its own dataset and
 * capacities (programs, total instructions); all device memory is allocated
 * at creation.  Case chunking depends only on a population's own case count,
 * so its fitness does not depend on which batch it is evaluated in.  Each
 * batch has its own stream; different batches run concurrently.
 * Generalises CudaEvaluator::evaluate_population (src/EvaluatorCuda.cu:298-469)
 * from one population to many; no single reference counterpart. */
typedef struct galop_batch galop_batch;
typedef struct {
    const galop_dataset* dataset;
    int64_t max_programs;
    int64_t max_words;
} galop_population_spec;

GALOP_API int galop_batch_create(galop_ctx* ctx, const galop_population_spec* pops, int32_t n_pops,
                                 galop_batch** out);
GALOP_API int galop_batch_destroy(galop_batch* b);
GALOP_API int64_t galop_batch_device_bytes(const galop_batch* b);
/* Host CSR programs of population `pop` for the next evaluation (H2D on the
 * batch's stream; pinned host memory makes it asynchronous). */
GALOP_API int galop_batch_set_population(galop_batch* b, int32_t pop, const uint32_t* words,
                                         const int64_t* offsets, int64_t n_programs);
/* Queue one generation on the batch's stream.  use_graph != 0: the device
 * work is captured as a CUDA graph the first time (and again whenever a
 * population's program count changes) and replayed afterwards. */
GALOP_API int galop_batch_evaluate(galop_batch* b, int32_t use_graph);
GALOP_API int galop_batch_synchronize(galop_batch* b);
/* D2H of one population's fitness (and SSE, may be NULL); waits. */
GALOP_API int galop_batch_get_fitness(galop_batch* b, int32_t pop, float* fitness_out, double* sse_out);
GALOP_API int galop_batch_last_stats(galop_batch* b, galop_stats* out);
/* The batch's cudaStream_t. */
GALOP_API void* galop_batch_stream(galop_batch* b);

/* Pooled batch: capacities are totals shared by whatever populations are
 * appended for the next evaluation (up to max_pops populations, max_programs
 * programs, max_words instructions, max_items work items -- a program has
 * ceil(cases / 16384) items, 1 in ORDERED mode).  All memory is allocated
 * here; galop_batch_clear + galop_batch_append recompose it every
 * generation without allocating.  append returns GALOP_E_CAPACITY when the
 * population does not fit. */
GALOP_API int galop_batch_create_pool(galop_ctx* ctx, int32_t max_pops, int64_t max_programs,
                                      int64_t max_words, int64_t max_items, galop_batch** out);
GALOP_API int galop_batch_clear(galop_batch* b);
GALOP_API int galop_batch_append(galop_batch* b, const galop_dataset* ds, const uint32_t* words,
                                 const int64_t* offsets, int64_t n_programs, int32_t* pop_out);
/* Fitness of every population, concatenated in population order, and the
 * interpreted instructions of each (eff_per_pop[n_pops], may be NULL); waits. */
GALOP_API int galop_batch_get_fitness_all(galop_batch* b, float* fitness_out, int64_t* eff_per_pop);
/* Interpreted (effective) instructions of population `pop` in the last
 * evaluation, summed over its programs; waits. */
GALOP_API int galop_batch_population_work(galop_batch* b, int32_t pop, int64_t* eff_instructions);

/* ---- serving: continuous batching for many independent GP runs ------------ */

/* A server owns a worker thread that admits submitted generations by HBM
 * footprint, packs them into pooled batches (one persistent launch each,
 * several batches in flight on their own streams) and completes them into
 * the callers' fitness buffers.  A run's dataset is uploaded when its first
 * request is admitted and stays resident while the run has work; datasets
 * of idle runs are evicted when the budget is needed.  A request's fitness
 * does not depend on what it was batched with. */
typedef struct galop_server galop_server;
typedef struct {
    int64_t hbm_budget_bytes;     /* resident datasets + slot buffers (default 150e9) */
    int32_t slots;                /* batches in flight (default 4) */
    int32_t max_pops_per_batch;   /* requests per batch (default 64) */
    int64_t slot_programs;        /* per-batch capacities (defaults 2^20, 2^27, 2^23) */
    int64_t slot_words;
    int64_t slot_items;
    int64_t pinned_bytes;         /* page-locked staging for submitted programs (1 GiB) */
} galop_server_options;

typedef struct {
    int32_t status;               /* GALOP_OK, or the error that ended the request */
    int32_t batch_requests;       /* requests in its batch */
    int64_t eff_instructions;     /* interpreted instructions of its programs */
    double queued_ms;             /* submit -> launch */
    double latency_ms;            /* submit -> fitness in the caller's buffer */
    double device_ms;             /* device time of its batch */
} galop_request_info;

typedef struct {
    int64_t completed, batches, pending;
    int64_t resident_bytes;       /* datasets + slot buffers on the device */
    int64_t case_ops;             /* sum over completed requests: eff. instructions x cases */
    double device_ms;
} galop_server_totals;

GALOP_API int galop_server_options_init(galop_server_options* opt);
GALOP_API int galop_server_create(galop_ctx* ctx, const galop_server_options* opt, galop_server** out);
/* Finishes queued work, then stops the worker and frees everything. */
GALOP_API int galop_server_destroy(galop_server* sv);
/* Registers a GP run; the dataset is copied (host) at this call. */
GALOP_API int galop_server_open_run(galop_server* sv, const float* inputs, const float* targets,
                                    int64_t n_cases, int32_t num_inputs, int32_t* run_id);
GALOP_API int galop_server_close_run(galop_server* sv, int32_t run_id);
/* One generation of a run: programs are copied at this call; fitness_out
 * (n_programs floats) must stay valid until galop_server_wait returns. */
GALOP_API int galop_server_submit(galop_server* sv, int32_t run_id, const uint32_t* words,
                                  const int64_t* offsets, int64_t n_programs, float* fitness_out,
                                  int64_t* request_id);
/* Waits for a request (timeout_s <= 0: no limit); GALOP_E_TIMEOUT if it is
 * not done in time (it stays queued and can be waited on again). */
GALOP_API int galop_server_wait(galop_server* sv, int64_t request_id, double timeout_s,
                                galop_request_info* info);
GALOP_API int galop_server_stats(galop_server* sv, galop_server_totals* out);

/* ---- evaluation without allocation --------------------------------------- */

/* Limits of galop_evaluate_csr_noalloc: programs and total instructions per
 * call.  Its working buffers are a fixed ~11 MiB __device__ array that every
 * GPU loading this library holds until the process exits. */
#define GALOP_NOALLOC_MAX_PROGRAMS 65536
#define GALOP_NOALLOC_MAX_WORDS 2097152

/* No counterpart in the reference.  For callers that cannot let a library
 * call cudaMalloc: hosts that own all device memory through their own pool
 * allocator (a framework's caching allocator, a server with a fixed budget
 * per model) and must never meet an out-of-memory failure or unaccounted
 * memory in the middle of a run, and loops that must not stall, since
 * cudaMalloc and cudaFree can synchronise the whole device.  It needs no
 * galop_ctx and allocates nothing -- no cudaMalloc, no cudaFree, no
 * allocating library routine; its scratch is the static array above.
 *
 * Same evaluation as galop_evaluate_csr_device, with the compact
 * interpreter (dispatch 2; results are identical): device pointers, CSR
 * programs (words, int64 offsets, total_words = offsets[n_programs]), the
 * dataset already feature-major on the device -- d_inputs[f*padded_cases +
 * c], d_targets[c], padded_cases a multiple of 1024 and >= n_cases (padding
 * values are never counted) -- opt as for galop_create (device and dispatch
 * ignored: the current device is used).  Work is queued on `stream` (NULL =
 * default stream) and the call returns without waiting.
 *
 * Limits: n_programs <= GALOP_NOALLOC_MAX_PROGRAMS and total_words <=
 * GALOP_NOALLOC_MAX_WORDS, else GALOP_E_CAPACITY with nothing queued.  The
 * offsets are checked on the device before any word is read: if offsets[0]
 * != 0, an offset decreases or offsets[n_programs] != total_words, nothing
 * beyond the stated sizes is read or written and every fitness (and SSE)
 * is NaN.  A CUDA error left pending by an earlier call of the caller is
 * not cleared: the call returns GALOP_E_CUDA and queues nothing.
 *
 * The first call on a device, with that device current, looks up the
 * scratch's device address and loads this entry point's kernels on that
 * device; make that first call before any stream capture.  Every call uses
 * the same scratch, which keeps the last call's contents (each call clears
 * what must start at zero): calls whose work overlaps on the GPU
 * (different streams, or different host threads, without ordering between
 * them) race and corrupt each other's results. */
GALOP_API int galop_evaluate_csr_noalloc(const galop_options* opt, const uint32_t* d_words,
                                         const int64_t* d_offsets, int64_t n_programs,
                                         int64_t total_words, const float* d_inputs,
                                         const float* d_targets, int64_t n_cases,
                                         int64_t padded_cases, int32_t num_inputs,
                                         float* d_fitness, double* d_sse, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GALOP_B200_H */
