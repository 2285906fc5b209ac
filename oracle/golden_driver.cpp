// golden_driver.cpp -- one golden cell (target, seed) through the reference's
// own LGPEngine, with a selectable evaluation backend.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles it against the
// reference's src/ (LGPEngine and friends, read in place) into
//   oracle/_ref/lgp_run_cpu     backend = the reference's CpuEvaluator
//   oracle/_ref/lgp_run_oracle  backend = the C restatement in oracle.c
//   oracle/_ref/lgp_run_b200    backend = galop::B200Evaluator (the product)
// Output files have the byte format of the reference's lgp_run
// (src/main.cpp:66-103), so they diff directly against golden/.
//
// usage: <bin> <train_csv> <test_csv> <target_name> <run_seed>
//              <results_csv> <program_txt> <history_csv>
//
// Runs that are not golden cells may change the evaluation ISA (the engine
// itself only moves instruction words, so it is unaffected):
//   GALOP_DRIVER_PROFILE=bj          BJ op set: EXP and protected LOG in
//                                    place of LT and GT (oracle and B200
//                                    backends only)
//   GALOP_DRIVER_CONSTANTS=<file>    NUM_REGISTERS whitespace-separated
//                                    floats replacing LGPConfig::CONSTANTS
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include "Dataset.h"
#include "EvalBackend.h"
#include "EvaluatorCpu.h"
#include "LGPConfig.h"
#include "LGPEngine.h"

// 0 = REF, 1 = BJ.
static int driver_profile() {
    const char* p = std::getenv("GALOP_DRIVER_PROFILE");
    return (p && std::string(p) == "bj") ? 1 : 0;
}

static std::vector<float> driver_constants() {
    std::vector<float> c(LGPConfig::CONSTANTS.begin(), LGPConfig::CONSTANTS.end());
    if (const char* path = std::getenv("GALOP_DRIVER_CONSTANTS")) {
        std::ifstream f(path);
        for (auto& v : c)
            if (!(f >> v)) {
                std::cerr << "GALOP_DRIVER_CONSTANTS: need " << c.size() << " floats in " << path << "\n";
                std::exit(2);
            }
    }
    return c;
}

#if defined(GOLDEN_BACKEND_B200)
#include "galop_b200_backend.hpp"
#elif defined(GOLDEN_BACKEND_ORACLE)
extern "C" {
typedef struct {
    int32_t profile, num_registers, input_protect, trig;  // trig 0: the C library's sinf/cosf
    const float* constants;
} orc_isa_t;
void orc_evaluate_population_dense(const orc_isa_t* isa, const uint32_t* instructions,
                                   const uint8_t* lengths, int64_t stride, int64_t n_programs,
                                   const float* inputs, const float* targets, int num_inputs,
                                   int64_t n_cases, float* fitness_out);
}
// EvalBackend over the C restatement, configured from this build's LGPConfig.
struct OracleBackend : EvalBackend {
    int profile = driver_profile();
    std::vector<float> constants = driver_constants();
    void evaluate_population(const uint32_t* instructions, const uint8_t* lengths, float* fitness_out,
                             int n_programs, const Dataset& ds) override {
        orc_isa_t isa{profile, LGPConfig::NUM_REGISTERS, LGPConfig::INPUT_PROTECT ? 1 : 0, 0, constants.data()};
        orc_evaluate_population_dense(&isa, instructions, lengths, LGPConfig::MAX_PROGRAM_SIZE, n_programs,
                                      ds.inputs.data(), ds.targets.data(), ds.num_inputs, ds.N, fitness_out);
    }
};
#endif

static std::unique_ptr<EvalBackend> make_backend() {
#if defined(GOLDEN_BACKEND_B200)
    const std::vector<float> constants = driver_constants();
    galop_options o = galop::B200Evaluator::options_from_config();
    o.profile = driver_profile() ? GALOP_PROFILE_BJ : GALOP_PROFILE_REF;
    o.constants = constants.data();                 // copied by galop_create
    return std::make_unique<galop::B200Evaluator>(o);
#elif defined(GOLDEN_BACKEND_ORACLE)
    return std::make_unique<OracleBackend>();
#else
    if (driver_profile() != 0 || std::getenv("GALOP_DRIVER_CONSTANTS")) {
        std::cerr << "the reference CpuEvaluator evaluates the REF ISA with LGPConfig::CONSTANTS only\n";
        std::exit(2);
    }
    return std::make_unique<CpuEvaluator>();
#endif
}

int main(int argc, char** argv) {
    if (argc != 8) {
        std::cerr << "usage: " << argv[0]
                  << " <train_csv> <test_csv> <target> <seed> <results_csv> <program_txt> <history_csv>\n";
        return 2;
    }
    const std::string target = argv[3];
    const uint32_t seed = static_cast<uint32_t>(std::stoul(argv[4]));
    Dataset train, test;
    try {
        train = load_csv_1d(argv[1]);
        test = load_csv_1d(argv[2]);
    } catch (const std::exception& e) {
        std::cerr << "dataset load failed: " << e.what() << "\n";
        return 1;
    }
    LGPEngine engine(seed, make_backend());
    try {
        engine.evolve_sr(train);
    } catch (const std::exception& e) {
        std::cerr << "evaluation failed: " << e.what() << "\n";
        return 1;
    }
    const float train_mse = engine.best_train_mse();
    const float test_mse = engine.best_test_mse(test);
    const int best_len = engine.best_length();
    {
        std::ofstream f(argv[5], std::ios::app);
        f << target << ",lgp," << seed << ',' << train_mse << ',' << test_mse << ',' << best_len << '\n';
    }
    {
        std::ofstream f(argv[6]);
        f << "# target=" << target << " seed=" << seed << " train_mse=" << train_mse
          << " test_mse=" << test_mse << " length=" << best_len << "\n";
        engine.print_best_program(f);
    }
    {
        std::ofstream f(argv[7]);
        f << "target,run_seed,generation,best_fitness,mean_fitness,best_length,mean_length\n";
        for (const auto& s : engine.history_view())
            f << target << ',' << seed << ',' << s.generation << ',' << s.best_fitness << ','
              << s.mean_fitness << ',' << s.best_length << ',' << s.mean_length << '\n';
    }
    return 0;
}
