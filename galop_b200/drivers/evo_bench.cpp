// evo_bench.cpp -- a whole evolutionary run: the reference's LGPEngine
// (selection and variation on the CPU, unchanged) with galop::B200Evaluator
// as its evaluation backend.
//
// Same command line and output row as the reference's whole-run benchmark
// (tests/cuda_evo_bench.cu:61-68), so the rows slot into its readouts:
//   usage: <bin> <D | dataset.csv> [seed]
//   stdout: b200,pop,D,gens,mean_size,seconds,gpops_s,best_mse
//   stderr: BREAKDOWN b200: total=..s eval=..s (..%) host+other=..s
// POPULATION_SIZE and MAX_GENERATIONS are compile-time settings of the
// engine (-DPOPULATION_SIZE_OVERRIDE, -DMAX_GENERATIONS_OVERRIDE), as there.
// GPops/s counts raw operations: sum over generations of P x mean length x D
// (tests/cuda_evo_bench.cu:52-58).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <string>

#include "Dataset.h"
#include "EvalBackend.h"
#include "LGPConfig.h"
#include "LGPEngine.h"
#include "galop_b200_backend.hpp"

namespace {

using Clock = std::chrono::steady_clock;

// The backend, with the time spent inside evaluate_population recorded.
class TimedB200 : public EvalBackend {
public:
    void evaluate_population(const uint32_t* instructions, const uint8_t* lengths, float* fitness_out,
                             int n_programs, const Dataset& ds) override {
        const auto t0 = Clock::now();
        inner_.evaluate_population(instructions, lengths, fitness_out, n_programs, ds);
        seconds_ += std::chrono::duration<double>(Clock::now() - t0).count();
    }
    double seconds() const { return seconds_; }

private:
    galop::B200Evaluator inner_{galop::B200Evaluator::options_from_config(GALOP_REDUCE_KAHAN32)};
    double seconds_ = 0.0;
};

Dataset load_any(const std::string& path) {
    std::ifstream f(path);
    std::string header;
    std::getline(f, header);
    const long cols = 1 + std::count(header.begin(), header.end(), ',');
    return cols > 2 ? load_csv_multi(path) : load_csv_1d(path);
}

}  // namespace

int main(int argc, char** argv) {
    const std::string arg1 = argc > 1 ? argv[1] : "32";
    Dataset ds;
    try {
        ds = arg1.find(".csv") != std::string::npos
                 ? load_any(arg1)
                 : make_sr_dataset_1d(std::atoi(arg1.c_str()), -1.f, 1.f, Nguyen::Nguyen_1, 1234);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "dataset: %s\n", e.what());
        return 1;
    }
    const uint32_t seed = argc > 2 ? (uint32_t)std::strtoul(argv[2], nullptr, 10) : 42u;

    auto backend = std::make_unique<TimedB200>();
    TimedB200* timed = backend.get();
    LGPEngine engine(seed, std::move(backend));
    const auto t0 = Clock::now();
    try {
        engine.evolve_sr(ds);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "evaluation failed: %s\n", e.what());
        return 1;
    }
    const double sec = std::chrono::duration<double>(Clock::now() - t0).count();

    double ops = 0.0, sbar_sum = 0.0;
    for (const auto& s : engine.history_view()) {
        ops += (double)LGPConfig::POPULATION_SIZE * s.mean_length * ds.N;
        sbar_sum += s.mean_length;
    }
    const int G = (int)engine.history_view().size();
    std::printf("b200,%d,%d,%d,%.2f,%.4f,%.3e,%.9e\n", LGPConfig::POPULATION_SIZE, ds.N, G,
                G ? sbar_sum / G : 0.0, sec, ops / sec, engine.best_train_mse());
    std::fflush(stdout);
    std::fprintf(stderr, "BREAKDOWN b200: total=%.3fs eval=%.3fs (%.1f%%) host+other=%.3fs\n", sec,
                 timed->seconds(), 100.0 * timed->seconds() / sec, sec - timed->seconds());
    return 0;
}
