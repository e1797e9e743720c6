// tuner.cuh — the project's own autotuner for the step, replacing KTT
// (reference: Tuner src/cuda/tuning/tuner.cpp:19-143, StepTuner parameter
// space step_tuner.cuh:79-121,326-357, TuningScheduler
// tuning_scheduler.h:12-26, load_config_json config_loader.cpp:8-54).
//
// Search space (StepConfig): warps per block of the three cell passes,
// neighbour-bitmask words (list capacity vs on-the-fly rescan), cell-size
// multiplier and hash-table multiplier, under the reference's constraint
// TABLE_SIZE_MULT >= uint64(1 / CELL_SIZE_MULT^3) (step_tuner.cuh:94-99).
// Searchers: MCMC (Metropolis walk over neighbouring configurations), random
// (uniform without replacement) and full (deterministic enumeration).
// Each tuning iteration times one real step with CUDA events.
#pragma once

#include <random>
#include <string>
#include <vector>

#include "simulator.cuh"

namespace wcsph {

struct TuneResult {
    StepConfig cfg;
    float total_ms = 0.f;
    std::vector<std::pair<const char*, float>> kernels;
};

class Tuner {
public:
    explicit Tuner(CUDASPHSimulator* sim);

    bool active() const { return budget_ > 0.f || frozen_; }
    // TuningScheduler::schedule: returns whether this step is a tuning iteration.
    bool before_step();
    void timed_step(float delta);
    void set(int searcher, float budget, const char* frozen_json);
    void reset();
    void save_config(const char* path) const;
    void save_results(const char* path) const;
    const StepConfig& best() const { return best_cfg_; }
    int searched() const { return static_cast<int>(results_.size()); }
    int space_size() const { return static_cast<int>(space_.size()); }

    static StepConfig parse_config_json(const std::string& text, const StepConfig& base);
    static std::string config_json(const StepConfig& c);

private:
    int next_candidate();
    CUDASPHSimulator* sim_;
    std::vector<StepConfig> space_;
    std::vector<char> visited_;
    int searcher_ = WCSPH_SEARCH_MCMC;
    float budget_ = 0.f;
    float accumulator_ = 0.f;
    bool frozen_ = false;
    StepConfig frozen_cfg_{};
    StepConfig best_cfg_{};
    float best_ms_ = 0.f;
    int current_ = -1;       // MCMC chain position
    float current_ms_ = 0.f;
    int full_cursor_ = 0;
    std::mt19937_64 rng_{0x5eedULL};
    std::vector<TuneResult> results_;
};

}  // namespace wcsph
