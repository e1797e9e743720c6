// tuner.cu — see tuner.cuh.
#include "tuner.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>

namespace wcsph {

namespace {
const int kWarps[] = {2, 4, 8};
const int kMaskWords[] = {8, 10, 11, 12, 16};
const int kChunk[] = {8, 16, 32};
const double kCellMult[] = {0.5, 2. / 3., 1., 1.5, 2.};  // step_tuner.cuh:88
const uint32_t kTableMult[] = {1, 2, 4, 8, 16, 32};      // step_tuner.cuh:251-256

// Minimal JSON reader for the KTT configuration schema: an array of
// {"Name": str, "Value": number|string|bool, "ValueType": str} objects, or an
// object holding such an array under "Configuration" (config_loader.cpp:23-29).
struct JsonCursor {
    const std::string& s;
    size_t i = 0;
    void ws() { while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) ++i; }
    bool eat(char c) { ws(); if (i < s.size() && s[i] == c) { ++i; return true; } return false; }
    void expect(char c) {
        if (!eat(c)) throw Error(WCSPH_ERR_CONFIG, std::string("config JSON: expected '") + c + "'");
    }
    std::string str() {
        ws();
        if (i >= s.size() || s[i] != '"') throw Error(WCSPH_ERR_CONFIG, "config JSON: expected string");
        ++i;
        std::string out;
        while (i < s.size() && s[i] != '"') {
            if (s[i] == '\\' && i + 1 < s.size()) { out += s[i + 1]; i += 2; continue; }
            out += s[i++];
        }
        if (i >= s.size()) throw Error(WCSPH_ERR_CONFIG, "config JSON: unterminated string");
        ++i;
        return out;
    }
    // scalar value as text (numbers, true/false/null) or string
    std::string scalar(bool* is_string) {
        ws();
        if (i < s.size() && s[i] == '"') { *is_string = true; return str(); }
        *is_string = false;
        size_t b = i;
        while (i < s.size() && s[i] != ',' && s[i] != '}' && s[i] != ']' && !std::isspace(static_cast<unsigned char>(s[i]))) ++i;
        return s.substr(b, i - b);
    }
    void skip_value() {
        ws();
        if (i >= s.size()) return;
        if (s[i] == '"') { str(); return; }
        if (s[i] == '{' || s[i] == '[') {
            int depth = 0;
            bool in_str = false;
            for (; i < s.size(); ++i) {
                const char c = s[i];
                if (in_str) { if (c == '\\') ++i; else if (c == '"') in_str = false; continue; }
                if (c == '"') in_str = true;
                else if (c == '{' || c == '[') ++depth;
                else if (c == '}' || c == ']') { if (--depth == 0) { ++i; return; } }
            }
            return;
        }
        bool dummy;
        scalar(&dummy);
    }
};

struct Entry { std::string name, value, type; };

std::vector<Entry> parse_entries(const std::string& text) {
    JsonCursor c{text};
    c.ws();
    if (c.eat('{')) {  // {"Configuration": [...], ...}
        bool found = false;
        while (!c.eat('}')) {
            const std::string key = c.str();
            c.expect(':');
            if (key == "Configuration") {
                found = true;
                c.ws();
                const size_t start = c.i;
                c.skip_value();
                const std::string sub = text.substr(start, c.i - start);
                return parse_entries(sub);
            }
            c.skip_value();
            c.eat(',');
        }
        if (!found) throw Error(WCSPH_ERR_CONFIG, "Config JSON must be an array or contain a 'Configuration' array");
    }
    c.expect('[');
    std::vector<Entry> out;
    while (!c.eat(']')) {
        c.expect('{');
        Entry e;
        bool has_name = false, has_value = false, has_type = false;
        while (!c.eat('}')) {
            const std::string key = c.str();
            c.expect(':');
            if (key == "Name") { e.name = c.str(); has_name = true; }
            else if (key == "Value") { bool s; e.value = c.scalar(&s); has_value = true; }
            else if (key == "ValueType") { e.type = c.str(); has_type = true; }
            else c.skip_value();
            c.eat(',');
        }
        if (!has_name || !has_value || !has_type)
            throw Error(WCSPH_ERR_CONFIG, "Config entry missing Name, Value, or ValueType");
        if (e.type != "Double" && e.type != "UnsignedInt" && e.type != "Int" && e.type != "Bool" && e.type != "String")
            throw Error(WCSPH_ERR_CONFIG, "Unknown ValueType: " + e.type);
        out.push_back(std::move(e));
        c.eat(',');
    }
    return out;
}

int warps_from_block(double block) {
    const int w = static_cast<int>(block) / 32;
    if (w <= 2) return 2;
    if (w >= 8) return 8;
    return 4;
}

bool config_allowed(const StepConfig& c) {
    // TABLE_SIZE_MULT >= uint64(1 / CELL_SIZE_MULT^3) (step_tuner.cuh:94-99)
    return c.table_size_mult >= static_cast<uint64_t>(1. / std::pow(static_cast<double>(c.cell_size_mult), 3.));
}
}  // namespace

Tuner::Tuner(CUDASPHSimulator* sim) : sim_(sim) {
    for (int wd : kWarps)
        for (int wf : kWarps)
            for (int ws : kWarps)
                for (int mw : kMaskWords)
                    for (int ch : kChunk)
                        for (double cm : kCellMult)
                            for (uint32_t tm : kTableMult) {
                                StepConfig c;
                                c.warps_density = wd; c.warps_force = wf; c.warps_surface = ws;
                                c.mask_words = mw; c.chunk = ch;
                                c.cell_size_mult = static_cast<float>(cm); c.table_size_mult = tm;
                                if (config_allowed(c)) space_.push_back(c);
                            }
    visited_.assign(space_.size(), 0);
    best_cfg_ = sim->config();
}

void Tuner::set(int searcher, float budget, const char* frozen_json) {
    if (searcher < WCSPH_SEARCH_MCMC || searcher > WCSPH_SEARCH_FULL)
        throw Error(WCSPH_ERR_INVALID_ARGUMENT, "unknown searcher");
    searcher_ = searcher;
    budget_ = budget < 0.f ? 0.f : budget;
    accumulator_ = 0.f;  // set_tune_iterations_per_frame resets the accumulator
    if (frozen_json) {
        std::ifstream f(frozen_json);
        if (!f) throw Error(WCSPH_ERR_IO, std::string("Cannot open config file: ") + frozen_json);
        std::stringstream ss;
        ss << f.rdbuf();
        frozen_cfg_ = parse_config_json(ss.str(), sim_->config());
        frozen_ = true;
        sim_->apply_config(frozen_cfg_);
        best_cfg_ = frozen_cfg_;
    }
}

void Tuner::reset() {
    results_.clear();
    std::fill(visited_.begin(), visited_.end(), 0);
    current_ = -1;
    full_cursor_ = 0;
    best_ms_ = 0.f;
}

bool Tuner::before_step() {
    if (frozen_) return false;
    accumulator_ += budget_;
    const int go = std::min(static_cast<int>(accumulator_), 1);
    accumulator_ -= static_cast<float>(go);
    if (go) return true;
    // non-tuning step: run the best configuration found so far
    if (!results_.empty()) sim_->apply_config(best_cfg_);
    return false;
}

int Tuner::next_candidate() {
    const int n = static_cast<int>(space_.size());
    if (searcher_ == WCSPH_SEARCH_FULL) {
        const int k = full_cursor_ % n;
        ++full_cursor_;
        return k;
    }
    if (searcher_ == WCSPH_SEARCH_RANDOM || current_ < 0) {
        int unvisited = 0;
        for (char v : visited_) unvisited += !v;
        if (unvisited == 0) std::fill(visited_.begin(), visited_.end(), 0), unvisited = n;
        std::uniform_int_distribution<int> d(0, unvisited - 1);
        int pick = d(rng_);
        for (int k = 0; k < n; ++k)
            if (!visited_[k] && pick-- == 0) return k;
        return 0;
    }
    // MCMC proposal: change one parameter of the current configuration to a
    // neighbouring value
    const StepConfig& cur = space_[current_];
    for (int attempt = 0; attempt < 64; ++attempt) {
        StepConfig c = cur;
        std::uniform_int_distribution<int> which(0, 6), dir(0, 1);
        const int p = which(rng_);
        const int step = dir(rng_) ? 1 : -1;
        auto shift = [&](auto& field, const auto* values, int count) {
            int idx = 0;
            for (int k = 0; k < count; ++k)
                if (static_cast<double>(values[k]) == static_cast<double>(field)) idx = k;
            idx = std::clamp(idx + step, 0, count - 1);
            field = static_cast<std::remove_reference_t<decltype(field)>>(values[idx]);
        };
        switch (p) {
        case 0: shift(c.warps_density, kWarps, 3); break;
        case 1: shift(c.warps_force, kWarps, 3); break;
        case 2: shift(c.warps_surface, kWarps, 3); break;
        case 3: shift(c.mask_words, kMaskWords, 5); break;
        case 6: shift(c.chunk, kChunk, 3); break;
        case 4: {
            int idx = 0;
            for (int k = 0; k < 5; ++k) if (static_cast<float>(kCellMult[k]) == c.cell_size_mult) idx = k;
            idx = std::clamp(idx + step, 0, 4);
            c.cell_size_mult = static_cast<float>(kCellMult[idx]);
            break;
        }
        default: shift(c.table_size_mult, kTableMult, 6); break;
        }
        for (int k = 0; k < n; ++k)
            if (space_[k] == c) return k;
    }
    return current_;
}

void Tuner::timed_step(float delta) {
    const int k = next_candidate();
    visited_[k] = 1;
    sim_->apply_config(space_[k]);
    TuneResult r;
    r.cfg = space_[k];
    r.total_ms = sim_->time_steps(1, delta);
    results_.push_back(r);
    if (best_ms_ == 0.f || r.total_ms < best_ms_) {
        best_ms_ = r.total_ms;
        best_cfg_ = r.cfg;
    }
    if (searcher_ == WCSPH_SEARCH_MCMC) {
        // Metropolis acceptance with a temperature of 5% of the current time
        bool accept = current_ < 0 || r.total_ms <= current_ms_;
        if (!accept) {
            const double T = 0.05 * current_ms_;
            std::uniform_real_distribution<double> u(0., 1.);
            accept = u(rng_) < std::exp(-(r.total_ms - current_ms_) / std::max(T, 1e-9));
        }
        if (accept) { current_ = k; current_ms_ = r.total_ms; }
    }
}

StepConfig Tuner::parse_config_json(const std::string& text, const StepConfig& base) {
    StepConfig c = base;
    for (const Entry& e : parse_entries(text)) {
        const double v = (e.type == "String") ? 0.0 : std::atof(e.value.c_str());
        if (e.name == "CELL_SIZE_MULT") c.cell_size_mult = static_cast<float>(v);
        else if (e.name == "TABLE_SIZE_MULT") c.table_size_mult = static_cast<uint32_t>(v);
        else if (e.name == "compute_rho_p_block") c.warps_density = warps_from_block(v);
        else if (e.name == "compute_pressure_accel_n_normal_block") c.warps_force = warps_from_block(v);
        else if (e.name == "compute_non_pressure_accel_block") c.warps_surface = warps_from_block(v);
        else if (e.name == "mask_words") c.mask_words = static_cast<int>(v);
        else if (e.name == "particles_per_warp") c.chunk = static_cast<int>(v);
        else if (e.name == "neighbour_list_width") c.nbr_width = static_cast<int>(v);
        // KTT-only parameters (KERNEL_DIR, *_u_n, *_nlist, *_shared, *_cache_log2,
        // MIN_TABLE_SIZE, EXTERNAL_FORCE ...) have no counterpart and are ignored.
    }
    if (!(c.cell_size_mult >= 0.5f && c.cell_size_mult <= 2.f))
        throw Error(WCSPH_ERR_CONFIG, "CELL_SIZE_MULT out of range [0.5, 2]");
    if (c.table_size_mult == 0 || (c.table_size_mult & (c.table_size_mult - 1)) || c.table_size_mult > 64)
        throw Error(WCSPH_ERR_CONFIG, "TABLE_SIZE_MULT must be a power of two <= 64");
    if (c.mask_words < 1 || c.mask_words > 16) throw Error(WCSPH_ERR_CONFIG, "mask_words must be in [1, 16]");
    if (c.chunk != 0 && c.chunk != 8 && c.chunk != 16 && c.chunk != 32)
        throw Error(WCSPH_ERR_CONFIG, "particles_per_warp must be 8, 16 or 32");
    if (c.nbr_width < 0 || c.nbr_width > 1024)
        throw Error(WCSPH_ERR_CONFIG, "neighbour_list_width must be in [0, 1024]");
    return c;
}

std::string Tuner::config_json(const StepConfig& c) {
    char buf[1024];
    std::snprintf(buf, sizeof(buf),
                  "[\n"
                  "  {\"Name\": \"CELL_SIZE_MULT\", \"Value\": %.17g, \"ValueType\": \"Double\"},\n"
                  "  {\"Name\": \"TABLE_SIZE_MULT\", \"Value\": %u, \"ValueType\": \"UnsignedInt\"},\n"
                  "  {\"Name\": \"compute_rho_p_block\", \"Value\": %d, \"ValueType\": \"UnsignedInt\"},\n"
                  "  {\"Name\": \"compute_pressure_accel_n_normal_block\", \"Value\": %d, \"ValueType\": \"UnsignedInt\"},\n"
                  "  {\"Name\": \"compute_non_pressure_accel_block\", \"Value\": %d, \"ValueType\": \"UnsignedInt\"},\n"
                  "  {\"Name\": \"mask_words\", \"Value\": %d, \"ValueType\": \"UnsignedInt\"},\n"
                  "  {\"Name\": \"particles_per_warp\", \"Value\": %d, \"ValueType\": \"UnsignedInt\"},\n"
                  "  {\"Name\": \"neighbour_list_width\", \"Value\": %d, \"ValueType\": \"UnsignedInt\"}\n"
                  "]\n",
                  static_cast<double>(c.cell_size_mult), c.table_size_mult, c.warps_density * 32,
                  c.warps_force * 32, c.warps_surface * 32, c.mask_words, c.chunk, c.nbr_width);
    return buf;
}

void Tuner::save_config(const char* path) const {
    std::ofstream f(path);
    if (!f) throw Error(WCSPH_ERR_IO, std::string("cannot open ") + path);
    f << config_json(frozen_ ? frozen_cfg_ : (results_.empty() ? sim_->config() : best_cfg_));
}

void Tuner::save_results(const char* path) const {
    // KTT results schema read by the reference's analysis scripts
    // (analysis/e3_distributions.py:13-45): Results[].TotalDuration (ns),
    // Results[].Configuration, Results[].ComputationResults[].{KernelFunction, Duration}.
    std::ofstream f(path);
    if (!f) throw Error(WCSPH_ERR_IO, std::string("cannot open ") + path);
    f << "{\n  \"Results\": [\n";
    for (size_t k = 0; k < results_.size(); ++k) {
        const TuneResult& r = results_[k];
        std::string cfg = config_json(r.cfg);
        f << "    {\"KernelName\": \"simulation_step\", \"TotalDuration\": "
          << static_cast<long long>(r.total_ms * 1e6) << ", \"CompilationOverhead\": 0, \"Configuration\": " << cfg
          << ", \"ComputationResults\": [{\"KernelFunction\": \"simulation_step\", \"Duration\": "
          << static_cast<long long>(r.total_ms * 1e6) << "}]}" << (k + 1 < results_.size() ? ",\n" : "\n");
    }
    f << "  ]\n}\n";
}

// ---- simulator hooks --------------------------------------------------------
void CUDASPHSimulator::set_tuning(int searcher, float budget, const char* frozen_json) {
    tuner_->set(searcher, budget, frozen_json);
}
void CUDASPHSimulator::save_config(const char* path) { tuner_->save_config(path); }
void CUDASPHSimulator::save_tuning_results(const char* path) { tuner_->save_results(path); }
void CUDASPHSimulator::reset_tuning() { tuner_->reset(); }

}  // namespace wcsph
