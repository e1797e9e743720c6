// cli_main.cpp — headless driver with the reference's command line
// (RunOptions/parse_cli src/cli.h:9-27, src/cli.cu:49-101;
// Application::init/run_headless/stop_reached src/application.cu:24-58,105-161).
// One executable serves every preset scene (--scene NAME) instead of one
// executable per app; all other flags keep the reference's meaning.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/wcsph.h"

namespace {

struct RunOptions {
    bool headless = false;
    std::optional<std::string> snapshot_load, snapshot_save, frozen_config;
    int searcher = WCSPH_SEARCH_MCMC;
    float tuning_budget = 0.1f;
    enum class StopKind { None, Iters, SimTime, WallTime } stop_kind = StopKind::None;
    double stop_value = 0.0;
    float fixed_dt = 0.01f;  // Application::DEFAULT_TIME_STEP (application.h:15)
    int warmup_iters = 0;
    std::optional<std::string> ktt_output, log_csv;
    bool log_metrics = false;
    std::string scene = "surface_tension";
    int device = -1;
    uint64_t seed = 0;
    // headless frames of the particle view (the reference's window contents)
    std::optional<std::string> frames_dir;
    int frame_every = 10;
    uint32_t frame_w = 640, frame_h = 480;
    float camera[5] = {0.f, 0.f, 2.5f, 270.f, 0.f};   // x, y, z, yaw deg, pitch deg (application.cu:16)
};

void print_usage(const char* prog) {
    std::cerr << "Usage: " << prog << " [OPTIONS]\n"
                 "  --scene NAME                    surface_tension | tilting_box | dam_break | mesh_obstacle |\n"
                 "                                  large_tilting | rollout_block (default surface_tension)\n"
                 "  --headless                      No window, no GUI, no render (always headless here)\n"
                 "  --snapshot-load FILE            Load snapshot after setup_scene\n"
                 "  --snapshot-save FILE            Save snapshot at stop\n"
                 "  --frozen-config FILE            JSON config; disables searcher\n"
                 "  --searcher {mcmc|random|full}   Default: mcmc\n"
                 "  --tuning-budget FLOAT           Default: 0.1 (0 disables tuning)\n"
                 "  --stop iters=N | sim-time=T | wall-time=T   Required in --headless\n"
                 "  --fixed-dt FLOAT                Default: 0.01\n"
                 "  --warmup-iters N                Default: 0\n"
                 "  --ktt-output PATH               Tuning results JSON (KTT schema)\n"
                 "  --log-csv FILE                  Per-step CSV log\n"
                 "  --log-metrics                   Add mean_speed,ke columns\n"
                 "  --device N                      CUDA device (default: current)\n"
                 "  --seed N                        Seed of the scene's jitter/velocities\n"
                 "  --frames DIR                    Write the particle view as PPM frames into DIR\n"
                 "  --frame-every N                 Frame interval in steps (default 10)\n"
                 "  --frame-size WxH                Default 640x480\n"
                 "  --camera x,y,z,yaw,pitch        Degrees; default 0,0,2.5,270,0\n";
}

int parse_searcher(const char* s) {
    if (!std::strcmp(s, "mcmc")) return WCSPH_SEARCH_MCMC;
    if (!std::strcmp(s, "random")) return WCSPH_SEARCH_RANDOM;
    if (!std::strcmp(s, "full")) return WCSPH_SEARCH_FULL;
    throw std::invalid_argument(std::string("Unknown searcher: ") + s);
}

// parse_stop (cli.cu:31-47)
void parse_stop(const char* s, RunOptions& o) {
    const char* eq = std::strchr(s, '=');
    if (!eq) throw std::invalid_argument("--stop must be iters=N, sim-time=T, or wall-time=T");
    const std::string key(s, eq - s);
    const char* val = eq + 1;
    char* end = nullptr;
    o.stop_value = std::strtod(val, &end);
    if (end == val || *end != '\0') throw std::invalid_argument(std::string("Invalid --stop value: ") + val);
    if (key == "iters") o.stop_kind = RunOptions::StopKind::Iters;
    else if (key == "sim-time") o.stop_kind = RunOptions::StopKind::SimTime;
    else if (key == "wall-time") o.stop_kind = RunOptions::StopKind::WallTime;
    else throw std::invalid_argument("Unknown --stop kind: " + key);
}

RunOptions parse_cli(int argc, char** argv) {
    RunOptions o;
    auto need = [&](int& i, const char* flag) -> const char* {
        if (++i >= argc) throw std::invalid_argument(std::string(flag) + " requires an argument");
        return argv[i];
    };
    for (int i = 1; i < argc; ++i) {
        const char* a = argv[i];
        if (!std::strcmp(a, "--headless")) o.headless = true;
        else if (!std::strcmp(a, "--snapshot-load")) o.snapshot_load = need(i, a);
        else if (!std::strcmp(a, "--snapshot-save")) o.snapshot_save = need(i, a);
        else if (!std::strcmp(a, "--frozen-config")) o.frozen_config = need(i, a);
        else if (!std::strcmp(a, "--searcher")) o.searcher = parse_searcher(need(i, a));
        else if (!std::strcmp(a, "--tuning-budget")) o.tuning_budget = std::strtof(need(i, a), nullptr);
        else if (!std::strcmp(a, "--stop")) parse_stop(need(i, a), o);
        else if (!std::strcmp(a, "--fixed-dt")) o.fixed_dt = std::strtof(need(i, a), nullptr);
        else if (!std::strcmp(a, "--warmup-iters")) o.warmup_iters = std::atoi(need(i, a));
        else if (!std::strcmp(a, "--ktt-output")) o.ktt_output = need(i, a);
        else if (!std::strcmp(a, "--log-csv")) o.log_csv = need(i, a);
        else if (!std::strcmp(a, "--log-metrics")) o.log_metrics = true;
        else if (!std::strcmp(a, "--scene")) o.scene = need(i, a);
        else if (!std::strcmp(a, "--device")) o.device = std::atoi(need(i, a));
        else if (!std::strcmp(a, "--seed")) o.seed = std::strtoull(need(i, a), nullptr, 10);
        else if (!std::strcmp(a, "--frames")) o.frames_dir = need(i, a);
        else if (!std::strcmp(a, "--frame-every")) o.frame_every = std::max(1, std::atoi(need(i, a)));
        else if (!std::strcmp(a, "--frame-size")) {
            const char* v = need(i, a);
            if (std::sscanf(v, "%ux%u", &o.frame_w, &o.frame_h) != 2 || !o.frame_w || !o.frame_h)
                throw std::invalid_argument(std::string("bad --frame-size: ") + v);
        } else if (!std::strcmp(a, "--camera")) {
            const char* v = need(i, a);
            if (std::sscanf(v, "%f,%f,%f,%f,%f", &o.camera[0], &o.camera[1], &o.camera[2], &o.camera[3],
                            &o.camera[4]) != 5)
                throw std::invalid_argument(std::string("bad --camera: ") + v);
        }
        else if (!std::strcmp(a, "--help") || !std::strcmp(a, "-h")) { print_usage(argv[0]); std::exit(EXIT_SUCCESS); }
        else throw std::invalid_argument(std::string("Unknown argument: ") + a);
    }
    if (o.headless && o.stop_kind == RunOptions::StopKind::None)
        throw std::invalid_argument("--stop is required in --headless mode");
    if (o.stop_kind == RunOptions::StopKind::None)
        throw std::invalid_argument("--stop is required (this driver has no interactive mode)");
    return o;
}

void check(int status, wcsph_ctx* ctx, const std::string& what) {
    if (status != WCSPH_OK)
        throw std::runtime_error(what + ": " + wcsph_status_string(status) + " (" + wcsph_last_error(ctx) + ")");
}

struct App {
    RunOptions opts;
    wcsph_ctx* ctx = nullptr;
    wcsph_preset_info info{};
    int64_t updates = 0;

    ~App() { if (ctx) wcsph_destroy(ctx); }

    void init() {
        // setup_scene
        int s = wcsph_preset(opts.scene.c_str(), opts.seed, &info, nullptr, nullptr, nullptr);
        if (s != WCSPH_OK) throw std::runtime_error("unknown or unavailable scene: " + opts.scene);
        std::vector<float> pos(4ull * info.fluid_n), vel(4ull * info.fluid_n), bpos(4ull * info.boundary_n);
        check(wcsph_preset(opts.scene.c_str(), opts.seed, &info, pos.data(), vel.data(), bpos.data()), nullptr,
              "preset");
        wcsph_scene sc{};
        sc.fluid_n = info.fluid_n;
        sc.fluid_pos = pos.data();
        sc.fluid_vel = vel.data();
        sc.boundary_n = info.boundary_n;
        sc.boundary_pos = info.boundary_n ? bpos.data() : nullptr;
        sc.box = info.box;
        check(wcsph_create(&info.params, &sc, opts.device, &ctx), nullptr, "create");
        // Application::init (application.cu:24-58)
        if (opts.snapshot_load) {
            s = wcsph_snapshot_load(ctx, opts.snapshot_load->c_str(), opts.scene.c_str());
            if (s != WCSPH_OK) throw std::runtime_error(std::string("Snapshot load failed: ") + wcsph_last_error(ctx));
        }
        if (opts.warmup_iters) {
            check(wcsph_set_tuning(ctx, opts.searcher, 0.f, nullptr), ctx, "set_tuning");
            for (int i = 0; i < opts.warmup_iters; ++i) update_objects(opts.fixed_dt);
            check(wcsph_reset_tuning(ctx), ctx, "reset_tuning");
        }
        const char* frozen = opts.frozen_config ? opts.frozen_config->c_str() : nullptr;
        check(wcsph_set_tuning(ctx, opts.searcher, opts.tuning_budget, frozen), ctx, "set_tuning");
    }

    void update_objects(float delta) {
        ++updates;
        if (info.moving_box) {
            wcsph_box b;
            check(wcsph_preset_box(opts.scene.c_str(), updates, delta, &b), ctx, "preset_box");
            check(wcsph_set_box(ctx, &b), ctx, "set_box");
        }
        check(wcsph_step(ctx, delta), ctx, "step");
    }

    bool stop_reached(int step, double sim_time, std::chrono::steady_clock::time_point t0) const {
        switch (opts.stop_kind) {
        case RunOptions::StopKind::Iters: return step >= static_cast<int>(opts.stop_value);
        case RunOptions::StopKind::SimTime: return sim_time >= opts.stop_value;
        case RunOptions::StopKind::WallTime:
            return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() >= opts.stop_value;
        default: return false;
        }
    }

    void run_headless() {
        using clock = std::chrono::steady_clock;
        const auto t0 = clock::now();
        double sim_time = 0.0;
        int step = 0;
        std::ofstream log;
        if (opts.log_csv) {
            log.open(*opts.log_csv);
            log << "step,sim_time,wall_dt_ms,scheduled_tune";
            if (opts.log_metrics) log << ",mean_speed,ke";
            log << '\n';
        }
        wcsph_camera cam{};
        wcsph_render_opts ropt{};
        std::vector<uint8_t> rgba;
        if (opts.frames_dir) {
            const float deg = 3.14159265358979f / 180.f;
            wcsph_camera_look(opts.camera, opts.camera[3] * deg, opts.camera[4] * deg, opts.frame_w, opts.frame_h, &cam);
            wcsph_default_render_opts(&ropt);
            ropt.width = opts.frame_w;
            ropt.height = opts.frame_h;
            ropt.radius = info.params.particle_radius;
            rgba.resize(static_cast<size_t>(opts.frame_w) * opts.frame_h * 4);
        }
        auto write_frame = [&](int k) {
            check(wcsph_render(ctx, &cam, &ropt, rgba.data(), nullptr), ctx, "render");
            char name[64];
            std::snprintf(name, sizeof(name), "/frame_%06d.ppm", k);
            std::ofstream f(*opts.frames_dir + name, std::ios::binary);
            if (!f) throw std::runtime_error("cannot write frame into " + *opts.frames_dir);
            f << "P6\n" << opts.frame_w << ' ' << opts.frame_h << "\n255\n";
            for (size_t px = 0; px < rgba.size(); px += 4) f.write(reinterpret_cast<const char*>(&rgba[px]), 3);
        };
        while (!stop_reached(step, sim_time, t0)) {
            const auto ts = clock::now();
            update_objects(opts.fixed_dt);
            check(wcsph_synchronize(ctx), ctx, "synchronize");
            sim_time += opts.fixed_dt;
            const double wall_dt = std::chrono::duration<double, std::milli>(clock::now() - ts).count();
            if (log) {
                int tuned = 0;
                wcsph_was_tuning_step(ctx, &tuned);
                log << step << ',' << sim_time << ',' << wall_dt << ',' << tuned;
                if (opts.log_metrics) {
                    float v = 0.f, ke = 0.f;
                    check(wcsph_metrics(ctx, &v, &ke), ctx, "metrics");
                    log << ',' << v << ',' << ke;
                }
                log << '\n';
            }
            if (opts.frames_dir && step % opts.frame_every == 0) write_frame(step);
            ++step;
        }
        if (opts.snapshot_save) {
            const int s = wcsph_snapshot_save(ctx, opts.snapshot_save->c_str(), opts.scene.c_str());
            if (s != WCSPH_OK) throw std::runtime_error(std::string("Snapshot save failed: ") + wcsph_last_error(ctx));
        }
        if (opts.ktt_output) check(wcsph_save_tuning_results(ctx, opts.ktt_output->c_str()), ctx, "save results");
    }
};

}  // namespace

int main(int argc, char** argv) {
    try {
        App app;
        app.opts = parse_cli(argc, argv);
        app.init();
        app.run_headless();
    } catch (const std::exception& e) {
        std::cerr << e.what() << std::endl;
        return EXIT_FAILURE;
    }
    return EXIT_SUCCESS;
}
