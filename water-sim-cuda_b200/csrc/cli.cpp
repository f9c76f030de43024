// mpm_run: the headless counterpart of the reference's program
// (main.cpp -> Simulation::Simulation + Simulation::run, Simulation.cpp:4-54)
// on the C ABI of libmpm_b200.so.
//
//   mpm_run CONFIG [options]
//
// Builds the scene from the config's WATER= / OBJECT= entries (model paths
// relative to --base-dir, default: the config file's directory), then runs
// --frames frames of SUBSTEPS substeps each, as the render loop does while
// the window is open and not paused.  Where the reference draws a frame, this
// program can append the positions (original particle order) to a file.
//
// Options:
//   --frames N          frames to run (default 100)
//   --device D          CUDA device (default 0)
//   --base-dir DIR      directory the model paths are relative to
//   --positions FILE    write positions every --every frames (default 1)
//   --checkpoint FILE   save a checkpoint after the last frame
//   --resume FILE       start from a checkpoint instead of the config
//   --corrector FILE    learned large steps: FILE holds MPM_CORRECTOR_PARAMS
//                       little-endian float32; a frame is SUBSTEPS / --ratio
//                       large steps (--ratio default 4, --threshold default
//                       0.02: the density-change fallback)
//   --render DIR        render frames headless (the SSF passes of the
//                       reference's renderer) to DIR/frame_NNNNN.ppm every
//                       --every frames; --render-size WxH (default 1920x1600)
//   --quiet             no per-frame lines
//
// Positions file: "MPMPOS01", int64 n, int64 frames, then per frame n x 3
// float32 (x, y, z per particle).  The summary is one JSON line on stdout.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "mpm_b200.h"

namespace {

int usage() {
    std::fprintf(stderr,
                 "usage: mpm_run CONFIG [--frames N] [--device D] [--base-dir DIR] [--positions FILE] [--every K]\n"
                 "               [--checkpoint FILE] [--resume FILE] [--corrector FILE] [--ratio R]\n"
                 "               [--threshold T] [--render DIR] [--render-size WxH] [--quiet]\n");
    return 2;
}

int fail(const char* what, mpm_status s, const char* detail) {
    std::fprintf(stderr, "mpm_run: %s: %s: %s\n", what, mpm_status_string(s), detail ? detail : "");
    return 1;
}

bool read_file(const std::string& path, std::string* out) {
    std::ifstream in(path, std::ios::binary);
    if (!in) return false;
    std::ostringstream ss;
    ss << in.rdbuf();
    *out = ss.str();
    return true;
}

std::string dir_of(const std::string& p) {
    const size_t k = p.find_last_of('/');
    return k == std::string::npos ? std::string(".") : p.substr(0, k);
}

}  // namespace

int main(int argc, char** argv) {
    std::string config, base_dir, pos_path, ckpt_out, resume, corrector, render_dir;
    int rw = 1920, rh = 1600;
    long frames = 100, every = 1;
    int device = 0, ratio = 4;
    float threshold = 0.02f;
    bool quiet = false;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto next = [&](const char* name) -> const char* {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "mpm_run: %s needs a value\n", name);
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "--frames") frames = std::atol(next("--frames"));
        else if (a == "--device") device = std::atoi(next("--device"));
        else if (a == "--base-dir") base_dir = next("--base-dir");
        else if (a == "--positions") pos_path = next("--positions");
        else if (a == "--every") every = std::atol(next("--every"));
        else if (a == "--checkpoint") ckpt_out = next("--checkpoint");
        else if (a == "--resume") resume = next("--resume");
        else if (a == "--corrector") corrector = next("--corrector");
        else if (a == "--ratio") ratio = std::atoi(next("--ratio"));
        else if (a == "--threshold") threshold = (float)std::atof(next("--threshold"));
        else if (a == "--render") render_dir = next("--render");
        else if (a == "--render-size") {
            if (std::sscanf(next("--render-size"), "%dx%d", &rw, &rh) != 2) return usage();
        } else if (a == "--quiet") quiet = true;
        else if (a == "-h" || a == "--help") return usage();
        else if (!a.empty() && a[0] == '-') return usage();
        else config = a;
    }
    if ((config.empty() && resume.empty()) || frames < 0 || every < 1) return usage();

    mpm_engine* eng = nullptr;
    mpm_config cfg{};
    std::string config_text;
    mpm_status s;
    const auto t0 = std::chrono::steady_clock::now();
    if (!resume.empty()) {
        if ((s = mpm_checkpoint_load(resume.c_str(), device, &eng)) != MPM_OK)
            return fail("resume", s, mpm_global_last_error());
        if ((s = mpm_checkpoint_info(resume.c_str(), &cfg, nullptr, nullptr, nullptr, 0)) != MPM_OK)
            return fail("resume", s, mpm_global_last_error());
    } else {
        if (!read_file(config, &config_text)) return fail("config", MPM_ERR_IO, config.c_str());
        char err[1024] = {0};
        int32_t nw = 0, no = 0;
        if ((s = mpm_config_parse_string(config_text.c_str(), &cfg, nullptr, 0, &nw, nullptr, 0, &no, err,
                                         sizeof(err))) != MPM_OK)
            return fail("config", s, err);
        mpm_scene_data* scene = nullptr;
        const std::string base = base_dir.empty() ? dir_of(config) : base_dir;
        if ((s = mpm_scene_build(config_text.c_str(), base.c_str(), device, &scene)) != MPM_OK)
            return fail("scene", s, mpm_scene_last_error());
        const int64_t n = mpm_scene_data_num_particles(scene), t = mpm_scene_data_num_triangles(scene);
        std::vector<float> state((size_t)MPM_PARTICLE_PLANES * n), tris((size_t)9 * t);
        mpm_scene_data_state(scene, state.data());
        mpm_scene_data_triangles(scene, tris.data());
        if (mpm_scene_data_log(scene)[0]) std::fprintf(stderr, "%s", mpm_scene_data_log(scene));
        mpm_scene_data_free(scene);
        if ((s = mpm_create(&cfg, device, &eng)) != MPM_OK) return fail("create", s, mpm_global_last_error());
        if ((s = mpm_init_particles(eng, n, state.data())) != MPM_OK) return fail("init", s, mpm_last_error(eng));
        if ((s = mpm_init_sdf(eng, t ? tris.data() : nullptr, t)) != MPM_OK)
            return fail("initSDF", s, mpm_last_error(eng));
    }
    const int64_t n = mpm_num_particles(eng);
    const double setup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

    int32_t large_per_frame = 0;
    if (!corrector.empty()) {
        std::string raw;
        if (!read_file(corrector, &raw) || raw.size() != MPM_CORRECTOR_PARAMS * sizeof(float))
            return fail("corrector", MPM_ERR_IO, "expected MPM_CORRECTOR_PARAMS float32 values");
        std::vector<float> w(MPM_CORRECTOR_PARAMS);
        std::memcpy(w.data(), raw.data(), raw.size());
        if (ratio < 1 || cfg.substeps % ratio != 0)
            return fail("corrector", MPM_ERR_INVALID_ARGUMENT, "SUBSTEPS must be a multiple of --ratio");
        if ((s = mpm_set_corrector(eng, w.data(), ratio, threshold)) != MPM_OK)
            return fail("corrector", s, mpm_last_error(eng));
        large_per_frame = cfg.substeps / ratio;
    }

    FILE* pf = nullptr;
    std::vector<float> xyz((size_t)3 * n);
    int64_t written = 0;
    if (!pos_path.empty()) {
        pf = std::fopen(pos_path.c_str(), "wb");
        if (!pf) return fail("positions", MPM_ERR_IO, pos_path.c_str());
        std::fwrite("MPMPOS01", 1, 8, pf);
        std::fwrite(&n, sizeof(n), 1, pf);
        std::fwrite(&written, sizeof(written), 1, pf);
    }
    mpm_renderer* ren = nullptr;
    std::vector<uint8_t> rgb8;
    int64_t rendered = 0;
    if (!render_dir.empty()) {
        mpm_render_params rp;
        mpm_render_params_default(&rp, cfg.size_x, cfg.size_y, cfg.size_z);
        rp.width = rw;
        rp.height = rh;
        if ((s = mpm_renderer_create(&rp, device, &ren)) != MPM_OK) return fail("render", s, mpm_global_last_error());
        rgb8.resize((size_t)rw * rh * 3);
    }
    mpm_learned_stats ls{};
    const auto t1 = std::chrono::steady_clock::now();
    for (long f = 0; f < frames; ++f) {
        s = large_per_frame ? mpm_step_learned(eng, large_per_frame, &ls) : mpm_step(eng, cfg.substeps);
        if (s != MPM_OK) return fail("step", s, mpm_last_error(eng));
        if (pf && (f + 1) % every == 0) {
            if ((s = mpm_get_positions(eng, xyz.data())) != MPM_OK) return fail("positions", s, mpm_last_error(eng));
            std::fwrite(xyz.data(), sizeof(float), xyz.size(), pf);
            ++written;
        }
        if (ren && (f + 1) % every == 0) {
            if ((s = mpm_render_frame(ren, eng)) != MPM_OK ||
                (s = mpm_renderer_get_image(ren, nullptr, rgb8.data())) != MPM_OK)
                return fail("render", s, mpm_renderer_last_error(ren));
            char name[64];
            std::snprintf(name, sizeof(name), "/frame_%05ld.ppm", f + 1);
            FILE* img = std::fopen((render_dir + name).c_str(), "wb");
            if (!img) return fail("render", MPM_ERR_IO, (render_dir + name).c_str());
            std::fprintf(img, "P6\n%d %d\n255\n", rw, rh);
            for (int y = rh - 1; y >= 0; --y) std::fwrite(rgb8.data() + (size_t)y * rw * 3, 1, (size_t)rw * 3, img);
            std::fclose(img);
            ++rendered;
        }
        if (!quiet) std::fprintf(stderr, "frame %ld/%ld\n", f + 1, frames);
    }
    if ((s = mpm_synchronize(eng)) != MPM_OK) return fail("step", s, mpm_last_error(eng));
    const double run_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
    if (pf) {
        std::fseek(pf, 16, SEEK_SET);
        std::fwrite(&written, sizeof(written), 1, pf);
        std::fclose(pf);
    }
    if (!ckpt_out.empty()) {
        if ((s = mpm_checkpoint_save(eng, ckpt_out.c_str(), config_text.c_str())) != MPM_OK)
            return fail("checkpoint", s, mpm_last_error(eng));
    }
    mpm_stats st{};
    mpm_get_stats(eng, &st, 0);
    const double substeps = (double)frames * cfg.substeps;
    std::printf(
        "{\"particles\": %lld, \"frames\": %ld, \"substeps_per_frame\": %d, \"setup_s\": %.3f, \"run_s\": %.4f, "
        "\"frames_per_s\": %.2f, \"particle_substeps_per_s\": %.4g, \"substeps_total\": %lld, "
        "\"large_steps\": %lld, \"fallbacks\": %lld, \"positions_frames\": %lld, \"rendered_frames\": %lld}\n",
        (long long)n, frames, cfg.substeps, setup_s, run_s, run_s > 0 ? frames / run_s : 0.0,
        run_s > 0 ? (double)n * substeps / run_s : 0.0, (long long)st.substeps, (long long)ls.large_steps,
        (long long)ls.fallbacks, (long long)written, (long long)rendered);
    mpm_renderer_destroy(ren);
    mpm_destroy(eng);
    return 0;
}
