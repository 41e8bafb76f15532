// fluidgpu_main.cpp -- the FluidGPU driver executable over the C ABI.
//
// Restates the reference's driver (main.cpp:9-58) and the set-up half of
// FluidSolver3D::init / run (FluidSolver3D.cu:81-199, 3100-3163):
//   1. read a config.json (argv[1], else the reference's fixed
//      InputData/config.json, main.cpp:11) with the keys of main.cpp:17-52 and
//      this library's additions (fp_config_load_json);
//   2. load the label file "inputLabelData" (default InputData/labels.txt);
//   3. with "activeBody", load the body: the analytic sphere when
//      "body_radius" > 0, else the SDF file "body_sdf" (the reference's fixed
//      InputData/ball.sdf, FluidSolver3D.cu:158);
//   4. seed "ppc" particles per FLUID cell and write them to
//      "initialParticles" (the reference's InputData/particles_-1.ply,
//      FluidSolver3D.cu:196; an empty string skips the file);
//   5. fp_run("frameAmount"): frames*iterPerFrame + 1 steps with a particle
//      frame every iterPerFrame steps, body_<frame>.ply and csvRes.csv beside
//      the frames when a body is active;
//   6. print the elapsed time and fps as run() does (FluidSolver3D.cu:3149-3162).
// Exit status 0 on success, 1 on any failure (with the library's message).
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>

#include "../../include/fluidprjct.h"

namespace {

// The one key the driver reads itself: "initialParticles" (a string), found
// textually; absent means the reference's path.
std::string initial_particles_path(const char* cfg_path) {
    std::ifstream f(cfg_path);
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string t = ss.str();
    const std::string key = "\"initialParticles\"";
    size_t p = t.find(key);
    if (p == std::string::npos) return "InputData/particles_-1.ply";
    p = t.find(':', p + key.size());
    if (p == std::string::npos) return "InputData/particles_-1.ply";
    p = t.find('"', p);
    if (p == std::string::npos) return "InputData/particles_-1.ply";
    const size_t e = t.find('"', p + 1);
    if (e == std::string::npos) return "InputData/particles_-1.ply";
    return t.substr(p + 1, e - p - 1);
}

int fail(fp_solver* s, const char* what, int rc) {
    std::fprintf(stderr, "FluidGPU: %s failed (status %d): %s\n", what, rc, s ? fp_last_error(s) : "");
    if (s) fp_destroy(s);
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc > 2 || (argc == 2 && (!std::strcmp(argv[1], "-h") || !std::strcmp(argv[1], "--help")))) {
        std::fprintf(stderr, "usage: FluidGPU [config.json]   (default InputData/config.json)\n");
        return argc == 2 ? 0 : 1;
    }
    const char* cfg_path = argc == 2 ? argv[1] : "InputData/config.json";
    fp_config cfg;
    fp_config_default(&cfg);
    char labels[1024];
    std::snprintf(labels, sizeof labels, "%s", "InputData/labels.txt");  // main.cpp:35
    int frames = 100;                                                     // main.cpp:39
    int rc = fp_config_load_json(cfg_path, &cfg, labels, sizeof labels, &frames);
    if (rc != FP_OK) return fail(nullptr, "reading the config", rc);
    if (!labels[0]) std::snprintf(labels, sizeof labels, "%s", "InputData/labels.txt");
    std::printf("alpha = %g\n", double(cfg.pic_weight));  // main.cpp:41

    fp_solver* s = nullptr;
    rc = fp_create(&cfg, &s);
    if (rc != FP_OK) return fail(nullptr, "fp_create", rc);
    rc = fp_load_labels(s, labels);
    if (rc != FP_OK) return fail(s, "loading the labels", rc);
    if (cfg.active_body) {
        rc = fp_load_sdf(s, cfg.body_radius > 0.0f ? nullptr : cfg.body_sdf);
        if (rc != FP_OK) return fail(s, "loading the body", rc);
    }
    rc = fp_seed_particles(s, cfg.ppc, cfg.seed);
    if (rc != FP_OK) return fail(s, "seeding particles", rc);
    std::printf("Number of particles is%lld\n", (long long)fp_num_particles(s));  // FluidSolver3D.cu:195
    const std::string init_ply = initial_particles_path(cfg_path);
    if (!init_ply.empty()) {
        rc = fp_save_ply(s, init_ply.c_str(), FP_OUT_PLY);
        if (rc != FP_OK) return fail(s, "writing the initial particles", rc);
    }

    const auto t0 = std::chrono::steady_clock::now();
    rc = fp_run(s, frames);
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rc != FP_OK) return fail(s, "fp_run", rc);
    fp_step_stats st;
    fp_stats(s, &st);
    const int ipf = cfg.iter_per_frame > 0 ? cfg.iter_per_frame : 1;
    std::printf("total  frames = %d\n", frames * ipf);
    std::printf("elapsed time = %g\n", el);
    std::printf("last step (ms): label %g p2g %g pressure %g (%d PCG iterations, residual %.3g) project %g "
                "body %g advect %g total %g\n",
                double(st.t_label), double(st.t_p2g), double(st.t_pressure), st.pcg_iters, st.residual,
                double(st.t_project), double(st.t_body), double(st.t_advect), double(st.t_total));
    std::printf("fps = %g\n", el > 0 ? double(frames) / el : 0.0);
    fp_destroy(s);
    return 0;
}
