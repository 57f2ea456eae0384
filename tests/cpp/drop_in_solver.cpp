// Uses physgrad_b200/mpm_solver.h exactly as code written against physgrad's
// src/mpm_solver.h would: config, addParticles, initialize, step/run,
// getParticles/getGrid/getMetrics.  Built by tests/test_cpp_dropin.py.
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "physgrad_b200/mpm_solver.h"

using namespace physgrad::mpm;

// compare mode: particles from <in> (int32 N, then x [N][3], v [N][3], m [N]
// as float32), initialize + 5 step() + run() (10 steps) on a 32^3 grid; the
// state is read back only through a const reference to the solver, with each
// container accessor the reference offers, and written to <out> as x [N][3],
// v [N][3] (float32) for the per-particle comparison with the FP64 oracle.
static int compare(const char* in_path, const char* out_path) {
    FILE* f = std::fopen(in_path, "rb");
    if (!f) return 10;
    int32_t n = 0;
    if (std::fread(&n, 4, 1, f) != 1 || n <= 0) return 11;
    std::vector<float> xin(3 * (size_t)n), vin(3 * (size_t)n), min((size_t)n);
    if (std::fread(xin.data(), 4, xin.size(), f) != xin.size() || std::fread(vin.data(), 4, vin.size(), f) != vin.size() ||
        std::fread(min.data(), 4, min.size(), f) != min.size())
        return 12;
    std::fclose(f);
    MPMSolverConfig cfg;
    cfg.grid_dimensions = {32, 32, 32};
    cfg.grid_spacing = {1.f / 32, 1.f / 32, 1.f / 32};
    cfg.time_step = 1e-4f;
    cfg.simulation_time = 1e-3f;  // run() = 10 steps
    cfg.gravity = {0.f, -9.8f, 0.f};
    cfg.max_particles = n;
    // fields of src/mpm_solver.h:53-65 that reference callers set
    cfg.enable_adaptive_timestep = false;
    cfg.min_timestep = 1e-6f;
    cfg.max_timestep = 1e-3f;
    cfg.enable_debug_output = false;
    cfg.verify_conservation = true;
    MPMSolver<float> solver(cfg);
    std::vector<T3> x((size_t)n), v((size_t)n);
    for (int32_t i = 0; i < n; ++i) {
        x[i] = T3{xin[3 * i], xin[3 * i + 1], xin[3 * i + 2]};
        v[i] = T3{vin[3 * i], vin[3 * i + 1], vin[3 * i + 2]};
    }
    solver.addParticles(x, v, min, MaterialType::ELASTIC);
    solver.initialize();
    for (int i = 0; i < 5; ++i) solver.step();
    solver.run();
    const MPMSolver<float>& cs = solver;
    const auto& P = cs.getParticles();
    if (P.size() != (size_t)n) return 13;
    const std::vector<std::array<float, 3>> pos = P.getPositions();
    const std::vector<std::array<float, 3>> vel = P.getVelocities();
    const std::vector<float> mass = P.getMasses();
    const float* pd = P.getPositionData();
    const float* vd = P.getVelocityData();
    for (int32_t i = 0; i < n; ++i) {
        float a, b, c;
        P.getPosition(i, a, b, c);
        if (a != pos[i][0] || b != pos[i][1] || c != pos[i][2] || pd[3 * i + 1] != b) return 14;
        P.getVelocity(i, a, b, c);
        if (a != vel[i][0] || b != vel[i][1] || c != vel[i][2] || vd[3 * i + 2] != c) return 15;
        if (mass[i] != min[i] || P.getMass(i) != min[i] || P.getMaterialType(i) != MaterialType::ELASTIC) return 16;
    }
    const auto& G = cs.getGrid();
    double gm = 0.0;
    for (size_t k = 0; k < G.getTotalNodes(); ++k) gm += G.getMassData()[k];
    double pm = 0.0;
    for (float q : mass) pm += q;
    if (std::fabs(gm - pm) > 1e-5 * pm) return 17;
    const auto& M = cs.getMetrics();
    if (M.total_steps != 15 || cs.getCurrentStep() != 15) return 18;
    FILE* o = std::fopen(out_path, "wb");
    if (!o) return 19;
    for (int32_t i = 0; i < n; ++i) std::fwrite(pos[i].data(), 4, 3, o);
    std::fwrite(vd, 4, 3 * (size_t)n, o);
    std::fclose(o);
    std::printf("{\"steps\": %d, \"grid_mass\": %.6e, \"particle_mass\": %.6e}\n", cs.getCurrentStep(), gm, pm);
    return 0;
}

int main(int argc, char** argv) {
    if (argc == 4 && std::string(argv[1]) == "compare") return compare(argv[2], argv[3]);
    if (argc > 1) {
        // output run: frames every 2.5e-4 s of simulated time into argv[1]
        MPMSolverConfig oc;
        oc.grid_dimensions = {32, 32, 32};
        oc.grid_spacing = {1.f / 32, 1.f / 32, 1.f / 32};
        oc.simulation_time = 1e-3f;
        oc.enable_output = true;
        oc.output_frequency = 2.5e-4f;
        oc.output_directory = argv[1];
        MPMSolver<float> os(oc);
        std::vector<T3> ox(512, T3{0.5f, 0.5f, 0.5f}), ov(512, T3{0.f, 0.f, 0.f});
        for (size_t i = 0; i < ox.size(); ++i) ox[i].x += 0.0005f * (float)(i % 64);
        os.addParticles(ox, ov, std::vector<float>(512, 1.25e-4f), MaterialType::ELASTIC);
        os.run();
        std::printf("{\"output_steps\": %d}\n", os.getCurrentStep());
        return 0;
    }
    MPMSolverConfig cfg;
    cfg.grid_dimensions = {32, 32, 32};
    cfg.grid_spacing = {1.f / 32, 1.f / 32, 1.f / 32};
    cfg.time_step = 1e-4f;
    cfg.simulation_time = 1e-3f;  // run() = 10 steps
    cfg.gravity = {0.f, -9.8f, 0.f};
    cfg.max_particles = 4096;
    MPMSolver<float> solver(cfg);
    std::mt19937 g(3);
    std::uniform_real_distribution<float> u(0.4f, 0.6f);
    std::vector<T3> x(2048), v(2048, T3{0.f, 0.f, 0.f});
    std::vector<float> m(2048, 1.25e-4f);
    for (auto& p : x) p = T3{u(g), u(g), u(g)};
    solver.addParticles(x, v, m, MaterialType::ELASTIC);
    bool threw = false;
    try {
        solver.step();
    } catch (const std::runtime_error&) {
        threw = true;  // "Solver not initialized", as the reference
    }
    if (!threw) return 2;
    solver.initialize();
    for (int i = 0; i < 5; ++i) solver.step();
    solver.run();
    const auto& P = solver.getParticles();
    double vy = 0.0;
    for (size_t i = 0; i < P.size(); ++i) {
        float a, b, c;
        P.getVelocity(i, a, b, c);
        if (!std::isfinite(a) || !std::isfinite(b) || !std::isfinite(c)) return 3;
        vy += b;
    }
    vy /= (double)P.size();
    const auto& G = solver.getGrid();
    double gm = 0.0;
    for (size_t n = 0; n < G.getTotalNodes(); ++n) gm += G.getMass(n);
    const auto& M = solver.getMetrics();
    std::printf("{\"steps\": %d, \"mean_vy\": %.6e, \"grid_mass\": %.6e, \"particle_mass\": %.6e, \"metric_steps\": %d}\n",
                solver.getCurrentStep(), vy, gm, 2048 * 1.25e-4, M.total_steps);
    // free fall for 15 steps of 1e-4 s: v_y = -9.8 * 1.5e-3 (elastic cube, no walls reached)
    if (std::fabs(vy + 9.8 * 1.5e-3) > 1e-4) return 4;
    if (std::fabs(gm - 2048 * 1.25e-4) > 1e-6) return 5;
    return 0;
}
