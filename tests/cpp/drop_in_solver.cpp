// Uses physgrad_b200/mpm_solver.h exactly as code written against physgrad's
// src/mpm_solver.h would: config, addParticles, initialize, step/run,
// getParticles/getGrid/getMetrics.  Built by tests/test_cpp_dropin.py.
#include <cmath>
#include <cstdio>
#include <random>
#include <stdexcept>

#include "physgrad_b200/mpm_solver.h"

using namespace physgrad::mpm;

int main(int argc, char** argv) {
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
