// The solver API that code written against physgrad's src/mpm_solver.h uses
// (src/mpm_solver.h:29-329, src/mpm_data_structures.h:79-96, 290-334, 412-427),
// in one translation unit that names its header as "mpm_solver.h" only, so
// the same file builds against either header by the include path alone.
// Compile-only: tests/test_cpp_dropin.py builds it with -fsyntax-only.
#include <array>
#include <cstddef>
#include <string>
#include <vector>

#include "mpm_solver.h"

using namespace physgrad::mpm;

double use_solver_api() {
    MPMSolverConfig cfg;
    cfg.grid_dimensions = {32, 32, 32};
    cfg.grid_spacing = {1.f / 32, 1.f / 32, 1.f / 32};
    cfg.domain_origin = {0.f, 0.f, 0.f};
    cfg.time_step = 1e-4f;
    cfg.simulation_time = 1e-3f;
    cfg.cfl_factor = 0.4f;
    cfg.max_particles = 1024;
    cfg.particle_radius = 0.005f;
    cfg.enable_gravity = true;
    cfg.gravity = {0.f, -9.8f, 0.f};
    cfg.enable_multi_material = true;
    cfg.max_materials = 8;
    cfg.cuda_block_size = 256;
    cfg.enable_g2p2g_fusion = true;
    cfg.enable_adaptive_timestep = false;
    cfg.min_timestep = 1e-6f;
    cfg.max_timestep = 1e-3f;
    cfg.enable_output = false;
    cfg.output_frequency = 0.01f;
    cfg.output_directory = std::string("./mpm_output");
    cfg.enable_profiling = false;
    cfg.enable_debug_output = false;
    cfg.verify_conservation = false;

    MPMSolver<float> solver(cfg);
    std::vector<T3> x(4), v(4);
    std::vector<float> m(4, 1e-3f);
    solver.addParticles(x, v, m, MaterialType::ELASTIC);
    solver.addParticles(x, v, m);
    solver.initialize();
    solver.step();
    solver.run();

    const MPMSolver<float>& cs = solver;
    const auto& P = cs.getParticles();
    const std::size_t n = P.size();
    const std::vector<std::array<float, 3>> pos = P.getPositions();
    const std::vector<std::array<float, 3>> vel = P.getVelocities();
    const std::vector<float> mass = P.getMasses();
    float px = 0.f, py = 0.f, pz = 0.f, vx = 0.f, vy = 0.f, vz = 0.f;
    P.getPosition(0, px, py, pz);
    P.getVelocity(0, vx, vy, vz);
    const float m0 = P.getMass(0);

    const auto& G = cs.getGrid();
    const std::array<float, 3> gs = G.getGridSpacing();
    const std::size_t nodes = G.getTotalNodes();
    const auto dims = G.getDimensions();
    const auto sp = G.getSpacing();
    const auto org = G.getOrigin();

    const MPMPerformanceMetrics& M = cs.getMetrics();
    M.print();
    double t = M.total_simulation_time + M.average_step_time + M.g2p_time + M.p2g_time + M.grid_update_time +
               M.particle_update_time;
    t += (double)(M.total_memory_usage + M.particle_memory + M.grid_memory);
    t += M.total_steps + M.rejected_steps + M.average_particles_per_second;
    t += cs.getCurrentTime() + cs.getCurrentStep();

    const MaterialParameters elastic = createElasticMaterial(1000.f, 1e4f, 0.3f);
    const MaterialParameters fluid = createFluidMaterial(1000.f, 1e-3f);
    t += elastic.youngs_modulus + fluid.density;
    return t + (double)n + pos.size() + vel.size() + mass.size() + px + py + pz + vx + vy + vz + m0 + gs[0] +
           (double)nodes + dims.x + sp.x + org.x;
}

int main() { return use_solver_api() > 0.0 ? 0 : 1; }
