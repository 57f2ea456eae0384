// Uses physgrad_b200/material_point_method.h and physgrad_b200/differentiable_mpm.h
// as code written against physgrad's src/material_point_method.h and
// src/differentiable_mpm.h would.  Built and run by tests/test_cpp_dropin.py,
// which writes the inputs and checks the outputs against the oracle.
//
//   drop_in_ref_diff ref  <in> <out>   MPMSolver<float, 64>: addParticles, steps, getParticles, getGrid
//   drop_in_ref_diff diff <in> <out>   DifferentiableMPMSystem<float>: steps with gradients, computeGradients
//
// Binary files: little-endian int32 / float32 records in the order read below.
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "physgrad_b200/differentiable_mpm.h"

using physgrad::ConceptVector3D;
using V3 = ConceptVector3D<float>;

namespace {

struct Reader {
    FILE* f;
    explicit Reader(const char* path) : f(std::fopen(path, "rb")) {
        if (!f) throw std::runtime_error("cannot open input");
    }
    ~Reader() { std::fclose(f); }
    int i32() {
        int v;
        if (std::fread(&v, 4, 1, f) != 1) throw std::runtime_error("short input");
        return v;
    }
    float f32() {
        float v;
        if (std::fread(&v, 4, 1, f) != 1) throw std::runtime_error("short input");
        return v;
    }
    std::vector<float> floats(size_t n) {
        std::vector<float> v(n);
        if (n && std::fread(v.data(), 4, n, f) != n) throw std::runtime_error("short input");
        return v;
    }
};

struct Writer {
    FILE* f;
    explicit Writer(const char* path) : f(std::fopen(path, "wb")) {
        if (!f) throw std::runtime_error("cannot open output");
    }
    ~Writer() { std::fclose(f); }
    void floats(const std::vector<float>& v) { std::fwrite(v.data(), 4, v.size(), f); }
};

// in: N, nx, ny, nz, steps, dx, origin[3], dt, gravity[3], x[N][3], v[N][3], m[N], vol[N]
// out: x[N][3], v[N][3], grid mass[nodes], grid velocity[nodes][3], grid momentum[nodes][3]
int run_ref(const char* in, const char* out) {
    Reader r(in);
    const int N = r.i32(), nx = r.i32(), ny = r.i32(), nz = r.i32(), steps = r.i32();
    const float dx = r.f32();
    V3 origin;
    for (int a = 0; a < 3; ++a) origin[a] = r.f32();
    physgrad::mpm::MPMSolver<float>::SimulationParams params;
    params.timestep = r.f32();
    for (int a = 0; a < 3; ++a) params.gravity[a] = r.f32();
    const std::vector<float> x = r.floats(3 * N), v = r.floats(3 * N), m = r.floats(N), vol = r.floats(N);
    std::vector<V3> pos(N), vel(N);
    for (int p = 0; p < N; ++p) {
        pos[p] = V3(x[3 * p], x[3 * p + 1], x[3 * p + 2]);
        vel[p] = V3(v[3 * p], v[3 * p + 1], v[3 * p + 2]);
    }
    physgrad::mpm::MPMSolver<float> solver(int3(nx, ny, nz), V3(dx, dx, dx), origin, params);
    // two batches of particles with the container read back in between, as
    // a caller that grows its scene would
    const int h = N / 2;
    solver.addParticles(std::vector<V3>(pos.begin(), pos.begin() + h), std::vector<V3>(vel.begin(), vel.begin() + h),
                        std::vector<float>(m.begin(), m.begin() + h), std::vector<float>(vol.begin(), vol.begin() + h));
    if (solver.getParticles().size() != (size_t)h) return 2;
    solver.addParticles(std::vector<V3>(pos.begin() + h, pos.end()), std::vector<V3>(vel.begin() + h, vel.end()),
                        std::vector<float>(m.begin() + h, m.end()), std::vector<float>(vol.begin() + h, vol.end()));
    for (int s = 0; s < steps; ++s) solver.step();
    if (solver.getStepCount() != (size_t)steps) return 3;
    const auto& P = solver.getParticles();
    std::vector<float> ox(3 * N), ov(3 * N);
    for (int p = 0; p < N; ++p) {
        const V3 a = P.getPosition(p), b = P.getVelocity(p);
        for (int k = 0; k < 3; ++k) {
            ox[3 * p + k] = a[k];
            ov[3 * p + k] = b[k];
        }
    }
    const auto& G = solver.getGrid();
    std::vector<float> gm(G.total_nodes), gv(3 * G.total_nodes), gp(3 * G.total_nodes);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const size_t n = G.getNodeIndex(i, j, k);
                gm[n] = G.mass[n];
                for (int a = 0; a < 3; ++a) {
                    gv[3 * n + a] = G.velocity[n][a];
                    gp[3 * n + a] = G.momentum[n][a];
                }
            }
    Writer w(out);
    w.floats(ox);
    w.floats(ov);
    w.floats(gm);
    w.floats(gv);
    w.floats(gp);
    std::printf("{\"ref_steps\": %zu, \"time\": %.6g}\n", solver.getStepCount(), (double)solver.getCurrentTime());
    return 0;
}

// in: N, nx, ny, nz, steps, checkpoint_interval, boundary, boundary_thickness,
//     dx, origin[3], dt, gravity[3], x[N][3], v[N][3], E[N], seed_x[N][3], seed_v[N][3]
// out: x[N][3], v[N][3] after the steps; dL/dx0[N][3], dL/dv0[N][3],
//      dL/dC0[N][9], dL/dF0[N][9]; then n_materials, (E, dL/dE) per material
int run_diff(const char* in, const char* out) {
    namespace D = physgrad::mpm::differentiable;
    Reader r(in);
    const int N = r.i32(), nx = r.i32(), ny = r.i32(), nz = r.i32(), steps = r.i32();
    D::DifferentiableMPMConfig<float> cfg;
    cfg.checkpoint_strategy = D::CheckpointStrategy::UNIFORM;
    cfg.checkpoint_interval = r.i32();
    cfg.boundary = r.i32();
    cfg.boundary_thickness = r.i32();
    const float dx = r.f32();
    V3 origin;
    for (int a = 0; a < 3; ++a) origin[a] = r.f32();
    const float dt = r.f32();
    V3 g;
    for (int a = 0; a < 3; ++a) g[a] = r.f32();
    const std::vector<float> x = r.floats(3 * N), v = r.floats(3 * N), E = r.floats(N), sx = r.floats(3 * N),
                             sv = r.floats(3 * N);
    D::DifferentiableMPMSystem<float> sys(cfg);
    bool threw = false;
    try {
        sys.simulationStep(dt, g);
    } catch (const std::runtime_error&) {
        threw = true;  // "System not initialized"
    }
    if (!threw) return 2;
    sys.initializeSystem(int3(nx, ny, nz), V3(dx, dx, dx), origin, (size_t)N);
    auto& P = sys.getParticles();
    for (int p = 0; p < N; ++p) {
        P.setPosition(p, V3(x[3 * p], x[3 * p + 1], x[3 * p + 2]));
        P.setVelocity(p, V3(v[3 * p], v[3 * p + 1], v[3 * p + 2]));
        P.young_modulus_chunks[p / 64][p % 64] = E[p];
    }
    threw = false;
    try {
        sys.computeGradients();
    } catch (const std::runtime_error&) {
        threw = true;  // "Gradient computation not enabled"
    }
    if (!threw) return 3;
    sys.enableGradientComputation(true);
    for (int s = 0; s < steps; ++s) sys.simulationStep(dt, g);
    if (sys.getGradientTapeSize() != (size_t)steps || sys.getCurrentStep() != (size_t)steps) return 4;
    const auto& Q = sys.getParticles();  // runs the recorded steps
    std::vector<float> ox(3 * N), ov(3 * N);
    for (int p = 0; p < N; ++p) {
        const V3 a = Q.getPosition(p), b = Q.getVelocity(p);
        for (int k = 0; k < 3; ++k) {
            ox[3 * p + k] = a[k];
            ov[3 * p + k] = b[k];
        }
    }
    auto& PG = sys.getParticleGradients();
    for (int p = 0; p < N; ++p) {
        PG.setPositionGradient(p, V3(sx[3 * p], sx[3 * p + 1], sx[3 * p + 2]));
        PG.setVelocityGradient(p, V3(sv[3 * p], sv[3 * p + 1], sv[3 * p + 2]));
    }
    sys.computeGradients();
    std::vector<float> gx(3 * N), gv(3 * N), gC(9 * N), gF(9 * N);
    for (int p = 0; p < N; ++p) {
        const V3 a = PG.getPositionGradient(p), b = PG.getVelocityGradient(p);
        for (int k = 0; k < 3; ++k) {
            gx[3 * p + k] = a[k];
            gv[3 * p + k] = b[k];
        }
        PG.getAffineGradient(p, &gC[9 * p]);
        PG.getDeformationGradientGradient(p, &gF[9 * p]);
    }
    Writer w(out);
    w.floats(ox);
    w.floats(ov);
    w.floats(gx);
    w.floats(gv);
    w.floats(gC);
    w.floats(gF);
    const auto& mats = sys.getMaterials();
    const auto& gE = sys.getYoungsModulusGradients();
    std::vector<float> tab;
    tab.push_back((float)mats.size());
    for (size_t i = 0; i < mats.size(); ++i) {
        tab.push_back(std::get<0>(mats[i]));
        tab.push_back(gE[i]);
    }
    w.floats(tab);
    // a changed step size inside a recording is refused
    threw = false;
    try {
        sys.simulationStep(dt * 2, g);
    } catch (const std::runtime_error&) {
        threw = true;
    }
    if (!threw) return 5;
    std::printf("{\"diff_steps\": %zu, \"materials\": %zu}\n", sys.getCurrentStep(), mats.size());
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s ref|diff <in> <out>\n", argv[0]);
        return 1;
    }
    try {
        const std::string mode = argv[1];
        if (mode == "ref") return run_ref(argv[2], argv[3]);
        if (mode == "diff") return run_diff(argv[2], argv[3]);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 10;
    }
    return 1;
}
