/*
 * ref_mpm_shim.cpp -- C entry points over the reference's OWN CPU MPM code,
 * compiled from its unmodified headers (pedroscortes/physgrad src/) by
 * oracle/Makefile into oracle/_ref/libref_mpm.so.  TEST INFRASTRUCTURE ONLY:
 * used to pin the oracle's REF_COMPAT restatement and as the timed CPU
 * baseline ("reference" arm of bench.py).  No reference source is copied
 * into this repository; this file only calls the reference's public API:
 *
 *   physgrad::mpm::MPMSolver<float,64>   src/material_point_method.h:430-676
 *     ctor (:450-453), addParticles (:455-477), step (:479-500),
 *     getParticles/getGrid (:503-504)
 *   physgrad::mpm::differentiable::DifferentiableMPMSystem<float>
 *     src/differentiable_mpm.h:689-879 (initializeSystem :711, simulationStep
 *     :748, computeGradients :772, getParticleGradients :791)
 */
#include <cstdint>
#include <cstring>
#include <vector>

#include "material_point_method.h"

using namespace physgrad;

// Stateful handle for timing: one reference solver instance per handle.
extern "C" void* ref_mpm_create(int64_t n, const float* x, const float* v, const float* m, const float* vol, int nx,
                                int ny, int nz, float dx, float dt, float gx, float gy, float gz) {
    try {
        mpm::MPMSolver<float>::SimulationParams p;
        p.timestep = dt;
        p.gravity = ConceptVector3D<float>(gx, gy, gz);
        auto* s = new mpm::MPMSolver<float>(int3(nx, ny, nz), ConceptVector3D<float>(dx, dx, dx),
                                            ConceptVector3D<float>(0, 0, 0), p);
        std::vector<ConceptVector3D<float>> X(n), V(n);
        std::vector<float> M(m, m + n), VOL(vol, vol + n);
        for (int64_t i = 0; i < n; ++i) {
            X[i] = ConceptVector3D<float>(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
            V[i] = ConceptVector3D<float>(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
        }
        s->addParticles(X, V, M, VOL);
        return s;
    } catch (...) {
        return nullptr;
    }
}

extern "C" int ref_mpm_step(void* h, int steps) {
    if (!h) return -1;
    auto* s = static_cast<mpm::MPMSolver<float>*>(h);
    for (int k = 0; k < steps; ++k) s->step();
    return 0;
}

extern "C" void ref_mpm_destroy(void* h) { delete static_cast<mpm::MPMSolver<float>*>(h); }

extern "C" int ref_mpm_run(int64_t n, const float* x, const float* v, const float* m, const float* vol,
                           int nx, int ny, int nz, float dx, float ox, float oy, float oz, float dt,
                           float gx, float gy, float gz, int steps, float* x_out, float* v_out,
                           float* grid_mass, float* grid_vel) {
    try {
        mpm::MPMSolver<float>::SimulationParams p;
        p.timestep = dt;
        p.gravity = ConceptVector3D<float>(gx, gy, gz);
        mpm::MPMSolver<float> s(int3(nx, ny, nz), ConceptVector3D<float>(dx, dx, dx),
                                ConceptVector3D<float>(ox, oy, oz), p);
        std::vector<ConceptVector3D<float>> X(n), V(n);
        std::vector<float> M(m, m + n), VOL(vol, vol + n);
        for (int64_t i = 0; i < n; ++i) {
            X[i] = ConceptVector3D<float>(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
            V[i] = ConceptVector3D<float>(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
        }
        s.addParticles(X, V, M, VOL);
        for (int k = 0; k < steps; ++k) s.step();
        const auto& P = s.getParticles();
        for (int64_t i = 0; i < n; ++i) {
            auto q = P.getPosition(i);
            auto w = P.getVelocity(i);
            for (int a = 0; a < 3; ++a) {
                if (x_out) x_out[3 * i + a] = q[a];
                if (v_out) v_out[3 * i + a] = w[a];
            }
        }
        const auto& G = s.getGrid();
        size_t nodes = (size_t)nx * ny * nz;
        for (size_t i = 0; i < nodes; ++i) {
            if (grid_mass) grid_mass[i] = G.mass[i];
            if (grid_vel)
                for (int a = 0; a < 3; ++a) grid_vel[3 * i + a] = G.velocity[i][a];
        }
    } catch (...) {
        return -1;
    }
    return 0;
}
