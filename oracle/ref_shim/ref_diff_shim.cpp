/*
 * ref_diff_shim.cpp -- C entry point over the reference's differentiable MPM
 * system (src/differentiable_mpm.h:689-879), compiled from its unmodified
 * headers into oracle/_ref/libref_diff.so.  TEST INFRASTRUCTURE ONLY.  It
 * runs the reference's forward with gradient recording enabled, calls
 * computeGradients() and returns the particle velocity/position gradients
 * the reference produces, so the tests can record what the reference's MPM
 * adjoint returns on the same inputs.
 */
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "differentiable_mpm.h"

using namespace physgrad;
using namespace physgrad::mpm;

extern "C" int ref_diff_run(int64_t n, const float* x, const float* v, const float* m, int nx, int ny, int nz,
                            float dx, float dt, int steps, float* x_out, float* grad_v, float* grad_x) {
    try {
        differentiable::DifferentiableMPMSystem<float> sys;
        sys.initializeSystem(int3(nx, ny, nz), ConceptVector3D<float>(dx, dx, dx),
                             ConceptVector3D<float>(0, 0, 0), (size_t)n);
        auto& P = sys.getParticles();
        for (int64_t i = 0; i < n; ++i) {
            P.setPosition(i, ConceptVector3D<float>(x[3 * i], x[3 * i + 1], x[3 * i + 2]));
            P.setVelocity(i, ConceptVector3D<float>(v[3 * i], v[3 * i + 1], v[3 * i + 2]));
            P.setMass(i, m[i]);
        }
        sys.enableGradientComputation(true);
        for (int s = 0; s < steps; ++s) sys.simulationStep(dt);
        sys.computeGradients();
        auto& G = sys.getParticleGradients();
        for (int64_t i = 0; i < n; ++i) {
            auto q = P.getPosition(i);
            auto gv = G.getVelocityGradient(i);
            auto gx = G.getPositionGradient(i);
            for (int a = 0; a < 3; ++a) {
                x_out[3 * i + a] = q[a];
                grad_v[3 * i + a] = gv[a];
                grad_x[3 * i + a] = gx[a];
            }
        }
    } catch (...) {
        return -1;
    }
    return 0;
}
