/*
 * ref_coupling_shim.cpp -- C entry point over the reference's SPH-MPM
 * coupling system (src/sph_mpm_coupling.h:413-579), compiled from its
 * unmodified headers into oracle/_ref/libref_coupling.so.  TEST
 * INFRASTRUCTURE ONLY.  It fills an SPHMPMCouplingSystem<float> with the
 * given SPH and MPM particles, runs findCouplingPairs() and
 * computeCouplingForces(), and returns what the reference computes: the
 * SPH particles' forces (which start at zero), the solid force of each pair
 * summed per MPM particle in pair order, the pair count and
 * getTotalCouplingEnergy().
 */
#include <cstdint>
#include <vector>

#include "sph_mpm_coupling.h"

using namespace physgrad;
using namespace physgrad::coupling::sph_mpm;

extern "C" int ref_sph_coupling(int64_t n_sph, const float* sph_x, const float* sph_v, int64_t n_mpm,
                                const float* mpm_x, const float* mpm_v, float stiffness, float damping,
                                float friction, float radius, int two_way, float* sph_force, float* mpm_force,
                                int64_t* n_pairs, float* energy) {
    try {
        CouplingConfig<float> cfg;
        cfg.coupling_stiffness = stiffness;
        cfg.coupling_damping = damping;
        cfg.friction_coefficient = friction;
        cfg.coupling_radius = radius;
        cfg.enable_two_way_coupling = two_way != 0;
        SPHMPMCouplingSystem<float> sys(cfg);
        sys.initializeSPHSystem((size_t)n_sph);
        sys.initializeMPMSystem(int3(4, 4, 4), ConceptVector3D<float>(1.f, 1.f, 1.f),
                                ConceptVector3D<float>(0.f, 0.f, 0.f), (size_t)n_mpm);
        auto& sp = sys.getSPHSystem().getParticles();
        for (int64_t i = 0; i < n_sph; ++i) {
            sp[i].position = ConceptVector3D<float>(sph_x[3 * i], sph_x[3 * i + 1], sph_x[3 * i + 2]);
            sp[i].velocity = ConceptVector3D<float>(sph_v[3 * i], sph_v[3 * i + 1], sph_v[3 * i + 2]);
            sp[i].force = ConceptVector3D<float>(0.f, 0.f, 0.f);
        }
        auto& mp = sys.getMPMParticles();
        for (int64_t i = 0; i < n_mpm; ++i) {
            mp.setPosition(i, ConceptVector3D<float>(mpm_x[3 * i], mpm_x[3 * i + 1], mpm_x[3 * i + 2]));
            mp.setVelocity(i, ConceptVector3D<float>(mpm_v[3 * i], mpm_v[3 * i + 1], mpm_v[3 * i + 2]));
        }
        sys.findCouplingPairs();
        sys.computeCouplingForces();
        for (int64_t i = 0; i < n_sph; ++i)
            for (int a = 0; a < 3; ++a) sph_force[3 * i + a] = sp[i].force[a];
        for (int64_t i = 0; i < 3 * n_mpm; ++i) mpm_force[i] = 0.f;
        for (const auto& f : sys.getCouplingForces())
            for (int a = 0; a < 3; ++a) mpm_force[3 * f.solid_particle_id + a] += f.solid_force[a];
        *n_pairs = (int64_t)sys.getNumCouplingPairs();
        *energy = sys.getTotalCouplingEnergy();
    } catch (...) {
        return -1;
    }
    return 0;
}
