/*
 * ref_fsi_shim.cpp -- C entry point over the reference's FSI simulation
 * manager (src/fsi_coupling.h:780-858), compiled from its unmodified headers
 * into oracle/_ref/libref_fsi.so.  TEST INFRASTRUCTURE ONLY.  It runs
 * FSISimulationManager::simulate for one time step with a coupling method
 * that leaves the particles as they are, so that the one entry of
 * getEnergyHistory() is the manager's computeTotalEnergy (the kinetic
 * energy of the fluid and the solid particle sets) of the given particles.
 */
#include <cstdint>
#include <memory>
#include <string>
#include <unordered_map>

#include "fsi_coupling.h"

using namespace physgrad;

namespace {
// A coupling step that changes nothing: simulate() then only measures.
class NoCoupling : public fsi::FSICouplingMethod<float> {
public:
    void couple(ParticleSet&, ParticleSet&, float, float) override {}
    ForceVector computeFluidForces(const ParticleSet&, const ParticleSet&) override { return {}; }
    ForceVector computeSolidForces(const ParticleSet&, const ParticleSet&) override { return {}; }
    void enforceNoSlipBoundary(ParticleSet&, const ParticleSet&) override {}
    void enforceContinuityConstraint(ParticleSet&, ParticleSet&) override {}
    void setParameters(const std::unordered_map<std::string, float>&) override {}
    std::unordered_map<std::string, float> getParameters() const override { return {}; }
};

void fill(mpm::ParticleAoSoA<float>& p, int64_t n, const float* v, const float* m) {
    p.resize((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        p.setVelocity(i, v[3 * i], v[3 * i + 1], v[3 * i + 2]);
        p.setMass(i, m[i]);
    }
}
}  // namespace

extern "C" int ref_fsi_energy(int64_t n_fluid, const float* v_fluid, const float* m_fluid, int64_t n_solid,
                              const float* v_solid, const float* m_solid, float* energy) {
    try {
        mpm::ParticleAoSoA<float> fluid, solid;
        fill(fluid, n_fluid, v_fluid, m_fluid);
        fill(solid, n_solid, v_solid, m_solid);
        fsi::FSISimulationManager<float> mgr(std::make_unique<NoCoupling>(), 1.0f, 1.0f);
        mgr.simulate(fluid, solid);
        if (mgr.getEnergyHistory().empty()) return -2;
        *energy = mgr.getEnergyHistory()[0];
    } catch (...) {
        return -1;
    }
    return 0;
}
