// physgrad_b200/differentiable_mpm.h -- drop-in C++ replacement for physgrad's
// differentiable MPM header (src/differentiable_mpm.h:41-340, 689-879),
// implemented over the C-ABI of libpgmpm.so (include/pgmpm.h): the MLS-MPM
// step with a checkpointed reverse pass.  Header-only; link -lpgmpm.
//
// Same names and argument meaning as the reference:
//   physgrad::mpm::differentiable::{GradientMode, CheckpointStrategy,
//   DifferentiableMPMConfig, ParticleGradients, GridGradients,
//   DifferentiableMPMSystem::{initializeSystem, enableGradientComputation,
//   simulationStep, computeGradients, getParticles, getGrid,
//   getParticleGradients, getGridGradients, getCurrentTime, getCurrentStep,
//   getGradientTapeSize, getGradientMemoryUsage, resetSimulation}}, with
//   std::runtime_error("System not initialized") and
//   std::runtime_error("Gradient computation not enabled") where the
//   reference throws them.
//
// The gradients.  The reference's tape records an empty backward
// (src/differentiable_mpm.h:871-876), so its computeGradients() yields zeros.
// Here computeGradients() reads dL/d(state after the last recorded step) from
// getParticleGradients() -- position, velocity and (additions) deformation
// gradient and affine matrix C -- and replaces it with dL/d(state when the
// recording began), plus dL/dE per material (getYoungsModulusGradients()).
// A recording begins at enableGradientComputation(true) or
// resetSimulation(), and covers every simulationStep() after it.
//
// The physics.  Each particle's Young's modulus, Poisson ratio and density
// come from its chunks (ParticleAoSoA of physgrad_b200/material_point_method.h);
// particles with equal values share one material of the model in
// config.constitutive_model.  initializeSystem() starts every particle with
// F = I, volume (cell/2)^3, E = config.youngs_modulus, nu =
// config.poisson_ratio, density 1000 and mass density x volume; positions and
// velocities start at zero (set them through getParticles()).  Walls: the
// outermost config.boundary_thickness node layers, sticky by default (the
// reference zeroes the outermost layer, MPMGrid::applyBoundaryConditions).
//
// Differences, each checked where it arises:
//   * T must be float (FP32 device path): static_assert.
//   * cell_size equal on the three axes: std::invalid_argument.
//   * dt and gravity must not change within one recording (the reverse pass
//     replays the steps with one dt): std::runtime_error.
//   * Particles changed through getParticles() while a recording holds steps:
//     std::runtime_error (the recorded trajectory would no longer match).
//   * CheckpointStrategy NONE (or use_checkpointing false) keeps every step
//     on the tape; UNIFORM, ADAPTIVE and LOGARITHMIC store the state every
//     config.checkpoint_interval steps and replay the segments between.
//   * Mass and stress gradients and the grid gradients stay zero (the
//     reverse pass keeps the grid adjoints on the device).
#pragma once

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <tuple>

#include "material_point_method.h"

namespace physgrad {
namespace mpm {
namespace differentiable {

enum class GradientMode { FORWARD, REVERSE, HYBRID };
enum class CheckpointStrategy { NONE, UNIFORM, ADAPTIVE, LOGARITHMIC };

template <typename T>
struct DifferentiableMPMConfig {
    GradientMode gradient_mode = GradientMode::REVERSE;
    CheckpointStrategy checkpoint_strategy = CheckpointStrategy::ADAPTIVE;
    T finite_difference_eps = T{1e-6};
    bool enable_second_order = false;
    bool use_checkpointing = true;
    size_t max_checkpoints = 100;
    T memory_budget_gb = T{4.0};
    T gradient_clip_threshold = T{1e3};
    bool enable_gradient_accumulation = true;
    bool parallelize_gradient_computation = true;
    size_t gradient_block_size = 256;
    // additions of this implementation
    int checkpoint_interval = 16;  // steps between stored states
    int constitutive_model = PGMPM_MODEL_FIXED_COROTATED;
    T youngs_modulus = T{1e4};     // initial per-particle E (bulk modulus K for EOS_FLUID)
    T poisson_ratio = T{0.3};
    int boundary = PGMPM_BC_STICKY;
    int boundary_thickness = 1;
    int device = 0;
};

// Per-particle gradients in the reference's chunked layout (chunks of 64).
template <typename T>
class ParticleGradients {
public:
    using vector_type = ConceptVector3D<T>;
    static constexpr size_t chunk_size = 64;

    ParticleGradients() = default;

    void resize(size_t n) {
        num_particles_ = n;
        const size_t c = (n + chunk_size - 1) / chunk_size;
        position_gradients_.assign(c, {});
        velocity_gradients_.assign(c, {});
        mass_gradients_.assign(c, {});
        deformation_grad_gradients_.assign(c, {});
        affine_gradients_.assign(c, {});
        volume_gradients_.assign(c, {});
        stress_gradients_.assign(c, {});
    }
    size_t size() const { return num_particles_; }

    vector_type getPositionGradient(size_t p) const { return get3(position_gradients_, p); }
    void setPositionGradient(size_t p, const vector_type& g) { set3(position_gradients_, p, g); }
    vector_type getVelocityGradient(size_t p) const { return get3(velocity_gradients_, p); }
    void setVelocityGradient(size_t p, const vector_type& g) { set3(velocity_gradients_, p, g); }
    T getMassGradient(size_t p) const { return mass_gradients_[p / chunk_size][p % chunk_size]; }
    void setMassGradient(size_t p, T g) { mass_gradients_[p / chunk_size][p % chunk_size] = g; }
    void accumulatePositionGradient(size_t p, const vector_type& g) {
        set3(position_gradients_, p, get3(position_gradients_, p) + g);
    }
    void accumulateVelocityGradient(size_t p, const vector_type& g) {
        set3(velocity_gradients_, p, get3(velocity_gradients_, p) + g);
    }
    // additions: dL/dF and dL/dC, 9 entries row-major
    void getDeformationGradientGradient(size_t p, T* g) const { get9(deformation_grad_gradients_, p, g); }
    void setDeformationGradientGradient(size_t p, const T* g) { set9(deformation_grad_gradients_, p, g); }
    void getAffineGradient(size_t p, T* g) const { get9(affine_gradients_, p, g); }
    void setAffineGradient(size_t p, const T* g) { set9(affine_gradients_, p, g); }

    void zero() { resize(num_particles_); }
    size_t getMemoryUsageBytes() const {
        const size_t c = position_gradients_.size();
        return c * sizeof(T) * chunk_size * (3 + 3 + 1 + 9 + 9 + 1 + 6);
    }

    // flat copies (particle order) used at the C-ABI boundary
    void gather(std::vector<float>& x, std::vector<float>& v, std::vector<float>& C, std::vector<float>& F) const {
        const size_t n = num_particles_;
        x.resize(3 * n);
        v.resize(3 * n);
        C.resize(9 * n);
        F.resize(9 * n);
        for (size_t p = 0; p < n; ++p) {
            const vector_type a = getPositionGradient(p), b = getVelocityGradient(p);
            for (int k = 0; k < 3; ++k) {
                x[3 * p + k] = a[k];
                v[3 * p + k] = b[k];
            }
            getAffineGradient(p, &C[9 * p]);
            getDeformationGradientGradient(p, &F[9 * p]);
        }
    }
    void scatter(const float* x, const float* v, const float* C, const float* F) {
        for (size_t p = 0; p < num_particles_; ++p) {
            setPositionGradient(p, {x[3 * p], x[3 * p + 1], x[3 * p + 2]});
            setVelocityGradient(p, {v[3 * p], v[3 * p + 1], v[3 * p + 2]});
            setAffineGradient(p, C + 9 * p);
            setDeformationGradientGradient(p, F + 9 * p);
        }
    }

private:
    size_t num_particles_ = 0;
    std::vector<std::array<T, chunk_size * 3>> position_gradients_, velocity_gradients_;
    std::vector<std::array<T, chunk_size>> mass_gradients_, volume_gradients_;
    std::vector<std::array<T, chunk_size * 9>> deformation_grad_gradients_, affine_gradients_;
    std::vector<std::array<T, chunk_size * 6>> stress_gradients_;

    template <class Ch>
    static vector_type get3(const Ch& ch, size_t p) {
        const auto& c = ch[p / chunk_size];
        const size_t l = p % chunk_size;
        return {c[l], c[l + chunk_size], c[l + 2 * chunk_size]};
    }
    template <class Ch>
    static void set3(Ch& ch, size_t p, const vector_type& g) {
        auto& c = ch[p / chunk_size];
        const size_t l = p % chunk_size;
        c[l] = g[0];
        c[l + chunk_size] = g[1];
        c[l + 2 * chunk_size] = g[2];
    }
    template <class Ch>
    static void get9(const Ch& ch, size_t p, T* g) {
        for (int i = 0; i < 9; ++i) g[i] = ch[p / chunk_size][p % chunk_size + i * chunk_size];
    }
    template <class Ch>
    static void set9(Ch& ch, size_t p, const T* g) {
        for (int i = 0; i < 9; ++i) ch[p / chunk_size][p % chunk_size + i * chunk_size] = g[i];
    }
};

// Per-node gradients (src/differentiable_mpm.h:262-340).  The reverse pass
// keeps the grid adjoints on the device, so these stay zero.
template <typename T>
class GridGradients {
public:
    using vector_type = ConceptVector3D<T>;
    explicit GridGradients(const int3& dims) : grid_dims_(dims) {
        resize(dims.x > 0 && dims.y > 0 && dims.z > 0 ? (size_t)dims.x * dims.y * dims.z : 0);
    }
    void resize(size_t n) {
        velocity_gradients_.assign(n, vector_type{});
        momentum_gradients_.assign(n, vector_type{});
    }
    vector_type getVelocityGradient(size_t i) const { return velocity_gradients_[i]; }
    void setVelocityGradient(size_t i, const vector_type& g) { velocity_gradients_[i] = g; }
    vector_type getMomentumGradient(size_t i) const { return momentum_gradients_[i]; }
    void setMomentumGradient(size_t i, const vector_type& g) { momentum_gradients_[i] = g; }
    void accumulateVelocityGradient(size_t i, const vector_type& g) { velocity_gradients_[i] = velocity_gradients_[i] + g; }
    void accumulateMomentumGradient(size_t i, const vector_type& g) { momentum_gradients_[i] = momentum_gradients_[i] + g; }
    void zero() { resize(velocity_gradients_.size()); }
    size_t getMemoryUsageBytes() const { return 2 * velocity_gradients_.size() * sizeof(vector_type); }

private:
    int3 grid_dims_;
    std::vector<vector_type> velocity_gradients_, momentum_gradients_;
};

template <typename T>
class DifferentiableMPMSystem {
    static_assert(std::is_same<T, float>::value, "the B200 path computes in FP32: use DifferentiableMPMSystem<float>");

public:
    using Particles = ParticleAoSoA<T, 64>;

    explicit DifferentiableMPMSystem(const DifferentiableMPMConfig<T>& config = DifferentiableMPMConfig<T>{})
        : config_(config) {}
    ~DifferentiableMPMSystem() { release(); }
    DifferentiableMPMSystem(const DifferentiableMPMSystem&) = delete;
    DifferentiableMPMSystem& operator=(const DifferentiableMPMSystem&) = delete;

    void initializeSystem(const int3& grid_dims, const ConceptVector3D<T>& cell_size,
                          const ConceptVector3D<T>& origin, size_t num_particles) {
        if (!(cell_size[0] == cell_size[1] && cell_size[1] == cell_size[2]))
            throw std::invalid_argument("initializeSystem: cell_size must be the same on the three axes");
        release();
        grid_.reset(new MPMGrid<T>(grid_dims, cell_size, origin));
        particles_.reset(new Particles());
        particles_->resize(num_particles);
        const T I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        const T vol = (cell_size[0] / 2) * (cell_size[0] / 2) * (cell_size[0] / 2);
        for (size_t p = 0; p < num_particles; ++p) {
            particles_->setDeformationGradient(p, I);
            particles_->volume_chunks[p / 64][p % 64] = vol;
            particles_->young_modulus_chunks[p / 64][p % 64] = config_.youngs_modulus;
            particles_->poisson_ratio_chunks[p / 64][p % 64] = config_.poisson_ratio;
            particles_->density_chunks[p / 64][p % 64] = T{1000};
            particles_->setMass(p, T{1000} * vol);
        }
        particle_gradients_.reset(new ParticleGradients<T>());
        particle_gradients_->resize(num_particles);
        grid_gradients_.reset(new GridGradients<T>(grid_dims));
        current_time_ = T{0};
        current_step_ = 0;
        rec_steps_ = rec_done_ = 0;
        device_stale_ = true;
    }

    void enableGradientComputation(bool enable = true) {
        if (enable == recording_) return;
        if (!enable) materialize();
        recording_ = enable;
        rec_steps_ = rec_done_ = 0;
    }

    // src/differentiable_mpm.h:748-766
    void simulationStep(T dt, const ConceptVector3D<T>& gravity = {T{0}, T{-9.81}, T{0}}) {
        if (!particles_ || !grid_) throw std::runtime_error("System not initialized");
        push();
        if (recording_ && rec_steps_ > 0 &&
            (dt != rec_dt_ || gravity[0] != rec_g_[0] || gravity[1] != rec_g_[1] || gravity[2] != rec_g_[2]))
            throw std::runtime_error("simulationStep: dt and gravity must stay fixed while gradients are recorded");
        if (dt != dev_dt_ || gravity[0] != dev_g_[0] || gravity[1] != dev_g_[1] || gravity[2] != dev_g_[2]) {
            const float g[3] = {gravity[0], gravity[1], gravity[2]};
            b200_detail::check(pgmpm_set_scene_params(h_, 0, dt, g));
            dev_dt_ = dt;
            dev_g_ = gravity;
        }
        if (recording_) {
            // the steps run when their result is needed (materialize)
            if (rec_steps_ == 0) {
                rec_dt_ = dt;
                rec_g_ = gravity;
            }
            ++rec_steps_;
        } else {
            b200_detail::check(pgmpm_step(h_, 1, nullptr));
            host_stale_ = grid_stale_ = true;
        }
        current_time_ += dt;
        ++current_step_;
    }

    // dL/d(final state) in getParticleGradients() -> dL/d(state when the
    // recording began); dL/dE per material in getYoungsModulusGradients()
    void computeGradients() {
        if (!recording_) throw std::runtime_error("Gradient computation not enabled");
        if (!particles_) throw std::runtime_error("System not initialized");
        materialize();
        grid_gradients_->zero();
        const size_t n = particles_->size();
        std::vector<float> gx, gv, gC, gF;
        particle_gradients_->gather(gx, gv, gC, gF);
        const size_t M = materials_.size();
        gE_.assign(M, 0.f);
        if (rec_steps_ > 0) {
            std::vector<float> ox(3 * n), ov(3 * n), oC(9 * n), oF(9 * n);
            b200_detail::check(pgmpm_backward(h_, gx.data(), gv.data(), gC.data(), gF.data(), ox.data(), ov.data(),
                                              oC.data(), oF.data(), gE_.data(), PGMPM_PTR_HOST, nullptr));
            particle_gradients_->zero();
            particle_gradients_->scatter(ox.data(), ov.data(), oC.data(), oF.data());
        }
    }

    Particles& getParticles() {
        sync();
        return *particles_;
    }
    const Particles& getParticles() const {
        const_cast<DifferentiableMPMSystem*>(this)->sync();
        return *particles_;
    }
    MPMGrid<T>& getGrid() {
        sync_grid();
        return *grid_;
    }
    const MPMGrid<T>& getGrid() const {
        const_cast<DifferentiableMPMSystem*>(this)->sync_grid();
        return *grid_;
    }
    ParticleGradients<T>& getParticleGradients() { return *particle_gradients_; }
    const ParticleGradients<T>& getParticleGradients() const { return *particle_gradients_; }
    GridGradients<T>& getGridGradients() { return *grid_gradients_; }
    const GridGradients<T>& getGridGradients() const { return *grid_gradients_; }

    T getCurrentTime() const { return current_time_; }
    size_t getCurrentStep() const { return current_step_; }
    size_t getGradientTapeSize() const { return recording_ ? (size_t)rec_steps_ : 0; }
    size_t getGradientMemoryUsage() const {
        // device checkpoints (6 float4 planes + key per particle) and the
        // per-step tape of one segment (~108 B per particle), plus the host
        // gradient arrays
        const size_t n = particles_ ? particles_->size() : 0;
        const size_t k = (size_t)std::max(1, interval());
        const size_t ck = rec_steps_ > 0 ? ((size_t)rec_steps_ + k - 1) / k : 0;
        const size_t dev = rec_steps_ > 0 ? n * (ck * 100 + std::min<size_t>(k, rec_steps_) * 108) : 0;
        return dev + (particle_gradients_ ? particle_gradients_->getMemoryUsageBytes() : 0) +
               (grid_gradients_ ? grid_gradients_->getMemoryUsageBytes() : 0);
    }

    // time and step count to zero; a recording restarts from the current state
    void resetSimulation() {
        materialize();
        current_time_ = T{0};
        current_step_ = 0;
        rec_steps_ = rec_done_ = 0;
        if (particle_gradients_) particle_gradients_->zero();
        if (grid_gradients_) grid_gradients_->zero();
    }

    // additions: the material table built from the particles' (E, nu,
    // density) and dL/dE of each entry after computeGradients()
    const std::vector<std::tuple<T, T, T>>& getMaterials() const { return materials_; }
    const std::vector<float>& getYoungsModulusGradients() const { return gE_; }

private:
    DifferentiableMPMConfig<T> config_;
    std::unique_ptr<Particles> particles_;
    std::unique_ptr<MPMGrid<T>> grid_;
    std::unique_ptr<ParticleGradients<T>> particle_gradients_;
    std::unique_ptr<GridGradients<T>> grid_gradients_;
    T current_time_ = T{0};
    size_t current_step_ = 0;

    pgmpm_solver h_ = nullptr;
    int64_t dev_count_ = -1;
    bool device_stale_ = true;  // host particles newer than the device
    bool host_stale_ = false;   // device state newer than the host copy
    bool grid_stale_ = false;
    T dev_dt_ = T{-1};
    ConceptVector3D<T> dev_g_{};
    std::vector<std::tuple<T, T, T>> materials_;
    std::vector<float> gE_;
    // the host state last exchanged with the device (to detect edits)
    std::vector<float> sx_, sv_, sF_, sm_, sV_, sE_, snu_, srho_;
    std::vector<int32_t> smat_;  // material id of each particle in the last upload

    bool recording_ = false;
    int rec_steps_ = 0;  // steps recorded
    int rec_done_ = 0;   // of them, run on the device by pgmpm_forward_checkpointed
    T rec_dt_ = T{0};
    ConceptVector3D<T> rec_g_{};
    std::vector<float> start_x_, start_v_, start_C_, start_F_;  // state when the recording began

    int interval() const {
        if (config_.checkpoint_strategy == CheckpointStrategy::NONE || !config_.use_checkpointing)
            return std::max(1, rec_steps_);
        return std::max(1, config_.checkpoint_interval);
    }

    void release() {
        if (h_) pgmpm_destroy(h_);
        h_ = nullptr;
        dev_count_ = -1;
        dev_dt_ = T{-1};
    }

    void snapshot(std::vector<float>& E, std::vector<float>& nu, std::vector<float>& rho) const {
        const size_t n = particles_->size();
        E.resize(n);
        nu.resize(n);
        rho.resize(n);
        for (size_t p = 0; p < n; ++p) {
            E[p] = particles_->young_modulus_chunks[p / 64][p % 64];
            nu[p] = particles_->poisson_ratio_chunks[p / 64][p % 64];
            rho[p] = particles_->density_chunks[p / 64][p % 64];
        }
    }

    // host -> device when the host particles differ from what the device has
    void push() {
        std::vector<float> x, v, F, m, V0, E, nu, rho;
        particles_->gatherFlat(x, v, F, m, V0);
        snapshot(E, nu, rho);
        if (!device_stale_ && x == sx_ && v == sv_ && F == sF_ && m == sm_ && V0 == sV_ && E == sE_ && nu == snu_ &&
            rho == srho_)
            return;
        if (recording_ && rec_steps_ > 0)
            throw std::runtime_error("particles changed while gradients are recorded");
        const int64_t n = (int64_t)particles_->size();
        // material table: one entry per distinct (E, nu, density)
        std::map<std::tuple<float, float, float>, int32_t> ids;
        std::vector<int32_t> mat(n);
        std::vector<std::tuple<T, T, T>> table;
        for (int64_t p = 0; p < n; ++p) {
            const auto key = std::make_tuple(E[p], nu[p], rho[p]);
            auto it = ids.find(key);
            if (it == ids.end()) {
                it = ids.emplace(key, (int32_t)table.size()).first;
                table.push_back(key);
            }
            mat[p] = it->second;
        }
        if (table.empty()) table.emplace_back(config_.youngs_modulus, config_.poisson_ratio, T{1000});
        std::vector<pgmpm_material> pm(table.size());
        for (size_t i = 0; i < table.size(); ++i) {
            pgmpm_material& q = pm[i];
            std::memset(&q, 0, sizeof(q));
            q.model = config_.constitutive_model;
            q.type = q.model == PGMPM_MODEL_EOS_FLUID ? PGMPM_MAT_FLUID : PGMPM_MAT_ELASTIC;
            q.youngs_modulus = std::get<0>(table[i]);
            q.poisson_ratio = std::get<1>(table[i]);
            q.density = std::get<2>(table[i]);
        }
        if (h_ && (dev_count_ != n || table.size() != materials_.size())) release();
        if (!h_) {
            pgmpm_scene_desc d{};
            d.n[0] = grid_->dimensions.x;
            d.n[1] = grid_->dimensions.y;
            d.n[2] = grid_->dimensions.z;
            for (int a = 0; a < 3; ++a) d.origin[a] = grid_->origin[a];
            d.gravity[1] = T{-9.81};
            d.dx = grid_->cell_size[0];
            d.dt = T{1e-4};
            d.physics = PGMPM_PHYSICS_MLS;
            d.boundary = config_.boundary;
            d.boundary_thickness = config_.boundary_thickness;
            b200_detail::check(pgmpm_create(&d, 1, &n, pm.data(), (int32_t)pm.size(), config_.device, &h_));
            dev_count_ = n;
            dev_dt_ = d.dt;
            dev_g_ = {d.gravity[0], d.gravity[1], d.gravity[2]};
        } else {
            b200_detail::check(pgmpm_set_materials(h_, pm.data(), (int32_t)pm.size()));
        }
        materials_ = table;
        b200_detail::check(pgmpm_upload(h_, x.data(), v.data(), nullptr, F.data(), m.data(), V0.data(), mat.data(),
                                        PGMPM_PTR_HOST, nullptr));
        smat_ = std::move(mat);
        sx_ = std::move(x);
        sv_ = std::move(v);
        sF_ = std::move(F);
        sm_ = std::move(m);
        sV_ = std::move(V0);
        sE_ = std::move(E);
        snu_ = std::move(nu);
        srho_ = std::move(rho);
        device_stale_ = false;
        host_stale_ = false;
        grid_stale_ = false;
    }

    // run the recorded steps that have not run yet: the whole recording from
    // its start state, so that one pgmpm_forward_checkpointed covers it
    void materialize() {
        if (!recording_ || rec_done_ == rec_steps_ || !h_) return;
        const size_t n = particles_->size();
        if (rec_done_ == 0) {
            start_x_.resize(3 * n);
            start_v_.resize(3 * n);
            start_C_.resize(9 * n);
            start_F_.resize(9 * n);
            b200_detail::check(pgmpm_download(h_, start_x_.data(), start_v_.data(), start_C_.data(), start_F_.data(),
                                              PGMPM_PTR_HOST, nullptr));
        } else {
            b200_detail::check(pgmpm_upload(h_, start_x_.data(), start_v_.data(), start_C_.data(), start_F_.data(),
                                            sm_.data(), sV_.data(), smat_.data(), PGMPM_PTR_HOST, nullptr));
        }
        b200_detail::check(pgmpm_forward_checkpointed(h_, rec_steps_, std::min(interval(), rec_steps_), nullptr));
        rec_done_ = rec_steps_;
        host_stale_ = grid_stale_ = true;
    }

    void sync() {
        if (!particles_) throw std::runtime_error("System not initialized");
        materialize();
        if (!host_stale_ || !h_) return;
        const size_t n = particles_->size();
        std::vector<float> x(3 * n), v(3 * n), F(9 * n);
        b200_detail::check(pgmpm_download(h_, x.data(), v.data(), nullptr, F.data(), PGMPM_PTR_HOST, nullptr));
        particles_->scatterFlat(x.data(), v.data(), F.data());
        sx_ = std::move(x);
        sv_ = std::move(v);
        sF_ = std::move(F);
        host_stale_ = false;
    }

    void sync_grid() {
        if (!grid_) throw std::runtime_error("System not initialized");
        materialize();
        if (!grid_stale_ || !h_) return;
        const size_t nodes = grid_->total_nodes;
        std::vector<float> m(nodes), v(3 * nodes);
        b200_detail::check(pgmpm_download_grid(h_, 0, m.data(), v.data(), PGMPM_PTR_HOST, nullptr));
        for (size_t i = 0; i < nodes; ++i) {
            grid_->mass[i] = m[i];
            grid_->velocity[i] = {v[3 * i], v[3 * i + 1], v[3 * i + 2]};
            grid_->momentum[i] = grid_->velocity[i] * m[i];
            grid_->force[i] = ConceptVector3D<T>{};
        }
        grid_stale_ = false;
    }
};

}  // namespace differentiable
}  // namespace mpm
}  // namespace physgrad
