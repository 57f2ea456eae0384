// physgrad_b200/mpm_solver.h -- drop-in C++ replacement for physgrad's GPU
// MPM solver header (src/mpm_solver.h:29-329 with the types of
// src/mpm_data_structures.h:54-96, 106-359, 617-627), implemented over the
// C-ABI of libpgmpm.so (include/pgmpm.h).  Header-only; link -lpgmpm.
//
// Same names, argument meaning and error behaviour as the reference:
//   MPMSolverConfig, MPMPerformanceMetrics, MaterialType, MaterialParameters,
//   createElasticMaterial, createFluidMaterial, ParticleAoSoA accessors,
//   MPMSolver<T>::{initialize, addParticles, step, run, getParticles, getGrid,
//   getMetrics, getCurrentTime, getCurrentStep}; std::runtime_error on the
//   reference's error paths ("Exceeded maximum particle count",
//   "Solver not initialized").  Physics: PGMPM_PHYSICS_MLS by default (set
//   config.physics = PGMPM_PHYSICS_REF_COMPAT for the reference CPU path).
//   Like the reference header it cannot share a translation unit with
//   material_point_method.h (both define physgrad::mpm::MPMSolver).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <filesystem>
#include <stdexcept>
#include <string>
#include <vector>

#include "../pgmpm.h"

namespace physgrad_b200_detail {
inline void check(int rc) {
    if (rc != PGMPM_OK) throw std::runtime_error(std::string("pgmpm: ") + pgmpm_last_error());
}
}  // namespace physgrad_b200_detail

template <typename T>
struct vec3 {
    T x, y, z;
    vec3() = default;
    vec3(T x_, T y_, T z_) : x(x_), y(y_), z(z_) {}
};
using T3 = vec3<float>;

namespace physgrad::mpm {

enum class MaterialType : uint32_t { ELASTIC = 0, ELASTOPLASTIC = 1, FLUID = 2, SAND = 3, SNOW = 4, JELLY = 5 };

enum class ConstitutiveModel : int32_t { FIXED_COROTATED = 0, NEO_HOOKEAN = 1, EOS_FLUID = 2 };

enum class BoundaryType : uint32_t {
    FREE = 0, DIRICHLET_X = 1, DIRICHLET_Y = 2, DIRICHLET_Z = 4, NEUMANN_X = 8, NEUMANN_Y = 16, NEUMANN_Z = 32,
    STICKY = 64, SLIP = 128
};

struct MaterialParameters {
    float density = 1000.0f;
    float youngs_modulus = 1e6f;  // bulk modulus for FLUID
    float poisson_ratio = 0.3f;
    float yield_stress = 1e5f;
    float hardening_coefficient = 0.0f;
    float viscosity = 0.001f;
    float friction_angle = 30.0f;
    float cohesion = 1000.0f;
    float critical_compression = 2.5e-2f;
    float critical_stretch = 7.5e-3f;
    MaterialType type = MaterialType::ELASTIC;
    ConstitutiveModel model = ConstitutiveModel::FIXED_COROTATED;
};

template <typename T>
MaterialParameters createElasticMaterial(T density, T youngs_modulus, T poisson_ratio) {
    MaterialParameters p;
    p.density = (float)density;
    p.youngs_modulus = (float)youngs_modulus;
    p.poisson_ratio = (float)poisson_ratio;
    p.type = MaterialType::ELASTIC;
    return p;
}

template <typename T>
MaterialParameters createFluidMaterial(T density, T viscosity, T gamma = 7.0f) {
    MaterialParameters p;
    p.density = (float)density;
    p.viscosity = (float)viscosity;
    p.youngs_modulus = (float)gamma;  // bulk modulus, as the reference stores it
    p.type = MaterialType::FLUID;
    p.model = ConstitutiveModel::EOS_FLUID;
    return p;
}

struct int3_ {
    int x, y, z;
};

struct MPMSolverConfig {
    int3_ grid_dimensions = {64, 64, 64};
    T3 grid_spacing = {0.01f, 0.01f, 0.01f};
    T3 domain_origin = {0.0f, 0.0f, 0.0f};
    float time_step = 1e-4f;
    float simulation_time = 1.0f;
    float cfl_factor = 0.4f;
    int max_particles = 1000000;
    float particle_radius = 0.005f;
    bool enable_gravity = true;
    T3 gravity = {0.0f, -9.81f, 0.0f};
    bool enable_multi_material = true;
    int max_materials = 8;
    int cuda_block_size = 256;
    bool enable_g2p2g_fusion = true;
    // Accepted as in src/mpm_solver.h:53-55.  The reference's adaptive step
    // (computeAdaptiveTimestep, :467-470) returns time_step unchanged and
    // never reads the bounds; so does this implementation.
    bool enable_adaptive_timestep = false;
    float min_timestep = 1e-6f;
    float max_timestep = 1e-3f;
    // output (src/mpm_solver.h:57-60): run() writes the particles every
    // output_frequency seconds of simulated time as
    // output_directory/frame_NNNNN.vtk (legacy binary VTK).  Off by default
    // here: the reference's outputData() only prints a line.
    bool enable_output = false;
    float output_frequency = 0.01f;
    std::string output_directory = "./mpm_output";
    // debug and profiling (src/mpm_solver.h:62-65).  enable_profiling times
    // each kernel group with events (getMetrics' p2g/g2p/grid times);
    // enable_debug_output and verify_conservation are accepted and, as in
    // the reference, not read.
    bool enable_profiling = false;
    bool enable_debug_output = false;
    bool verify_conservation = false;
    // additions of this implementation
    int physics = PGMPM_PHYSICS_MLS;
    int boundary = PGMPM_BC_STICKY;
    int boundary_thickness = 3;
    int device = 0;
    std::vector<MaterialParameters> materials = {createElasticMaterial(1000.0f, 1e4f, 0.3f)};
};

struct MPMPerformanceMetrics {
    double total_simulation_time = 0.0;
    double average_step_time = 0.0;
    double g2p_time = 0.0;
    double p2g_time = 0.0;
    double grid_update_time = 0.0;
    double particle_update_time = 0.0;
    size_t total_memory_usage = 0;
    size_t particle_memory = 0;
    size_t grid_memory = 0;
    int total_steps = 0;
    int rejected_steps = 0;
    float average_particles_per_second = 0.0f;
    void reset() { *this = MPMPerformanceMetrics{}; }
    // a summary on stdout (src/mpm_solver.h:92-100 has one of the same name)
    void print() const {
        const double t = total_simulation_time > 0.0 ? total_simulation_time : 1.0;
        std::printf("MPM metrics: %d steps in %.6f s (%.4f ms per step), %.3f M particle-steps/s, %zu MB on the "
                    "device; P2G %.1f%%, grid %.1f%%, G2P %.1f%%\n",
                    total_steps, total_simulation_time, average_step_time * 1e3,
                    average_particles_per_second / 1e6, total_memory_usage >> 20, 100.0 * p2g_time / t,
                    100.0 * grid_update_time / t, 100.0 * g2p_time / t);
    }
};

// Host copy of the particle state with the accessors of the reference's
// chunked container (src/mpm_data_structures.h:106-359).  Arrays are sized
// to whole chunks, so get*Data() returns the same layout as the reference's
// chunk arrays: per particle x, y, z (positions, velocities), one value
// (mass, volume), F row-major (9), stress xx, yy, zz, xy, xz, yz (6).
// MPMSolver::getParticles() fills positions, velocities, masses, volumes,
// F, the APIC matrix C (getAffineMatrix) and material types; the stress is
// not a state of the MLS step and stays as set.
template <typename T = float, size_t ChunkSize = 256>
class ParticleAoSoA {
public:
    static constexpr size_t chunk_size = ChunkSize;
    using scalar_type = T;

    ParticleAoSoA() = default;
    explicit ParticleAoSoA(size_t num_particles) { resize(num_particles); }

    void resize(size_t num_particles) {
        n_ = num_particles;
        chunks_ = (num_particles + chunk_size - 1) / chunk_size;
        const size_t cap = chunks_ * chunk_size;
        x_.resize(3 * cap);
        v_.resize(3 * cap);
        m_.resize(cap);
        V_.resize(cap);
        F_.resize(9 * cap);
        C_.resize(9 * cap);
        stress_.resize(6 * cap);
        type_.resize(cap, MaterialType::ELASTIC);
        active_.resize(cap, 1u);
    }
    size_t size() const { return n_; }
    size_t num_chunks() const { return chunks_; }

    void setPosition(size_t i, T x, T y, T z) { x_[3 * i] = x; x_[3 * i + 1] = y; x_[3 * i + 2] = z; }
    void getPosition(size_t i, T& x, T& y, T& z) const { x = x_[3 * i]; y = x_[3 * i + 1]; z = x_[3 * i + 2]; }
    void setVelocity(size_t i, T x, T y, T z) { v_[3 * i] = x; v_[3 * i + 1] = y; v_[3 * i + 2] = z; }
    void getVelocity(size_t i, T& x, T& y, T& z) const { x = v_[3 * i]; y = v_[3 * i + 1]; z = v_[3 * i + 2]; }
    void setMass(size_t i, T m) { m_[i] = m; }
    T getMass(size_t i) const { return m_[i]; }
    void setVolume(size_t i, T v) { V_[i] = v; }
    T getVolume(size_t i) const { return V_[i]; }
    void setDeformationGradient(size_t i, const T F[9]) {
        for (int k = 0; k < 9; ++k) F_[9 * i + k] = F[k];
    }
    void getDeformationGradient(size_t i, T F[9]) const {
        for (int k = 0; k < 9; ++k) F[k] = F_[9 * i + k];
    }
    void getAffineMatrix(size_t i, T C[9]) const {
        for (int k = 0; k < 9; ++k) C[k] = C_[9 * i + k];
    }
    void setStress(size_t i, const T s[6]) {
        for (int k = 0; k < 6; ++k) stress_[6 * i + k] = s[k];
    }
    void getStress(size_t i, T s[6]) const {
        for (int k = 0; k < 6; ++k) s[k] = stress_[6 * i + k];
    }
    void setMaterialType(size_t i, MaterialType t) { type_[i] = t; }
    MaterialType getMaterialType(size_t i) const { return type_[i]; }
    void setActive(size_t i, bool a) { active_[i] = a ? 1u : 0u; }
    bool isActive(size_t i) const { return active_[i] != 0u; }

    // bulk operations (src/mpm_data_structures.h:274-322)
    void setPositions(const std::vector<std::array<T, 3>>& p) {
        for (size_t i = 0; i < std::min(p.size(), size()); ++i) setPosition(i, p[i][0], p[i][1], p[i][2]);
    }
    void setVelocities(const std::vector<std::array<T, 3>>& p) {
        for (size_t i = 0; i < std::min(p.size(), size()); ++i) setVelocity(i, p[i][0], p[i][1], p[i][2]);
    }
    void setMasses(const std::vector<T>& m) {
        for (size_t i = 0; i < std::min(m.size(), size()); ++i) setMass(i, m[i]);
    }
    std::vector<std::array<T, 3>> getPositions() const { return triples(x_); }
    std::vector<std::array<T, 3>> getVelocities() const { return triples(v_); }
    std::vector<T> getMasses() const { return std::vector<T>(m_.begin(), m_.begin() + (ptrdiff_t)n_); }

    // raw arrays (src/mpm_data_structures.h:325-342)
    T* getPositionData() { return x_.data(); }
    T* getVelocityData() { return v_.data(); }
    T* getMassData() { return m_.data(); }
    T* getVolumeData() { return V_.data(); }
    T* getDeformationGradientData() { return F_.data(); }
    T* getStressData() { return stress_.data(); }
    MaterialType* getMaterialTypeData() { return type_.data(); }
    uint32_t* getActiveData() { return active_.data(); }
    const T* getPositionData() const { return x_.data(); }
    const T* getVelocityData() const { return v_.data(); }
    const T* getMassData() const { return m_.data(); }
    const T* getVolumeData() const { return V_.data(); }
    const T* getDeformationGradientData() const { return F_.data(); }
    const T* getStressData() const { return stress_.data(); }
    const MaterialType* getMaterialTypeData() const { return type_.data(); }
    const uint32_t* getActiveData() const { return active_.data(); }
    size_t getMemoryFootprint() const {
        return chunks_ * chunk_size * (sizeof(T) * (3 + 3 + 1 + 1 + 9 + 6 + 9) + sizeof(MaterialType) + 2 * sizeof(uint32_t));
    }

private:
    std::vector<std::array<T, 3>> triples(const std::vector<T>& a) const {
        std::vector<std::array<T, 3>> r(n_);
        for (size_t i = 0; i < n_; ++i) r[i] = {{a[3 * i], a[3 * i + 1], a[3 * i + 2]}};
        return r;
    }

public:
    // storage, filled by MPMSolver::getParticles() (also reachable through
    // the get*Data() accessors above)
    size_t n_ = 0, chunks_ = 0;
    std::vector<T> x_, v_, m_, V_, F_, C_, stress_;
    std::vector<MaterialType> type_;
    std::vector<uint32_t> active_;
};

// Host copy of the grid after the last step's grid update, with the
// reference's accessors (src/mpm_data_structures.h:369-530): index k nx ny +
// j nx + i, masses, velocities, momentum (mass times velocity); forces are
// not a state of the MLS step (the stress enters the momentum in P2G) and
// read as zero, boundary flags as set.
template <typename T = float>
class MPMGrid {
public:
    using scalar_type = T;
    MPMGrid() = default;
    MPMGrid(int3_ dims, vec3<T> spacing, vec3<T> origin = {T(0), T(0), T(0)}) { reset(dims, spacing, origin); }

    void reset(int3_ dims, vec3<T> spacing, vec3<T> origin) {
        dims_ = dims;
        spacing_ = spacing;
        origin_ = origin;
        const size_t n = (size_t)dims.x * dims.y * dims.z;
        mass_.assign(n, T(0));
        vel_.assign(3 * n, T(0));
        force_.assign(3 * n, T(0));
        mom_.assign(3 * n, T(0));
        bc_.assign(n, 0u);
    }
    void clearGrid() {
        std::fill(mass_.begin(), mass_.end(), T(0));
        std::fill(vel_.begin(), vel_.end(), T(0));
        std::fill(force_.begin(), force_.end(), T(0));
        std::fill(mom_.begin(), mom_.end(), T(0));
    }
    std::array<T, 3> getGridSpacing() const { return {{spacing_.x, spacing_.y, spacing_.z}}; }
    int3_ getDimensions() const { return dims_; }
    vec3<T> getSpacing() const { return spacing_; }
    vec3<T> getOrigin() const { return origin_; }
    size_t getTotalNodes() const { return mass_.size(); }
    size_t getLinearIndex(int i, int j, int k) const {
        return (size_t)k * dims_.x * dims_.y + (size_t)j * dims_.x + (size_t)i;
    }
    int3_ getGridIndex(size_t l) const {
        const size_t layer = (size_t)dims_.x * dims_.y;
        const int k = (int)(l / layer), r = (int)(l % layer);
        return {r % dims_.x, r / dims_.x, k};
    }
    vec3<T> getWorldPosition(int i, int j, int k) const {
        return {origin_.x + i * spacing_.x, origin_.y + j * spacing_.y, origin_.z + k * spacing_.z};
    }
    int3_ getGridPosition(T x, T y, T z) const {
        return {(int)std::floor((x - origin_.x) / spacing_.x), (int)std::floor((y - origin_.y) / spacing_.y),
                (int)std::floor((z - origin_.z) / spacing_.z)};
    }
    void setMass(size_t n, T m) { mass_[n] = m; }
    T getMass(size_t n) const { return mass_[n]; }
    void setVelocity(size_t n, T vx, T vy, T vz) { vel_[3 * n] = vx; vel_[3 * n + 1] = vy; vel_[3 * n + 2] = vz; }
    void getVelocity(size_t n, T& vx, T& vy, T& vz) const { vx = vel_[3 * n]; vy = vel_[3 * n + 1]; vz = vel_[3 * n + 2]; }
    void addVelocity(size_t n, T dx, T dy, T dz) { vel_[3 * n] += dx; vel_[3 * n + 1] += dy; vel_[3 * n + 2] += dz; }
    void setForce(size_t n, T fx, T fy, T fz) { force_[3 * n] = fx; force_[3 * n + 1] = fy; force_[3 * n + 2] = fz; }
    void addForce(size_t n, T fx, T fy, T fz) { force_[3 * n] += fx; force_[3 * n + 1] += fy; force_[3 * n + 2] += fz; }
    void setBoundaryCondition(size_t n, uint32_t f) { bc_[n] = f; }
    uint32_t getBoundaryCondition(size_t n) const { return bc_[n]; }
    T* getMassData() { return mass_.data(); }
    T* getVelocityData() { return vel_.data(); }
    T* getForceData() { return force_.data(); }
    T* getMomentumData() { return mom_.data(); }
    uint32_t* getBoundaryConditionData() { return bc_.data(); }
    const T* getMassData() const { return mass_.data(); }
    const T* getVelocityData() const { return vel_.data(); }
    const T* getForceData() const { return force_.data(); }
    const T* getMomentumData() const { return mom_.data(); }
    const uint32_t* getBoundaryConditionData() const { return bc_.data(); }
    size_t getMemoryFootprint() const {
        return sizeof(T) * (mass_.size() + vel_.size() + force_.size() + mom_.size()) + sizeof(uint32_t) * bc_.size();
    }

    // storage, filled by MPMSolver::getGrid()
    int3_ dims_{0, 0, 0};
    vec3<T> spacing_{T(0), T(0), T(0)}, origin_{T(0), T(0), T(0)};
    std::vector<T> mass_, vel_, force_, mom_;
    std::vector<uint32_t> bc_;
};

template <typename T = float>
class MPMSolver {
    static_assert(sizeof(T) == 4, "the B200 path computes in FP32");

public:
    using scalar_type = T;
    using particle_container = ParticleAoSoA<T>;
    using grid_container = MPMGrid<T>;

    explicit MPMSolver(const MPMSolverConfig& config = MPMSolverConfig{}) : config_(config) {}
    ~MPMSolver() {
        if (h_) pgmpm_destroy(h_);
    }
    MPMSolver(const MPMSolver&) = delete;
    MPMSolver& operator=(const MPMSolver&) = delete;

    void initialize() {
        if (initialized_) return;
        pgmpm_scene_desc d{};
        d.n[0] = config_.grid_dimensions.x;
        d.n[1] = config_.grid_dimensions.y;
        d.n[2] = config_.grid_dimensions.z;
        d.physics = config_.physics;
        d.boundary = config_.physics == PGMPM_PHYSICS_MLS ? config_.boundary : PGMPM_BC_NONE;
        d.boundary_thickness = config_.boundary_thickness;
        d.dx = config_.grid_spacing.x;
        d.origin[0] = config_.domain_origin.x;
        d.origin[1] = config_.domain_origin.y;
        d.origin[2] = config_.domain_origin.z;
        d.dt = config_.time_step;
        const T3 g = config_.enable_gravity ? config_.gravity : T3{0.f, 0.f, 0.f};
        d.gravity[0] = g.x;
        d.gravity[1] = g.y;
        d.gravity[2] = g.z;
        std::vector<pgmpm_material> mats;
        for (const auto& m : config_.materials)
            mats.push_back(pgmpm_material{(int32_t)m.type, (int32_t)m.model, m.youngs_modulus, m.poisson_ratio,
                                          m.density, m.yield_stress, m.viscosity});
        const int64_t n = (int64_t)m_.size();
        physgrad_b200_detail::check(
            pgmpm_create(&d, 1, &n, mats.data(), (int32_t)mats.size(), config_.device, &h_));
        if (n)
            physgrad_b200_detail::check(pgmpm_upload(h_, x_.data(), v_.data(), nullptr, nullptr, m_.data(),
                                                     V_.data(), mats.size() > 1 ? mat_.data() : nullptr,
                                                     PGMPM_PTR_HOST, nullptr));
        physgrad_b200_detail::check(pgmpm_set_profiling(h_, config_.enable_profiling ? 1 : 0));
        initialized_ = true;
    }

    // src/mpm_solver.h:190-226 (V = m / density of the material)
    void addParticles(const std::vector<T3>& positions, const std::vector<T3>& velocities,
                      const std::vector<T>& masses, MaterialType material_type = MaterialType::ELASTIC) {
        if (initialized_) throw std::runtime_error("addParticles after initialize() is not supported");
        if (m_.size() + positions.size() > (size_t)config_.max_particles)
            throw std::runtime_error("Exceeded maximum particle count");
        int mid = -1;
        for (size_t i = 0; i < config_.materials.size(); ++i)
            if (config_.materials[i].type == material_type) {
                mid = (int)i;
                break;
            }
        if (mid < 0) throw std::runtime_error("material type not in config.materials");
        const float rho = config_.materials[mid].density;
        for (size_t i = 0; i < positions.size(); ++i) {
            x_.insert(x_.end(), {positions[i].x, positions[i].y, positions[i].z});
            v_.insert(v_.end(), {velocities[i].x, velocities[i].y, velocities[i].z});
            m_.push_back(masses[i]);
            V_.push_back(masses[i] / rho);
            mat_.push_back(mid);
        }
    }

    void step() {
        if (!initialized_) throw std::runtime_error("Solver not initialized");
        physgrad_b200_detail::check(pgmpm_step(h_, 1, nullptr));
        time_ += config_.time_step;
        ++step_;
    }

    void run() {
        initialize();
        const int n = (int)(config_.simulation_time / config_.time_step + 0.5f);
        if (!config_.enable_output) {
            physgrad_b200_detail::check(pgmpm_step(h_, n, nullptr));
            time_ += n * config_.time_step;
            step_ += n;
            return;
        }
        // the steps between outputs run as one call; a frame is written after
        // each step that crosses a multiple of output_frequency (the
        // reference's test, src/mpm_solver.h:306-311)
        std::filesystem::create_directories(config_.output_directory);
        int done = 0, frame = 0;
        while (done < n) {
            int k = 1;
            while (done + k < n && !crosses_output(time_ + k * config_.time_step)) ++k;
            physgrad_b200_detail::check(pgmpm_step(h_, k, nullptr));
            done += k;
            step_ += k;
            time_ += k * config_.time_step;
            if (crosses_output(time_)) {
                char name[32];
                std::snprintf(name, sizeof(name), "/frame_%05d.vtk", frame++);
                physgrad_b200_detail::check(pgmpm_write_vtk(h_, (config_.output_directory + name).c_str(), time_,
                                                            nullptr));
            }
        }
    }

    // Data access (src/mpm_solver.h:324-326), callable on a const solver:
    // the host copies are refreshed from the device on each call.
    const particle_container& getParticles() const {
        const size_t n = m_.size();
        particles_.resize(n);
        std::copy(m_.begin(), m_.end(), particles_.m_.begin());
        std::copy(V_.begin(), V_.end(), particles_.V_.begin());
        for (size_t i = 0; i < n; ++i) particles_.type_[i] = config_.materials[(size_t)mat_[i]].type;
        if (initialized_ && n)
            physgrad_b200_detail::check(pgmpm_download(h_, particles_.x_.data(), particles_.v_.data(),
                                                       particles_.C_.data(), particles_.F_.data(), PGMPM_PTR_HOST,
                                                       nullptr));
        return particles_;
    }

    const grid_container& getGrid() const {
        grid_.reset(config_.grid_dimensions, {config_.grid_spacing.x, config_.grid_spacing.y, config_.grid_spacing.z},
                    {config_.domain_origin.x, config_.domain_origin.y, config_.domain_origin.z});
        if (initialized_) {
            physgrad_b200_detail::check(
                pgmpm_download_grid(h_, 0, grid_.mass_.data(), grid_.vel_.data(), PGMPM_PTR_HOST, nullptr));
            for (size_t n = 0; n < grid_.mass_.size(); ++n)
                for (int a = 0; a < 3; ++a) grid_.mom_[3 * n + a] = grid_.mass_[n] * grid_.vel_[3 * n + a];
        }
        return grid_;
    }

    const MPMPerformanceMetrics& getMetrics() const {
        if (initialized_) {
            pgmpm_metrics m{};
            physgrad_b200_detail::check(pgmpm_get_metrics(h_, &m));
            metrics_.total_steps = (int)m.total_steps;
            metrics_.average_step_time = m.average_step_ms * 1e-3;
            metrics_.p2g_time = m.p2g_ms * 1e-3;
            metrics_.g2p_time = m.g2p_ms * 1e-3;
            metrics_.grid_update_time = m.grid_ms * 1e-3;
            metrics_.average_particles_per_second = (float)m.particle_steps_per_s;
            metrics_.particle_memory = m_.size() * (6 * 16 + 8 + 4);
            metrics_.grid_memory = (size_t)config_.grid_dimensions.x * config_.grid_dimensions.y *
                                   config_.grid_dimensions.z * 32;
            metrics_.total_memory_usage = metrics_.particle_memory + metrics_.grid_memory;
        }
        return metrics_;
    }

    float getCurrentTime() const { return time_; }
    // Write the particles now (legacy binary VTK; see pgmpm_write_vtk).
    void outputData(const std::string& path) {
        physgrad_b200_detail::check(pgmpm_write_vtk(h_, path.c_str(), time_, nullptr));
    }
    int getCurrentStep() const { return step_; }
    pgmpm_solver handle() const { return h_; }

private:
    MPMSolverConfig config_;
    pgmpm_solver h_ = nullptr;
    bool initialized_ = false;
    std::vector<float> x_, v_, m_, V_;
    std::vector<int32_t> mat_;
    // host copies refreshed by the const getters
    mutable particle_container particles_;
    mutable grid_container grid_;
    mutable MPMPerformanceMetrics metrics_;
    // the step that ended at simulated time t crossed a multiple of output_frequency
    bool crosses_output(float t) const {
        return config_.output_frequency > 0.f && (int)(t / config_.output_frequency) >
                                                     (int)((t - config_.time_step) / config_.output_frequency);
    }
    float time_ = 0.f;
    int step_ = 0;
};

}  // namespace physgrad::mpm
