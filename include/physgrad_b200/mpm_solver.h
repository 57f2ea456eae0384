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
    bool enable_adaptive_timestep = false;
    bool enable_profiling = false;
    // output (src/mpm_solver.h:57-60): run() writes the particles every
    // output_frequency seconds of simulated time as
    // output_directory/frame_NNNNN.vtk (legacy binary VTK).  Off by default
    // here: the reference's outputData() only prints a line.
    bool enable_output = false;
    float output_frequency = 0.01f;
    std::string output_directory = "./mpm_output";
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
};

// Host copy of the particle state with ParticleAoSoA's accessors
// (src/mpm_data_structures.h:165-258); filled by MPMSolver::getParticles().
template <typename T = float>
class ParticleAoSoA {
public:
    size_t size() const { return x_.size() / 3; }
    void getPosition(size_t i, T& x, T& y, T& z) const { x = x_[3 * i]; y = x_[3 * i + 1]; z = x_[3 * i + 2]; }
    void getVelocity(size_t i, T& x, T& y, T& z) const { x = v_[3 * i]; y = v_[3 * i + 1]; z = v_[3 * i + 2]; }
    T getMass(size_t i) const { return m_[i]; }
    T getVolume(size_t i) const { return V_[i]; }
    void getDeformationGradient(size_t i, T F[9]) const {
        for (int k = 0; k < 9; ++k) F[k] = F_[9 * i + k];
    }
    void getAffineMatrix(size_t i, T C[9]) const {
        for (int k = 0; k < 9; ++k) C[k] = C_[9 * i + k];
    }
    std::vector<T> x_, v_, C_, F_, m_, V_;
};

template <typename T = float>
class MPMGrid {
public:
    int3_ getDimensions() const { return dims_; }
    size_t getTotalNodes() const { return mass_.size(); }
    size_t getLinearIndex(int i, int j, int k) const {
        return (size_t)k * dims_.x * dims_.y + (size_t)j * dims_.x + (size_t)i;
    }
    T getMass(size_t n) const { return mass_[n]; }
    void getVelocity(size_t n, T& vx, T& vy, T& vz) const { vx = vel_[3 * n]; vy = vel_[3 * n + 1]; vz = vel_[3 * n + 2]; }
    int3_ dims_{0, 0, 0};
    std::vector<T> mass_, vel_;
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

    const particle_container& getParticles() {
        const size_t n = m_.size();
        particles_.x_.resize(3 * n);
        particles_.v_.resize(3 * n);
        particles_.C_.resize(9 * n);
        particles_.F_.resize(9 * n);
        particles_.m_ = m_;
        particles_.V_ = V_;
        if (initialized_ && n)
            physgrad_b200_detail::check(pgmpm_download(h_, particles_.x_.data(), particles_.v_.data(),
                                                       particles_.C_.data(), particles_.F_.data(), PGMPM_PTR_HOST,
                                                       nullptr));
        return particles_;
    }

    const grid_container& getGrid() {
        const size_t nodes = (size_t)config_.grid_dimensions.x * config_.grid_dimensions.y * config_.grid_dimensions.z;
        grid_.dims_ = config_.grid_dimensions;
        grid_.mass_.assign(nodes, 0.f);
        grid_.vel_.assign(3 * nodes, 0.f);
        if (initialized_)
            physgrad_b200_detail::check(
                pgmpm_download_grid(h_, 0, grid_.mass_.data(), grid_.vel_.data(), PGMPM_PTR_HOST, nullptr));
        return grid_;
    }

    const MPMPerformanceMetrics& getMetrics() {
        if (initialized_) {
            pgmpm_metrics m{};
            physgrad_b200_detail::check(pgmpm_get_metrics(h_, &m));
            metrics_.total_steps = (int)m.total_steps;
            metrics_.average_step_time = m.average_step_ms * 1e-3;
            metrics_.p2g_time = m.p2g_ms * 1e-3;
            metrics_.g2p_time = m.g2p_ms * 1e-3;
            metrics_.grid_update_time = m.grid_ms * 1e-3;
            metrics_.average_particles_per_second = (float)m.particle_steps_per_s;
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
    particle_container particles_;
    grid_container grid_;
    MPMPerformanceMetrics metrics_;
    // the step that ended at simulated time t crossed a multiple of output_frequency
    bool crosses_output(float t) const {
        return config_.output_frequency > 0.f && (int)(t / config_.output_frequency) >
                                                     (int)((t - config_.time_step) / config_.output_frequency);
    }
    float time_ = 0.f;
    int step_ = 0;
};

}  // namespace physgrad::mpm
