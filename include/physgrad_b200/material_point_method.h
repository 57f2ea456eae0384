// physgrad_b200/material_point_method.h -- drop-in C++ replacement for
// physgrad's CPU MPM solver header (src/material_point_method.h:45-263 and
// 430-506, with ConceptVector3D of src/common_types.h), implemented over the
// C-ABI of libpgmpm.so (include/pgmpm.h).  Header-only; link -lpgmpm.
//
// Same names, member layout and argument meaning as the reference:
//   physgrad::ConceptVector3D<T>, int3 (CUDA's when CUDA headers are in use),
//   physgrad::mpm::ParticleAoSoA<T, ChunkSize> (the chunked arrays and their
//   accessors), MPMGrid<T> (mass / velocity / momentum / force per node, index
//   k*nx*ny + j*nx + i), MPMSolver<T, ChunkSize>::{SimulationParams,
//   MPMSolver(int3, cell_size, origin, params), addParticles, step,
//   getParticles, getGrid, getCurrentTime, getStepCount}.
// The step is the reference's own PIC step (floor-based 3-node quadratic
// stencil, 1e-10 weight and mass thresholds, gravity added to the nodal
// momentum, no stress), run on the GPU as PGMPM_PHYSICS_REF_COMPAT.
//
// Differences, each checked where it arises:
//   * T must be float (the B200 path computes in FP32): static_assert.
//   * cell_size must be the same on the three axes, and interpolation_order
//     must be 2 (the reference default): std::invalid_argument otherwise.
//   * use_affine_pic, use_flip, flip_ratio and cfl_factor are accepted and
//     unused, as in the reference step.
//   * getGrid() holds the last step's nodal mass and velocity; momentum is
//     mass x velocity where the mass exceeds 1e-10 (the device keeps the
//     velocity), force is zero (the reference step writes none).
//   * addParticles also stores volumes, Young's modulus, Poisson ratio and
//     density in their chunks (the reference leaves them zero).
// Like the reference header it cannot share a translation unit with
// physgrad_b200/mpm_solver.h (both define physgrad::mpm::MPMSolver).
#pragma once

#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../pgmpm.h"

#if defined(__CUDACC__) || defined(__VECTOR_TYPES_H__)
#include <vector_types.h>
#else
struct int3 {
    int x, y, z;
    int3() : x(0), y(0), z(0) {}
    int3(int x_, int y_, int z_) : x(x_), y(y_), z(z_) {}
};
#endif

namespace physgrad {

template <typename T>
class ConceptVector3D {
public:
    using value_type = T;
    T x, y, z;
    constexpr ConceptVector3D() : x(T{0}), y(T{0}), z(T{0}) {}
    constexpr ConceptVector3D(T x_, T y_, T z_) : x(x_), y(y_), z(z_) {}
    constexpr T& operator[](size_t i) { return i == 0 ? x : (i == 1 ? y : z); }
    constexpr const T& operator[](size_t i) const { return i == 0 ? x : (i == 1 ? y : z); }
    static constexpr size_t size() { return 3; }
    ConceptVector3D operator+(const ConceptVector3D& o) const { return {x + o.x, y + o.y, z + o.z}; }
    ConceptVector3D operator-(const ConceptVector3D& o) const { return {x - o.x, y - o.y, z - o.z}; }
    ConceptVector3D operator*(T s) const { return {x * s, y * s, z * s}; }
};

namespace b200_detail {
inline void check(int rc) {
    if (rc != PGMPM_OK) throw std::runtime_error(std::string("pgmpm: ") + pgmpm_last_error());
}
}  // namespace b200_detail

namespace mpm {

// Host particle container with the reference's chunked layout: chunk c holds
// particles [c * ChunkSize, (c + 1) * ChunkSize); a vector field stores its
// components as ChunkSize x's, then ChunkSize y's, then ChunkSize z's, and
// F its 9 entries (row-major) the same way.
template <typename T, size_t ChunkSize = 64>
struct ParticleAoSoA {
    static constexpr size_t chunk_size = ChunkSize;
    using value_type = T;

    std::vector<std::array<T, chunk_size * 3>> position_chunks;
    std::vector<std::array<T, chunk_size * 3>> velocity_chunks;
    std::vector<std::array<T, chunk_size>> mass_chunks;
    std::vector<std::array<T, chunk_size>> volume_chunks;
    std::vector<std::array<T, chunk_size * 9>> deformation_gradient_chunks;
    std::vector<std::array<T, chunk_size * 6>> stress_chunks;
    std::vector<std::array<T, chunk_size>> young_modulus_chunks;
    std::vector<std::array<T, chunk_size>> poisson_ratio_chunks;
    std::vector<std::array<T, chunk_size>> density_chunks;

    size_t num_particles = 0;
    size_t num_chunks = 0;

    size_t size() const { return num_particles; }

    void resize(size_t new_size) {
        num_particles = new_size;
        num_chunks = (new_size + chunk_size - 1) / chunk_size;
        position_chunks.resize(num_chunks);
        velocity_chunks.resize(num_chunks);
        mass_chunks.resize(num_chunks);
        volume_chunks.resize(num_chunks);
        deformation_gradient_chunks.resize(num_chunks);
        stress_chunks.resize(num_chunks);
        young_modulus_chunks.resize(num_chunks);
        poisson_ratio_chunks.resize(num_chunks);
        density_chunks.resize(num_chunks);
    }

    ConceptVector3D<T> getPosition(size_t p) const { return get3(position_chunks, p); }
    void setPosition(size_t p, const ConceptVector3D<T>& v) { set3(position_chunks, p, v); }
    ConceptVector3D<T> getVelocity(size_t p) const { return get3(velocity_chunks, p); }
    void setVelocity(size_t p, const ConceptVector3D<T>& v) { set3(velocity_chunks, p, v); }
    T getMass(size_t p) const { return mass_chunks[p / chunk_size][p % chunk_size]; }
    void setMass(size_t p, T m) { mass_chunks[p / chunk_size][p % chunk_size] = m; }
    void getDeformationGradient(size_t p, T* F) const {
        const auto& c = deformation_gradient_chunks[p / chunk_size];
        for (int i = 0; i < 9; ++i) F[i] = c[p % chunk_size + i * chunk_size];
    }
    void setDeformationGradient(size_t p, const T* F) {
        auto& c = deformation_gradient_chunks[p / chunk_size];
        for (int i = 0; i < 9; ++i) c[p % chunk_size + i * chunk_size] = F[i];
    }

    // flat copies (upload order) used at the C-ABI boundary
    void gatherFlat(std::vector<float>& x, std::vector<float>& v, std::vector<float>& F, std::vector<float>& m,
                    std::vector<float>& V0) const {
        const size_t n = num_particles;
        x.resize(3 * n);
        v.resize(3 * n);
        F.resize(9 * n);
        m.resize(n);
        V0.resize(n);
        for (size_t p = 0; p < n; ++p) {
            const auto xp = getPosition(p), vp = getVelocity(p);
            for (int a = 0; a < 3; ++a) {
                x[3 * p + a] = xp[a];
                v[3 * p + a] = vp[a];
            }
            getDeformationGradient(p, &F[9 * p]);
            m[p] = getMass(p);
            V0[p] = volume_chunks[p / chunk_size][p % chunk_size];
        }
    }
    void scatterFlat(const float* x, const float* v, const float* F) {
        for (size_t p = 0; p < num_particles; ++p) {
            if (x) setPosition(p, {x[3 * p], x[3 * p + 1], x[3 * p + 2]});
            if (v) setVelocity(p, {v[3 * p], v[3 * p + 1], v[3 * p + 2]});
            if (F) setDeformationGradient(p, F + 9 * p);
        }
    }

private:
    template <class Chunks>
    static ConceptVector3D<T> get3(const Chunks& ch, size_t p) {
        const auto& c = ch[p / chunk_size];
        const size_t l = p % chunk_size;
        return {c[l], c[l + chunk_size], c[l + 2 * chunk_size]};
    }
    template <class Chunks>
    static void set3(Chunks& ch, size_t p, const ConceptVector3D<T>& v) {
        auto& c = ch[p / chunk_size];
        const size_t l = p % chunk_size;
        c[l] = v[0];
        c[l + chunk_size] = v[1];
        c[l + 2 * chunk_size] = v[2];
    }
};

// Background grid (src/material_point_method.h:186-263): dense node arrays,
// index k*nx*ny + j*nx + i.
template <typename T>
struct MPMGrid {
    std::vector<T> mass;
    std::vector<ConceptVector3D<T>> velocity;
    std::vector<ConceptVector3D<T>> momentum;
    std::vector<ConceptVector3D<T>> force;

    int3 dimensions;
    int3 dims;
    ConceptVector3D<T> cell_size;
    ConceptVector3D<T> origin;
    size_t total_nodes = 0;

    MPMGrid(const int3& d, const ConceptVector3D<T>& cell, const ConceptVector3D<T>& orig)
        : dimensions(d), dims(d), cell_size(cell), origin(orig) {
        total_nodes = d.x > 0 && d.y > 0 && d.z > 0 ? (size_t)d.x * d.y * d.z : 0;
        resize();
    }

    void resize() {
        mass.assign(total_nodes, T{0});
        velocity.assign(total_nodes, ConceptVector3D<T>{});
        momentum.assign(total_nodes, ConceptVector3D<T>{});
        force.assign(total_nodes, ConceptVector3D<T>{});
    }
    void clear() { resize(); }
    void clearGridData() { clear(); }

    // v = p / m above the reference's 1e-10 mass threshold, else 0
    void updateGridVelocities() {
        for (size_t i = 0; i < total_nodes; ++i)
            velocity[i] = mass[i] > T{1e-10} ? momentum[i] * (T{1} / mass[i]) : ConceptVector3D<T>{};
    }
    // the outermost node layer at rest
    void applyBoundaryConditions() {
        for (int k = 0; k < dimensions.z; ++k)
            for (int j = 0; j < dimensions.y; ++j)
                for (int i = 0; i < dimensions.x; ++i)
                    if (i == 0 || j == 0 || k == 0 || i == dimensions.x - 1 || j == dimensions.y - 1 ||
                        k == dimensions.z - 1) {
                        velocity[getNodeIndex(i, j, k)] = ConceptVector3D<T>{};
                        momentum[getNodeIndex(i, j, k)] = ConceptVector3D<T>{};
                    }
    }

    size_t getNodeIndex(int i, int j, int k) const {
        return (size_t)k * dimensions.x * dimensions.y + (size_t)j * dimensions.x + (size_t)i;
    }
    ConceptVector3D<T> getNodePosition(int i, int j, int k) const {
        return {origin[0] + i * cell_size[0], origin[1] + j * cell_size[1], origin[2] + k * cell_size[2]};
    }
};

template <typename T, size_t ChunkSize = 64>
class MPMSolver {
    static_assert(std::is_same<T, float>::value, "the B200 path computes in FP32: use MPMSolver<float>");

public:
    using ParticleData = ParticleAoSoA<T, ChunkSize>;
    using Grid = MPMGrid<T>;

    struct SimulationParams {
        T timestep = T{1e-4};
        ConceptVector3D<T> gravity = {T{0}, T{-9.81}, T{0}};
        T cfl_factor = T{0.4};
        bool use_affine_pic = true;
        bool use_flip = true;
        T flip_ratio = T{0.95};
        int interpolation_order = 2;
        int device = 0;  // CUDA ordinal (addition of this implementation)
    };

    MPMSolver(const int3& grid_dims, const ConceptVector3D<T>& cell_size, const ConceptVector3D<T>& origin,
              const SimulationParams& params = {})
        : grid_(grid_dims, cell_size, origin), params_(params) {
        if (!(cell_size[0] == cell_size[1] && cell_size[1] == cell_size[2]))
            throw std::invalid_argument("MPMSolver: cell_size must be the same on the three axes");
        if (params.interpolation_order != 2)
            throw std::invalid_argument("MPMSolver: only interpolation_order 2 (quadratic) is implemented");
    }
    ~MPMSolver() {
        if (h_) pgmpm_destroy(h_);
    }
    MPMSolver(const MPMSolver&) = delete;
    MPMSolver& operator=(const MPMSolver&) = delete;

    // src/material_point_method.h:455-477: appended particles start with F = I
    void addParticles(const std::vector<ConceptVector3D<T>>& positions,
                      const std::vector<ConceptVector3D<T>>& velocities, const std::vector<T>& masses,
                      const std::vector<T>& volumes, T young_modulus = T{1e6}, T poisson_ratio = T{0.3},
                      T density = T{1000}) {
        if (velocities.size() < positions.size() || masses.size() < positions.size())
            throw std::invalid_argument("addParticles: velocities and masses must cover every position");
        pull();  // keep particles stepped so far
        const size_t old = particles_.num_particles;
        particles_.resize(old + positions.size());
        const T I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        for (size_t i = 0; i < positions.size(); ++i) {
            const size_t p = old + i;
            particles_.setPosition(p, positions[i]);
            particles_.setVelocity(p, velocities[i]);
            particles_.setMass(p, masses[i]);
            particles_.setDeformationGradient(p, I);
            particles_.volume_chunks[p / ChunkSize][p % ChunkSize] = i < volumes.size() ? volumes[i] : T{0};
            particles_.young_modulus_chunks[p / ChunkSize][p % ChunkSize] = young_modulus;
            particles_.poisson_ratio_chunks[p / ChunkSize][p % ChunkSize] = poisson_ratio;
            particles_.density_chunks[p / ChunkSize][p % ChunkSize] = density;
        }
        device_stale_ = true;
    }

    // src/material_point_method.h:479-500
    void step() { advance(1); }
    // n steps in one call (one CUDA graph per step, no host synchronisation in between)
    void step(int n) { advance(n); }

    const ParticleData& getParticles() const {
        pull();
        return particles_;
    }
    const Grid& getGrid() const {
        if (grid_stale_ && h_) {
            const size_t n = grid_.total_nodes;
            std::vector<float> m(n), v(3 * n);
            b200_detail::check(pgmpm_download_grid(h_, 0, m.data(), v.data(), PGMPM_PTR_HOST, nullptr));
            for (size_t i = 0; i < n; ++i) {
                grid_.mass[i] = m[i];
                grid_.velocity[i] = {v[3 * i], v[3 * i + 1], v[3 * i + 2]};
                grid_.momentum[i] = m[i] > T{1e-10} ? grid_.velocity[i] * m[i] : ConceptVector3D<T>{};
                grid_.force[i] = ConceptVector3D<T>{};
            }
        }
        grid_stale_ = false;
        return grid_;
    }
    T getCurrentTime() const { return current_time_; }
    size_t getStepCount() const { return step_count_; }

private:
    mutable ParticleData particles_;
    mutable Grid grid_;
    SimulationParams params_;
    T current_time_ = T{0};
    size_t step_count_ = 0;
    pgmpm_solver h_ = nullptr;
    int64_t device_count_ = -1;      // particles in the device solver
    bool device_stale_ = true;       // host particles changed since the upload
    mutable bool host_stale_ = false;  // device state newer than the host copy
    mutable bool grid_stale_ = false;

    void advance(int n) {
        if (n <= 0) return;
        push();
        b200_detail::check(pgmpm_step(h_, n, nullptr));
        host_stale_ = grid_stale_ = true;
        for (int i = 0; i < n; ++i) current_time_ += params_.timestep;
        step_count_ += (size_t)n;
    }

    // host -> device: (re)create the solver when the particle count changed
    void push() {
        if (!device_stale_) return;
        const int64_t n = (int64_t)particles_.num_particles;
        if (h_ && device_count_ != n) {
            pgmpm_destroy(h_);
            h_ = nullptr;
        }
        if (!h_) {
            pgmpm_scene_desc d{};
            d.n[0] = grid_.dimensions.x;
            d.n[1] = grid_.dimensions.y;
            d.n[2] = grid_.dimensions.z;
            for (int a = 0; a < 3; ++a) {
                d.origin[a] = grid_.origin[a];
                d.gravity[a] = params_.gravity[a];
            }
            d.dx = grid_.cell_size[0];
            d.dt = params_.timestep;
            d.physics = PGMPM_PHYSICS_REF_COMPAT;
            d.boundary = PGMPM_BC_NONE;
            d.boundary_thickness = 0;
            // the material is not used by the reference's PIC step
            pgmpm_material mat{};
            mat.type = PGMPM_MAT_ELASTIC;
            mat.model = PGMPM_MODEL_FIXED_COROTATED;
            mat.youngs_modulus = 1e6f;
            mat.poisson_ratio = 0.3f;
            mat.density = 1000.f;
            b200_detail::check(pgmpm_create(&d, 1, &n, &mat, 1, params_.device, &h_));
            device_count_ = n;
        }
        std::vector<float> x, v, F, m, V0;
        particles_.gatherFlat(x, v, F, m, V0);
        b200_detail::check(pgmpm_upload(h_, x.data(), v.data(), nullptr, F.data(), m.data(), V0.data(), nullptr,
                                        PGMPM_PTR_HOST, nullptr));
        device_stale_ = false;
    }

    // device -> host when the device holds newer particles
    void pull() const {
        if (!host_stale_ || !h_) return;
        const size_t n = particles_.num_particles;
        std::vector<float> x(3 * n), v(3 * n), F(9 * n);
        b200_detail::check(pgmpm_download(h_, x.data(), v.data(), nullptr, F.data(), PGMPM_PTR_HOST, nullptr));
        particles_.scatterFlat(x.data(), v.data(), F.data());
        host_stale_ = false;
    }
};

}  // namespace mpm
}  // namespace physgrad
