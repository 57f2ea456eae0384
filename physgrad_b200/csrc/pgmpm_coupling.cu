// pgmpm_coupling.cu -- consumers of the solver's particles on the device:
//   * pgmpm_sph_coupling: the SPH-MPM contact coupling of
//     SPHMPMCouplingSystem (src/sph_mpm_coupling.h:453-575), with the
//     solver's particles as the MPM side.  Candidate MPM particles of each
//     SPH particle come from the spatial hash grid (pgmpm_hashgrid_*, the
//     reference's SpatialHashGrid) built on the current positions with a
//     cell of one coupling radius; one thread per SPH particle keeps the
//     pairs closer than the radius and forms their forces in the reference's
//     float operations, in the same order, so pair membership is bit-exact;
//     only the order in which a particle's pair forces are summed differs.
//   * pgmpm_kinetic_energy: the energy monitor of FSISimulationManager
//     (computeTotalEnergy, src/fsi_coupling.h:837-858), per material.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "pgmpm_solver_impl.h"

using namespace pgmpm;

namespace {

// positions and velocities of the state (physical order) as [N][3]
// physical-order float4 sums -> the caller's [N][3] array in upload order
__global__ void k_mforce_out(const float4* __restrict__ mf, const uint32_t* __restrict__ user_of_phys, int64_t N,
                             float* __restrict__ out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += stride) {
        const float4 f = mf[p];
        const size_t u = user_of_phys[p];
        out[3 * u] = f.x;
        out[3 * u + 1] = f.y;
        out[3 * u + 2] = f.z;
    }
}

__global__ void k_state_xv(const float4* __restrict__ q, int64_t N, float* __restrict__ x, float* __restrict__ v) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += stride) {
        const float4 a = q[p];
        x[3 * p] = a.x;
        x[3 * p + 1] = a.y;
        x[3 * p + 2] = a.z;
        if (v) {
            const float4 b = q[3 * N + p];
            v[3 * p] = b.x;
            v[3 * p + 1] = b.y;
            v[3 * p + 2] = b.z;
        }
    }
}

// One SPH particle per thread over its candidate MPM particles (physical
// indices): the pairs closer than r, their contact forces (normal spring and
// damping, friction along the tangential velocity), the fluid force summed
// into sph_force (two-way), the solid force into mpm_force (upload order),
// the pair count and k (r - d)^2 / 2 summed over pairs.
// One warp per SPH particle: the lanes take its candidates in turn (the
// candidate list is read coalesced and the long lists of particles inside
// the solid are shared by 32 lanes), and the warp sums the lanes' fluid
// forces at the end.
// The MPM side is read from the state planes (x from plane 0, v from plane
// 3, one 16-byte load each), and each pair's solid force is added to
// mforce[p] (physical order, float4) with one vector atomic.
__global__ void k_sph_pairs(const float* __restrict__ sx, const float* __restrict__ sv, int64_t nq,
                            const int64_t* __restrict__ off, const uint32_t* __restrict__ cand,
                            const float4* __restrict__ state, int64_t N, pgmpm_sph_coupling_config cfg,
                            float* __restrict__ sph_force, float4* __restrict__ mforce,
                            unsigned long long* __restrict__ npairs, double* __restrict__ energy) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    const float k = cfg.coupling_stiffness, c = cfg.coupling_damping, mu = cfg.friction_coefficient,
                r = cfg.coupling_radius;
    unsigned long long cnt = 0;
    double e = 0.0;
    for (int64_t q = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < nq; q += warps) {
        const float y0 = sx[3 * q], y1 = sx[3 * q + 1], y2 = sx[3 * q + 2];
        const float w0 = sv[3 * q], w1 = sv[3 * q + 1], w2 = sv[3 * q + 2];
        float f0 = 0.f, f1 = 0.f, f2 = 0.f;
        const int64_t end = off[q + 1];
        for (int64_t ci = off[q] + lane; ci < end; ci += 32) {
            const uint32_t p = cand[ci];
            const float4 xp = state[p];
            // distance as the reference forms it (no contraction)
            const float r0 = __fsub_rn(xp.x, y0), r1 = __fsub_rn(xp.y, y1), r2 = __fsub_rn(xp.z, y2);
            const float d = sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(r0, r0), __fmul_rn(r1, r1)), __fmul_rn(r2, r2)));
            if (!(d < r)) continue;
            ++cnt;
            const float pen = __fsub_rn(r, d);
            e += (double)__fmul_rn(__fmul_rn(__fmul_rn(0.5f, k), pen), pen);
            if (d < 1e-6f) continue;
            const float inv = __fdiv_rn(1.f, d);
            const float n0 = __fmul_rn(r0, inv), n1 = __fmul_rn(r1, inv), n2 = __fmul_rn(r2, inv);
            const float4 vp = state[3 * N + p];
            const float d0 = __fsub_rn(vp.x, w0), d1 = __fsub_rn(vp.y, w1), d2 = __fsub_rn(vp.z, w2);
            const float fn = __fmul_rn(k, pen);
            const float vn = __fadd_rn(__fadd_rn(__fmul_rn(d0, n0), __fmul_rn(d1, n1)), __fmul_rn(d2, n2));
            const float ft = __fadd_rn(fn, __fmul_rn(c, vn));
            float s0 = __fmul_rn(n0, ft), s1 = __fmul_rn(n1, ft), s2 = __fmul_rn(n2, ft);
            const float t0 = __fsub_rn(d0, __fmul_rn(n0, vn)), t1 = __fsub_rn(d1, __fmul_rn(n1, vn)),
                        t2 = __fsub_rn(d2, __fmul_rn(n2, vn));
            const float ts = sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(t0, t0), __fmul_rn(t1, t1)), __fmul_rn(t2, t2)));
            if (ts > 1e-6f) {
                const float it = __fdiv_rn(1.f, ts), fm = -__fmul_rn(mu, fn);
                s0 = __fadd_rn(s0, __fmul_rn(__fmul_rn(t0, it), fm));
                s1 = __fadd_rn(s1, __fmul_rn(__fmul_rn(t1, it), fm));
                s2 = __fadd_rn(s2, __fmul_rn(__fmul_rn(t2, it), fm));
            }
            f0 = __fadd_rn(f0, -s0);
            f1 = __fadd_rn(f1, -s1);
            f2 = __fadd_rn(f2, -s2);
            if (mforce) atomicAdd(&mforce[p], make_float4(s0, s1, s2, 0.f));
        }
        if (cfg.enable_two_way_coupling) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                f0 += __shfl_down_sync(0xFFFFFFFFu, f0, o);
                f1 += __shfl_down_sync(0xFFFFFFFFu, f1, o);
                f2 += __shfl_down_sync(0xFFFFFFFFu, f2, o);
            }
            if (lane == 0) {
                sph_force[3 * q] += f0;
                sph_force[3 * q + 1] += f1;
                sph_force[3 * q + 2] += f2;
            }
        }
    }
    // warp sums of the pair count and the energy, one atomic each per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_down_sync(0xFFFFFFFFu, cnt, o);
        e += __shfl_down_sync(0xFFFFFFFFu, e, o);
    }
    if (lane == 0) {
        if (cnt) atomicAdd(npairs, cnt);
        if (e != 0.0) atomicAdd(energy, e);
    }
}

// Per-material sums of m |v|^2 / 2 in FP64.  Up to KE_REG_MATS materials each
// thread keeps one register sum per material, and each warp adds its sums
// with one atomic per material; with more, per-block shared-memory sums take
// the particles' terms.  (One global atomic per particle on a handful of
// addresses serialises: 3 ms for 2 M particles of two materials.)
constexpr int KE_REG_MATS = 8;
constexpr int KE_SMEM_MATS = 64;
template <int MR>
__global__ void k_kinetic(const float4* __restrict__ q, const float2* __restrict__ mV, const int32_t* __restrict__ mat,
                          int64_t N, int M, double* __restrict__ out) {
    __shared__ double s_acc[KE_SMEM_MATS];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    double acc[MR > 0 ? MR : 1];
#pragma unroll
    for (int m = 0; m < (MR > 0 ? MR : 1); ++m) acc[m] = 0.0;
    if (MR == 0) {
        for (int m = threadIdx.x; m < KE_SMEM_MATS; m += blockDim.x) s_acc[m] = 0.0;
        __syncthreads();
    }
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += stride) {
        const float4 v = q[3 * N + p];
        const double ke = 0.5 * (double)mV[p].x * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
        const int id = mat ? min(max(mat[p], 0), M - 1) : 0;
        if (MR > 0) {
#pragma unroll
            for (int m = 0; m < (MR > 0 ? MR : 1); ++m) acc[m] += id == m ? ke : 0.0;
        } else if (M <= KE_SMEM_MATS) {
            atomicAdd(&s_acc[id], ke);
        } else {
            atomicAdd(&out[id], ke);
        }
    }
    if (MR > 0) {
#pragma unroll
        for (int m = 0; m < (MR > 0 ? MR : 1); ++m) {
            double e = acc[m];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xFFFFFFFFu, e, o);
            if ((threadIdx.x & 31) == 0 && e != 0.0 && m < M) atomicAdd(&out[m], e);
        }
    } else if (M <= KE_SMEM_MATS) {
        __syncthreads();
        for (int m = threadIdx.x; m < M; m += blockDim.x)
            if (s_acc[m] != 0.0) atomicAdd(&out[m], s_acc[m]);
    }
}

int nblocks(int64_t n, int t, int cap) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + t - 1) / t, cap)); }

}  // namespace

extern "C" {

int pgmpm_sph_coupling(pgmpm_solver s, const pgmpm_sph_coupling_config* cfg, const float* sph_x, const float* sph_v,
                       int64_t n_sph, float* sph_force, float* mpm_force, int64_t* n_pairs, double* energy,
                       int32_t ptr_kind, void* stream) {
    if (!s || !cfg || n_sph < 0) return fail(PGMPM_ERR_ARG, "pgmpm_sph_coupling: bad arguments");
    if (!s->uploaded) return fail(PGMPM_ERR_STATE, "no particles uploaded");
    if (s->S != 1) return fail(PGMPM_ERR_UNSUPPORTED, "pgmpm_sph_coupling: one scene");
    if (!(cfg->coupling_radius > 0.f) || !std::isfinite(cfg->coupling_radius))
        return fail(PGMPM_ERR_ARG, "pgmpm_sph_coupling: coupling_radius must be positive");
    if (n_sph > 0 && (!sph_x || !sph_v || (cfg->enable_two_way_coupling && !sph_force)))
        return fail(PGMPM_ERR_ARG, "pgmpm_sph_coupling: sph_x, sph_v (and sph_force when two-way) are required");
    if (ptr_kind != PGMPM_PTR_HOST && ptr_kind != PGMPM_PTR_DEVICE) return fail(PGMPM_ERR_ARG, "bad ptr_kind");
    DeviceGuard dg(s->device);
    cudaStream_t st = ST(stream);
    const int64_t N = s->N;
    const size_t Nz = (size_t)std::max<int64_t>(N, 1), Qz = (size_t)std::max<int64_t>(n_sph, 1);
    // the MPM side: current positions (physical order, [N][3]) for the hash
    // grid build; the pair kernel reads the state planes
    CK(s->cpl_xv.ensure(sizeof(float) * 3 * Nz));
    float* mx = s->cpl_xv.as<float>();
    if (N > 0) k_state_xv<<<nblocks(N, 256, 148 * 16), 256, 0, st>>>(s->q.as<float4>(), N, mx, nullptr);
    CK(cudaGetLastError());
    // the SPH side on the device
    const float *dsx = sph_x, *dsv = sph_v;
    float* dsf = sph_force;
    float* dmf = mpm_force;
    if (ptr_kind == PGMPM_PTR_HOST) {
        CK(s->cpl_stage.ensure(sizeof(float) * (9 * Qz + 3 * Nz)));
        float* b = s->cpl_stage.as<float>();
        if (n_sph > 0) {
            CK(cudaMemcpyAsync(b, sph_x, sizeof(float) * 3 * n_sph, cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(b + 3 * Qz, sph_v, sizeof(float) * 3 * n_sph, cudaMemcpyHostToDevice, st));
            if (cfg->enable_two_way_coupling)
                CK(cudaMemcpyAsync(b + 6 * Qz, sph_force, sizeof(float) * 3 * n_sph, cudaMemcpyHostToDevice, st));
        }
        dsx = b;
        dsv = b + 3 * Qz;
        dsf = b + 6 * Qz;
        dmf = mpm_force ? b + 9 * Qz : nullptr;
    }
    float4* mf = nullptr;  // the solid forces, physical order
    if (dmf && N > 0) {
        CK(s->cpl_mf.ensure(sizeof(float4) * Nz));
        mf = s->cpl_mf.as<float4>();
        CK(cudaMemsetAsync(mf, 0, sizeof(float4) * N, st));
    }
    CK(s->cpl_acc.ensure(sizeof(double) * 2));
    CK(cudaMemsetAsync(s->cpl_acc.p, 0, sizeof(double) * 2, st));
    unsigned long long* d_pairs = s->cpl_acc.as<unsigned long long>();
    double* d_energy = s->cpl_acc.as<double>() + 1;
    if (N > 0 && n_sph > 0) {
        // candidates: the MPM particles of the hash cells within one radius
        // of each SPH particle, over the scene's domain.  Cells of half a
        // radius (125 around a particle) hold 42% fewer candidates than cells
        // of one radius (27), unless that makes more than 4 cells per MPM
        // particle (or 2^20, if more).
        const pgmpm_scene_desc& d = s->desc[0];
        float lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
            lo[a] = d.origin[a];
            hi[a] = d.origin[a] + (float)(d.n[a] - 1) * d.dx;
        }
        double cells_half = 1.0;
        for (int a = 0; a < 3; ++a) cells_half *= std::ceil((hi[a] - lo[a]) / (0.5 * cfg->coupling_radius));
        const float cell = cells_half <= std::max(4.0 * (double)N, (double)(1 << 20)) ? 0.5f * cfg->coupling_radius
                                                                                      : cfg->coupling_radius;
        if (!s->cpl_grid || s->cpl_cell != cell || s->cpl_cap < N) {
            if (s->cpl_grid) pgmpm_hashgrid_destroy(s->cpl_grid);
            s->cpl_grid = nullptr;
            int rc = pgmpm_hashgrid_create(cell, lo, hi, N, s->device, &s->cpl_grid);
            if (rc) return rc;
            s->cpl_cell = cell;
            s->cpl_cap = N;
        }
        int rc = pgmpm_hashgrid_build(s->cpl_grid, mx, N, PGMPM_PTR_DEVICE, stream);
        if (rc) return rc;
        CK(s->cpl_off.ensure(sizeof(int64_t) * (Qz + 1)));
        int64_t total = 0;
        rc = pgmpm_hashgrid_neighbors(s->cpl_grid, dsx, n_sph, cfg->coupling_radius, s->cpl_off.as<int64_t>(),
                                      nullptr, 0, &total, PGMPM_PTR_DEVICE, stream);
        if (rc) return rc;
        CK(s->cpl_idx.ensure(sizeof(uint32_t) * (size_t)std::max<int64_t>(total, 1)));
        rc = pgmpm_hashgrid_neighbors(s->cpl_grid, dsx, n_sph, cfg->coupling_radius, s->cpl_off.as<int64_t>(),
                                      s->cpl_idx.as<uint32_t>(), total, &total, PGMPM_PTR_DEVICE, stream);
        if (rc) return rc;
        k_sph_pairs<<<nblocks(n_sph * 32, 256, 148 * 16), 256, 0, st>>>(
            dsx, dsv, n_sph, s->cpl_off.as<int64_t>(), s->cpl_idx.as<uint32_t>(), s->q.as<float4>(), N, *cfg, dsf, mf,
            d_pairs, d_energy);
        CK(cudaGetLastError());
    }
    if (mf)
        k_mforce_out<<<nblocks(N, 256, 148 * 16), 256, 0, st>>>(mf, s->user_of_phys.as<uint32_t>(), N, dmf);
    CK(cudaGetLastError());
    if (ptr_kind == PGMPM_PTR_HOST) {
        if (cfg->enable_two_way_coupling && n_sph > 0)
            CK(cudaMemcpyAsync(sph_force, dsf, sizeof(float) * 3 * n_sph, cudaMemcpyDeviceToHost, st));
        if (mpm_force && N > 0) CK(cudaMemcpyAsync(mpm_force, dmf, sizeof(float) * 3 * N, cudaMemcpyDeviceToHost, st));
    }
    unsigned long long h_pairs = 0;
    double h_energy = 0.0;
    CK(cudaMemcpyAsync(&h_pairs, d_pairs, sizeof(h_pairs), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&h_energy, d_energy, sizeof(h_energy), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (n_pairs) *n_pairs = (int64_t)h_pairs;
    if (energy) *energy = h_energy;
    return PGMPM_OK;
}

int pgmpm_kinetic_energy(pgmpm_solver s, double* per_material, double* total, void* stream) {
    if (!s) return fail(PGMPM_ERR_ARG, "null solver");
    if (!s->uploaded) return fail(PGMPM_ERR_STATE, "no particles uploaded");
    DeviceGuard dg(s->device);
    cudaStream_t st = ST(stream);
    const int M = s->M;
    CK(s->cpl_acc.ensure(sizeof(double) * std::max(2, M)));
    CK(cudaMemsetAsync(s->cpl_acc.p, 0, sizeof(double) * M, st));
    if (s->N > 0) {
        const int nb = nblocks(s->N, 256, 148 * 8);
        const int32_t* mt = s->pf.multi_mat ? s->mat.as<int32_t>() : nullptr;
        if (!mt)
            k_kinetic<1><<<nb, 256, 0, st>>>(s->q.as<float4>(), s->mV.as<float2>(), nullptr, s->N, M,
                                             s->cpl_acc.as<double>());
        else if (M <= 2)
            k_kinetic<2><<<nb, 256, 0, st>>>(s->q.as<float4>(), s->mV.as<float2>(), mt, s->N, M,
                                             s->cpl_acc.as<double>());
        else if (M <= KE_REG_MATS)
            k_kinetic<KE_REG_MATS><<<nb, 256, 0, st>>>(s->q.as<float4>(), s->mV.as<float2>(), mt, s->N, M,
                                                       s->cpl_acc.as<double>());
        else
            k_kinetic<0><<<nb, 256, 0, st>>>(s->q.as<float4>(), s->mV.as<float2>(), mt, s->N, M,
                                             s->cpl_acc.as<double>());
    }
    CK(cudaGetLastError());
    std::vector<double> h(M);
    CK(cudaMemcpyAsync(h.data(), s->cpl_acc.p, sizeof(double) * M, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double t = 0.0;
    for (int i = 0; i < M; ++i) {
        if (per_material) per_material[i] = h[i];
        t += h[i];
    }
    if (total) *total = t;
    return PGMPM_OK;
}

}  // extern "C"
