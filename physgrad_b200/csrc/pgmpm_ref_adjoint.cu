// pgmpm_ref_adjoint.cu -- reverse of one REF_COMPAT step (the reference's PIC
// step, src/material_point_method.h:479-666) for launch_mpm_timestep_backward
// (src/pytorch_autograd.cu:384-402).
//
// Forward (per particle p, node i, REF weights w_pi of x_p, thresholded at
// 1e-10 and cut at the grid bounds):
//   m_i = sum_p w m_p,  P_i = sum_p w m_p v_p
//   v_i = (P_i + m_i g dt) / m_i = P_i / m_i + g dt     (m_i > 1e-10, else 0)
//   v'_p = sum_i w v_i,  x'_p = x_p + dt v'_p
// Reverse, given gx' = dL/dx', gv' = dL/dv':
//   1. k_ref_adj_scatter  a_p = gv' + dt gx';  Gv_i += w a_p
//   2. k_ref_adj_grid     gP_i = Gv_i / m_i, gm_i = -Gv_i . (P_i / m_i) / m_i,
//                         dL/dg += dt sum_i Gv_i
//   3. k_ref_adj_gather   dL/dx = gx' + sum_i grad w (a_p . v_i + m_p gm_i + m_p gP_i . v_p)
//                         dL/dv = sum_i w m_p gP_i
//                         dL/dm = sum_i w (gm_i + gP_i . v_p)
// Particles are read in the caller's order (upload order); the grid is the
// solver's tiled grid after the recomputed forward step.
#include <algorithm>

#include "pgmpm_internal.h"

namespace pgmpm {
namespace {

// d/dr of the reference quadratic B-spline (ref_quadratic)
__device__ __forceinline__ float ref_quadratic_d(float r) {
    const float a = r < 0.f ? -r : r;
    if (a >= 1.5f) return 0.f;
    if (a < 0.5f) return -2.f * r;
    const float t = 1.5f - a;
    return r < 0.f ? t : -t;
}

// REF stencil of x with the weight derivatives (d/dx, per axis and node)
struct RefStencil {
    Stencil st;
    float dw[3][3];
};

__device__ __forceinline__ void ref_stencil(const SceneDev& sc, const float x[3], RefStencil& r, uint32_t& flags) {
    make_stencil<PHYS_REF>(sc, x, r.st, flags);
    const float idx = 1.f / sc.dx;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int k = 0; k < 3; ++k) r.dw[a][k] = ref_quadratic_d(r.st.f[a] - (float)(k - 1)) * idx;
}

__global__ void k_ref_adj_scatter(View V, const float* __restrict__ x, const float* __restrict__ gx,
                                  const float* __restrict__ gv, float4* __restrict__ G, int64_t n) {
    const SceneDev& sc = V.scenes[0];
    uint32_t flags = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
        const float xp[3] = {x[3 * p], x[3 * p + 1], x[3 * p + 2]};
        Stencil st;
        make_stencil<PHYS_REF>(sc, xp, st, flags);
        float a[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) a[c] = gv[3 * p + c] + sc.dt * gx[3 * p + c];
#pragma unroll
        for (int ii = 0; ii < 3; ++ii) {
            const int gi = st.b[0] + ii;
            if (gi < 0 || gi >= sc.n[0]) continue;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const int gj = st.b[1] + j;
                if (gj < 0 || gj >= sc.n[1]) continue;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const int gk = st.b[2] + k;
                    if (gk < 0 || gk >= sc.n[2]) continue;
                    const float w = __fmul_rn(__fmul_rn(st.w[0][ii], st.w[1][j]), st.w[2][k]);
                    if (!(w > 1e-10f)) continue;
                    float* g = reinterpret_cast<float*>(&G[node_index(sc, gi, gj, gk)]);
                    atomicAdd(g, w * a[0]);
                    atomicAdd(g + 1, w * a[1]);
                    atomicAdd(g + 2, w * a[2]);
                }
            }
        }
    }
}

// over the step's active node tiles (the only nodes a stencil reaches)
__global__ void k_ref_adj_grid(View V, float4* __restrict__ G, float* __restrict__ ggrav) {
    const SceneDev& sc = V.scenes[0];
    const uint32_t count = V.counters[CNT_TILES];
    const int tiles_per_block = blockDim.x >> 6;
    const int l = threadIdx.x & 63;
    float acc[3] = {0.f, 0.f, 0.f};
    for (uint32_t w = blockIdx.x * tiles_per_block + (threadIdx.x >> 6); w < count;
         w += gridDim.x * tiles_per_block) {
        const uint32_t nt = V.tile_list[w];
        if (nt >= (uint32_t)V.total_nt) continue;
        const int64_t idx = ((int64_t)nt << 6) + l;
        const float4 g = G[idx];
        const float4 vm = V.grid_v[idx];  // (v, m) of the forward step
        float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
        if (vm.w > 1e-10f) {
            const float im = 1.f / vm.w;
            const float pm0 = vm.x - sc.gravity[0] * sc.dt, pm1 = vm.y - sc.gravity[1] * sc.dt,
                        pm2 = vm.z - sc.gravity[2] * sc.dt;  // P / m
            out = make_float4(g.x * im, g.y * im, g.z * im, -(g.x * pm0 + g.y * pm1 + g.z * pm2) * im);
            acc[0] += g.x;
            acc[1] += g.y;
            acc[2] += g.z;
        }
        G[idx] = out;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float s = acc[c] * sc.dt;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, o);
        if (ggrav && (threadIdx.x & 31) == 0 && s != 0.f) atomicAdd(&ggrav[c], s);
    }
}

__global__ void k_ref_adj_gather(View V, const float* __restrict__ x, const float* __restrict__ v,
                                 const float* __restrict__ m, const float* __restrict__ gx,
                                 const float* __restrict__ gv, const float4* __restrict__ G,
                                 float* __restrict__ gx_in, float* __restrict__ gv_in, float* __restrict__ gm_in,
                                 int64_t n) {
    const SceneDev& sc = V.scenes[0];
    uint32_t flags = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
        const float xp[3] = {x[3 * p], x[3 * p + 1], x[3 * p + 2]};
        const float vp[3] = {v[3 * p], v[3 * p + 1], v[3 * p + 2]};
        const float mp = m[p];
        RefStencil r;
        ref_stencil(sc, xp, r, flags);
        float a[3], ox[3], ov[3] = {0.f, 0.f, 0.f}, om = 0.f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            ox[c] = gx[3 * p + c];
            a[c] = gv[3 * p + c] + sc.dt * ox[c];
        }
#pragma unroll
        for (int ii = 0; ii < 3; ++ii) {
            const int gi = r.st.b[0] + ii;
            if (gi < 0 || gi >= sc.n[0]) continue;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const int gj = r.st.b[1] + j;
                if (gj < 0 || gj >= sc.n[1]) continue;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const int gk = r.st.b[2] + k;
                    if (gk < 0 || gk >= sc.n[2]) continue;
                    const float wx = r.st.w[0][ii], wy = r.st.w[1][j], wz = r.st.w[2][k];
                    const float w = __fmul_rn(__fmul_rn(wx, wy), wz);
                    if (!(w > 1e-10f)) continue;
                    const int64_t idx = node_index(sc, gi, gj, gk);
                    const float4 vi = V.grid_v[idx];
                    const float4 g = G[idx];  // (gP, gm)
                    const float gPv = g.x * vp[0] + g.y * vp[1] + g.z * vp[2];
                    const float s = a[0] * vi.x + a[1] * vi.y + a[2] * vi.z + mp * (g.w + gPv);
                    ox[0] += r.dw[0][ii] * wy * wz * s;
                    ox[1] += wx * r.dw[1][j] * wz * s;
                    ox[2] += wx * wy * r.dw[2][k] * s;
                    ov[0] += w * mp * g.x;
                    ov[1] += w * mp * g.y;
                    ov[2] += w * mp * g.z;
                    om += w * (g.w + gPv);
                }
            }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (gx_in) gx_in[3 * p + c] = ox[c];
            if (gv_in) gv_in[3 * p + c] = ov[c];
        }
        if (gm_in) gm_in[p] = om;
    }
}

inline int blocks_for(int64_t n, int block) {
    int64_t g = (n + block - 1) / block;
    return (int)(g < 1 ? 1 : (g > 148 * 64 ? 148 * 64 : g));
}

}  // namespace

cudaError_t launch_ref_adjoint(const View& V, const float* x, const float* v, const float* m, const float* gx,
                               const float* gv, float4* G, float* gx_in, float* gv_in, float* gm_in, float* ggrav,
                               int num_sms, cudaStream_t st) {
    if (V.N == 0) return cudaSuccess;
    k_ref_adj_scatter<<<blocks_for(V.N, 256), 256, 0, st>>>(V, x, gx, gv, G, V.N);
    int nb = (int)std::min<int64_t>(((int64_t)V.total_nt + 3) / 4, (int64_t)num_sms * 8);
    k_ref_adj_grid<<<nb < 1 ? 1 : nb, 256, 0, st>>>(V, G, ggrav);
    k_ref_adj_gather<<<blocks_for(V.N, 256), 256, 0, st>>>(V, x, v, m, gx, gv, G, gx_in, gv_in, gm_in, V.N);
    return cudaGetLastError();
}

}  // namespace pgmpm
