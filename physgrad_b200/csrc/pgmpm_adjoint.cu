// pgmpm_adjoint.cu -- reverse-mode kernels of one MLS-MPM step.
//
// Forward step (per particle p, node i, weights w_pi of x_p):
//   P2G   m_i = sum w m_p,  p_i = sum w (m_p v_p + A_p d_i),  d_i = x_i - x_p,
//         A_p = -dt V0_p D tau(F_p) + m_p C_p
//   grid  vpre_i = p_i/m_i + dt g,  v_i = walls(vpre_i)
//   G2P   v'_p = sum w v_i,  C'_p = D sum w v_i d_i^T,  F'_p = (I + dt C') F,
//         x'_p = x_p + dt v'_p   (fluid: F' = cbrt(det F') I)
// Reverse, given the adjoint of (x', v', C', F'):
//   1. scatter (k_p2g_tiles, MODE_ADJ): gv_i += w (gv' + dt gx' + D gC d_i)
//      with gC = gC' + dt gF'raw F^T   -- the "cell-sorted scatter"
//   2. k_adj_grid: walls^T, gp_i = gv_i / m_i, gm_i = -gv_i . (p_i/m_i) / m_i
//   3. k_adj_gather: per particle, gather v_i, gp_i, gm_i over the stencil and
//      form gx, gv, gC, gF (with the stress adjoint) and dL/dE -- the gather
//      that is the reverse of P2G.
#include "pgmpm_internal.h"

namespace pgmpm {
namespace {

__device__ __forceinline__ const SceneDev& scene_ref(const View& V, int s) { return V.scenes[s]; }

__global__ void k_adj_grid(View V, AdjView A) {
    // the scatter has finished with the work cursor: leave it at zero, as the
    // forward's grid update does, so that a later replay of this step that
    // keeps its recorded sort (no counter reset) starts its P2G from zero
    if (blockIdx.x == 0 && threadIdx.x == 0) V.counters[CNT_P2G_CURSOR] = 0u;
    const uint32_t count = V.counters[CNT_TILES];
    const int tiles_per_block = blockDim.x >> 6;
    const int l = threadIdx.x & 63;
    for (uint32_t w = blockIdx.x * tiles_per_block + (threadIdx.x >> 6); w < count;
         w += gridDim.x * tiles_per_block) {
        const uint32_t nt = V.tile_list[w];
        if (nt >= (uint32_t)V.total_nt) continue;
        const int s = V.S == 1 ? 0 : scene_of_node_tile(V.scenes, V.S, (int)nt);
        const SceneDev& sc = scene_ref(V, s);
        const int lt = (int)nt - sc.nt_base;
        const int i = 4 * (lt % sc.nt[0]) + (l & 3);
        const int j = 4 * ((lt / sc.nt[0]) % sc.nt[1]) + ((l >> 2) & 3);
        const int k = 4 * (lt / (sc.nt[0] * sc.nt[1])) + (l >> 4);
        const int64_t idx = ((int64_t)nt << 6) + l;
        const float4 g = A.grid_gv[idx];
        const float4 vp = V.grid_vpre[idx];
        float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
        if (vp.w > 0.f) {
            float gv[3] = {g.y, g.z, g.w};
            float v[3] = {vp.x, vp.y, vp.z};
            const uint32_t zeroed = apply_bc(sc, i, j, k, v);
#pragma unroll
            for (int a = 0; a < 3; ++a)
                if (zeroed & (1u << a)) gv[a] = 0.f;
            const float im = 1.f / vp.w;
            const float pm0 = vp.x - sc.dt * sc.gravity[0], pm1 = vp.y - sc.dt * sc.gravity[1],
                        pm2 = vp.z - sc.dt * sc.gravity[2];
            out = make_float4(gv[0] * im, gv[1] * im, gv[2] * im, -(gv[0] * pm0 + gv[1] * pm1 + gv[2] * pm2) * im);
        }
        A.grid_gpm[idx] = out;
        A.grid_gv[idx] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

constexpr int GATHER_T = 128;
constexpr int MAX_SMEM_MATS = 64;

template <bool MULTI, bool FLUID>
__global__ void __launch_bounds__(GATHER_T, 3) k_adj_gather(View V, AdjView A) {
    __shared__ float sE[MAX_SMEM_MATS];
    const bool smem_e = V.M <= MAX_SMEM_MATS;
    for (int m = threadIdx.x; m < MAX_SMEM_MATS; m += blockDim.x) sE[m] = 0.f;
    __syncthreads();
    const int64_t N = V.N;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    uint32_t flags = 0;
    // particles in physical order (the order of the state planes)
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += stride) {
        const int s = V.S == 1 ? 0 : scene_of_particle(V.scenes, V.S, (int)p);
        const SceneDev& sc = scene_ref(V, s);
        const int mid = MULTI ? V.mat[p] : 0;
        const MatDev mt = V.mats[mid];
        float x[3], F[9], v[3], C[9], Cn[9], vdum[3];
        unpack_xF(V.q[p], V.q[N + p], V.q[2 * N + p], x, F);
        unpack_vC(V.q[3 * N + p], V.q[4 * N + p], V.q[5 * N + p], v, C);
        unpack_vC(A.q_next[3 * N + p], A.q_next[4 * N + p], A.q_next[5 * N + p], vdum, Cn);
        float gx[3], gF[9], gv[3], gC[9];
        unpack_xF(A.g[p], A.g[N + p], A.g[2 * N + p], gx, gF);
        unpack_vC(A.g[3 * N + p], A.g[4 * N + p], A.g[5 * N + p], gv, gC);
        const float2 mv = V.mV[p];
        const float m = mv.x;
        Stencil st;
        make_stencil<PHYS_MLS>(sc, x, st, flags);
        float dw[3][3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            mls_dweights(st.f[a], dw[a]);
            // a clamped (escaped) coordinate has zero weight derivative
            const float raw = __fsub_rn(__fmul_rn(__fsub_rn(x[a], sc.origin[a]), sc.inv_dx), (float)st.s[a]);
            if (raw < 0.5f || raw > 1.5f) dw[a][0] = dw[a][1] = dw[a][2] = 0.f;
        }
        // adjoint through the fluid reset and the F update
        float M[9];
#pragma unroll
        for (int a = 0; a < 9; ++a) M[a] = sc.dt * Cn[a] + ((a % 4 == 0) ? 1.f : 0.f);
        if (FLUID && mt.model == MODEL_EOS) {
            float Fr[9], cof[9];
            m3_mul(M, F, Fr);
            m3_cof(Fr, cof);
            const float J = Fr[0] * cof[0] + Fr[1] * cof[1] + Fr[2] * cof[2];
            const float c = cbrtf(J) / (3.f * J) * (gF[0] + gF[4] + gF[8]);
#pragma unroll
            for (int a = 0; a < 9; ++a) gF[a] = c * cof[a];
        }
        float gvt[3], gCt[9], gFFt[9];
        m3_mulT(gF, F, gFFt);
#pragma unroll
        for (int a = 0; a < 3; ++a) gvt[a] = gv[a] + sc.dt * gx[a];
#pragma unroll
        for (int a = 0; a < 9; ++a) gCt[a] = gC[a] + sc.dt * gFFt[a];
        // forward affine matrix (R kept for the stress adjoint)
        float tau[9], Am[9], R[9];
        kirchhoff<true>(F, mt, tau, R);
        if (FLUID) add_viscous(F, C, mt, tau);
        const float kk = -sc.dt * mv.y * sc.D;
#pragma unroll
        for (int a = 0; a < 9; ++a) Am[a] = kk * tau[a] + m * C[a];
        const float dx = sc.dx, D = sc.D, idx_ = 1.f / dx;
        // Per node i (offset o, d_i = (o - f) dx, weight w_i, gradient gw_i):
        //   wb_i = m gm_i + v_i . (gvt + D gCt d_i) + gp_i . (m v + Am d_i)
        //   gx  += wb_i gw_i - w_i (D gCt^T v_i + Am^T gp_i)
        //   gv  += w_i m gp_i,   Ab += w_i gp_i d_i^T
        // The bracketed vectors are affine in o: they start at o = 0 and
        // advance by one matrix column per node step.  The second gx term,
        // gv and Ab need only sum w v, sum w gp and sum w gp o^T.
        float Gp[9], Ap[9];  // dx D gCt, dx Am (gCt and Am are not needed past this point)
#pragma unroll
        for (int a = 0; a < 9; ++a) {
            Gp[a] = dx * D * gCt[a];
            Ap[a] = dx * Am[a];
        }
        // F' = M F  ->  gF_in = M^T gF'raw (the stress adjoint adds to it after the loop)
        float oF[9];
        m3_Tmul(M, gF, oF);
        float b1[3], b2[3];  // at o = 0: gvt - Gp f,  m v - Ap f
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            b1[a] = gvt[a] - (Gp[3 * a] * st.f[0] + Gp[3 * a + 1] * st.f[1] + Gp[3 * a + 2] * st.f[2]);
            b2[a] = m * v[a] - (Ap[3 * a] * st.f[0] + Ap[3 * a + 1] * st.f[1] + Ap[3 * a + 2] * st.f[2]);
        }
        // separable tiled node index: idx = X[i] + Y[j] + Z[k]
        int X[3], Y[3], Z[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int gi = st.s[0] + a, gj = st.s[1] + a, gk = st.s[2] + a;
            X[a] = ((gi >> 2) << 6) + (gi & 3);
            Y[a] = (gj >> 2) * (sc.nt[0] << 6) + ((gj & 3) << 2);
            Z[a] = (gk >> 2) * ((sc.nt[0] * sc.nt[1]) << 6) + ((gk & 3) << 4) + (sc.nt_base << 6);
        }
        // The node loop keeps the x, y components of its 3-vectors as float2
        // pairs and z alone.  In wb = v . h1 + gp . h2 + m gm the loaded
        // (v_z, m_i) and (gp_z, gm_i) pairs meet (h1_z, 0) and (h2_z, m), so
        // wb is four pair operations and one add.
        const float2 G0a = make_float2(Gp[0], Gp[3]), G0b = make_float2(Gp[6], 0.f);  // Gp column 0
        const float2 A0a = make_float2(Ap[0], Ap[3]), A0b = make_float2(Ap[6], 0.f);  // Ap column 0
        float ox[3] = {gx[0], gx[1], gx[2]};
        // sums over the stencil: (x, y) pairs and z scalars
        float2 SWva = f2(0.f), SWga = f2(0.f), Sg0a = f2(0.f), Sg1a = f2(0.f), Sg2a = f2(0.f);
        float SWvz = 0.f, SWgz = 0.f, Sg0z = 0.f, Sg1z = 0.f, Sg2z = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const float fj = (float)j, fk = (float)k;
                float2 H1a = make_float2(b1[0] + fj * Gp[1] + fk * Gp[2], b1[1] + fj * Gp[4] + fk * Gp[5]);
                float2 H1b = make_float2(b1[2] + fj * Gp[7] + fk * Gp[8], 0.f);
                float2 H2a = make_float2(b2[0] + fj * Ap[1] + fk * Ap[2], b2[1] + fj * Ap[4] + fk * Ap[5]);
                float2 H2b = make_float2(b2[2] + fj * Ap[7] + fk * Ap[8], m);
                float P0 = 0.f, P1 = 0.f;
                float2 RVa = f2(0.f), RGa = f2(0.f), RXa = f2(0.f);
                float RVz = 0.f, RGz = 0.f, RXz = 0.f;
                const int row = Y[j] + Z[k];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const int64_t n = (int64_t)(row + X[i]);
                    const float4 vi = __ldg(&V.grid_v[n]);
                    const float4 gpm = A.grid_gpm[n];
                    const float2 Va = make_float2(vi.x, vi.y), Vb = make_float2(vi.z, vi.w);
                    const float2 Ga = make_float2(gpm.x, gpm.y), Gb = make_float2(gpm.z, gpm.w);
                    float2 wb2 = f2_mul(Va, H1a);
                    wb2 = f2_fma(Vb, H1b, wb2);
                    wb2 = f2_fma(Ga, H2a, wb2);
                    wb2 = f2_fma(Gb, H2b, wb2);
                    const float wb = wb2.x + wb2.y;
                    const float wx = st.w[0][i];
                    const float2 W = f2(wx);
                    P0 += dw[0][i] * wb;
                    P1 += wx * wb;
                    RVa = f2_fma(W, Va, RVa);
                    RVz += wx * vi.z;
                    const float2 Ta = f2_mul(W, Ga);
                    const float Tz = wx * gpm.z;
                    RGa = f2_add(RGa, Ta);
                    RGz += Tz;
                    if (i) {
                        RXa = f2_fma(f2((float)i), Ta, RXa);
                        RXz += (float)i * Tz;
                    }
                    if (i < 2) {
                        H1a = f2_add(H1a, G0a);
                        H1b = f2_add(H1b, G0b);
                        H2a = f2_add(H2a, A0a);
                        H2b = f2_add(H2b, A0b);
                    }
                }
                const float wyz = st.w[1][j] * st.w[2][k];
                const float R0 = wyz * idx_, R1 = dw[1][j] * st.w[2][k] * idx_, R2 = st.w[1][j] * dw[2][k] * idx_;
                ox[0] += P0 * R0;
                ox[1] += P1 * R1;
                ox[2] += P1 * R2;
                const float2 WYZ = f2(wyz);
                SWva = f2_fma(WYZ, RVa, SWva);
                SWvz += wyz * RVz;
                SWga = f2_fma(WYZ, RGa, SWga);
                SWgz += wyz * RGz;
                Sg0a = f2_fma(WYZ, RXa, Sg0a);
                Sg0z += wyz * RXz;
                if (j) {
                    const float jw = fj * wyz;
                    Sg1a = f2_fma(f2(jw), RGa, Sg1a);
                    Sg1z += jw * RGz;
                }
                if (k) {
                    const float kw = fk * wyz;
                    Sg2a = f2_fma(f2(kw), RGa, Sg2a);
                    Sg2z += kw * RGz;
                }
            }
        }
        const float SWv[3] = {SWva.x, SWva.y, SWvz}, SWg[3] = {SWga.x, SWga.y, SWgz};
        const float Sg[3][3] = {{Sg0a.x, Sg0a.y, Sg0z}, {Sg1a.x, Sg1a.y, Sg1z}, {Sg2a.x, Sg2a.y, Sg2z}};
        float ogv[3], Ab[9];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            // D gCt^T sum(w v) + Am^T sum(w gp), from Gp = dx D gCt and Ap = dx Am
            const float t1 = Gp[a] * SWv[0] + Gp[3 + a] * SWv[1] + Gp[6 + a] * SWv[2];
            const float t2 = Ap[a] * SWg[0] + Ap[3 + a] * SWg[1] + Ap[6 + a] * SWg[2];
            ox[a] -= (t1 + t2) * idx_;
            ogv[a] = m * SWg[a];
#pragma unroll
            for (int bb = 0; bb < 3; ++bb) Ab[3 * a + bb] = dx * (Sg[bb][a] - SWg[a] * st.f[bb]);
        }
        // plus the stress adjoint
        float tb[9];
#pragma unroll
        for (int a = 0; a < 9; ++a) tb[a] = kk * Ab[a];
        const float dE = kirchhoff_adjoint(F, R, mt, tb, oF);
        float oC[9];
#pragma unroll
        for (int a = 0; a < 9; ++a) oC[a] = m * Ab[a];
        if (FLUID) add_viscous_adjoint(F, C, mt, tb, oF, oC);
        float4 g0, g1, g2, g3, g4, g5;
        pack_xF(ox, oF, g0, g1, g2);
        pack_vC(ogv, oC, g3, g4, g5);
        A.g[p] = g0;
        A.g[N + p] = g1;
        A.g[2 * N + p] = g2;
        A.g[3 * N + p] = g3;
        A.g[4 * N + p] = g4;
        A.g[5 * N + p] = g5;
        if (smem_e) {
            // lanes of one material combine before one shared atomic
            const unsigned peers = __match_any_sync(__activemask(), mid);
            const float e = dE;
            const int leader = __ffs(peers) - 1;
            // every peer reads every peer's value; the leader adds the sum once
            float sum = 0.f;
            unsigned rest = peers;
            while (rest) {
                const int src = __ffs(rest) - 1;
                rest &= rest - 1;
                sum += __shfl_sync(peers, e, src);
            }
            if ((int)(threadIdx.x & 31) == leader) atomicAdd(&sE[mid], sum);
        } else {
            atomicAdd(&A.gE[mid], dE);
        }
    }
    __syncthreads();
    if (smem_e)
        for (int m = threadIdx.x; m < V.M; m += blockDim.x)
            if (sE[m] != 0.f) atomicAdd(&A.gE[m], sE[m]);
    if (flags) atomicOr(&V.counters[CNT_FLAGS], flags);
}

__global__ void k_state_to_planes(const float* __restrict__ x, const float* __restrict__ v,
                                  const float* __restrict__ C, const float* __restrict__ F,
                                  const uint32_t* __restrict__ user_of_phys, float4* __restrict__ g, int64_t N) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
        const int64_t u = user_of_phys[i];
        if (u >= N) continue;
        float xx[3], vv[3], CC[9], FF[9];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            xx[a] = x ? x[3 * u + a] : 0.f;
            vv[a] = v ? v[3 * u + a] : 0.f;
        }
#pragma unroll
        for (int a = 0; a < 9; ++a) {
            CC[a] = C ? C[9 * u + a] : 0.f;
            FF[a] = F ? F[9 * u + a] : 0.f;
        }
        float4 o0, o1, o2, o3, o4, o5;
        pack_xF(xx, FF, o0, o1, o2);
        pack_vC(vv, CC, o3, o4, o5);
        g[i] = o0;
        g[N + i] = o1;
        g[2 * N + i] = o2;
        g[3 * N + i] = o3;
        g[4 * N + i] = o4;
        g[5 * N + i] = o5;
    }
}

__global__ void k_planes_to_state(const float4* __restrict__ g, const uint32_t* __restrict__ phys_of_user,
                                  float* __restrict__ x, float* __restrict__ v, float* __restrict__ C,
                                  float* __restrict__ F, int64_t N) {
    // upload order: contiguous writes of the caller's records, gathered planes
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < N; u += stride) {
        const int64_t i = phys_of_user[u];
        if (i >= N) continue;
        float xx[3], FF[9], vv[3], CC[9];
        unpack_xF(g[i], g[N + i], g[2 * N + i], xx, FF);
        unpack_vC(g[3 * N + i], g[4 * N + i], g[5 * N + i], vv, CC);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (x) x[3 * u + a] = xx[a];
            if (v) v[3 * u + a] = vv[a];
        }
#pragma unroll
        for (int a = 0; a < 9; ++a) {
            if (C) C[9 * u + a] = CC[a];
            if (F) F[9 * u + a] = FF[a];
        }
    }
}

inline int blocks_for(int64_t n, int block) {
    int64_t g = (n + block - 1) / block;
    return (int)(g < 1 ? 1 : (g > 148 * 64 ? 148 * 64 : g));
}

}  // namespace

cudaError_t launch_adj_grid(const View& V, const AdjView& A, const Tuning& t, int num_sms, cudaStream_t st) {
    if (V.N == 0) return cudaSuccess;
    const int tiles_per_block = t.grid_block / 64;
    int64_t nb = ((int64_t)V.total_nt + tiles_per_block - 1) / tiles_per_block;
    if (nb > num_sms * 8) nb = num_sms * 8;
    if (nb < 1) nb = 1;
    k_adj_grid<<<(int)nb, t.grid_block, 0, st>>>(V, A);
    return cudaGetLastError();
}

cudaError_t launch_adj_gather(const View& V, const AdjView& A, const PhysFlags& pf, const Tuning& t,
                              cudaStream_t st) {
    (void)t;
    if (V.N == 0) return cudaSuccess;
    const int nb = blocks_for(V.N, GATHER_T);
    if (pf.multi_mat) {
        if (pf.has_fluid)
            k_adj_gather<true, true><<<nb, GATHER_T, 0, st>>>(V, A);
        else
            k_adj_gather<true, false><<<nb, GATHER_T, 0, st>>>(V, A);
    } else {
        if (pf.has_fluid)
            k_adj_gather<false, true><<<nb, GATHER_T, 0, st>>>(V, A);
        else
            k_adj_gather<false, false><<<nb, GATHER_T, 0, st>>>(V, A);
    }
    return cudaGetLastError();
}

cudaError_t launch_state_to_planes(const float* x, const float* v, const float* C, const float* F,
                                   const uint32_t* user_of_phys, float4* g, int64_t N, cudaStream_t st) {
    if (N == 0) return cudaSuccess;
    k_state_to_planes<<<blocks_for(N, 256), 256, 0, st>>>(x, v, C, F, user_of_phys, g, N);
    return cudaGetLastError();
}

cudaError_t launch_planes_to_state(const float4* g, const uint32_t* phys_of_user, float* x, float* v, float* C,
                                   float* F, int64_t N, cudaStream_t st) {
    if (N == 0) return cudaSuccess;
    k_planes_to_state<<<blocks_for(N, 256), 256, 0, st>>>(g, phys_of_user, x, v, C, F, N);
    return cudaGetLastError();
}

}  // namespace pgmpm
