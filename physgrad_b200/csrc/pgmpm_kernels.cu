// pgmpm_kernels.cu -- the forward MLS-MPM step on sm_100a.
//
// Per step (all on one stream, captured as one CUDA graph):
//   [sort]   bin sort of the cell keys written by the previous G2P
//            (pgmpm_sort.cu): occupied cell tiles, their sorted ranges, each
//            cell's range, and the active node tiles
//   P2G      default k_p2g_cells: one 64-thread block per occupied 4^3 cell
//            tile, thread c owns cell c and the 27 nodes of its stencil (108
//            register accumulators), walks its cell's particles and adds the
//            payload (m, b, affine matrix, stencil fraction) precomputed by
//            the previous G2P; the block then sums the 6^3 nodes the tile
//            touches in shared memory and flushes each with one vector atomic
//            (red.global.add.v4.f32) into grid_mp.  k_p2g_tiles (cell x
//            z-slice) and k_p2g (chunks, shared atomics) are the other
//            variants.
//   k_grid   active node tiles only: v = p/m + dt g, walls, (v, m) -> grid_v,
//            grid_mp cleared for the next step.
//   G2P      default k_g2p_phys: one thread per particle in physical order:
//            27-node gather of v, APIC C, F <- (I + dt C) F, x <- x + dt v,
//            the particle's next key and next P2G payload.
// HBM- and latency-bound: no tensor-core work exists on this path (a
// scatter/gather stencil, not a dense contraction).
#include "pgmpm_internal.h"

namespace pgmpm {

namespace {

constexpr int TN = 6;              // smem tile edge in nodes (4 cells + 2)
constexpr int TILE_NODES = TN * TN * TN;

__device__ __forceinline__ const SceneDev& scene_ref(const View& V, int s) { return V.scenes[s]; }

// ------------------------------------------------------------------ keys
template <int PHYS>
__global__ void k_keys(View V) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    uint32_t flags = 0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < V.N; p += stride) {
        const int s = V.S == 1 ? 0 : scene_of_particle(V.scenes, V.S, (int)p);
        const SceneDev& sc = scene_ref(V, s);
        const float4 q0 = V.q[p];
        const float x[3] = {q0.x, q0.y, q0.z};
        int so[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float u;
            so[a] = stencil_origin(x[a], sc.origin[a], sc.dx, sc.inv_dx, sc.n[a], PHYS, u, flags);
        }
        if (V.sp.cap) {  // sparse grid: the slot of the cell's tile, claimed if new
            const uint32_t slot = sp_find_or_insert(V.sp, sp_code(so[0] >> 2, so[1] >> 2, so[2] >> 2), flags);
            V.keys[p] = slot == SP_NONE ? SP_NONE
                                        : slot * 64u + (uint32_t)((so[2] & 3) * 16 + (so[1] & 3) * 4 + (so[0] & 3));
        } else {
            V.keys[p] = cell_key(sc, so);
        }
    }
    if (flags) atomicOr(&V.counters[CNT_FLAGS], flags);
}

// Lowest node of cell tile ct (dense: from its index; sparse: from the
// slot's coordinates).
__device__ __forceinline__ void tile_origin(const View& V, const SceneDev& sc, uint32_t ct, int& ox, int& oy,
                                            int& oz) {
    if (V.sp.cap) {
        sp_decode(V.sp.code[ct], ox, oy, oz);
    } else {
        const int lt = (int)ct - sc.ct_base;
        ox = lt % sc.ct[0];
        oy = (lt / sc.ct[0]) % sc.ct[1];
        oz = lt / (sc.ct[0] * sc.ct[1]);
    }
    ox *= 4;
    oy *= 4;
    oz *= 4;
}

// --------------------------------------------------------------- payload
// P2G payload of the current MLS state (after an upload, a material change,
// or at the start of a replayed segment); G2P keeps it current afterwards.
template <bool MULTI>
__global__ void k_payload(View V) {
    const int64_t N = V.N;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    uint32_t flags = 0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += stride) {
        const int s = V.S == 1 ? 0 : scene_of_particle(V.scenes, V.S, (int)p);
        const SceneDev& sc = scene_ref(V, s);
        float x[3], F[9], v[3], C[9];
        unpack_xF(V.q[p], V.q[N + p], V.q[2 * N + p], x, F);
        unpack_vC(V.q[3 * N + p], V.q[4 * N + p], V.q[5 * N + p], v, C);
        Stencil st;
        make_stencil<PHYS_MLS>(sc, x, st, flags);
        const float2 mv = V.mV[p];
        float4 a0, a1, a2, a3;
        mls_payload(sc, V.mats[MULTI ? V.mat[p] : 0], st.f, F, v, C, mv.x, mv.y, a0, a1, a2, a3);
        V.pay[p] = a0;
        V.pay[N + p] = a1;
        V.pay[2 * N + p] = a2;
        V.pay[3 * N + p] = a3;
    }
    if (flags) atomicOr(&V.counters[CNT_FLAGS], flags);
}

// ------------------------------------------------------------------ mark
__global__ void k_mark(View V) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < V.N; i += stride) {
        const uint32_t ct = V.skeys[i] >> 6;
        const bool first = i == 0 || (V.skeys[i - 1] >> 6) != ct;
        const bool last = i + 1 == V.N || (V.skeys[i + 1] >> 6) != ct;
        if (!first && !last) continue;
        if (ct >= (uint32_t)V.total_ct) {
            atomicOr(&V.counters[CNT_FLAGS], FLAG_TILE_RANGE);
            continue;
        }
        // first / last particle of cell tile ct: record the tile's sorted
        // range; the first one also lists the tile and marks its node tiles
        uint32_t* rng = reinterpret_cast<uint32_t*>(&V.ctile_range[ct]);
        if (last) rng[1] = (uint32_t)(i + 1);
        if (!first) continue;
        rng[0] = (uint32_t)i;
        {
            const uint32_t slot = atomicAdd(&V.counters[CNT_CTILES], 1u);
            V.ctile_list[slot] = ct;
        }
        const int s = V.S == 1 ? 0 : scene_of_cell_tile(V.scenes, V.S, (int)ct);
        const SceneDev& sc = scene_ref(V, s);
        const int lt = (int)ct - sc.ct_base;
        const int tx = lt % sc.ct[0], ty = (lt / sc.ct[0]) % sc.ct[1], tz = lt / (sc.ct[0] * sc.ct[1]);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int nx = tx + (c & 1), ny = ty + ((c >> 1) & 1), nz = tz + (c >> 2);
            const uint32_t nt = (uint32_t)(sc.nt_base + (nz * sc.nt[1] + ny) * sc.nt[0] + nx);
            if (atomicExch(&V.tile_flags[nt], 1u) == 0u) {
                const uint32_t slot = atomicAdd(&V.counters[CNT_TILES], 1u);
                V.tile_list[slot] = nt;
            }
        }
    }
}

// ------------------------------------------------------------------- P2G
template <int PHYS, bool MULTI>
__global__ void __launch_bounds__(512) k_p2g(View V, int ppt) {
    __shared__ float tile[4 * TILE_NODES];
    for (int i = threadIdx.x; i < 4 * TILE_NODES; i += blockDim.x) tile[i] = 0.f;
    __syncthreads();
    const int64_t N = V.N;
    const int64_t c0 = (int64_t)blockIdx.x * ppt;
    if (c0 >= N) return;
    const int64_t cend = min(N, c0 + (int64_t)ppt);
    uint32_t flags = 0;
    int64_t seg = c0;
    while (seg < cend) {
        const uint32_t ct = V.skeys[seg] >> 6;
        // end of this cell tile's run inside the chunk (keys are sorted)
        int64_t lo = seg + 1, hi = cend;
        const uint32_t target = (ct + 1u) << 6;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (V.skeys[mid] < target) lo = mid + 1; else hi = mid;
        }
        const int64_t send = lo;
        if (ct >= (uint32_t)V.total_ct) {  // corrupt key: skip the run, report
            flags |= FLAG_TILE_RANGE;
            seg = send;
            continue;
        }
        const int s = V.S == 1 ? 0 : scene_of_cell_tile(V.scenes, V.S, (int)ct);
        const SceneDev& sc = scene_ref(V, s);
        const int lt = (int)ct - sc.ct_base;
        const int ox = 4 * (lt % sc.ct[0]), oy = 4 * ((lt / sc.ct[0]) % sc.ct[1]),
                  oz = 4 * (lt / (sc.ct[0] * sc.ct[1]));
        const int L = (int)(send - seg);
        const int R = (L + 31) >> 5;
        for (int slot = threadIdx.x; slot < 32 * R; slot += blockDim.x) {
            const int jj = (slot & 31) * R + (slot >> 5);
            if (jj >= L) continue;
            const uint32_t p = V.order[seg + jj];
            if (p >= (uint32_t)N) {
                flags |= FLAG_TILE_RANGE;
                continue;
            }
            const float4 q0 = V.q[p];
            const float x[3] = {q0.x, q0.y, q0.z};
            const float2 mv = V.mV[p];
            Stencil st;
            make_stencil<PHYS>(sc, x, st, flags);
            if (PHYS == PHYS_MLS) {
                const float4 q1 = V.q[N + p], q2 = V.q[2 * N + p];
                const float4 q3 = V.q[3 * N + p], q4 = V.q[4 * N + p], q5 = V.q[5 * N + p];
                float xx[3], F[9], v[3], C[9];
                unpack_xF(q0, q1, q2, xx, F);
                unpack_vC(q3, q4, q5, v, C);
                const MatDev mt = V.mats[MULTI ? V.mat[p] : 0];
                float tau[9];
                kirchhoff(F, mt, tau);
                add_viscous(F, C, mt, tau);
                const float kk = -sc.dt * mv.y * sc.D;
                float A[9];
#pragma unroll
                for (int i = 0; i < 9; ++i) A[i] = kk * tau[i] + mv.x * C[i];
                const int lx = st.s[0] - ox, ly = st.s[1] - oy, lz = st.s[2] - oz;
                if ((unsigned)lx > 3u || (unsigned)ly > 3u || (unsigned)lz > 3u) {
                    flags |= FLAG_TILE_RANGE;
                    continue;
                }
                const float dx = sc.dx;
                float d0[3], d1[3], d2[3];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    d0[i] = ((float)i - st.f[0]) * dx;
                    d1[i] = ((float)i - st.f[1]) * dx;
                    d2[i] = ((float)i - st.f[2]) * dx;
                }
                const float m = mv.x;
                const float mvx = m * v[0], mvy = m * v[1], mvz = m * v[2];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        const float wjk = st.w[1][j] * st.w[2][k];
                        const float bx = mvx + A[1] * d1[j] + A[2] * d2[k];
                        const float by = mvy + A[4] * d1[j] + A[5] * d2[k];
                        const float bz = mvz + A[7] * d1[j] + A[8] * d2[k];
                        const int row = (lx) + TN * (ly + j) + TN * TN * (lz + k);
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            const float w = st.w[0][i] * wjk;
                            const int nidx = row + i;
                            atomicAdd(&tile[nidx], w * m);
                            atomicAdd(&tile[TILE_NODES + nidx], w * (bx + A[0] * d0[i]));
                            atomicAdd(&tile[2 * TILE_NODES + nidx], w * (by + A[3] * d0[i]));
                            atomicAdd(&tile[3 * TILE_NODES + nidx], w * (bz + A[6] * d0[i]));
                        }
                    }
                }
            } else {
                const float4 q3 = V.q[3 * N + p];
                const float vel[3] = {q3.x, q3.y, q3.z};
                const float mass = mv.x;
                // reference loop order: x outer, z inner (material_point_method.h:535-566)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const int gi = st.b[0] + i;
                    if (gi < 0 || gi >= sc.n[0]) continue;
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        const int gj = st.b[1] + j;
                        if (gj < 0 || gj >= sc.n[1]) continue;
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            const int gk = st.b[2] + k;
                            if (gk < 0 || gk >= sc.n[2]) continue;
                            const float weight = __fmul_rn(__fmul_rn(st.w[0][i], st.w[1][j]), st.w[2][k]);
                            if (!(weight > 1e-10f)) continue;
                            const int lx = gi - ox, ly = gj - oy, lz = gk - oz;
                            if ((unsigned)lx >= (unsigned)TN || (unsigned)ly >= (unsigned)TN ||
                                (unsigned)lz >= (unsigned)TN) {
                                flags |= FLAG_TILE_RANGE;
                                continue;
                            }
                            const int nidx = lx + TN * ly + TN * TN * lz;
                            const float wm = __fmul_rn(weight, mass);
                            atomicAdd(&tile[nidx], wm);
                            atomicAdd(&tile[TILE_NODES + nidx], __fmul_rn(wm, vel[0]));
                            atomicAdd(&tile[2 * TILE_NODES + nidx], __fmul_rn(wm, vel[1]));
                            atomicAdd(&tile[3 * TILE_NODES + nidx], __fmul_rn(wm, vel[2]));
                        }
                    }
                }
            }
        }
        __syncthreads();
        // flush: one vector atomic per touched node, then clear the tile
        for (int nidx = threadIdx.x; nidx < TILE_NODES; nidx += blockDim.x) {
            const float m = tile[nidx];
            if (m != 0.f) {
                const float4 val = make_float4(m, tile[TILE_NODES + nidx], tile[2 * TILE_NODES + nidx],
                                               tile[3 * TILE_NODES + nidx]);
                tile[nidx] = 0.f;
                tile[TILE_NODES + nidx] = 0.f;
                tile[2 * TILE_NODES + nidx] = 0.f;
                tile[3 * TILE_NODES + nidx] = 0.f;
                const int lx = nidx % TN, ly = (nidx / TN) % TN, lz = nidx / (TN * TN);
                const int gi = ox + lx, gj = oy + ly, gk = oz + lz;
                if (gi < sc.n[0] && gj < sc.n[1] && gk < sc.n[2]) atomicAdd(&V.grid_mp[node_index(sc, gi, gj, gk)], val);
            }
        }
        __syncthreads();
        seg = send;
    }
    if (flags) atomicOr(&V.counters[CNT_FLAGS], flags);
}

// ---------------------------------------------------- P2G over cell tiles
// One block per occupied 4^3 cell tile (work taken from an atomic cursor).
// Thread t owns cell t/3 and z-slice oz = t%3 of that cell's 3x3x3 stencil:
// 9 nodes x (m, p) = 36 register accumulators.  Per sub-chunk of P2G_SC
// sorted particles:
//   phase A (thread = particle, coalesced): stress, affine matrix, axis
//            weights -> shared-memory payload (SoA);
//   phase B (thread = (cell, oz)): loop over the cell's particles of the
//            sub-chunk, accumulate its 9 nodes in registers.
// Flush: accumulators are transposed through shared memory (plain stores,
// no atomics), each of the 6^3 tile nodes sums the <= 27 cells that touch
// it, and non-empty nodes get ONE vector atomic (red.global.add.v4.f32).
constexpr int P2G_T = 192;
constexpr int P2G_SC = 256;
constexpr int PAY_W = 0;    // wx0..2, wy0..2, wz0..2
constexpr int PAY_M = 9;
constexpr int PAY_B = 10;   // MLS: m v - (A dx) f ;  REF: v
constexpr int PAY_A = 13;   // MLS: A dx (row-major)
constexpr int PAY_MLS = 22;

// MODE: forward MLS, forward REF_COMPAT, or the reverse of G2P (dL/dv_i
// scatter, same accumulation skeleton with an adjoint payload and no mass
// channel).
enum { MODE_MLS = 0, MODE_REF = 1, MODE_ADJ = 2 };

template <int MODE, bool MULTI, bool FLUID>
__global__ void __launch_bounds__(P2G_T, 3) k_p2g_tiles(View V, AdjView AV) {
    constexpr int PHYS = MODE == MODE_REF ? PHYS_REF : PHYS_MLS;
    __shared__ float sm[27 * 4 * 64];  // payload [22][P2G_SC], then transpose [27][4][64]
    __shared__ uint32_t cb[64], ce[64];
    __shared__ uint32_t s_work;
    static_assert(PAY_MLS * P2G_SC <= 27 * 4 * 64, "payload must fit the transpose buffer");
    const int t = threadIdx.x;
    const int cell = t / 3, oz = t - 3 * (t / 3);
    const int64_t N = V.N;
    uint32_t flags = 0;
    const uint32_t ntiles = V.counters[CNT_CTILES];
    for (;;) {
        if (t == 0) s_work = atomicAdd(&V.counters[CNT_P2G_CURSOR], 1u);
        if (t < 64) {
            cb[t] = 0u;
            ce[t] = 0u;
        }
        __syncthreads();
        const uint32_t w = s_work;
        if (w >= ntiles) break;
        const uint32_t ct = V.ptile_list ? V.ptile_list[w] : V.ctile_list[w];  // largest tiles first
        const uint2 rg = V.ctile_range[ct];
        const int s = V.S == 1 ? 0 : scene_of_cell_tile(V.scenes, V.S, (int)ct);
        const SceneDev& sc = scene_ref(V, s);
        const int lt = (int)ct - sc.ct_base;
        const int ox = 4 * (lt % sc.ct[0]), oy = 4 * ((lt / sc.ct[0]) % sc.ct[1]),
                  oz0 = 4 * (lt / (sc.ct[0] * sc.ct[1]));
        // per-cell sorted ranges inside the tile (keys are sorted by local cell)
        for (uint32_t i = rg.x + t; i < rg.y; i += P2G_T) {
            const uint32_t k = V.skeys[i] & 63u;
            if (i == rg.x || (V.skeys[i - 1] & 63u) != k) cb[k] = i;
            if (i + 1 == rg.y || (V.skeys[i + 1] & 63u) != k) ce[k] = i + 1;
        }
        __syncthreads();
        const uint32_t my_b = cb[cell], my_e = ce[cell];
        float am[3][3], apx[3][3], apy[3][3], apz[3][3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) am[a][b] = apx[a][b] = apy[a][b] = apz[a][b] = 0.f;
        for (uint32_t s0 = rg.x; s0 < rg.y; s0 += P2G_SC) {
            const uint32_t s1 = min(rg.y, s0 + (uint32_t)P2G_SC);
            // ---- phase A: per-particle payload
            for (uint32_t i = s0 + t; i < s1; i += P2G_T) {
                const int j = (int)(i - s0);
                const uint32_t p = V.order[i];
                if (p >= (uint32_t)N) {
                    flags |= FLAG_TILE_RANGE;
#pragma unroll
                    for (int f = 0; f < PAY_MLS; ++f) sm[f * P2G_SC + j] = 0.f;
                    continue;
                }
                const float4 q0 = V.q[p];
                const float x[3] = {q0.x, q0.y, q0.z};
                const float2 mv = V.mV[p];
                Stencil st;
                make_stencil<PHYS>(sc, x, st, flags);
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int k = 0; k < 3; ++k) sm[(PAY_W + 3 * a + k) * P2G_SC + j] = st.w[a][k];
                if (MODE == MODE_ADJ) {
                    // reverse of G2P: dL/dv_i += w_i (gv + D gC d_i), with
                    // gv = dL/dv' + dt dL/dx' and gC = dL/dC' + dt dL/dF'raw F^T
                    const float4 q1 = V.q[N + p], q2 = V.q[2 * N + p];
                    float xx[3], F[9];
                    unpack_xF(q0, q1, q2, xx, F);
                    float gx[3], gF[9], gv[3], gC[9];
                    unpack_xF(AV.g[p], AV.g[N + p], AV.g[2 * N + p], gx, gF);
                    unpack_vC(AV.g[3 * N + p], AV.g[4 * N + p], AV.g[5 * N + p], gv, gC);
                    if (FLUID && V.mats[MULTI ? V.mat[p] : 0].model == MODEL_EOS) {
                        // F' = cbrt(det Fraw) I, Fraw = (I + dt C') F
                        float Cn[9], vdum[3], M[9], Fr[9], cof[9];
                        unpack_vC(AV.q_next[3 * N + p], AV.q_next[4 * N + p], AV.q_next[5 * N + p], vdum, Cn);
#pragma unroll
                        for (int a = 0; a < 9; ++a) M[a] = sc.dt * Cn[a] + ((a % 4 == 0) ? 1.f : 0.f);
                        m3_mul(M, F, Fr);
                        m3_cof(Fr, cof);
                        const float J = Fr[0] * cof[0] + Fr[1] * cof[1] + Fr[2] * cof[2];
                        const float c = cbrtf(J) / (3.f * J) * (gF[0] + gF[4] + gF[8]);
#pragma unroll
                        for (int a = 0; a < 9; ++a) gF[a] = c * cof[a];
                    }
                    float gFFt[9];
                    m3_mulT(gF, F, gFFt);
                    const float sD = sc.D * sc.dx;
                    float Ad[9];
#pragma unroll
                    for (int a = 0; a < 9; ++a) Ad[a] = sD * (gC[a] + sc.dt * gFFt[a]);
                    sm[PAY_M * P2G_SC + j] = 0.f;
#pragma unroll
                    for (int a = 0; a < 3; ++a)
                        sm[(PAY_B + a) * P2G_SC + j] = (gv[a] + sc.dt * gx[a]) -
                                                       (Ad[3 * a] * st.f[0] + Ad[3 * a + 1] * st.f[1] +
                                                        Ad[3 * a + 2] * st.f[2]);
#pragma unroll
                    for (int a = 0; a < 9; ++a) sm[(PAY_A + a) * P2G_SC + j] = Ad[a];
                } else if (PHYS == PHYS_MLS) {
                    // precomputed payload (G2P of the previous step / k_payload)
                    const float4 a0 = V.pay[p], a1 = V.pay[N + p], a2 = V.pay[2 * N + p], a3 = V.pay[3 * N + p];
                    float m, b[3], Ad[9], f[3];
                    unpack_payload(a0, a1, a2, a3, m, b, Ad, f);
                    sm[PAY_M * P2G_SC + j] = m;
                    sm[(PAY_B + 0) * P2G_SC + j] = b[0];
                    sm[(PAY_B + 1) * P2G_SC + j] = b[1];
                    sm[(PAY_B + 2) * P2G_SC + j] = b[2];
#pragma unroll
                    for (int a = 0; a < 9; ++a) sm[(PAY_A + a) * P2G_SC + j] = Ad[a];
                } else {
                    const float4 q3 = V.q[3 * N + p];
                    const bool regular = st.b[0] == st.s[0] && st.b[1] == st.s[1] && st.b[2] == st.s[2];
                    sm[PAY_M * P2G_SC + j] = regular ? mv.x : 0.f;
                    sm[(PAY_B + 0) * P2G_SC + j] = q3.x;
                    sm[(PAY_B + 1) * P2G_SC + j] = q3.y;
                    sm[(PAY_B + 2) * P2G_SC + j] = q3.z;
                    if (!regular) {
                        // stencil partly outside the grid: scatter this particle
                        // directly (per-node bounds checks as the reference)
                        const float vel[3] = {q3.x, q3.y, q3.z};
                        for (int ii = 0; ii < 3; ++ii) {
                            const int gi = st.b[0] + ii;
                            if (gi < 0 || gi >= sc.n[0]) continue;
                            for (int jj = 0; jj < 3; ++jj) {
                                const int gj = st.b[1] + jj;
                                if (gj < 0 || gj >= sc.n[1]) continue;
                                for (int kq = 0; kq < 3; ++kq) {
                                    const int gk = st.b[2] + kq;
                                    if (gk < 0 || gk >= sc.n[2]) continue;
                                    const float wgt = __fmul_rn(__fmul_rn(st.w[0][ii], st.w[1][jj]), st.w[2][kq]);
                                    if (!(wgt > 1e-10f)) continue;
                                    const float wm = __fmul_rn(wgt, mv.x);
                                    float* g = reinterpret_cast<float*>(&V.grid_mp[node_index(sc, gi, gj, gk)]);
                                    atomicAdd(g, wm);
                                    atomicAdd(g + 1, __fmul_rn(wm, vel[0]));
                                    atomicAdd(g + 2, __fmul_rn(wm, vel[1]));
                                    atomicAdd(g + 3, __fmul_rn(wm, vel[2]));
                                }
                            }
                        }
                    }
                }
            }
            __syncthreads();
            // ---- phase B: this thread's cell, slice oz
            const uint32_t ib = max(my_b, s0), ie = min(my_e, s1);
            for (uint32_t i = ib; i < ie; ++i) {
                const int j = (int)(i - s0);
                const float wz = sm[(PAY_W + 6 + oz) * P2G_SC + j];
                const float m = sm[PAY_M * P2G_SC + j];
                const float wx[3] = {sm[(PAY_W + 0) * P2G_SC + j], sm[(PAY_W + 1) * P2G_SC + j],
                                     sm[(PAY_W + 2) * P2G_SC + j]};
                const float wy[3] = {sm[(PAY_W + 3) * P2G_SC + j], sm[(PAY_W + 4) * P2G_SC + j],
                                     sm[(PAY_W + 5) * P2G_SC + j]};
                const float b0 = sm[(PAY_B + 0) * P2G_SC + j], b1 = sm[(PAY_B + 1) * P2G_SC + j],
                            b2 = sm[(PAY_B + 2) * P2G_SC + j];
                if (PHYS == PHYS_MLS) {
                    float Ad[9];
#pragma unroll
                    for (int a = 0; a < 9; ++a) Ad[a] = sm[(PAY_A + a) * P2G_SC + j];
                    const float fz = (float)oz;
                    const float bz0 = b0 + Ad[2] * fz, bz1 = b1 + Ad[5] * fz, bz2 = b2 + Ad[8] * fz;
#pragma unroll
                    for (int yy = 0; yy < 3; ++yy) {
                        const float wyz = wy[yy] * wz;
                        float v0 = bz0 + Ad[1] * (float)yy, v1 = bz1 + Ad[4] * (float)yy,
                              v2 = bz2 + Ad[7] * (float)yy;
#pragma unroll
                        for (int xx = 0; xx < 3; ++xx) {
                            const float wgt = wx[xx] * wyz;
                            am[yy][xx] += wgt * m;
                            apx[yy][xx] += wgt * v0;
                            apy[yy][xx] += wgt * v1;
                            apz[yy][xx] += wgt * v2;
                            v0 += Ad[0];
                            v1 += Ad[3];
                            v2 += Ad[6];
                        }
                    }
                } else {
#pragma unroll
                    for (int yy = 0; yy < 3; ++yy)
#pragma unroll
                        for (int xx = 0; xx < 3; ++xx) {
                            const float wgt = __fmul_rn(__fmul_rn(wx[xx], wy[yy]), wz);
                            if (wgt > 1e-10f) {
                                const float wm = __fmul_rn(wgt, m);
                                am[yy][xx] += wm;
                                apx[yy][xx] += __fmul_rn(wm, b0);
                                apy[yy][xx] += __fmul_rn(wm, b1);
                                apz[yy][xx] += __fmul_rn(wm, b2);
                            }
                        }
                }
            }
            __syncthreads();
        }
        // ---- flush: transpose through shared memory, one vector atomic per node
#pragma unroll
        for (int yy = 0; yy < 3; ++yy)
#pragma unroll
            for (int xx = 0; xx < 3; ++xx) {
                const int o = xx + 3 * yy + 9 * oz;
                sm[(o * 4 + 0) * 64 + cell] = am[yy][xx];
                sm[(o * 4 + 1) * 64 + cell] = apx[yy][xx];
                sm[(o * 4 + 2) * 64 + cell] = apy[yy][xx];
                sm[(o * 4 + 3) * 64 + cell] = apz[yy][xx];
            }
        __syncthreads();
        for (int n = t; n < TILE_NODES; n += P2G_T) {
            const int nx = n % TN, ny = (n / TN) % TN, nz = n / (TN * TN);
            float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
            for (int zz = max(0, nz - 3); zz <= min(2, nz); ++zz)
                for (int yy = max(0, ny - 3); yy <= min(2, ny); ++yy)
                    for (int xx = max(0, nx - 3); xx <= min(2, nx); ++xx) {
                        const int c = (nx - xx) + 4 * (ny - yy) + 16 * (nz - zz);
                        const int o = xx + 3 * yy + 9 * zz;
                        acc.x += sm[(o * 4 + 0) * 64 + c];
                        acc.y += sm[(o * 4 + 1) * 64 + c];
                        acc.z += sm[(o * 4 + 2) * 64 + c];
                        acc.w += sm[(o * 4 + 3) * 64 + c];
                    }
            const int gi = ox + nx, gj = oy + ny, gk = oz0 + nz;
            const bool any = MODE == MODE_ADJ ? (acc.y != 0.f || acc.z != 0.f || acc.w != 0.f) : acc.x != 0.f;
            if (any && gi < sc.n[0] && gj < sc.n[1] && gk < sc.n[2])
                atomicAdd(&V.grid_mp[node_index(sc, gi, gj, gk)], acc);
        }
        __syncthreads();
    }
    if (flags) atomicOr(&V.counters[CNT_FLAGS], flags);
}

// Reverse of G2P for one particle (MLS): the scatter payload of dL/dv_i
// and dL/dm_i contributions, node o gets w_o (b + Ad o).  Also fills the
// stencil (f, w) of the particle's position.
template <bool MULTI, bool FLUID>
__device__ __forceinline__ void adj_payload(const View& V, const AdjView& AV, const SceneDev& sc, int64_t p,
                                            Stencil& st, uint32_t& flags, float b[3], float Ad[9]) {
    const int64_t N = V.N;
    const float4 q0 = V.q[p];
    const float x[3] = {q0.x, q0.y, q0.z};
    make_stencil<PHYS_MLS>(sc, x, st, flags);
    const float4 q1 = V.q[N + p], q2 = V.q[2 * N + p];
    float xx[3], F[9];
    unpack_xF(q0, q1, q2, xx, F);
    float gx[3], gF[9], gv[3], gC[9];
    unpack_xF(AV.g[p], AV.g[N + p], AV.g[2 * N + p], gx, gF);
    unpack_vC(AV.g[3 * N + p], AV.g[4 * N + p], AV.g[5 * N + p], gv, gC);
    if (FLUID && V.mats[MULTI ? V.mat[p] : 0].model == MODEL_EOS) {
        float Cn[9], vdum[3], M[9], Fr[9], cof[9];
        unpack_vC(AV.q_next[3 * N + p], AV.q_next[4 * N + p], AV.q_next[5 * N + p], vdum, Cn);
#pragma unroll
        for (int a = 0; a < 9; ++a) M[a] = sc.dt * Cn[a] + ((a % 4 == 0) ? 1.f : 0.f);
        m3_mul(M, F, Fr);
        m3_cof(Fr, cof);
        const float J = Fr[0] * cof[0] + Fr[1] * cof[1] + Fr[2] * cof[2];
        const float cc = cbrtf(J) / (3.f * J) * (gF[0] + gF[4] + gF[8]);
#pragma unroll
        for (int a = 0; a < 9; ++a) gF[a] = cc * cof[a];
    }
    float gFFt[9];
    m3_mulT(gF, F, gFFt);
    const float sD = sc.D * sc.dx;
#pragma unroll
    for (int a = 0; a < 9; ++a) Ad[a] = sD * (gC[a] + sc.dt * gFFt[a]);
#pragma unroll
    for (int a = 0; a < 3; ++a)
        b[a] = (gv[a] + sc.dt * gx[a]) - (Ad[3 * a] * st.f[0] + Ad[3 * a + 1] * st.f[1] + Ad[3 * a + 2] * st.f[2]);
}

// Sum of the contributions to node (nx, ny, nz) of the 6^3 node block of a
// 4^3 cell tile, from T4[o * 64 + cell] = cell's accumulators for its
// stencil offset o.  Every offset is walked (compile-time shared offsets,
// no divergence); an offset whose cell falls outside the tile reads slot 0
// and is not added, so the address stays inside the table.
__device__ __forceinline__ float4 tile_node_sum(const float4* T4, int nx, int ny, int nz) {
    // bit d of vx: cell x = nx - d lies in the tile (0..3); same for y, z
    const uint32_t vx = (nx <= 3 ? 1u : 0u) | (nx >= 1 && nx <= 4 ? 2u : 0u) | (nx >= 2 ? 4u : 0u);
    const uint32_t vy = (ny <= 3 ? 1u : 0u) | (ny >= 1 && ny <= 4 ? 2u : 0u) | (ny >= 2 ? 4u : 0u);
    const uint32_t vz = (nz <= 3 ? 1u : 0u) | (nz >= 1 && nz <= 4 ? 2u : 0u) | (nz >= 2 ? 4u : 0u);
    const int cn = nx + 4 * ny + 16 * nz;
    float4 a4 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int zz = 0; zz < 3; ++zz)
#pragma unroll
        for (int yy = 0; yy < 3; ++yy)
#pragma unroll
            for (int xx = 0; xx < 3; ++xx) {
                const bool valid = ((vx >> xx) & (vy >> yy) & (vz >> zz) & 1u) != 0u;
                const int cell = valid ? cn - (xx + 4 * yy + 16 * zz) : 0;
                const float4 t = T4[(xx + 3 * yy + 9 * zz) * 64 + cell];
                if (valid) {
                    a4.x += t.x;
                    a4.y += t.y;
                    a4.z += t.z;
                    a4.w += t.w;
                }
            }
    return a4;
}

// ------------------------------------------------ P2G, one thread per cell
// Variant 2: one 64-thread block per occupied cell tile, thread c owns cell
// c and all 27 nodes of its stencil (108 register accumulators).  The
// thread walks its cell's particles (sorted, contiguous) and accumulates
// their payloads (precomputed by G2P for MLS; computed here from the state
// for REF and the adjoint): no shared payload staging and no barriers until
// the flush, a shared-memory transpose + one vector atomic per tile node.
constexpr int P2GC_T = 64;

template <int MODE, bool MULTI, bool FLUID>
__global__ void __launch_bounds__(P2GC_T, 6) k_p2g_cells(View V, AdjView AV) {
    constexpr int PHYS = MODE == MODE_REF ? PHYS_REF : PHYS_MLS;
    __shared__ float4 T4[27 * 64];  // [offset o][cell]: the 4 channels of cell's node o
    __shared__ uint32_t s_work;
    const int c = threadIdx.x;
    const int64_t N = V.N;
    uint32_t flags = 0;
    const uint32_t ntiles = V.counters[CNT_CTILES];
    // Few occupied tiles (a small, dense scene) leave most blocks idle: then
    // each cell's run is split into S interleaved slices, one work item per
    // (tile, slice), each flushing its own partial sums.  S stops at 4: a
    // work item's flush (216 node sums) outweighs a handful of particles
    // per thread.
    const uint32_t S = ntiles ? min(4u, max(1u, (gridDim.x + ntiles - 1) / ntiles)) : 1u;
    const uint32_t nwork = ntiles * S;
    // with at least two work items per block, the next one is claimed while
    // this one runs (thread 0 holds it); with fewer, claiming early would
    // leave blocks idle, so it is claimed at the end of the item
    const bool early = nwork >= 2u * gridDim.x;
    uint32_t next_work = 0;
    if (c == 0) s_work = atomicAdd(&V.counters[CNT_P2G_CURSOR], 1u);
    for (;;) {
        __syncthreads();
        const uint32_t w = s_work;
        if (w >= nwork) break;
        if (early && c == 0) next_work = atomicAdd(&V.counters[CNT_P2G_CURSOR], 1u);
        const uint32_t wt = w / S, slice = w - wt * S;
        const uint32_t ct = V.ptile_list ? V.ptile_list[wt] : V.ctile_list[wt];  // largest tiles first
        const uint2 rg = V.ctile_range[ct];
        const int s = V.S == 1 ? 0 : scene_of_cell_tile(V.scenes, V.S, (int)ct);
        const SceneDev& sc = scene_ref(V, s);
        const int lt = (int)ct - sc.ct_base;
        const int ox = 4 * (lt % sc.ct[0]), oy = 4 * ((lt / sc.ct[0]) % sc.ct[1]),
                  oz0 = 4 * (lt / (sc.ct[0] * sc.ct[1]));
        // this cell's sorted range: from the sort's cell table, else a
        // search of the tile's keys (ordered by local cell)
        uint32_t cb, ce;
        if (V.cell_range) {
            const uint2 cr = V.cell_range[(size_t)ct * 64 + c];
            cb = max(cr.x, rg.x);
            ce = min(cr.y, rg.y);
        } else {
            const uint32_t kc = (ct << 6) | (uint32_t)c;
            uint32_t lo = rg.x, hi = rg.y;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (V.skeys[mid] < kc) lo = mid + 1; else hi = mid;
            }
            cb = lo;
            hi = rg.y;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (V.skeys[mid] <= kc) lo = mid + 1; else hi = mid;
            }
            ce = lo;
        }
        float acc[27][4];
#pragma unroll
        for (int o = 0; o < 27; ++o) acc[o][0] = acc[o][1] = acc[o][2] = acc[o][3] = 0.f;
        for (uint32_t i = cb + slice; i < ce; i += S) {
            const uint32_t p = V.order[i];
            if (p >= (uint32_t)N) {
                flags |= FLAG_TILE_RANGE;
                continue;
            }
            Stencil st;
            float m, b[3], Ad[9];
            if (MODE == MODE_MLS) {
                // precomputed payload (G2P of the previous step / k_payload)
                const float4 a0 = V.pay[p], a1 = V.pay[N + p], a2 = V.pay[2 * N + p], a3 = V.pay[3 * N + p];
                unpack_payload(a0, a1, a2, a3, m, b, Ad, st.f);
#pragma unroll
                for (int a = 0; a < 3; ++a) mls_weights(st.f[a], st.w[a]);
            } else if (MODE == MODE_ADJ) {
                adj_payload<MULTI, FLUID>(V, AV, sc, p, st, flags, b, Ad);
                m = 0.f;
            } else {
                const float4 q0 = V.q[p];
                const float x[3] = {q0.x, q0.y, q0.z};
                make_stencil<PHYS>(sc, x, st, flags);
                const float4 q3 = V.q[3 * N + p];
                const float2 mv = V.mV[p];
                const bool regular = st.b[0] == st.s[0] && st.b[1] == st.s[1] && st.b[2] == st.s[2];
                if (!regular) {
                    // stencil partly outside the grid: scatter directly with
                    // the reference's per-node bounds checks
                    const float vel[3] = {q3.x, q3.y, q3.z};
                    for (int ii = 0; ii < 3; ++ii) {
                        const int gi = st.b[0] + ii;
                        if (gi < 0 || gi >= sc.n[0]) continue;
                        for (int jj = 0; jj < 3; ++jj) {
                            const int gj = st.b[1] + jj;
                            if (gj < 0 || gj >= sc.n[1]) continue;
                            for (int kq = 0; kq < 3; ++kq) {
                                const int gk = st.b[2] + kq;
                                if (gk < 0 || gk >= sc.n[2]) continue;
                                const float wgt = __fmul_rn(__fmul_rn(st.w[0][ii], st.w[1][jj]), st.w[2][kq]);
                                if (!(wgt > 1e-10f)) continue;
                                const float wm = __fmul_rn(wgt, mv.x);
                                float* g = reinterpret_cast<float*>(&V.grid_mp[node_index(sc, gi, gj, gk)]);
                                atomicAdd(g, wm);
                                atomicAdd(g + 1, __fmul_rn(wm, vel[0]));
                                atomicAdd(g + 2, __fmul_rn(wm, vel[1]));
                                atomicAdd(g + 3, __fmul_rn(wm, vel[2]));
                            }
                        }
                    }
                    continue;
                }
#pragma unroll
                for (int zz = 0; zz < 3; ++zz)
#pragma unroll
                    for (int yy = 0; yy < 3; ++yy)
#pragma unroll
                        for (int xx = 0; xx < 3; ++xx) {
                            const float wgt = __fmul_rn(__fmul_rn(st.w[0][xx], st.w[1][yy]), st.w[2][zz]);
                            if (wgt > 1e-10f) {
                                const int o = xx + 3 * yy + 9 * zz;
                                const float wm = __fmul_rn(wgt, mv.x);
                                acc[o][0] += wm;
                                acc[o][1] += __fmul_rn(wm, q3.x);
                                acc[o][2] += __fmul_rn(wm, q3.y);
                                acc[o][3] += __fmul_rn(wm, q3.z);
                            }
                        }
                continue;
            }
            // MLS / adjoint: node o gets w_o (m, b + Ad o)
#pragma unroll
            for (int zz = 0; zz < 3; ++zz) {
                const float bz0 = b[0] + Ad[2] * (float)zz, bz1 = b[1] + Ad[5] * (float)zz,
                            bz2 = b[2] + Ad[8] * (float)zz;
#pragma unroll
                for (int yy = 0; yy < 3; ++yy) {
                    const float wyz = st.w[1][yy] * st.w[2][zz];
                    float v0 = bz0 + Ad[1] * (float)yy, v1 = bz1 + Ad[4] * (float)yy, v2 = bz2 + Ad[7] * (float)yy;
#pragma unroll
                    for (int xx = 0; xx < 3; ++xx) {
                        const int o = xx + 3 * yy + 9 * zz;
                        const float wgt = st.w[0][xx] * wyz;
                        if (MODE != MODE_ADJ) acc[o][0] += wgt * m;
                        acc[o][1] += wgt * v0;
                        acc[o][2] += wgt * v1;
                        acc[o][3] += wgt * v2;
                        v0 += Ad[0];
                        v1 += Ad[3];
                        v2 += Ad[6];
                    }
                }
            }
        }
        // flush: the thread stores its cell's node o as T4[o][c]; then node n
        // sums T4[o][n - o] over the offsets whose cell lies in the tile and
        // issues one vector atomic (see k_p2g_pairs)
#pragma unroll
        for (int o = 0; o < 27; ++o) T4[o * 64 + c] = make_float4(acc[o][0], acc[o][1], acc[o][2], acc[o][3]);
        __syncthreads();
        for (int n = c; n < TILE_NODES; n += P2GC_T) {
            const int nx = n % TN, ny = (n / TN) % TN, nz = n / (TN * TN);
            const float4 a4 = tile_node_sum(T4, nx, ny, nz);
            const int gi = ox + nx, gj = oy + ny, gk = oz0 + nz;
            const bool any = MODE == MODE_ADJ ? (a4.y != 0.f || a4.z != 0.f || a4.w != 0.f) : a4.x != 0.f;
            if (any && gi < sc.n[0] && gj < sc.n[1] && gk < sc.n[2])
                atomicAdd(&V.grid_mp[node_index(sc, gi, gj, gk)], a4);
        }
        __syncthreads();
        if (c == 0) s_work = early ? next_work : atomicAdd(&V.counters[CNT_P2G_CURSOR], 1u);
    }
    if (flags) atomicOr(&V.counters[CNT_FLAGS], flags);
}

// ------------------------------------- P2G, two threads per cell (MLS)
// Variant 3: variant 2 with each cell's 108 accumulators split over a pair
// of adjacent lanes -- lane 2c+0 holds (m, p_x), lane 2c+1 holds (p_y, p_z)
// of the 27 nodes -- so that a 128-thread block of ~100 registers per
// thread fits 5 times per SM (20 warps against variant 2's 12).  Both lanes
// of a pair read the same payload (one memory request), compute the
// weights, and accumulate their two channels; the flush is variant 2's.
constexpr int P2GP_T = 128;

__global__ void __launch_bounds__(P2GP_T, 5) k_p2g_pairs(View V) {
    __shared__ float4 T4[27 * 64];  // [offset o][cell]: the 4 channels of cell's node o
    __shared__ uint32_t s_work;
    const int c = threadIdx.x >> 1, h = threadIdx.x & 1;
    const int64_t N = V.N;
    uint32_t flags = 0;
    const uint32_t ntiles = V.counters[CNT_CTILES];
    // slices of a cell's run when tiles are few (see k_p2g_cells)
    const uint32_t S = ntiles ? min(4u, max(1u, (gridDim.x + ntiles - 1) / ntiles)) : 1u;
    const uint32_t nwork = ntiles * S;
    // with at least two work items per block, the next one is claimed while
    // this one runs (thread 0 holds it); with fewer, claiming early would
    // leave blocks idle, so it is claimed at the end of the item
    const bool early = nwork >= 2u * gridDim.x;
    uint32_t next_work = 0;
    if (threadIdx.x == 0) s_work = atomicAdd(&V.counters[CNT_P2G_CURSOR], 1u);
    for (;;) {
        __syncthreads();
        const uint32_t w = s_work;
        if (w >= nwork) break;
        if (early && threadIdx.x == 0) next_work = atomicAdd(&V.counters[CNT_P2G_CURSOR], 1u);
        const uint32_t wt = w / S, slice = w - wt * S;
        const uint32_t ct = V.ptile_list ? V.ptile_list[wt] : V.ctile_list[wt];
        const uint2 rg = V.ctile_range[ct];
        const int s = V.S == 1 ? 0 : scene_of_cell_tile(V.scenes, V.S, (int)ct);
        const SceneDev& sc = scene_ref(V, s);
        const int lt = (int)ct - sc.ct_base;
        const int ox = 4 * (lt % sc.ct[0]), oy = 4 * ((lt / sc.ct[0]) % sc.ct[1]),
                  oz0 = 4 * (lt / (sc.ct[0] * sc.ct[1]));
        uint32_t cb, ce;
        if (V.cell_range) {
            const uint2 cr = V.cell_range[(size_t)ct * 64 + c];
            cb = max(cr.x, rg.x);
            ce = min(cr.y, rg.y);
        } else {
            const uint32_t kc = (ct << 6) | (uint32_t)c;
            uint32_t lo = rg.x, hi = rg.y;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (V.skeys[mid] < kc) lo = mid + 1; else hi = mid;
            }
            cb = lo;
            hi = rg.y;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (V.skeys[mid] <= kc) lo = mid + 1; else hi = mid;
            }
            ce = lo;
        }
        float accA[27], accB[27];
#pragma unroll
        for (int o = 0; o < 27; ++o) accA[o] = accB[o] = 0.f;
        for (uint32_t i = cb + slice; i < ce; i += S) {
            const uint32_t p = V.order[i];
            if (p >= (uint32_t)N) {
                flags |= FLAG_TILE_RANGE;
                continue;
            }
            const float4 a0 = V.pay[p], a1 = V.pay[N + p], a2 = V.pay[2 * N + p], a3 = V.pay[3 * N + p];
            // channel value at offset o: beta + gamma . o
            //   lane 0: A = m (gamma 0), B = p_x (b_x, Ad row 0)
            //   lane 1: A = p_y (b_y, Ad row 1), B = p_z (b_z, Ad row 2)
            const float bA = h ? a0.y : a0.w, bB = h ? a0.z : a0.x;
            const float gAx = h ? a1.w : 0.f, gAy = h ? a2.x : 0.f, gAz = h ? a2.y : 0.f;
            const float gBx = h ? a2.z : a1.x, gBy = h ? a2.w : a1.y, gBz = h ? a3.x : a1.z;
            float wt[3][3];
            mls_weights(a3.y, wt[0]);
            mls_weights(a3.z, wt[1]);
            mls_weights(a3.w, wt[2]);
#pragma unroll
            for (int zz = 0; zz < 3; ++zz) {
                const float zA = bA + gAz * (float)zz, zB = bB + gBz * (float)zz;
#pragma unroll
                for (int yy = 0; yy < 3; ++yy) {
                    const float wyz = wt[1][yy] * wt[2][zz];
                    float vA = zA + gAy * (float)yy, vB = zB + gBy * (float)yy;
#pragma unroll
                    for (int xx = 0; xx < 3; ++xx) {
                        const int o = xx + 3 * yy + 9 * zz;
                        const float wgt = wt[0][xx] * wyz;
                        accA[o] += wgt * vA;
                        accB[o] += wgt * vB;
                        vA += gAx;
                        vB += gBx;
                    }
                }
            }
        }
        // flush: each lane stores its two channels of node o as one float2 of
        // T4[o][c]; then node n sums T4[o][n - o] over the offsets o whose
        // cell lies in the tile (all 27 offsets walked by every lane, the
        // shared-memory offsets compile-time) and issues one vector atomic
#pragma unroll
        for (int o = 0; o < 27; ++o)
            reinterpret_cast<float2*>(&T4[o * 64 + c])[h] = make_float2(accA[o], accB[o]);
        __syncthreads();
        for (int n = threadIdx.x; n < TILE_NODES; n += P2GP_T) {
            const int nx = n % TN, ny = (n / TN) % TN, nz = n / (TN * TN);
            const float4 a4 = tile_node_sum(T4, nx, ny, nz);
            const int gi = ox + nx, gj = oy + ny, gk = oz0 + nz;
            if (a4.x != 0.f && gi < sc.n[0] && gj < sc.n[1] && gk < sc.n[2])
                atomicAdd(&V.grid_mp[node_index(sc, gi, gj, gk)], a4);
        }
        __syncthreads();
        if (threadIdx.x == 0) s_work = early ? next_work : atomicAdd(&V.counters[CNT_P2G_CURSOR], 1u);
    }
    if (flags) atomicOr(&V.counters[CNT_FLAGS], flags);
}

// ------------------------------------ P2G, balanced particle runs (MLS)
// Variant 4: variant 3's lane pairs and accumulators, with the work split by
// particles instead of by cells.  A work item's sorted particles (a tile, or
// a slice of one) are cut into 4 warp parts at the cell boundaries nearest
// the quarter points, and each warp cuts its part into 16 equal runs, one per
// lane pair.  A pair walks its run in key order; when it passes the last
// particle of a cell it owns that cell and writes the cell's 27 node sums to
// the flush table (one writer per cell).  A run that ends inside a cell
// leaves a partial sum: after the walk, a segmented scan over the warp's
// pairs (shuffles) gathers each cell's partials into the last of them, which
// adds them to the owner's entry.  Warp parts end at cell boundaries, so a
// cell never spans two warps.  A tile's longest walk is then about its
// particle count / 64 instead of its fullest cell's count.  Needs the sort's
// cell table (contiguous ranges of the tile's 64 cells).
constexpr int P2GR_T = 128;

__device__ __forceinline__ void runs_store(float4* T4, uint32_t c, int h, const float* accA, const float* accB) {
#pragma unroll
    for (int o = 0; o < 27; ++o) reinterpret_cast<float2*>(&T4[o * 64 + c])[h] = make_float2(accA[o], accB[o]);
}

template <bool SPARSE>
__global__ void __launch_bounds__(P2GR_T, 5) k_p2g_runs(View V) {
    __shared__ float4 T4[27 * 64];                // [offset o][cell]: the 4 channels of cell's node o
    __shared__ uint32_t s_end[P2GR_T / 32][64];   // per warp: end of each cell's range in the item
    __shared__ uint32_t s_work;
    constexpr uint32_t FULL = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int q = lane >> 1, h = lane & 1;
    const int64_t N = V.N;
    uint32_t flags = 0;
    uint32_t* const wend = s_end[wp];
    const uint32_t ntiles = V.counters[CNT_CTILES];
    // slices of a tile's particles when tiles are few (see k_p2g_cells)
    const uint32_t S = ntiles ? min(4u, max(1u, (gridDim.x + ntiles - 1) / ntiles)) : 1u;
    const uint32_t nwork = ntiles * S;
    const bool early = nwork >= 2u * gridDim.x;
    uint32_t next_work = 0;
    if (threadIdx.x == 0) s_work = atomicAdd(&V.counters[CNT_P2G_CURSOR], 1u);
    for (;;) {
        __syncthreads();
        const uint32_t w = s_work;
        if (w >= nwork) break;
        if (early && threadIdx.x == 0) next_work = atomicAdd(&V.counters[CNT_P2G_CURSOR], 1u);
        const uint32_t wt = w / S, slice = w - wt * S;
        const uint32_t ct = V.ptile_list ? V.ptile_list[wt] : V.ctile_list[wt];
        const uint2 rg = V.ctile_range[ct];
        const int s = V.S == 1 ? 0 : scene_of_cell_tile(V.scenes, V.S, (int)ct);
        const SceneDev& sc = scene_ref(V, s);
        int ox, oy, oz0;
        tile_origin(V, sc, ct, ox, oy, oz0);
        // the item's particles [lo, hi) and its cells' ranges clamped to them
        // (lane holds cells lane and lane + 32)
        const uint32_t P = rg.y > rg.x ? rg.y - rg.x : 0u;
        const uint32_t lo = rg.x + (uint32_t)(((uint64_t)P * slice) / S);
        const uint32_t hi = rg.x + (uint32_t)(((uint64_t)P * (slice + 1)) / S);
        const uint2 r0 = V.cell_range[(size_t)ct * 64 + lane], r1 = V.cell_range[(size_t)ct * 64 + 32 + lane];
        const uint32_t s0 = min(max(r0.x, lo), hi), s1 = min(max(r1.x, lo), hi);
        const uint32_t e0 = min(max(r0.y, lo), hi), e1 = min(max(r1.y, lo), hi);
        if ((lane == 0 && s0 != lo) || (lane == 31 && e1 != hi)) flags |= FLAG_TILE_RANGE;
        wend[lane] = e0;
        wend[lane + 32] = e1;
        // warp part [b0, b1): the cell starts nearest the quarter points
        auto bound = [&](int k) -> uint32_t {
            if (k == 0) return lo;
            if (k == 4) return hi;
            const uint32_t t = lo + (uint32_t)(((uint64_t)(hi - lo) * (uint32_t)k) / 4u);
            const uint32_t a = __reduce_max_sync(FULL, max(s0 <= t ? s0 : lo, s1 <= t ? s1 : lo));
            const uint32_t b = __reduce_min_sync(FULL, min(s0 >= t ? s0 : hi, s1 >= t ? s1 : hi));
            return t - a <= b - t ? a : b;
        };
        const uint32_t b0 = bound(wp), b1 = max(bound(wp + 1), b0);
        const uint32_t len = (b1 - b0 + 15u) >> 4;
        const uint32_t i0 = min(b0 + (uint32_t)q * len, b1), i1 = min(i0 + len, b1);
        __syncwarp();
        // cells without particles in the item get a zero entry (warp wp: cells
        // 16 wp .. 16 wp + 15, the half-warps take alternate offsets)
        {
            const int zc = 16 * wp + (lane & 15);
            const uint32_t zs = zc == 0 ? lo : wend[zc - 1];
            if (wend[zc] == zs)
                for (int o = lane >> 4; o < 27; o += 2) T4[o * 64 + zc] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        float accA[27], accB[27];
#pragma unroll
        for (int o = 0; o < 27; ++o) accA[o] = accB[o] = 0.f;
        // the cell of particle i0: the first cell whose range ends after it
        uint32_t c = 0, cend = 0;
        if (i0 < i1) {
            uint32_t l = 0, r = 63;
            while (l < r) {
                const uint32_t m = (l + r) >> 1;
                if (wend[m] > i0) r = m; else l = m + 1;
            }
            c = l;
            cend = wend[c];
        }
        // the next particle's index is loaded one iteration ahead, so an
        // iteration's payload loads do not wait on its index load (P2G of the
        // two-material drop: 110.5 -> 107.4 us)
        uint32_t pn = i0 < i1 ? V.order[i0] : 0u;
        for (uint32_t i = i0; i < i1; ++i) {
            const uint32_t p = pn;
            if (i + 1 < i1) pn = V.order[i + 1];
            if (i == cend) {
                // the run passed the last particle of cell c: its sums are final
                runs_store(T4, c, h, accA, accB);
#pragma unroll
                for (int o = 0; o < 27; ++o) accA[o] = accB[o] = 0.f;
                while (c < 63) {  // next cell with particles (c stays a cell index)
                    ++c;
                    if (wend[c] > i) break;
                }
                cend = wend[c];
            }
            if (p >= (uint32_t)N) {
                flags |= FLAG_TILE_RANGE;
                continue;
            }
            const float4 a0 = V.pay[p], a1 = V.pay[N + p], a2 = V.pay[2 * N + p], a3 = V.pay[3 * N + p];
            // channels as in k_p2g_pairs (lane 0: m, p_x; lane 1: p_y, p_z)
            const float bA = h ? a0.y : a0.w, bB = h ? a0.z : a0.x;
            const float gAx = h ? a1.w : 0.f, gAy = h ? a2.x : 0.f, gAz = h ? a2.y : 0.f;
            const float gBx = h ? a2.z : a1.x, gBy = h ? a2.w : a1.y, gBz = h ? a3.x : a1.z;
            float wt[3][3];
            mls_weights(a3.y, wt[0]);
            mls_weights(a3.z, wt[1]);
            mls_weights(a3.w, wt[2]);
#pragma unroll
            for (int zz = 0; zz < 3; ++zz) {
                const float zA = bA + gAz * (float)zz, zB = bB + gBz * (float)zz;
#pragma unroll
                for (int yy = 0; yy < 3; ++yy) {
                    const float wyz = wt[1][yy] * wt[2][zz];
                    float vA = zA + gAy * (float)yy, vB = zB + gBy * (float)yy;
#pragma unroll
                    for (int xx = 0; xx < 3; ++xx) {
                        const int o = xx + 3 * yy + 9 * zz;
                        const float wgt = wt[0][xx] * wyz;
                        accA[o] += wgt * vA;
                        accB[o] += wgt * vB;
                        vA += gAx;
                        vB += gBx;
                    }
                }
            }
        }
        // a run that ends where its cell ends owns that cell; otherwise the
        // cell's owner is a later pair of this warp and the sum is partial
        const bool open = i0 < i1 && i1 != cend;
        if (i0 < i1 && !open) runs_store(T4, c, h, accA, accB);
        __syncwarp();
        // segmented inclusive scan of the partial sums over consecutive pairs
        // of the same cell; the last pair of a segment then holds its total
        const uint32_t key = open ? c : FULL;
        const uint32_t pkey = __shfl_up_sync(FULL, key, 2), nkey = __shfl_down_sync(FULL, key, 2);
        const bool head = open && (q == 0 || pkey != key);
        const uint32_t heads = __ballot_sync(FULL, head && h == 0);
        const int dist = open ? q - ((31 - __clz(heads & (FULL >> (31 - lane)))) >> 1) : 0;
        const int maxd = __reduce_max_sync(FULL, dist);
        for (int d = 1; d <= maxd; d <<= 1) {
            const bool take = dist >= d;
#pragma unroll
            for (int o = 0; o < 27; ++o) {
                const float a = __shfl_up_sync(FULL, accA[o], 2 * d);
                const float b = __shfl_up_sync(FULL, accB[o], 2 * d);
                if (take) {
                    accA[o] += a;
                    accB[o] += b;
                }
            }
        }
        if (open && (q == 15 || nkey != key)) {
#pragma unroll
            for (int o = 0; o < 27; ++o) {
                float2* t = reinterpret_cast<float2*>(&T4[o * 64 + c]) + h;
                const float2 v = *t;
                *t = make_float2(v.x + accA[o], v.y + accB[o]);
            }
        }
        __syncthreads();
        uint32_t nb[8];  // sparse: the slots of the 8 node tiles of the tile's node block
        if (SPARSE) sp_load_nbr(V.sp, ct, nb);
        for (int n = threadIdx.x; n < TILE_NODES; n += P2GR_T) {
            const int nx = n % TN, ny = (n / TN) % TN, nz = n / (TN * TN);
            const float4 a4 = tile_node_sum(T4, nx, ny, nz);
            const int gi = ox + nx, gj = oy + ny, gk = oz0 + nz;
            if (a4.x != 0.f && gi < sc.n[0] && gj < sc.n[1] && gk < sc.n[2]) {
                if (SPARSE)
                    atomicAdd(&V.grid_mp[sp_node(nb, gi, gj, gk, ox, oy, oz0)], a4);
                else
                    atomicAdd(&V.grid_mp[node_index(sc, gi, gj, gk)], a4);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) s_work = early ? next_work : atomicAdd(&V.counters[CNT_P2G_CURSOR], 1u);
    }
    if (flags) atomicOr(&V.counters[CNT_FLAGS], flags);
}

// ------------------------------ adjoint scatter, balanced particle runs
// Reverse of G2P (the adjoint payload scattered to the grid adjoint) with
// k_p2g_runs' work split at one lane per run: a particle's adjoint payload
// takes a whole thread's registers.  A 64-thread block takes a tile (or a
// slice of one); its two warps take the halves split at the cell boundary
// nearest the midpoint, and each lane an equal run of its half.  A run
// stores the sums of each cell whose last particle it passes (one writer
// per cell); partial sums of runs that end inside a cell are gathered by a
// segmented scan over the warp's lanes into the last of them, which adds
// them to the owner's entry.  Against one thread per cell, a tile's longest
// walk drops from its fullest cell's count to about count/64.
constexpr int ADJR_T = 64;

__device__ __forceinline__ void adj_runs_store(float4* T4, uint32_t c, const float (*acc)[3]) {
#pragma unroll
    for (int o = 0; o < 27; ++o) T4[o * 64 + c] = make_float4(0.f, acc[o][0], acc[o][1], acc[o][2]);
}

template <bool MULTI, bool FLUID>
__global__ void __launch_bounds__(ADJR_T, 6) k_adj_runs(View V, AdjView AV) {
    __shared__ float4 T4[27 * 64];                // [offset o][cell]: (0, adjoint of p) of cell's node o
    __shared__ uint32_t s_end[ADJR_T / 32][64];   // per warp: end of each cell's range in the item
    __shared__ uint32_t s_work;
    constexpr uint32_t FULL = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int64_t N = V.N;
    uint32_t flags = 0;
    uint32_t* const wend = s_end[wp];
    const uint32_t ntiles = V.counters[CNT_CTILES];
    // slices of a tile's particles when tiles are few (see k_p2g_cells)
    const uint32_t S = ntiles ? min(4u, max(1u, (gridDim.x + ntiles - 1) / ntiles)) : 1u;
    const uint32_t nwork = ntiles * S;
    const bool early = nwork >= 2u * gridDim.x;
    uint32_t next_work = 0;
    if (threadIdx.x == 0) s_work = atomicAdd(&V.counters[CNT_P2G_CURSOR], 1u);
    for (;;) {
        __syncthreads();
        const uint32_t w = s_work;
        if (w >= nwork) break;
        if (early && threadIdx.x == 0) next_work = atomicAdd(&V.counters[CNT_P2G_CURSOR], 1u);
        const uint32_t wt = w / S, slice = w - wt * S;
        const uint32_t ct = V.ptile_list ? V.ptile_list[wt] : V.ctile_list[wt];
        const uint2 rg = V.ctile_range[ct];
        const int s = V.S == 1 ? 0 : scene_of_cell_tile(V.scenes, V.S, (int)ct);
        const SceneDev& sc = scene_ref(V, s);
        const int lt = (int)ct - sc.ct_base;
        const int ox = 4 * (lt % sc.ct[0]), oy = 4 * ((lt / sc.ct[0]) % sc.ct[1]),
                  oz0 = 4 * (lt / (sc.ct[0] * sc.ct[1]));
        // the item's particles [lo, hi) and its cells' ranges clamped to them
        // (lane holds cells lane and lane + 32)
        const uint32_t P = rg.y > rg.x ? rg.y - rg.x : 0u;
        const uint32_t lo = rg.x + (uint32_t)(((uint64_t)P * slice) / S);
        const uint32_t hi = rg.x + (uint32_t)(((uint64_t)P * (slice + 1)) / S);
        const uint2 r0 = V.cell_range[(size_t)ct * 64 + lane], r1 = V.cell_range[(size_t)ct * 64 + 32 + lane];
        const uint32_t s0 = min(max(r0.x, lo), hi), s1 = min(max(r1.x, lo), hi);
        const uint32_t e0 = min(max(r0.y, lo), hi), e1 = min(max(r1.y, lo), hi);
        if ((lane == 0 && s0 != lo) || (lane == 31 && e1 != hi)) flags |= FLAG_TILE_RANGE;
        wend[lane] = e0;
        wend[lane + 32] = e1;
        // warp half [b0, b1): split at the cell start nearest the midpoint
        uint32_t mid;
        {
            const uint32_t t = lo + ((hi - lo) >> 1);
            const uint32_t a = __reduce_max_sync(FULL, max(s0 <= t ? s0 : lo, s1 <= t ? s1 : lo));
            const uint32_t b = __reduce_min_sync(FULL, min(s0 >= t ? s0 : hi, s1 >= t ? s1 : hi));
            mid = t - a <= b - t ? a : b;
        }
        const uint32_t b0 = wp == 0 ? lo : mid, b1 = wp == 0 ? mid : hi;
        const uint32_t len = (b1 - b0 + 31u) >> 5;
        const uint32_t i0 = min(b0 + (uint32_t)lane * len, b1), i1 = min(i0 + len, b1);
        __syncwarp();
        // cells without particles in the item get a zero entry (warp wp:
        // cells 32 wp .. 32 wp + 31)
        {
            const int zc = 32 * wp + lane;
            const uint32_t zs = zc == 0 ? lo : wend[zc - 1];
            if (wend[zc] == zs)
                for (int o = 0; o < 27; ++o) T4[o * 64 + zc] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        float acc[27][3];
#pragma unroll
        for (int o = 0; o < 27; ++o) acc[o][0] = acc[o][1] = acc[o][2] = 0.f;
        // the cell of particle i0: the first cell whose range ends after it
        uint32_t c = 0, cend = 0;
        if (i0 < i1) {
            uint32_t l = 0, r = 63;
            while (l < r) {
                const uint32_t m = (l + r) >> 1;
                if (wend[m] > i0) r = m; else l = m + 1;
            }
            c = l;
            cend = wend[c];
        }
        for (uint32_t i = i0; i < i1; ++i) {
            if (i == cend) {
                // the run passed the last particle of cell c: its sums are final
                adj_runs_store(T4, c, acc);
#pragma unroll
                for (int o = 0; o < 27; ++o) acc[o][0] = acc[o][1] = acc[o][2] = 0.f;
                while (c < 63) {  // next cell with particles (c stays a cell index)
                    ++c;
                    if (wend[c] > i) break;
                }
                cend = wend[c];
            }
            const uint32_t p = V.order[i];
            if (p >= (uint32_t)N) {
                flags |= FLAG_TILE_RANGE;
                continue;
            }
            Stencil st;
            float b[3], Ad[9];
            adj_payload<MULTI, FLUID>(V, AV, sc, p, st, flags, b, Ad);
            // node o gets w_o (b + Ad o)
#pragma unroll
            for (int zz = 0; zz < 3; ++zz) {
                const float bz0 = b[0] + Ad[2] * (float)zz, bz1 = b[1] + Ad[5] * (float)zz,
                            bz2 = b[2] + Ad[8] * (float)zz;
#pragma unroll
                for (int yy = 0; yy < 3; ++yy) {
                    const float wyz = st.w[1][yy] * st.w[2][zz];
                    float v0 = bz0 + Ad[1] * (float)yy, v1 = bz1 + Ad[4] * (float)yy, v2 = bz2 + Ad[7] * (float)yy;
#pragma unroll
                    for (int xx = 0; xx < 3; ++xx) {
                        const int o = xx + 3 * yy + 9 * zz;
                        const float wgt = st.w[0][xx] * wyz;
                        acc[o][0] += wgt * v0;
                        acc[o][1] += wgt * v1;
                        acc[o][2] += wgt * v2;
                        v0 += Ad[0];
                        v1 += Ad[3];
                        v2 += Ad[6];
                    }
                }
            }
        }
        // a run that ends where its cell ends owns that cell; otherwise the
        // cell's owner is a later lane of this warp and the sum is partial
        const bool open = i0 < i1 && i1 != cend;
        if (i0 < i1 && !open) adj_runs_store(T4, c, acc);
        __syncwarp();
        // segmented inclusive scan of the partial sums over consecutive lanes
        // of the same cell; the last lane of a segment then holds its total
        const uint32_t key = open ? c : FULL;
        const uint32_t pkey = __shfl_up_sync(FULL, key, 1), nkey = __shfl_down_sync(FULL, key, 1);
        const bool head = open && (lane == 0 || pkey != key);
        const uint32_t heads = __ballot_sync(FULL, head);
        const int dist = open ? lane - (31 - __clz(heads & (FULL >> (31 - lane)))) : 0;
        const int maxd = __reduce_max_sync(FULL, dist);
        for (int d = 1; d <= maxd; d <<= 1) {
            const bool take = dist >= d;
#pragma unroll
            for (int o = 0; o < 27; ++o) {
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float a = __shfl_up_sync(FULL, acc[o][k], d);
                    if (take) acc[o][k] += a;
                }
            }
        }
        if (open && (lane == 31 || nkey != key)) {
#pragma unroll
            for (int o = 0; o < 27; ++o) {
                float4 t = T4[o * 64 + c];
                t.y += acc[o][0];
                t.z += acc[o][1];
                t.w += acc[o][2];
                T4[o * 64 + c] = t;
            }
        }
        __syncthreads();
        for (int n = threadIdx.x; n < TILE_NODES; n += ADJR_T) {
            const int nx = n % TN, ny = (n / TN) % TN, nz = n / (TN * TN);
            const float4 a4 = tile_node_sum(T4, nx, ny, nz);
            const int gi = ox + nx, gj = oy + ny, gk = oz0 + nz;
            if ((a4.y != 0.f || a4.z != 0.f || a4.w != 0.f) && gi < sc.n[0] && gj < sc.n[1] && gk < sc.n[2])
                atomicAdd(&V.grid_mp[node_index(sc, gi, gj, gk)], a4);
        }
        __syncthreads();
        if (threadIdx.x == 0) s_work = early ? next_work : atomicAdd(&V.counters[CNT_P2G_CURSOR], 1u);
    }
    if (flags) atomicOr(&V.counters[CNT_FLAGS], flags);
}

// ------------------------------------------------------------ grid update
template <int PHYS>
__global__ void k_grid(View V) {
    // P2G has finished with its work cursor: leave it at zero for the reverse
    // of this step, whose scatter takes work from the same cursor
    if (blockIdx.x == 0 && threadIdx.x == 0) V.counters[CNT_P2G_CURSOR] = 0u;
    const uint32_t count = V.counters[CNT_TILES];
    const int tiles_per_block = blockDim.x >> 6;
    const int l = threadIdx.x & 63;
    uint32_t active = 0;
    for (uint32_t w = blockIdx.x * tiles_per_block + (threadIdx.x >> 6); w < count;
         w += gridDim.x * tiles_per_block) {
        const uint32_t nt = V.tile_list[w];
        if (nt >= (uint32_t)V.total_nt) continue;
        const int s = V.S == 1 ? 0 : scene_of_node_tile(V.scenes, V.S, (int)nt);
        const SceneDev& sc = scene_ref(V, s);
        int i, j, k;
        if (V.sp.cap) {  // sparse: the slot's coordinates
            sp_decode(V.sp.code[nt], i, j, k);
        } else {
            const int lt = (int)nt - sc.nt_base;
            i = lt % sc.nt[0];
            j = (lt / sc.nt[0]) % sc.nt[1];
            k = lt / (sc.nt[0] * sc.nt[1]);
        }
        i = 4 * i + (l & 3);
        j = 4 * j + ((l >> 2) & 3);
        k = 4 * k + (l >> 4);
        const int64_t idx = ((int64_t)nt << 6) + l;
        const float4 mp = V.grid_mp[idx];
        float v[3] = {0.f, 0.f, 0.f};
        if (PHYS == PHYS_MLS) {
            if (mp.x > 0.f) {
                v[0] = __fdiv_rn(mp.y, mp.x) + sc.dt * sc.gravity[0];
                v[1] = __fdiv_rn(mp.z, mp.x) + sc.dt * sc.gravity[1];
                v[2] = __fdiv_rn(mp.w, mp.x) + sc.dt * sc.gravity[2];
                ++active;
            }
            if (V.grid_vpre) V.grid_vpre[idx] = make_float4(v[0], v[1], v[2], mp.x);
            apply_bc(sc, i, j, k, v);
        } else {
            // material_point_method.h:572-597: p += (m g) dt, v = p / m
            if (mp.x > 1e-10f) {
                v[0] = __fdiv_rn(__fadd_rn(mp.y, __fmul_rn(__fmul_rn(mp.x, sc.gravity[0]), sc.dt)), mp.x);
                v[1] = __fdiv_rn(__fadd_rn(mp.z, __fmul_rn(__fmul_rn(mp.x, sc.gravity[1]), sc.dt)), mp.x);
                v[2] = __fdiv_rn(__fadd_rn(mp.w, __fmul_rn(__fmul_rn(mp.x, sc.gravity[2]), sc.dt)), mp.x);
            }
            if (mp.x > 0.f) ++active;
        }
        V.grid_v[idx] = make_float4(v[0], v[1], v[2], mp.x);
        V.grid_mp[idx] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (V.sp.cap) {
            // sparse: into the node block of every occupied cell tile that
            // holds this node (offset q: the node tile is q above the cell
            // tile; the node lies in its 6^3 block when its local
            // coordinate is below 2 along each axis of q)
            const uint32_t stamp = V.counters[CNT_STAMP];
            const int lx = l & 3, ly = (l >> 2) & 3, lz = l >> 4;
            const float4 gv = make_float4(v[0], v[1], v[2], mp.x);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int dx = q & 1, dy = (q >> 1) & 1, dz = q >> 2;
                if ((dx && lx > 1) || (dy && ly > 1) || (dz && lz > 1)) continue;
                const uint2 r = V.sp.rev[8 * (size_t)nt + q];
                if (r.y != stamp) continue;
                V.sp.box[216 * (size_t)r.x + (lx + 4 * dx) + TN * ((ly + 4 * dy) + TN * (lz + 4 * dz))] = gv;
            }
        }
    }
    // active node count: warp sums, then one atomic per block (a single
    // counter word takes every block's add)
    __shared__ uint32_t s_active;
    if (threadIdx.x == 0) s_active = 0u;
    __syncthreads();
    uint32_t a = active;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xFFFFFFFFu, a, o);
    if ((threadIdx.x & 31) == 0 && a) atomicAdd(&s_active, a);
    __syncthreads();
    if (threadIdx.x == 0 && s_active)
        atomicAdd(reinterpret_cast<unsigned long long*>(&V.counters[CNT_ACTIVE]), (unsigned long long)s_active);
}

// ------------------------------------------------------------------- G2P
// APIC sums of one MLS particle over its 27 stencil nodes: nv = sum w v and
// S = sum w v o^T (o the integer stencil offset, so B = sum w v d^T =
// dx (S - nv f^T)).  row(j, k, g0, g1, g2) fetches the (v, m) float4 of the
// three nodes (0..2, j, k) of the stencil.
template <class Row>
__device__ __forceinline__ void mls_gather(const Stencil& st, const Row& row, float nv[3], float S[9]) {
    nv[0] = nv[1] = nv[2] = 0.f;
#pragma unroll
    for (int a = 0; a < 9; ++a) S[a] = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float wjk = st.w[1][j] * st.w[2][k];
            float4 g0, g1, g2;
            row(j, k, g0, g1, g2);
            const float w0 = st.w[0][0] * wjk, w1 = st.w[0][1] * wjk, w2 = st.w[0][2] * wjk;
            const float r1x = w1 * g1.x, r1y = w1 * g1.y, r1z = w1 * g1.z;
            const float r2x = w2 * g2.x, r2y = w2 * g2.y, r2z = w2 * g2.z;
            const float sx = w0 * g0.x + r1x + r2x, sy = w0 * g0.y + r1y + r2y, sz = w0 * g0.z + r1z + r2z;
            nv[0] += sx; nv[1] += sy; nv[2] += sz;
            S[0] += r1x + 2.f * r2x; S[3] += r1y + 2.f * r2y; S[6] += r1z + 2.f * r2z;
            if (j) {
                const float fj = (float)j;
                S[1] += fj * sx; S[4] += fj * sy; S[7] += fj * sz;
            }
            if (k) {
                const float fk = (float)k;
                S[2] += fk * sx; S[5] += fk * sy; S[8] += fk * sz;
            }
        }
    }
}

// APIC matrix C = D B = D dx (S - nv f^T) from the gathered sums.
__device__ __forceinline__ void mls_affine(const SceneDev& sc, const Stencil& st, const float nv[3], const float S[9],
                                           float C[9]) {
    const float dx = sc.dx;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) C[3 * a + b] = sc.D * dx * (S[3 * a + b] - nv[a] * st.f[b]);
}

// F <- (I + dt C) F (a fluid's F reset to its volumetric part, cbrt(J) I)
// and x <- x + dt v.
// mid: the particle's material id (0 with one material).
template <bool FLUID>
__device__ __forceinline__ void mls_advance(const View& V, const SceneDev& sc, int mid, const float nv[3],
                                            const float C[9], const float F[9], float x[3], float Fn[9]) {
    float M[9];
#pragma unroll
    for (int a = 0; a < 9; ++a) M[a] = sc.dt * C[a] + (a % 4 == 0 ? 1.f : 0.f);
    m3_mul(M, F, Fn);
    if (FLUID) {
        if (V.mats[mid].model == MODEL_EOS) {
            const float c = cbrtf(m3_det(Fn));
#pragma unroll
            for (int a = 0; a < 9; ++a) Fn[a] = (a % 4 == 0) ? c : 0.f;
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) x[a] = x[a] + sc.dt * nv[a];
}

// Per-particle G2P update shared by both G2P variants; `fetch(i, j, k)`
// returns the (v, m) float4 of grid node (i, j, k) of scene sc.
// PLASTIC: the payload's stress includes the von Mises cap (launched when an
// ELASTOPLASTIC material is present).
// SPARSE (MLS, physical order, live solver only): the grid is the slot pool
// of V.sp; the particle's tile is the slot of the key it was sorted by (read
// before the new key overwrites it).
// CHECK (MLS, dense, replaying recorded steps): V.keys holds the keys the
// forward recorded for the next step; a new key that differs replaces it and
// sets *V.resort, so that the next step sorts again instead of keeping the
// recorded sort.
template <int PHYS, bool MULTI, bool FLUID, bool PLASTIC, class Fetch, bool SPARSE = false, bool CHECK = false>
__device__ __forceinline__ void g2p_particle(const View& V, const SceneDev& sc, uint32_t p, const Fetch& fetch,
                                             uint32_t& flags) {
    const int64_t N = V.N;
    const float4 q0 = V.q[p];
    float x[3] = {q0.x, q0.y, q0.z};
    Stencil st;
    make_stencil<PHYS>(sc, x, st, flags);
    if (PHYS == PHYS_MLS) {
        const float4 q1 = V.q[N + p], q2 = V.q[2 * N + p];
        float xx[3], F[9];
        unpack_xF(q0, q1, q2, xx, F);
        float nv[3], S[9];
        uint32_t oslot = 0;
        int ox = 0, oy = 0, oz = 0;
        if (SPARSE) {
            const uint32_t okey = V.keys[p];
            if (okey >= (uint32_t)V.total_ct * 64u) {  // no slot (a full pool): the particle is left as is
                flags |= FLAG_TILE_POOL;
                return;
            }
            oslot = okey >> 6;
            sp_decode(V.sp.code[oslot], ox, oy, oz);
            ox *= 4;
            oy *= 4;
            oz *= 4;
            int l[3] = {st.s[0] - ox, st.s[1] - oy, st.s[2] - oz};
            if ((unsigned)l[0] > 3u || (unsigned)l[1] > 3u || (unsigned)l[2] > 3u) {
                // not in the tile it was sorted into: keep the gather inside
                // that tile's node block and report it
                flags |= FLAG_TILE_RANGE;
#pragma unroll
                for (int a = 0; a < 3; ++a) l[a] = min(max(l[a], 0), 3);
            }
            // the tile's node block, written by this step's grid update
            const float4* box = V.sp.box + 216 * (size_t)oslot + l[0] + TN * (l[1] + TN * l[2]);
            mls_gather(st, [&](int j, int k, float4& g0, float4& g1, float4& g2) {
                const float4* r = box + TN * (j + TN * k);
                g0 = __ldg(r);
                g1 = __ldg(r + 1);
                g2 = __ldg(r + 2);
            }, nv, S);
        } else {
            // separable tiled node index: idx = X[i] + Y[j] + Z[k]
            int X[3], Y[3], Z[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const int gi = st.s[0] + a, gj = st.s[1] + a, gk = st.s[2] + a;
                X[a] = ((gi >> 2) << 6) + (gi & 3);
                Y[a] = (gj >> 2) * (sc.nt[0] << 6) + ((gj & 3) << 2);
                Z[a] = (gk >> 2) * ((sc.nt[0] * sc.nt[1]) << 6) + ((gk & 3) << 4) + (sc.nt_base << 6);
            }
            mls_gather(st, [&](int j, int k, float4& g0, float4& g1, float4& g2) {
                const int row = Y[j] + Z[k];
                g0 = fetch(st.s[0], st.s[1] + j, st.s[2] + k, row + X[0]);
                g1 = fetch(st.s[0] + 1, st.s[1] + j, st.s[2] + k, row + X[1]);
                g2 = fetch(st.s[0] + 2, st.s[1] + j, st.s[2] + k, row + X[2]);
            }, nv, S);
        }
        float C[9], Fn[9];
        mls_affine(sc, st, nv, S, C);
        float4* qo = V.q_out;
        if (V.write_vc) {  // else the next step of the call reads v, C from the payload only
            float4 o3, o4, o5;
            pack_vC(nv, C, o3, o4, o5);
            qo[3 * N + p] = o3;
            qo[4 * N + p] = o4;
            qo[5 * N + p] = o5;
        }
        mls_advance<FLUID>(V, sc, MULTI ? V.mat[p] : 0, nv, C, F, x, Fn);
        float4 o0, o1, o2;
        pack_xF(x, Fn, o0, o1, o2);
        qo[p] = o0;
        qo[N + p] = o1;
        qo[2 * N + p] = o2;
        // key and P2G payload of the new state for the next step
        int so[3];
        float fn[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float u;
            so[a] = stencil_origin(x[a], sc.origin[a], sc.dx, sc.inv_dx, sc.n[a], PHYS, u, flags);
            fn[a] = fminf(fmaxf(__fsub_rn(u, (float)so[a]), 0.5f), 1.5f);
        }
        if (SPARSE) {
            const int tx = so[0] >> 2, ty = so[1] >> 2, tz = so[2] >> 2;
            const uint32_t slot = (4 * tx == ox && 4 * ty == oy && 4 * tz == oz)
                                      ? oslot
                                      : sp_find_or_insert(V.sp, sp_code(tx, ty, tz), flags);
            V.keys[p] = slot == SP_NONE ? SP_NONE
                                        : slot * 64u + (uint32_t)((so[2] & 3) * 16 + (so[1] & 3) * 4 + (so[0] & 3));
        } else if (CHECK) {
            const uint32_t nk = cell_key(sc, so);
            if (V.keys[p] != nk) {  // rare: the replay rounded across a cell face
                V.keys[p] = nk;
                atomicOr(V.resort, 1u);
            }
        } else {
            V.keys[p] = cell_key(sc, so);
        }
        if (V.pay_out) {
            const float2 mv = V.mV[p];
            float4 a0, a1, a2, a3;
            mls_payload<PLASTIC>(sc, V.mats[MULTI ? V.mat[p] : 0], fn, Fn, nv, C, mv.x, mv.y, a0, a1, a2, a3);
            V.pay_out[p] = a0;
            V.pay_out[N + p] = a1;
            V.pay_out[2 * N + p] = a2;
            V.pay_out[3 * N + p] = a3;
        }
        return;
    } else {
        // material_point_method.h:599-666 in the same order of operations
        float nv[3] = {0.f, 0.f, 0.f};
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
                    const float weight = __fmul_rn(__fmul_rn(st.w[0][ii], st.w[1][j]), st.w[2][k]);
                    if (!(weight > 1e-10f)) continue;
                    const float4 g = fetch(gi, gj, gk, (int)node_index(sc, gi, gj, gk));
                    nv[0] = __fadd_rn(nv[0], __fmul_rn(weight, g.x));
                    nv[1] = __fadd_rn(nv[1], __fmul_rn(weight, g.y));
                    nv[2] = __fadd_rn(nv[2], __fmul_rn(weight, g.z));
                }
            }
        }
        const float4 q3 = V.q[3 * N + p];
#pragma unroll
        for (int a = 0; a < 3; ++a) x[a] = __fadd_rn(x[a], __fmul_rn(nv[a], sc.dt));
        V.q[p] = make_float4(x[0], x[1], x[2], q0.w);
        V.q[3 * N + p] = make_float4(nv[0], nv[1], nv[2], q3.w);
    }
    // key of the new position for the next step's sort
    int so[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float u;
        so[a] = stencil_origin(x[a], sc.origin[a], sc.dx, sc.inv_dx, sc.n[a], PHYS, u, flags);
    }
    V.keys[p] = cell_key(sc, so);
}

// G2P variants 1 and 2: one thread per particle, 27 gathers through L1.
// Variant 1 visits particles in the step's sorted order; variant 2 in
// physical order (p = i): a gather needs no grouping, the physical order was
// sorted at upload and particles drift less than a cell per step, so
// neighbouring threads still share grid nodes, and the state loads are fully
// coalesced with no dependent load of the order array.
template <int PHYS, bool MULTI, bool FLUID, bool PHYS_ORDER, bool PLASTIC, bool SPARSE = false, bool CHECK = false>
__device__ __forceinline__ void k_g2p_impl(const View& V) {
    const int64_t N = V.N;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    uint32_t flags = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
        const uint32_t p = PHYS_ORDER ? (uint32_t)i : V.order[i];
        if (p >= (uint32_t)N) {
            flags |= FLAG_TILE_RANGE;
            continue;
        }
        const int s = V.S == 1 ? 0 : scene_of_particle(V.scenes, V.S, (int)p);
        const SceneDev& sc = scene_ref(V, s);
        const float4* gv = V.grid_v;
        auto fetch = [&](int, int, int, int idx) { return __ldg(&gv[idx]); };
        g2p_particle<PHYS, MULTI, FLUID, PLASTIC, decltype(fetch), SPARSE, CHECK>(V, sc, p, fetch, flags);
    }
    if (flags) atomicOr(&V.counters[CNT_FLAGS], flags);
}

template <int PHYS, bool MULTI, bool FLUID>
__global__ void k_g2p(View V) {
    k_g2p_impl<PHYS, MULTI, FLUID, false, true>(V);
}
// 64 registers (4 blocks of 256 threads per SM): the gathers' latency wants
// the occupancy more than the few spilled words cost
template <int PHYS, bool MULTI, bool FLUID>
__global__ void __launch_bounds__(512, 2) k_g2p_phys(View V) {
    k_g2p_impl<PHYS, MULTI, FLUID, true, false>(V);
}
// the same with the von Mises cap (an ELASTOPLASTIC material is present)
template <int PHYS, bool MULTI, bool FLUID>
__global__ void __launch_bounds__(512, 2) k_g2p_phys_vm(View V) {
    k_g2p_impl<PHYS, MULTI, FLUID, true, true>(V);
}
// replay of recorded steps (MLS, dense): the new keys are checked against
// the recorded ones (see g2p_particle's CHECK)
template <bool MULTI, bool FLUID, bool PLASTIC>
__global__ void __launch_bounds__(512, 2) k_g2p_check(View V) {
    k_g2p_impl<PHYS_MLS, MULTI, FLUID, true, PLASTIC, false, true>(V);
}
// sparse grids (MLS)
template <bool MULTI, bool FLUID, bool PLASTIC>
__global__ void __launch_bounds__(512, 2) k_g2p_sparse(View V) {
    k_g2p_impl<PHYS_MLS, MULTI, FLUID, true, PLASTIC, true>(V);
}

// G2P variant 0: one block per occupied cell tile; the tile's 6^3 node
// velocities are staged in shared memory once and every particle of the tile
// gathers its 27 nodes from there.
template <int PHYS, bool MULTI, bool FLUID>
__global__ void __launch_bounds__(256) k_g2p_tiles(View V) {
    __shared__ float4 gsm[TILE_NODES];
    __shared__ uint32_t s_work;
    const int64_t N = V.N;
    uint32_t flags = 0;
    const uint32_t ntiles = V.counters[CNT_CTILES];
    for (;;) {
        if (threadIdx.x == 0) s_work = atomicAdd(&V.counters[CNT_G2P_CURSOR], 1u);
        __syncthreads();
        const uint32_t w = s_work;
        if (w >= ntiles) break;
        const uint32_t ct = V.ctile_list[w];
        const uint2 rg = V.ctile_range[ct];
        const int s = V.S == 1 ? 0 : scene_of_cell_tile(V.scenes, V.S, (int)ct);
        const SceneDev& sc = scene_ref(V, s);
        const int lt = (int)ct - sc.ct_base;
        const int ox = 4 * (lt % sc.ct[0]), oy = 4 * ((lt / sc.ct[0]) % sc.ct[1]),
                  oz = 4 * (lt / (sc.ct[0] * sc.ct[1]));
        for (int n = threadIdx.x; n < TILE_NODES; n += blockDim.x) {
            const int gi = ox + n % TN, gj = oy + (n / TN) % TN, gk = oz + n / (TN * TN);
            gsm[n] = (gi < sc.n[0] && gj < sc.n[1] && gk < sc.n[2]) ? V.grid_v[node_index(sc, gi, gj, gk)]
                                                                     : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        __syncthreads();
        const float4* gv = V.grid_v;
        auto fetch = [&](int gi, int gj, int gk, int idx) {
            const unsigned lx = (unsigned)(gi - ox), ly = (unsigned)(gj - oy), lz = (unsigned)(gk - oz);
            if (lx < (unsigned)TN && ly < (unsigned)TN && lz < (unsigned)TN) return gsm[lx + TN * (ly + TN * lz)];
            return __ldg(&gv[idx]);
        };
        for (uint32_t i = rg.x + threadIdx.x; i < rg.y; i += blockDim.x) {
            const uint32_t p = V.order[i];
            if (p >= (uint32_t)N) {
                flags |= FLAG_TILE_RANGE;
                continue;
            }
            g2p_particle<PHYS, MULTI, FLUID, true>(V, sc, p, fetch, flags);
        }
        __syncthreads();
    }
    if (flags) atomicOr(&V.counters[CNT_FLAGS], flags);
}

// ------------------------------------------ fused G2P -> P2G (MLS, variant 5)
// One pass over the particles that does the G2P of this step and the P2G of
// the next: the P2G payload never leaves the SM (the split path writes it to
// HBM in G2P and reads it back in P2G).  Work items are the occupied cell
// tiles of this step's sort (or slices of them when tiles are few), largest
// first, taken from the G2P work cursor (P2G's is left for the reverse
// scatter).  Per item:
//   * the tile's 6^3 node velocities are staged in shared memory: every
//     particle of the tile gathers its 27 nodes from there;
//   * the item's sorted particles are cut into two warp halves at the cell
//     boundary nearest the midpoint and each lane walks an equal run of its
//     half (one lane per run: 27 nodes x 4 channels of register
//     accumulators);
//   * per particle: G2P (v, C, F, x), the new state stored, the next cell
//     key, the stress and the payload of the new state, accumulated into the
//     run's sums.  Particles move less than a cell per step, so a particle's
//     new cell is nearly always its cell of this step's sort: the run's sums
//     stay one cell's sums.  A particle that changed cell adds its 27 nodes
//     to the grid with vector atomics instead;
//   * a run that passes a cell's last particle stores the cell's sums (one
//     writer per cell); runs that end inside a cell are merged by a
//     segmented scan over the warp's lanes; each of the 6^3 nodes the tile
//     touches then sums its <= 27 cells and gets one vector atomic
//     (red.global.add.v4.f32) into grid_mp, which the next grid update
//     reads.
// grid_mp must hold no other contributions on entry (the grid update of
// this step cleared it).  Needs the bin sort's cell table.
// MINB: resident blocks per SM the register budget is cut for (4: up to 255
// registers, no spills; 6: 168 registers, some spilled).
constexpr int G2_T = 64;

// Asynchronous global -> shared copies (cp.async, no registers held while
// the copy is in flight); completion per thread with cp_async_wait<n>.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N_>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N_) : "memory");
}

// One particle's G2P inputs staged in shared memory: q0..q2 (x, F), then
// (m, V0) and the material id.
struct G2Stage {
    float4 q[3];
    float2 mv;
    int32_t mat;
    int32_t pad;
};

template <bool MULTI, bool FLUID, bool PLASTIC, int MINB>
__global__ void __launch_bounds__(G2_T, MINB) k_g2p2g(View V) {
    __shared__ float4 box[TILE_NODES];           // grid_v of the tile's node block
    __shared__ float4 T4[27 * 64];                // [offset o][cell]: (m, p) of cell's node o
    __shared__ uint32_t s_end[G2_T / 32][64];     // per warp: end of each cell's range in the item
    __shared__ G2Stage s_in[2][G2_T];             // per lane: inputs of this and the next particle
    __shared__ uint32_t s_work;
    constexpr uint32_t FULL = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int64_t N = V.N;
    uint32_t flags = 0;
    uint32_t* const wend = s_end[wp];
    const uint32_t ntiles = V.counters[CNT_CTILES];
    // stage particle q's inputs into buffer b of this lane (copies in flight
    // until the matching cp_async_wait)
    auto stage = [&](uint32_t q, int b) {
        if (q >= (uint32_t)N) return;
        G2Stage& d = s_in[b][threadIdx.x];
        cp_async16(&d.q[0], &V.q[q]);
        cp_async16(&d.q[1], &V.q[N + q]);
        cp_async16(&d.q[2], &V.q[2 * N + q]);
        cp_async8(&d.mv, &V.mV[q]);
        if (MULTI) cp_async4(&d.mat, &V.mat[q]);
    };
    // slices of a tile's particles when tiles are few (each slice flushes the
    // tile's whole node block)
    const uint32_t S = ntiles ? min(8u, max(1u, (gridDim.x + ntiles - 1) / ntiles)) : 1u;
    const uint32_t nwork = ntiles * S;
    const bool early = nwork >= 2u * gridDim.x;
    uint32_t next_work = 0;
    if (threadIdx.x == 0) s_work = atomicAdd(&V.counters[CNT_G2P_CURSOR], 1u);
    for (;;) {
        __syncthreads();
        const uint32_t w = s_work;
        if (w >= nwork) break;
        if (early && threadIdx.x == 0) next_work = atomicAdd(&V.counters[CNT_G2P_CURSOR], 1u);
        const uint32_t wt = w / S, slice = w - wt * S;
        const uint32_t ct = V.ptile_list ? V.ptile_list[wt] : V.ctile_list[wt];
        const uint2 rg = V.ctile_range[ct];
        const int s = V.S == 1 ? 0 : scene_of_cell_tile(V.scenes, V.S, (int)ct);
        const SceneDev& sc = scene_ref(V, s);
        const int lt = (int)ct - sc.ct_base;
        const int ox = 4 * (lt % sc.ct[0]), oy = 4 * ((lt / sc.ct[0]) % sc.ct[1]),
                  oz0 = 4 * (lt / (sc.ct[0] * sc.ct[1]));
        for (int n = threadIdx.x; n < TILE_NODES; n += G2_T) {
            const int gi = ox + n % TN, gj = oy + (n / TN) % TN, gk = oz0 + n / (TN * TN);
            box[n] = (gi < sc.n[0] && gj < sc.n[1] && gk < sc.n[2]) ? V.grid_v[node_index(sc, gi, gj, gk)]
                                                                    : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        // the item's particles [lo, hi) and its cells' ranges clamped to them
        // (lane holds cells lane and lane + 32)
        const uint32_t P = rg.y > rg.x ? rg.y - rg.x : 0u;
        const uint32_t lo = rg.x + (uint32_t)(((uint64_t)P * slice) / S);
        const uint32_t hi = rg.x + (uint32_t)(((uint64_t)P * (slice + 1)) / S);
        const uint2 r0 = V.cell_range[(size_t)ct * 64 + lane], r1 = V.cell_range[(size_t)ct * 64 + 32 + lane];
        const uint32_t s0 = min(max(r0.x, lo), hi), s1 = min(max(r1.x, lo), hi);
        const uint32_t e0 = min(max(r0.y, lo), hi), e1 = min(max(r1.y, lo), hi);
        if ((lane == 0 && s0 != lo) || (lane == 31 && e1 != hi)) flags |= FLAG_TILE_RANGE;
        wend[lane] = e0;
        wend[lane + 32] = e1;
        // warp half [b0, b1): split at the cell start nearest the midpoint
        uint32_t mid;
        {
            const uint32_t t = lo + ((hi - lo) >> 1);
            const uint32_t a = __reduce_max_sync(FULL, max(s0 <= t ? s0 : lo, s1 <= t ? s1 : lo));
            const uint32_t b = __reduce_min_sync(FULL, min(s0 >= t ? s0 : hi, s1 >= t ? s1 : hi));
            mid = t - a <= b - t ? a : b;
        }
        const uint32_t b0 = wp == 0 ? lo : mid, b1 = wp == 0 ? mid : hi;
        const uint32_t len = (b1 - b0 + 31u) >> 5;
        const uint32_t i0 = min(b0 + (uint32_t)lane * len, b1), i1 = min(i0 + len, b1);
        __syncwarp();
        // cells without particles in the item get a zero entry (warp wp:
        // cells 32 wp .. 32 wp + 31)
        {
            const int zc = 32 * wp + lane;
            const uint32_t zs = zc == 0 ? lo : wend[zc - 1];
            if (wend[zc] == zs)
                for (int o = 0; o < 27; ++o) T4[o * 64 + zc] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        __syncthreads();  // the node block is staged
        float acc[27][4];
#pragma unroll
        for (int o = 0; o < 27; ++o) acc[o][0] = acc[o][1] = acc[o][2] = acc[o][3] = 0.f;
        // the cell of particle i0: the first cell whose range ends after it
        uint32_t c = 0, cend = 0;
        if (i0 < i1) {
            uint32_t l = 0, r = 63;
            while (l < r) {
                const uint32_t m = (l + r) >> 1;
                if (wend[m] > i0) r = m; else l = m + 1;
            }
            c = l;
            cend = wend[c];
        }
        // Software pipeline over the run: the inputs of particle i + 1 are
        // copied to shared memory while particle i is computed, and the
        // sorted index two ahead is loaded, so an iteration does not wait on
        // HBM for its own particle.
        uint32_t pc = i0 < i1 ? V.order[i0] : 0u;
        uint32_t pn = i0 + 1 < i1 ? V.order[i0 + 1] : 0u;
        if (i0 < i1) stage(pc, 0);
        cp_async_commit();
        for (uint32_t i = i0; i < i1; ++i) {
            const uint32_t p = pc;
            const int cur = (int)((i - i0) & 1u);
            if (i + 1 < i1) stage(pn, cur ^ 1);
            cp_async_commit();
            pc = pn;
            if (i + 2 < i1) pn = V.order[i + 2];
            if (i == cend) {
                // the run passed the last particle of cell c: its sums are final
#pragma unroll
                for (int o = 0; o < 27; ++o) {
                    T4[o * 64 + c] = make_float4(acc[o][0], acc[o][1], acc[o][2], acc[o][3]);
                    acc[o][0] = acc[o][1] = acc[o][2] = acc[o][3] = 0.f;
                }
                while (c < 63) {  // next cell with particles (c stays a cell index)
                    ++c;
                    if (wend[c] > i) break;
                }
                cend = wend[c];
            }
            if (p >= (uint32_t)N) {
                flags |= FLAG_TILE_RANGE;
                continue;
            }
            cp_async_wait<1>();  // this particle's copies are done (the next one's may not be)
            const G2Stage& in = s_in[cur][threadIdx.x];
            // ---- G2P of this step
            float x[3], F[9];
            unpack_xF(in.q[0], in.q[1], in.q[2], x, F);
            Stencil st;
            make_stencil<PHYS_MLS>(sc, x, st, flags);
            const int lx = st.s[0] - ox, ly = st.s[1] - oy, lz = st.s[2] - oz0;
            const bool in_tile = (unsigned)lx <= 3u && (unsigned)ly <= 3u && (unsigned)lz <= 3u;
            // the particle's stencil origin is the run's cell (its sorted key)
            const bool own = in_tile && (uint32_t)(lx + 4 * ly + 16 * lz) == c;
            if (!own) flags |= FLAG_TILE_RANGE;
            float nv[3], Sg[9];
            if (in_tile) {
                const int base = lx + TN * (ly + TN * lz);
                mls_gather(st, [&](int j, int k, float4& g0, float4& g1, float4& g2) {
                    const float4* r = &box[base + TN * (j + TN * k)];
                    g0 = r[0];
                    g1 = r[1];
                    g2 = r[2];
                }, nv, Sg);
            } else {
                // not a particle of this tile's cells (the sort said otherwise):
                // gather from the grid (reported above)
                mls_gather(st, [&](int j, int k, float4& g0, float4& g1, float4& g2) {
                    g0 = __ldg(&V.grid_v[node_index(sc, st.s[0], st.s[1] + j, st.s[2] + k)]);
                    g1 = __ldg(&V.grid_v[node_index(sc, st.s[0] + 1, st.s[1] + j, st.s[2] + k)]);
                    g2 = __ldg(&V.grid_v[node_index(sc, st.s[0] + 2, st.s[1] + j, st.s[2] + k)]);
                }, nv, Sg);
            }
            float C[9], Fn[9];
            mls_affine(sc, st, nv, Sg, C);
            float4* qo = V.q_out;
            if (V.write_vc) {
                float4 o3, o4, o5;
                pack_vC(nv, C, o3, o4, o5);
                qo[3 * N + p] = o3;
                qo[4 * N + p] = o4;
                qo[5 * N + p] = o5;
            }
            mls_advance<FLUID>(V, sc, MULTI ? in.mat : 0, nv, C, F, x, Fn);
            {
                float4 o0, o1, o2;
                pack_xF(x, Fn, o0, o1, o2);
                qo[p] = o0;
                qo[N + p] = o1;
                qo[2 * N + p] = o2;
            }
            // ---- next cell key and the payload of the new state
            int so[3];
            float fn[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                float u;
                so[a] = stencil_origin(x[a], sc.origin[a], sc.dx, sc.inv_dx, sc.n[a], PHYS_MLS, u, flags);
                fn[a] = fminf(fmaxf(__fsub_rn(u, (float)so[a]), 0.5f), 1.5f);
            }
            V.keys[p] = cell_key(sc, so);
            const float2 mv = in.mv;
            float4 a0, a1, a2, a3;
            mls_payload<PLASTIC>(sc, V.mats[MULTI ? in.mat : 0], fn, Fn, nv, C, mv.x, mv.y, a0, a1, a2, a3);
            float m, b[3], Ad[9], f[3];
            unpack_payload(a0, a1, a2, a3, m, b, Ad, f);
            float wt[3][3];
            mls_weights(f[0], wt[0]);
            mls_weights(f[1], wt[1]);
            mls_weights(f[2], wt[2]);
            // ---- P2G of the next step: node o gets w_o (m, b + Ad o)
            if (own && so[0] == st.s[0] && so[1] == st.s[1] && so[2] == st.s[2]) {
#pragma unroll
                for (int zz = 0; zz < 3; ++zz) {
                    const float bz0 = b[0] + Ad[2] * (float)zz, bz1 = b[1] + Ad[5] * (float)zz,
                                bz2 = b[2] + Ad[8] * (float)zz;
#pragma unroll
                    for (int yy = 0; yy < 3; ++yy) {
                        const float wyz = wt[1][yy] * wt[2][zz];
                        float v0 = bz0 + Ad[1] * (float)yy, v1 = bz1 + Ad[4] * (float)yy,
                              v2 = bz2 + Ad[7] * (float)yy;
#pragma unroll
                        for (int xx = 0; xx < 3; ++xx) {
                            const int o = xx + 3 * yy + 9 * zz;
                            const float wgt = wt[0][xx] * wyz;
                            acc[o][0] += wgt * m;
                            acc[o][1] += wgt * v0;
                            acc[o][2] += wgt * v1;
                            acc[o][3] += wgt * v2;
                            v0 += Ad[0];
                            v1 += Ad[3];
                            v2 += Ad[6];
                        }
                    }
                }
            } else {
                // the particle changed cell: its nodes are not the run's cell's
                // (nor are they after an inconsistent sort, reported above)
#pragma unroll
                for (int zz = 0; zz < 3; ++zz)
#pragma unroll
                    for (int yy = 0; yy < 3; ++yy)
#pragma unroll
                        for (int xx = 0; xx < 3; ++xx) {
                            const float wgt = wt[0][xx] * wt[1][yy] * wt[2][zz];
                            const float4 add =
                                make_float4(wgt * m, wgt * (b[0] + Ad[0] * xx + Ad[1] * yy + Ad[2] * zz),
                                            wgt * (b[1] + Ad[3] * xx + Ad[4] * yy + Ad[5] * zz),
                                            wgt * (b[2] + Ad[6] * xx + Ad[7] * yy + Ad[8] * zz));
                            atomicAdd(&V.grid_mp[node_index(sc, so[0] + xx, so[1] + yy, so[2] + zz)], add);
                        }
            }
        }
        cp_async_wait<0>();  // no copy into the stage buffers outlives the item
        // a run that ends where its cell ends owns that cell; otherwise the
        // cell's owner is a later lane of this warp and the sum is partial
        const bool open = i0 < i1 && i1 != cend;
        if (i0 < i1 && !open)
#pragma unroll
            for (int o = 0; o < 27; ++o) T4[o * 64 + c] = make_float4(acc[o][0], acc[o][1], acc[o][2], acc[o][3]);
        __syncwarp();
        // segmented inclusive scan of the partial sums over consecutive lanes
        // of the same cell; the last lane of a segment then holds its total
        const uint32_t key = open ? c : FULL;
        const uint32_t pkey = __shfl_up_sync(FULL, key, 1), nkey = __shfl_down_sync(FULL, key, 1);
        const bool head = open && (lane == 0 || pkey != key);
        const uint32_t heads = __ballot_sync(FULL, head);
        const int dist = open ? lane - (31 - __clz(heads & (FULL >> (31 - lane)))) : 0;
        const int maxd = __reduce_max_sync(FULL, dist);
        for (int d = 1; d <= maxd; d <<= 1) {
            const bool take = dist >= d;
#pragma unroll
            for (int o = 0; o < 27; ++o) {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float a = __shfl_up_sync(FULL, acc[o][k], d);
                    if (take) acc[o][k] += a;
                }
            }
        }
        if (open && (lane == 31 || nkey != key)) {
#pragma unroll
            for (int o = 0; o < 27; ++o) {
                float4 t = T4[o * 64 + c];
                t.x += acc[o][0];
                t.y += acc[o][1];
                t.z += acc[o][2];
                t.w += acc[o][3];
                T4[o * 64 + c] = t;
            }
        }
        __syncthreads();
        for (int n = threadIdx.x; n < TILE_NODES; n += G2_T) {
            const int nx = n % TN, ny = (n / TN) % TN, nz = n / (TN * TN);
            const float4 a4 = tile_node_sum(T4, nx, ny, nz);
            const int gi = ox + nx, gj = oy + ny, gk = oz0 + nz;
            if (a4.x != 0.f && gi < sc.n[0] && gj < sc.n[1] && gk < sc.n[2])
                atomicAdd(&V.grid_mp[node_index(sc, gi, gj, gk)], a4);
        }
        __syncthreads();
        if (threadIdx.x == 0) s_work = early ? next_work : atomicAdd(&V.counters[CNT_G2P_CURSOR], 1u);
    }
    if (flags) atomicOr(&V.counters[CNT_FLAGS], flags);
}

// ------------------------------------------------------------ pack / unpack
__global__ void k_pack(View V, const float* __restrict__ x, const float* __restrict__ v,
                       const float* __restrict__ C, const float* __restrict__ F, const float* __restrict__ m,
                       const float* __restrict__ V0, const int32_t* __restrict__ mat,
                       const uint32_t* __restrict__ order, uint32_t* __restrict__ user_of_phys,
                       uint32_t* __restrict__ phys_of_user, float2* __restrict__ mV_out,
                       int32_t* __restrict__ mat_out) {
    const int64_t N = V.N;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
        const uint32_t u = order[i];
        if (u >= (uint32_t)N) {
            atomicOr(&V.counters[CNT_FLAGS], FLAG_TILE_RANGE);
            continue;
        }
        float xx[3], vv[3], CC[9], FF[9];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            xx[a] = x[3 * (int64_t)u + a];
            vv[a] = v ? v[3 * (int64_t)u + a] : 0.f;
        }
#pragma unroll
        for (int a = 0; a < 9; ++a) {
            CC[a] = C ? C[9 * (int64_t)u + a] : 0.f;
            FF[a] = F ? F[9 * (int64_t)u + a] : ((a % 4 == 0) ? 1.f : 0.f);
        }
        float4 o0, o1, o2, o3, o4, o5;
        pack_xF(xx, FF, o0, o1, o2);
        pack_vC(vv, CC, o3, o4, o5);
        V.q[i] = o0;
        V.q[N + i] = o1;
        V.q[2 * N + i] = o2;
        V.q[3 * N + i] = o3;
        V.q[4 * N + i] = o4;
        V.q[5 * N + i] = o5;
        mV_out[i] = make_float2(m[u], V0 ? V0[u] : 0.f);
        if (mat_out) {
            int32_t mid = mat ? mat[u] : 0;
            if (mid < 0 || mid >= V.M) {  // invalid material id: use 0 and report
                atomicOr(&V.counters[CNT_FLAGS], FLAG_BAD_MATERIAL);
                mid = 0;
            }
            mat_out[i] = mid;
        }
        user_of_phys[i] = u;
        phys_of_user[u] = (uint32_t)i;
    }
}

// Walks the upload order: the caller's records are written contiguously and
// the state planes are gathered (scattered partial-sector writes cost more).
__global__ void k_unpack(View V, const uint32_t* __restrict__ phys_of_user, float* __restrict__ x,
                         float* __restrict__ v, float* __restrict__ C, float* __restrict__ F) {
    const int64_t N = V.N;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < N; u += stride) {
        const int64_t i = phys_of_user[u];
        if (i >= N) continue;
        float xx[3], FF[9], vv[3], CC[9];
        unpack_xF(V.q[i], V.q[N + i], V.q[2 * N + i], xx, FF);
        unpack_vC(V.q[3 * N + i], V.q[4 * N + i], V.q[5 * N + i], vv, CC);
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

__global__ void k_grid_download(View V, SceneDev sc, float* __restrict__ mass, float* __restrict__ vel) {
    const int64_t nodes = (int64_t)sc.n[0] * sc.n[1] * sc.n[2];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t li = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; li < nodes; li += stride) {
        const int i = (int)(li % sc.n[0]);
        const int j = (int)((li / sc.n[0]) % sc.n[1]);
        const int k = (int)(li / ((int64_t)sc.n[0] * sc.n[1]));
        const int t = ((k >> 2) * sc.nt[1] + (j >> 2)) * sc.nt[0] + (i >> 2);
        float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
        if (V.tile_flags[sc.nt_base + t]) g = V.grid_v[node_index(sc, i, j, k)];
        if (mass) mass[li] = g.w;
        if (vel) {
            vel[3 * li] = g.x;
            vel[3 * li + 1] = g.y;
            vel[3 * li + 2] = g.z;
        }
    }
}

// Sparse grids: every node of the node tiles active in the last step (flag
// equal to the step stamp) into the zeroed reference layout.
__global__ void k_grid_download_sparse(View V, SceneDev sc, float* __restrict__ mass, float* __restrict__ vel) {
    const uint32_t stamp = V.counters[CNT_STAMP];
    const int64_t total = (int64_t)V.total_nt * 64;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += stride) {
        const uint32_t slot = (uint32_t)(g >> 6);
        if (V.tile_flags[slot] != stamp || V.sp.code[slot] == SP_EMPTY) continue;
        const int l = (int)(g & 63);
        int tx, ty, tz;
        sp_decode(V.sp.code[slot], tx, ty, tz);
        const int i = 4 * tx + (l & 3), j = 4 * ty + ((l >> 2) & 3), k = 4 * tz + (l >> 4);
        if (i >= sc.n[0] || j >= sc.n[1] || k >= sc.n[2]) continue;
        const int64_t li = ((int64_t)k * sc.n[1] + j) * sc.n[0] + i;
        const float4 v = V.grid_v[g];
        if (mass) mass[li] = v.w;
        if (vel) {
            vel[3 * li] = v.x;
            vel[3 * li + 1] = v.y;
            vel[3 * li + 2] = v.z;
        }
    }
}

inline int grid_for(int64_t n, int block, int cap = 148 * 32) {
    int64_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    return (int)(g < cap ? g : cap);
}

}  // namespace

cudaError_t launch_keys(const View& V, const PhysFlags& pf, cudaStream_t st) {
    if (V.N == 0) return cudaSuccess;
    if (pf.physics == PHYS_MLS)
        k_keys<PHYS_MLS><<<grid_for(V.N, 256), 256, 0, st>>>(V);
    else
        k_keys<PHYS_REF><<<grid_for(V.N, 256), 256, 0, st>>>(V);
    return cudaGetLastError();
}

cudaError_t launch_payload(const View& V, const PhysFlags& pf, cudaStream_t st) {
    if (V.N == 0 || pf.physics != PHYS_MLS) return cudaSuccess;
    if (!V.pay) return cudaErrorInvalidValue;
    if (pf.multi_mat)
        k_payload<true><<<grid_for(V.N, 256), 256, 0, st>>>(V);
    else
        k_payload<false><<<grid_for(V.N, 256), 256, 0, st>>>(V);
    return cudaGetLastError();
}

cudaError_t launch_mark(const View& V, cudaStream_t st) {
    if (V.N == 0) return cudaSuccess;
    k_mark<<<grid_for(V.N, 256), 256, 0, st>>>(V);
    return cudaGetLastError();
}

cudaError_t launch_adj_scatter(const View& V, const AdjView& A, const PhysFlags& pf, const Tuning& t, int num_sms,
                               cudaStream_t st) {
    if (V.N == 0) return cudaSuccess;
    if (pf.physics != PHYS_MLS) return cudaErrorNotSupported;
    if (t.p2g_variant >= 4 && V.cell_range) {  // balanced runs over the sort's cell table
        const int nb = num_sms * 6;
        if (pf.multi_mat) {
            if (pf.has_fluid)
                k_adj_runs<true, true><<<nb, ADJR_T, 0, st>>>(V, A);
            else
                k_adj_runs<true, false><<<nb, ADJR_T, 0, st>>>(V, A);
        } else {
            if (pf.has_fluid)
                k_adj_runs<false, true><<<nb, ADJR_T, 0, st>>>(V, A);
            else
                k_adj_runs<false, false><<<nb, ADJR_T, 0, st>>>(V, A);
        }
        return cudaGetLastError();
    }
    if (t.p2g_variant >= 2) {  // the adjoint scatter of variant 3 (and of 4 without a cell table) is variant 2's
        const int nb = num_sms * t.cell_blocks_per_sm;
        if (pf.multi_mat) {
            if (pf.has_fluid)
                k_p2g_cells<MODE_ADJ, true, true><<<nb, P2GC_T, 0, st>>>(V, A);
            else
                k_p2g_cells<MODE_ADJ, true, false><<<nb, P2GC_T, 0, st>>>(V, A);
        } else {
            if (pf.has_fluid)
                k_p2g_cells<MODE_ADJ, false, true><<<nb, P2GC_T, 0, st>>>(V, A);
            else
                k_p2g_cells<MODE_ADJ, false, false><<<nb, P2GC_T, 0, st>>>(V, A);
        }
        return cudaGetLastError();
    }
    const int nb = num_sms * t.tile_blocks_per_sm;
    if (pf.multi_mat) {
        if (pf.has_fluid)
            k_p2g_tiles<MODE_ADJ, true, true><<<nb, P2G_T, 0, st>>>(V, A);
        else
            k_p2g_tiles<MODE_ADJ, true, false><<<nb, P2G_T, 0, st>>>(V, A);
    } else {
        if (pf.has_fluid)
            k_p2g_tiles<MODE_ADJ, false, true><<<nb, P2G_T, 0, st>>>(V, A);
        else
            k_p2g_tiles<MODE_ADJ, false, false><<<nb, P2G_T, 0, st>>>(V, A);
    }
    return cudaGetLastError();
}

cudaError_t launch_p2g(const View& V, const PhysFlags& pf, const Tuning& t, int num_sms, cudaStream_t st) {
    if (V.N == 0) return cudaSuccess;
    if (t.p2g_variant >= 3 && pf.physics == PHYS_MLS) {
        if (!V.pay) return cudaErrorInvalidValue;
        if (t.p2g_variant >= 4 && V.cell_range)  // without the sort's cell table: variant 3
            if (V.sp.cap)
                k_p2g_runs<true><<<num_sms * t.pair_blocks_per_sm, P2GR_T, 0, st>>>(V);
            else
                k_p2g_runs<false><<<num_sms * t.pair_blocks_per_sm, P2GR_T, 0, st>>>(V);
        else
            k_p2g_pairs<<<num_sms * t.pair_blocks_per_sm, P2GP_T, 0, st>>>(V);
        return cudaGetLastError();
    }
    if (t.p2g_variant >= 2) {  // REF physics: variants 3 to 5 run variant 2
        const int nb = num_sms * t.cell_blocks_per_sm;
        const AdjView none{};
        if (pf.physics == PHYS_MLS) {
            if (pf.multi_mat)
                k_p2g_cells<MODE_MLS, true, false><<<nb, P2GC_T, 0, st>>>(V, none);
            else
                k_p2g_cells<MODE_MLS, false, false><<<nb, P2GC_T, 0, st>>>(V, none);
        } else {
            k_p2g_cells<MODE_REF, false, false><<<nb, P2GC_T, 0, st>>>(V, none);
        }
        return cudaGetLastError();
    }
    if (t.p2g_variant == 0) {
        const int nb = num_sms * t.tile_blocks_per_sm;
        const AdjView none{};
        if (pf.physics == PHYS_MLS) {
            if (pf.multi_mat)
                k_p2g_tiles<MODE_MLS, true, false><<<nb, P2G_T, 0, st>>>(V, none);
            else
                k_p2g_tiles<MODE_MLS, false, false><<<nb, P2G_T, 0, st>>>(V, none);
        } else {
            k_p2g_tiles<MODE_REF, false, false><<<nb, P2G_T, 0, st>>>(V, none);
        }
        return cudaGetLastError();
    }
    const int64_t nb = (V.N + t.ppt - 1) / t.ppt;
    if (nb > 0x7FFFFFFF) return cudaErrorInvalidValue;
    if (pf.physics == PHYS_MLS) {
        if (pf.multi_mat)
            k_p2g<PHYS_MLS, true><<<(int)nb, t.p2g_block, 0, st>>>(V, t.ppt);
        else
            k_p2g<PHYS_MLS, false><<<(int)nb, t.p2g_block, 0, st>>>(V, t.ppt);
    } else {
        k_p2g<PHYS_REF, false><<<(int)nb, t.p2g_block, 0, st>>>(V, t.ppt);
    }
    return cudaGetLastError();
}

cudaError_t launch_grid(const View& V, const PhysFlags& pf, const Tuning& t, int num_sms, cudaStream_t st) {
    if (V.N == 0) return cudaSuccess;
    const int tiles_per_block = t.grid_block / 64;
    int64_t nb = ((int64_t)V.total_nt + tiles_per_block - 1) / tiles_per_block;
    const int cap = num_sms * 8;
    if (nb > cap) nb = cap;
    if (nb < 1) nb = 1;
    if (pf.physics == PHYS_MLS)
        k_grid<PHYS_MLS><<<(int)nb, t.grid_block, 0, st>>>(V);
    else
        k_grid<PHYS_REF><<<(int)nb, t.grid_block, 0, st>>>(V);
    return cudaGetLastError();
}

#define PGMPM_G2P_DISPATCH(KERNEL, GRID, BLOCK)                                  \
    do {                                                                         \
        if (pf.physics == PHYS_MLS) {                                            \
            if (pf.multi_mat) {                                                  \
                if (pf.has_fluid)                                                \
                    KERNEL<PHYS_MLS, true, true><<<GRID, BLOCK, 0, st>>>(V);     \
                else                                                             \
                    KERNEL<PHYS_MLS, true, false><<<GRID, BLOCK, 0, st>>>(V);    \
            } else {                                                             \
                if (pf.has_fluid)                                                \
                    KERNEL<PHYS_MLS, false, true><<<GRID, BLOCK, 0, st>>>(V);    \
                else                                                             \
                    KERNEL<PHYS_MLS, false, false><<<GRID, BLOCK, 0, st>>>(V);   \
            }                                                                    \
        } else {                                                                 \
            KERNEL<PHYS_REF, false, false><<<GRID, BLOCK, 0, st>>>(V);           \
        }                                                                        \
    } while (0)

cudaError_t launch_g2p(const View& V, const PhysFlags& pf, const Tuning& t, int num_sms, cudaStream_t st) {
    if (V.N == 0) return cudaSuccess;
    if (V.sp.cap) {  // sparse grids run the physical-order MLS G2P only
        if (pf.physics != PHYS_MLS) return cudaErrorNotSupported;
        const int nb = grid_for(V.N, t.g2p_block, 1 << 30);
#define PGMPM_G2PS(M_, F_, P_) k_g2p_sparse<M_, F_, P_><<<nb, t.g2p_block, 0, st>>>(V)
        if (pf.multi_mat) {
            if (pf.has_fluid) {
                if (pf.has_plastic) PGMPM_G2PS(true, true, true); else PGMPM_G2PS(true, true, false);
            } else {
                if (pf.has_plastic) PGMPM_G2PS(true, false, true); else PGMPM_G2PS(true, false, false);
            }
        } else {
            if (pf.has_fluid) {
                if (pf.has_plastic) PGMPM_G2PS(false, true, true); else PGMPM_G2PS(false, true, false);
            } else {
                if (pf.has_plastic) PGMPM_G2PS(false, false, true); else PGMPM_G2PS(false, false, false);
            }
        }
#undef PGMPM_G2PS
        return cudaGetLastError();
    }
    if (V.resort) {  // a replay of recorded steps: physical order, keys checked
        if (pf.physics != PHYS_MLS) return cudaErrorNotSupported;
        const int nb = grid_for(V.N, t.g2p_block, 1 << 30);
#define PGMPM_G2PC(M_, F_, P_) k_g2p_check<M_, F_, P_><<<nb, t.g2p_block, 0, st>>>(V)
        if (pf.multi_mat) {
            if (pf.has_fluid) {
                if (pf.has_plastic) PGMPM_G2PC(true, true, true); else PGMPM_G2PC(true, true, false);
            } else {
                if (pf.has_plastic) PGMPM_G2PC(true, false, true); else PGMPM_G2PC(true, false, false);
            }
        } else {
            if (pf.has_fluid) {
                if (pf.has_plastic) PGMPM_G2PC(false, true, true); else PGMPM_G2PC(false, true, false);
            } else {
                if (pf.has_plastic) PGMPM_G2PC(false, false, true); else PGMPM_G2PC(false, false, false);
            }
        }
#undef PGMPM_G2PC
        return cudaGetLastError();
    }
    if (t.g2p_variant == 0) {
        const int nb = num_sms * t.g2p_tiles_per_sm;
        PGMPM_G2P_DISPATCH(k_g2p_tiles, nb, 256);
    } else if (t.g2p_variant == 1) {
        const int nb = grid_for(V.N, t.g2p_block, 1 << 30);
        PGMPM_G2P_DISPATCH(k_g2p, nb, t.g2p_block);
    } else {
        const int nb = grid_for(V.N, t.g2p_block, 1 << 30);
        if (pf.has_plastic)
            PGMPM_G2P_DISPATCH(k_g2p_phys_vm, nb, t.g2p_block);
        else
            PGMPM_G2P_DISPATCH(k_g2p_phys, nb, t.g2p_block);
    }
    return cudaGetLastError();
}

cudaError_t launch_g2p2g(const View& V, const PhysFlags& pf, const Tuning& t, int num_sms, cudaStream_t st) {
    if (V.N == 0) return cudaSuccess;
    if (pf.physics != PHYS_MLS || !V.cell_range) return cudaErrorNotSupported;
    const int minb = t.g2p2g_blocks_per_sm == 6 ? 6 : 4;
    const int nb = num_sms * minb;
#define PGMPM_G2P2G(M_, F_, P_)                                          \
    do {                                                                 \
        if (minb == 6)                                                   \
            k_g2p2g<M_, F_, P_, 6><<<nb, G2_T, 0, st>>>(V);              \
        else                                                             \
            k_g2p2g<M_, F_, P_, 4><<<nb, G2_T, 0, st>>>(V);              \
    } while (0)
    if (pf.multi_mat) {
        if (pf.has_fluid) {
            if (pf.has_plastic) PGMPM_G2P2G(true, true, true); else PGMPM_G2P2G(true, true, false);
        } else {
            if (pf.has_plastic) PGMPM_G2P2G(true, false, true); else PGMPM_G2P2G(true, false, false);
        }
    } else {
        if (pf.has_fluid) {
            if (pf.has_plastic) PGMPM_G2P2G(false, true, true); else PGMPM_G2P2G(false, true, false);
        } else {
            if (pf.has_plastic) PGMPM_G2P2G(false, false, true); else PGMPM_G2P2G(false, false, false);
        }
    }
#undef PGMPM_G2P2G
    return cudaGetLastError();
}

cudaError_t launch_pack(const View& V, const float* x, const float* v, const float* C, const float* F,
                        const float* m, const float* V0, const int32_t* mat, const uint32_t* order,
                        uint32_t* user_of_phys, uint32_t* phys_of_user, float2* mV_out, int32_t* mat_out,
                        cudaStream_t st) {
    if (V.N == 0) return cudaSuccess;
    k_pack<<<grid_for(V.N, 256), 256, 0, st>>>(V, x, v, C, F, m, V0, mat, order, user_of_phys, phys_of_user, mV_out,
                                               mat_out);
    return cudaGetLastError();
}

cudaError_t launch_unpack(const View& V, const uint32_t* phys_of_user, float* x, float* v, float* C, float* F,
                          cudaStream_t st) {
    if (V.N == 0) return cudaSuccess;
    k_unpack<<<grid_for(V.N, 256), 256, 0, st>>>(V, phys_of_user, x, v, C, F);
    return cudaGetLastError();
}

namespace {
__global__ void k_merge_flags(uint32_t* c, int slots, uint32_t* live) {
    uint32_t f = 0;
    for (int j = threadIdx.x; j < slots; j += blockDim.x) {
        f |= c[(size_t)j * CNT_WORDS + CNT_FLAGS];
        c[(size_t)j * CNT_WORDS + CNT_FLAGS] = 0u;
    }
    if (f) atomicOr(&live[CNT_FLAGS], f);
}
}  // namespace

cudaError_t launch_merge_flags(uint32_t* slots_counters, int slots, uint32_t* live, cudaStream_t st) {
    if (slots <= 0) return cudaSuccess;
    k_merge_flags<<<1, 128, 0, st>>>(slots_counters, slots, live);
    return cudaGetLastError();
}

cudaError_t launch_grid_download(const View& V, int scene, const SceneDev& sc, float* mass, float* vel,
                                 cudaStream_t st) {
    (void)scene;
    const int64_t nodes = (int64_t)sc.n[0] * sc.n[1] * sc.n[2];
    if (V.sp.cap) {  // the untouched nodes are zero
        if (mass) {
            cudaError_t e = cudaMemsetAsync(mass, 0, sizeof(float) * (size_t)nodes, st);
            if (e != cudaSuccess) return e;
        }
        if (vel) {
            cudaError_t e = cudaMemsetAsync(vel, 0, sizeof(float) * 3 * (size_t)nodes, st);
            if (e != cudaSuccess) return e;
        }
        k_grid_download_sparse<<<grid_for((int64_t)V.total_nt * 64, 256), 256, 0, st>>>(V, sc, mass, vel);
        return cudaGetLastError();
    }
    k_grid_download<<<grid_for(nodes, 256), 256, 0, st>>>(V, sc, mass, vel);
    return cudaGetLastError();
}

}  // namespace pgmpm
