// pgmpm_device.cuh -- device-side data layout and per-particle physics of the
// MLS-MPM step (sm_100a).  Included by the kernel translation units only.
//
// Layouts (HBM):
//   particle state: 6 float4 planes, plane-major SoA, one float4 per particle
//   per plane, packed so that G2P reads exactly x and F (planes 0-2) and
//   P2G reads x, F, v, C (planes 0-5) with no padding:
//     q0 = (x.x, x.y, x.z, F00)   q1 = (F01, F02, F10, F11)   q2 = (F12, F20, F21, F22)
//     q3 = (v.x, v.y, v.z, C00)   q4 = (C01, C02, C10, C11)   q5 = (C12, C20, C21, C22)
//   static per-particle data: mV float2 (mass, initial volume), mat int32.
//   grid: dense per scene, 4x4x4-node tiles stored tile-major (64 nodes =
//   1 KB per float4 array), node local index lx + 4 ly + 16 lz.
//     grid_mp float4 (mass, momentum) -- P2G accumulator, zero between steps
//     grid_v  float4 (velocity, mass) -- written by the grid update
//   cell keys: stencil origin s (lowest node of the 3x3x3 stencil) per axis,
//   cell tile t = s >> 2, key = scene cell base + t_linear*64 + local cell.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace pgmpm {

enum { PHYS_MLS = 0, PHYS_REF = 1 };
enum { BC_NONE = 0, BC_STICKY = 1, BC_SLIP = 2, BC_SEPARATE = 3 };
enum { MODEL_FCR = 0, MODEL_NH = 1, MODEL_EOS = 2, MODEL_VM = 3 };  // VM: neo-Hookean + von Mises
enum { FLAG_ESCAPE = 1u, FLAG_NONFINITE = 2u, FLAG_TILE_RANGE = 4u, FLAG_BAD_MATERIAL = 8u, FLAG_TILE_POOL = 16u };

struct SceneDev {
    int n[3];       // grid nodes per axis
    int ct[3];      // cell tiles per axis: ((n - 3) >> 2) + 1
    int nt[3];      // node tiles per axis: ct + 1
    int ct_base;    // first global cell tile of this scene
    int nt_base;    // first global node tile of this scene
    int physics, boundary, bthick;
    int p_begin, p_end;  // particle range (physical order)
    float dx, D;    // D = 4 / dx^2 (inverse APIC inertia of the quadratic spline)
    float origin[3];
    float dt;
    float gravity[3];
    float inv_dx;   // 1/dx rounded to float (MLS stencil coordinate)
};

struct MatDev {
    int model;
    float mu, lam, E, dmu_dE, dlam_dE;
    float yield;  // MODEL_VM: von Mises yield stress of the Cauchy stress
    float visc;   // MODEL_EOS: dynamic viscosity (0: inviscid)
};

// ------------------------------------------------------------- 3x3 algebra
__device__ __forceinline__ void m3_mul(const float A[9], const float B[9], float C[9]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}
__device__ __forceinline__ void m3_mulT(const float A[9], const float B[9], float C[9]) {  // A B^T
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            C[3 * i + j] = A[3 * i] * B[3 * j] + A[3 * i + 1] * B[3 * j + 1] + A[3 * i + 2] * B[3 * j + 2];
}
__device__ __forceinline__ void m3_Tmul(const float A[9], const float B[9], float C[9]) {  // A^T B
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C[3 * i + j] = A[i] * B[j] + A[3 + i] * B[3 + j] + A[6 + i] * B[6 + j];
}
// cofactor matrix: cof(A) = det(A) A^{-T}
__device__ __forceinline__ void m3_cof(const float A[9], float R[9]) {
    R[0] = A[4] * A[8] - A[5] * A[7];
    R[1] = A[5] * A[6] - A[3] * A[8];
    R[2] = A[3] * A[7] - A[4] * A[6];
    R[3] = A[2] * A[7] - A[1] * A[8];
    R[4] = A[0] * A[8] - A[2] * A[6];
    R[5] = A[1] * A[6] - A[0] * A[7];
    R[6] = A[1] * A[5] - A[2] * A[4];
    R[7] = A[2] * A[3] - A[0] * A[5];
    R[8] = A[0] * A[4] - A[1] * A[3];
}
__device__ __forceinline__ float m3_det(const float A[9]) {
    return A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
           A[2] * (A[3] * A[7] - A[4] * A[6]);
}

// ------------------------------------------------------ packed FP32 pairs
// sm_100 issues an FP32 add, multiply or FMA on a pair of floats as one
// instruction (per component the same rounding as the scalar operation), so
// loops over 3-vectors keep two components per float2 and cut their FP issue.
__device__ __forceinline__ float2 f2(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 f2_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 f2_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 f2_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }

// ------------------------------------------------------------ state packing
__device__ __forceinline__ void unpack_xF(const float4 q0, const float4 q1, const float4 q2, float x[3], float F[9]) {
    x[0] = q0.x; x[1] = q0.y; x[2] = q0.z;
    F[0] = q0.w; F[1] = q1.x; F[2] = q1.y; F[3] = q1.z; F[4] = q1.w;
    F[5] = q2.x; F[6] = q2.y; F[7] = q2.z; F[8] = q2.w;
}
__device__ __forceinline__ void unpack_vC(const float4 q3, const float4 q4, const float4 q5, float v[3], float C[9]) {
    v[0] = q3.x; v[1] = q3.y; v[2] = q3.z;
    C[0] = q3.w; C[1] = q4.x; C[2] = q4.y; C[3] = q4.z; C[4] = q4.w;
    C[5] = q5.x; C[6] = q5.y; C[7] = q5.z; C[8] = q5.w;
}
__device__ __forceinline__ void pack_xF(const float x[3], const float F[9], float4& q0, float4& q1, float4& q2) {
    q0 = make_float4(x[0], x[1], x[2], F[0]);
    q1 = make_float4(F[1], F[2], F[3], F[4]);
    q2 = make_float4(F[5], F[6], F[7], F[8]);
}
__device__ __forceinline__ void pack_vC(const float v[3], const float C[9], float4& q3, float4& q4, float4& q5) {
    q3 = make_float4(v[0], v[1], v[2], C[0]);
    q4 = make_float4(C[1], C[2], C[3], C[4]);
    q5 = make_float4(C[5], C[6], C[7], C[8]);
}

// --------------------------------------------------------------- stencils
// Stencil origin of one coordinate.  The grid coordinate u is formed with
// correctly rounded operations (no contraction) so the cell keys are
// bit-identical to the CPU definition: MLS u = (x - o) * inv_dx (inv_dx =
// 1/dx rounded to float); REF_COMPAT u = (x - o) / dx as the reference.
__device__ __forceinline__ int stencil_origin(float xa, float oa, float dx, float inv_dx, int n, int physics,
                                              float& u, uint32_t& flags) {
    u = physics == PHYS_MLS ? __fmul_rn(__fsub_rn(xa, oa), inv_dx) : __fdiv_rn(__fsub_rn(xa, oa), dx);
    float s = physics == PHYS_MLS ? floorf(__fsub_rn(u, 0.5f)) : __fsub_rn(floorf(u), 1.0f);
    if (!(s == s)) {
        flags |= FLAG_NONFINITE;
        s = 0.f;
    }
    const float hi = (float)(n - 3);
    if (s < 0.f || s > hi) {
        if (physics == PHYS_MLS) flags |= FLAG_ESCAPE;
        s = fminf(fmaxf(s, 0.f), hi);
    }
    return (int)s;
}

// MLS quadratic B-spline weights at f in [0.5, 1.5) and d/df.
__device__ __forceinline__ void mls_weights(float f, float w[3]) {
    const float a = 1.5f - f, b = f - 1.0f, c = f - 0.5f;
    w[0] = 0.5f * a * a;
    w[1] = 0.75f - b * b;
    w[2] = 0.5f * c * c;
}
__device__ __forceinline__ void mls_dweights(float f, float dw[3]) {
    dw[0] = f - 1.5f;
    dw[1] = -2.0f * (f - 1.0f);
    dw[2] = f - 0.5f;
}

// Reference quadratic B-spline (src/material_point_method.h:288-293).
__device__ __forceinline__ float ref_quadratic(float x) {
    float abs_x = x < 0.f ? -x : x;
    if (abs_x >= 1.5f) return 0.f;
    if (abs_x < 0.5f) return __fsub_rn(0.75f, __fmul_rn(x, x));
    float t = __fsub_rn(1.5f, abs_x);
    return __fmul_rn(__fmul_rn(0.5f, t), t);
}

struct Stencil {
    int s[3];      // stencil origin (lowest node), clamped
    float f[3];    // MLS: u - s in [0.5, 1.5);  REF: u - floor(u) in [0, 1)
    int b[3];      // REF: unclamped floor(u) - 1 (actual lowest node)
    float w[3][3];
};

template <int PHYS>
__device__ __forceinline__ void make_stencil(const SceneDev& sc, const float x[3], Stencil& st, uint32_t& flags) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float u;
        st.s[a] = stencil_origin(x[a], sc.origin[a], sc.dx, sc.inv_dx, sc.n[a], PHYS, u, flags);
        if (PHYS == PHYS_MLS) {
            // f is clamped to the stencil's support so that a particle that
            // left the grid (flagged ESCAPE) transfers as if at the wall
            // instead of with extrapolated, negative weights.
            st.f[a] = fminf(fmaxf(__fsub_rn(u, (float)st.s[a]), 0.5f), 1.5f);
            st.b[a] = st.s[a];
            mls_weights(st.f[a], st.w[a]);
        } else {
            float fl = floorf(u);
            if (!(fl == fl)) fl = 0.f;
            fl = fminf(fmaxf(fl, -4.f), (float)sc.n[a] + 4.f);
            st.b[a] = (int)fl - 1;
            st.f[a] = __fsub_rn(u, fl);
#pragma unroll
            for (int k = 0; k < 3; ++k) st.w[a][k] = ref_quadratic(__fsub_rn(st.f[a], (float)(k - 1)));
        }
    }
}

__device__ __forceinline__ uint32_t cell_key(const SceneDev& sc, const int s[3]) {
    const uint32_t t = (uint32_t)(((s[2] >> 2) * sc.ct[1] + (s[1] >> 2)) * sc.ct[0] + (s[0] >> 2));
    const uint32_t l = (uint32_t)((s[2] & 3) * 16 + (s[1] & 3) * 4 + (s[0] & 3));
    return ((uint32_t)sc.ct_base + t) * 64u + l;
}

// Tiled node index of node (i,j,k) of scene sc.
__device__ __forceinline__ int64_t node_index(const SceneDev& sc, int i, int j, int k) {
    const int t = ((k >> 2) * sc.nt[1] + (j >> 2)) * sc.nt[0] + (i >> 2);
    return ((int64_t)(sc.nt_base + t) << 6) + ((k & 3) << 4) + ((j & 3) << 2) + (i & 3);
}

// ------------------------------------------------------------ sparse grid
// A sparse grid stores only the 4^3 tiles that particles reach, in a pool
// of `cap` slots found through an open-addressing hash of the tile's
// coordinates (linear probing, slot = bucket).  One slot is both the cell
// tile (cell keys slot * 64 + local cell) and the node tile (grid nodes
// slot * 64 + local node) with those coordinates.  Slots are claimed with
// atomicCAS and never released, so a slot's grid words stay at the zero
// the grid update leaves them at.  nbr[c] lists, for an occupied cell tile c,
// the slots of the 8 node tiles c + {0,1}^3 its particles' stencils reach
// (rebuilt after every sort).
// The grid update also writes each occupied cell tile's 6^3 node velocities
// contiguously (box[c]), so that G2P gathers them with dense local indices:
// rev[n][q] = (c, stamp) names, for node tile n, the cell tile c = n - off(q)
// whose box holds it, when c was occupied in the step of that stamp.
struct SparseTiles {
    uint32_t* code;  // [cap] packed tile coordinates of each slot, SP_EMPTY when free
    uint4* nbr;      // [cap][2]: 8 node-tile slots (x + 2y + 4z offset order)
    float4* box;     // [cap][216]: (v, m) of the cell tile's 6^3 node block, after the grid update
    uint2* rev;      // [cap][8]: (cell tile, step stamp) whose box holds this node tile at offset q
    uint32_t cap;    // power of two (0: the grid is dense)
    int shift;       // 32 - log2(cap)
};
constexpr uint32_t SP_EMPTY = 0xFFFFFFFFu;
constexpr uint32_t SP_NONE = 0xFFFFFFFFu;
constexpr int SP_MAX_PROBES = 64;
constexpr int SP_AXIS_BITS = 10;  // tile coordinates < 1024 per axis (grids up to 4095 nodes)

__device__ __forceinline__ uint32_t sp_code(int tx, int ty, int tz) {
    return (uint32_t)tx | ((uint32_t)ty << SP_AXIS_BITS) | ((uint32_t)tz << (2 * SP_AXIS_BITS));
}
__device__ __forceinline__ void sp_decode(uint32_t code, int& tx, int& ty, int& tz) {
    const uint32_t m = (1u << SP_AXIS_BITS) - 1u;
    tx = (int)(code & m);
    ty = (int)((code >> SP_AXIS_BITS) & m);
    tz = (int)(code >> (2 * SP_AXIS_BITS));
}
// Slot of the tile with this code, claiming a free bucket when it has none;
// SP_NONE (and FLAG_TILE_POOL) when SP_MAX_PROBES buckets were all taken.
// Concurrent callers with one code get one slot: a bucket's code is written
// once, by atomicCAS, and never changes.
__device__ __forceinline__ uint32_t sp_find_or_insert(const SparseTiles& sp, uint32_t code, uint32_t& flags) {
    uint32_t b = (code * 0x9E3779B1u) >> sp.shift;
    for (int probe = 0; probe < SP_MAX_PROBES; ++probe) {
        uint32_t k = *reinterpret_cast<volatile uint32_t*>(&sp.code[b]);
        if (k == code) return b;
        if (k == SP_EMPTY) {
            k = atomicCAS(&sp.code[b], SP_EMPTY, code);
            if (k == SP_EMPTY || k == code) return b;
        }
        b = (b + 1u) & (sp.cap - 1u);
    }
    flags |= FLAG_TILE_POOL;
    return SP_NONE;
}
// Slot of node (i, j, k) from the 8 node-tile slots nb[] of the cell tile
// whose lowest node is (ox, oy, oz); the node lies in [o, o + 6) per axis.
__device__ __forceinline__ int64_t sp_node(const uint32_t nb[8], int i, int j, int k, int ox, int oy, int oz) {
    const int lx = i - ox, ly = j - oy, lz = k - oz;
    const int sel = (lx >> 2) | ((ly >> 2) << 1) | ((lz >> 2) << 2);
    uint32_t slot = nb[0];
#pragma unroll
    for (int q = 1; q < 8; ++q)
        if (sel == q) slot = nb[q];
    return ((int64_t)slot << 6) + ((lz & 3) << 4) + ((ly & 3) << 2) + (lx & 3);
}
__device__ __forceinline__ void sp_load_nbr(const SparseTiles& sp, uint32_t c, uint32_t nb[8]) {
    const uint4 a = sp.nbr[2 * (size_t)c], b = sp.nbr[2 * (size_t)c + 1];
    nb[0] = a.x; nb[1] = a.y; nb[2] = a.z; nb[3] = a.w;
    nb[4] = b.x; nb[5] = b.y; nb[6] = b.z; nb[7] = b.w;
}

// ----------------------------------------------------------- scene lookup
__device__ __forceinline__ int scene_of_cell_tile(const SceneDev* sc, int S, int ct) {
    int lo = 0, hi = S - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(&sc[mid].ct_base) <= ct) lo = mid; else hi = mid - 1;
    }
    return lo;
}
__device__ __forceinline__ int scene_of_node_tile(const SceneDev* sc, int S, int nt) {
    int lo = 0, hi = S - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(&sc[mid].nt_base) <= nt) lo = mid; else hi = mid - 1;
    }
    return lo;
}
__device__ __forceinline__ int scene_of_particle(const SceneDev* sc, int S, int p) {
    int lo = 0, hi = S - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(&sc[mid].p_begin) <= p) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ------------------------------------------------------ constitutive laws
// Rotation of the polar decomposition F = R S by the determinant-scaled
// Newton iteration X <- (zeta X + (zeta X)^{-T}) / 2, zeta = |det X|^{-1/3}
// (Higham 1986).  Converges quadratically; F is close to a rotation in
// elastic MPM so a few iterations suffice.  For det F < 0 it converges to the
// orthogonal factor (det R = -1).
__device__ __forceinline__ void polar_rotation(const float F[9], float R[9]) {
#pragma unroll
    for (int i = 0; i < 9; ++i) R[i] = F[i];
#pragma unroll 1
    for (int it = 0; it < 8; ++it) {
        float cof[9];
        m3_cof(R, cof);
        const float det = R[0] * cof[0] + R[1] * cof[1] + R[2] * cof[2];
        if (!(fabsf(det) > 1e-30f)) break;
        const float zeta = rcbrtf(fabsf(det));
        const float a = 0.5f * zeta, b = 0.5f / (zeta * det);
        float diff = 0.f, nrm = 0.f;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const float xn = a * R[i] + b * cof[i];
            const float d = xn - R[i];
            diff += d * d;
            nrm += xn * xn;
            R[i] = xn;
        }
        if (diff <= 1e-13f * nrm) break;
    }
}

// Kirchhoff stress tau = P F^T.
//   FCR: 2 mu (F - R) F^T + lam (J - 1) J I
//   NH : mu (F F^T - I) + lam ln(J) I   (J times the Cauchy form of
//        src/mpm_kernels.cu:113-127)
//   EOS: K J (J - 1) I  with K carried in E (p = -K (J - 1))
// R receives the rotation of F's polar decomposition for the fixed-corotated
// model (and is left unset otherwise), for kirchhoff_adjoint to reuse.
// PLASTIC = false leaves out the von Mises cap (kernels launched only when no
// ELASTOPLASTIC material is present, and the adjoint, which excludes it).
template <bool PLASTIC = true>
__device__ __forceinline__ void kirchhoff(const float F[9], const MatDev& m, float tau[9], float R[9]) {
    const float J = m3_det(F);
    if (m.model == MODEL_FCR) {
        float D[9];
        polar_rotation(F, R);
#pragma unroll
        for (int i = 0; i < 9; ++i) D[i] = F[i] - R[i];
        m3_mulT(D, F, tau);
        const float c = 2.f * m.mu, t = m.lam * (J - 1.f) * J;
#pragma unroll
        for (int i = 0; i < 9; ++i) tau[i] = c * tau[i] + ((i % 4 == 0) ? t : 0.f);
    } else if (m.model == MODEL_NH || m.model == MODEL_VM) {
        float B[9];
        m3_mulT(F, F, B);
        const float t = m.lam * logf(J);
#pragma unroll
        for (int i = 0; i < 9; ++i) tau[i] = m.mu * (B[i] - ((i % 4 == 0) ? 1.f : 0.f)) + ((i % 4 == 0) ? t : 0.f);
        if (PLASTIC && m.model == MODEL_VM) {
            // von Mises return mapping (src/material_point_method.h:375-402) on
            // the Cauchy stress sigma = tau / J: above the yield stress Y its
            // deviatoric part is scaled by Y / vm(sigma); vm(tau) = J vm(sigma)
            const float p = (tau[0] + tau[4] + tau[8]) * (1.f / 3.f);
            float ss = 0.f;
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                const float d = tau[i] - ((i % 4 == 0) ? p : 0.f);
                ss += d * d;
            }
            const float vm = sqrtf(1.5f * ss);
            if (vm > J * m.yield) {
                const float sc = J * m.yield / vm;
#pragma unroll
                for (int i = 0; i < 9; ++i)
                    tau[i] = (i % 4 == 0) ? p + sc * (tau[i] - p) : sc * tau[i];
            }
        }
    } else {
        const float t = m.E * J * (J - 1.f);
#pragma unroll
        for (int i = 0; i < 9; ++i) tau[i] = (i % 4 == 0) ? t : 0.f;
    }
}

// Viscous fluid: the Newtonian stress 2 mu_v sym(grad v) of
// src/mpm_kernels.cu:131-149 with the APIC C as grad v, added as Kirchhoff
// stress J mu_v (C + C^T) to the EOS pressure.
__device__ __forceinline__ void add_viscous(const float F[9], const float C[9], const MatDev& m, float tau[9]) {
    if (m.model != MODEL_EOS || !(m.visc > 0.f)) return;
    const float Jv = m3_det(F) * m.visc;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) tau[3 * i + j] += Jv * (C[3 * i + j] + C[3 * j + i]);
}

template <bool PLASTIC = true>
__device__ __forceinline__ void kirchhoff(const float F[9], const MatDev& m, float tau[9]) {
    float R[9];
    kirchhoff<PLASTIC>(F, m, tau, R);
}

// Adjoint of kirchhoff(): gF += d<tb, tau(F)>/dF; returns d<tb, tau>/dE.
// The rotation's derivative follows from F = R S: with M = R^T dF,
// Omega = R^T dR is skew with axial vector (tr(S) I - S)^{-1} axial(M - M^T),
// so a cotangent Rb maps to gF += R skew(z), z = (tr(S) I - S)^{-1}
// axial(R^T Rb - Rb^T R).  tr(S) I - S has eigenvalues s_i + s_j (sums of
// singular values) and stays invertible for det F > 0; no 1/(s_i^2 - s_j^2)
// terms appear.
// R: the rotation kirchhoff(F, m, tau, R) returned (fixed-corotated only).
// MODEL_VM (neo-Hookean predictor e with the von Mises cap): above the
// yield stress tau = p I + s dev(e), s = J Y / vm(e), p = tr(e)/3, and
//   <tb, dtau> = <tb_e, de> + s <tb, dev e> dJ / J,
//   tb_e = tr(tb)/3 I + s dev(tb) - s <tb, dev e> / |dev e|^2 dev e,
// so the neo-Hookean adjoint runs with tb_e (below the yield stress, tb).
__device__ __forceinline__ float kirchhoff_adjoint(const float F[9], const float R[9], const MatDev& m,
                                                   const float tb_in[9], float gF[9]) {
    float cofF[9];
    m3_cof(F, cofF);
    const float J = F[0] * cofF[0] + F[1] * cofF[1] + F[2] * cofF[2];  // cof = J F^{-T}
    float tb[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) tb[i] = tb_in[i];
    if (m.model == MODEL_VM) {
        float B[9], d[9];
        m3_mulT(F, F, B);
        const float t = m.lam * logf(J);
        float pe = 0.f;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            d[i] = m.mu * (B[i] - ((i % 4 == 0) ? 1.f : 0.f)) + ((i % 4 == 0) ? t : 0.f);
            if (i % 4 == 0) pe += d[i];
        }
        pe *= (1.f / 3.f);
        float ss = 0.f;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            d[i] -= (i % 4 == 0) ? pe : 0.f;
            ss += d[i] * d[i];
        }
        const float vm = sqrtf(1.5f * ss);
        if (vm > J * m.yield) {
            const float sc = J * m.yield / vm;
            const float pt = (tb[0] + tb[4] + tb[8]) * (1.f / 3.f);
            float tbd = 0.f;
#pragma unroll
            for (int i = 0; i < 9; ++i) tbd += tb[i] * d[i];
            const float k = sc * tbd / ss;
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                const float dg = (i % 4 == 0) ? pt : 0.f;
                tb[i] = dg + sc * (tb[i] - dg) - k * d[i];
            }
            const float cj = sc * tbd / J;  // times dJ/dF = cof F
#pragma unroll
            for (int i = 0; i < 9; ++i) gF[i] += cj * cofF[i];
        }
    }
    const float trt = tb[0] + tb[4] + tb[8];
    if (m.model == MODEL_FCR) {
        float D[9], tbF[9], tbTD[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) D[i] = F[i] - R[i];
        m3_mul(tb, F, tbF);
        m3_Tmul(tb, D, tbTD);
        const float c2 = 2.f * m.mu;
#pragma unroll
        for (int i = 0; i < 9; ++i) gF[i] += c2 * (tbF[i] + tbTD[i]);
        // polar adjoint with Rb = -2 mu tb F
        float Rb[9], RtRb[9], S[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) Rb[i] = -c2 * tbF[i];
        m3_Tmul(R, Rb, RtRb);
        m3_Tmul(R, F, S);
        const float y0 = RtRb[7] - RtRb[5], y1 = RtRb[2] - RtRb[6], y2 = RtRb[3] - RtRb[1];
        const float s01 = 0.5f * (S[1] + S[3]), s02 = 0.5f * (S[2] + S[6]), s12 = 0.5f * (S[5] + S[7]);
        const float trS = S[0] + S[4] + S[8];
        float G[9] = {trS - S[0], -s01, -s02, -s01, trS - S[4], -s12, -s02, -s12, trS - S[8]};
        float cG[9];
        m3_cof(G, cG);
        const float dG = G[0] * cG[0] + G[1] * cG[1] + G[2] * cG[2];
        const float idG = 1.f / dG;
        // G symmetric: G^{-1} = cof(G)^T / det = cof(G) / det
        const float z0 = (cG[0] * y0 + cG[1] * y1 + cG[2] * y2) * idG;
        const float z1 = (cG[3] * y0 + cG[4] * y1 + cG[5] * y2) * idG;
        const float z2 = (cG[6] * y0 + cG[7] * y1 + cG[8] * y2) * idG;
        const float Z[9] = {0.f, -z2, z1, z2, 0.f, -z0, -z1, z0, 0.f};
        float RZ[9];
        m3_mul(R, Z, RZ);
        const float cl = m.lam * (2.f * J - 1.f) * trt;  // times J F^{-T} = cofF
#pragma unroll
        for (int i = 0; i < 9; ++i) gF[i] += RZ[i] + cl * cofF[i];
        float tmu[9];
        m3_mulT(D, F, tmu);
        float dmu = 0.f;
#pragma unroll
        for (int i = 0; i < 9; ++i) dmu += tb[i] * 2.f * tmu[i];
        const float dlam = trt * (J - 1.f) * J;
        return dmu * m.dmu_dE + dlam * m.dlam_dE;
    } else if (m.model == MODEL_NH || m.model == MODEL_VM) {
        float a[9], b[9], B[9];
        m3_mul(tb, F, a);
        m3_Tmul(tb, F, b);
        const float cl = m.lam * trt / J;  // lam tr(tb) F^{-T} = lam tr(tb) cof / J
#pragma unroll
        for (int i = 0; i < 9; ++i) gF[i] += m.mu * (a[i] + b[i]) + cl * cofF[i];
        m3_mulT(F, F, B);
        float dmu = 0.f;
#pragma unroll
        for (int i = 0; i < 9; ++i) dmu += tb[i] * (B[i] - ((i % 4 == 0) ? 1.f : 0.f));
        const float dlam = trt * logf(J);
        return dmu * m.dmu_dE + dlam * m.dlam_dE;
    } else {
        const float c = m.E * (2.f * J - 1.f) * trt;  // times J F^{-T}
#pragma unroll
        for (int i = 0; i < 9; ++i) gF[i] += c * cofF[i];
        return trt * J * (J - 1.f);
    }
}

// Adjoint of add_viscous: with tau_v = J mu_v (C + C^T), gC += J mu_v
// (tb + tb^T) and gF += mu_v <tb, C + C^T> cof F (dJ/dF = cof F).
__device__ __forceinline__ void add_viscous_adjoint(const float F[9], const float C[9], const MatDev& m,
                                                    const float tb[9], float gF[9], float gC[9]) {
    if (m.model != MODEL_EOS || !(m.visc > 0.f)) return;
    float cofF[9];
    m3_cof(F, cofF);
    const float Jv = (F[0] * cofF[0] + F[1] * cofF[1] + F[2] * cofF[2]) * m.visc;
    float tc = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            gC[3 * i + j] += Jv * (tb[3 * i + j] + tb[3 * j + i]);
            tc += tb[3 * i + j] * (C[3 * i + j] + C[3 * j + i]);
        }
    const float c = m.visc * tc;
#pragma unroll
    for (int i = 0; i < 9; ++i) gF[i] += c * cofF[i];
}

__device__ __forceinline__ float kirchhoff_adjoint(const float F[9], const MatDev& m, const float tb[9], float gF[9]) {
    float R[9];
    if (m.model == MODEL_FCR) polar_rotation(F, R);
    return kirchhoff_adjoint(F, R, m, tb, gF);
}

// --------------------------------------------------------- P2G payload
// What P2G needs of one MLS particle, computed where the state is already in
// registers (G2P of the previous step, or k_payload after an upload):
//   node o of the stencil receives w_o(f) * (m, b + Ad o) with
//   Ad = dx * A, A = -dt V0 D tau(F) + m C, b = m v - Ad f.
// Packed as 4 float4 planes: p0 = (b, m), p1 = Ad[0..3], p2 = Ad[4..7],
// p3 = (Ad[8], f).
template <bool PLASTIC = true>
__device__ __forceinline__ void mls_payload(const SceneDev& sc, const MatDev& mt, const float f[3], const float F[9],
                                            const float v[3], const float C[9], float m, float V0, float4& p0,
                                            float4& p1, float4& p2, float4& p3) {
    float tau[9];
    kirchhoff<PLASTIC>(F, mt, tau);
    add_viscous(F, C, mt, tau);
    const float kk = -sc.dt * V0 * sc.D;
    float Ad[9];
#pragma unroll
    for (int a = 0; a < 9; ++a) Ad[a] = (kk * tau[a] + m * C[a]) * sc.dx;
    float b[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) b[a] = m * v[a] - (Ad[3 * a] * f[0] + Ad[3 * a + 1] * f[1] + Ad[3 * a + 2] * f[2]);
    p0 = make_float4(b[0], b[1], b[2], m);
    p1 = make_float4(Ad[0], Ad[1], Ad[2], Ad[3]);
    p2 = make_float4(Ad[4], Ad[5], Ad[6], Ad[7]);
    p3 = make_float4(Ad[8], f[0], f[1], f[2]);
}

// The whole payload of one particle from its 4 planes (see mls_payload).
__device__ __forceinline__ void unpack_payload(const float4& p0, const float4& p1, const float4& p2, const float4& p3,
                                               float& m, float b[3], float Ad[9], float f[3]) {
    m = p0.w;
    b[0] = p0.x;
    b[1] = p0.y;
    b[2] = p0.z;
    Ad[0] = p1.x; Ad[1] = p1.y; Ad[2] = p1.z; Ad[3] = p1.w;
    Ad[4] = p2.x; Ad[5] = p2.y; Ad[6] = p2.z; Ad[7] = p2.w;
    Ad[8] = p3.x;
    f[0] = p3.y;
    f[1] = p3.z;
    f[2] = p3.w;
}

// ----------------------------------------------------------- grid update
__device__ __forceinline__ bool in_wall(const SceneDev& sc, int a, int idx, int& side) {
    if (idx < sc.bthick) { side = -1; return true; }
    if (idx >= sc.n[a] - sc.bthick) { side = 1; return true; }
    return false;
}

// Boundary condition on a pre-BC velocity; returns a per-component mask of
// the components it zeroed (bit a).
__device__ __forceinline__ uint32_t apply_bc(const SceneDev& sc, int i, int j, int k, float v[3]) {
    if (sc.boundary == BC_NONE) return 0u;
    const int id[3] = {i, j, k};
    uint32_t zeroed = 0u;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int side;
        if (!in_wall(sc, a, id[a], side)) continue;
        if (sc.boundary == BC_STICKY) {
            zeroed = 7u;
        } else if (sc.boundary == BC_SLIP) {
            zeroed |= 1u << a;
        } else if ((side < 0 && v[a] < 0.f) || (side > 0 && v[a] > 0.f)) {
            zeroed |= 1u << a;
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
        if (zeroed & (1u << a)) v[a] = 0.f;
    return zeroed;
}

}  // namespace pgmpm
