/*
 * oracle.cpp -- CPU oracle for the MLS-MPM step.  TEST INFRASTRUCTURE ONLY:
 * the checker for the CUDA kernels, never the thing measured or shipped.
 * See oracle.h for what is restated from which reference file:line.
 *
 * Build: oracle/Makefile (g++ -O2 -pthread -ffp-contract=off).  FMA
 * contraction is off so the float REF_COMPAT instance performs exactly the
 * float operations the reference's own CPU solver performs.
 */
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace {

// ------------------------------------------------------- host parallelism
// std::thread range split (the image has no OpenMP runtime) and CAS-based
// floating-point atomic add for the scatter loops.  The worker count is per
// calling thread, so that several host threads may run the oracle at once
// (each spawning its own workers); it is read only on the calling thread.
thread_local int g_threads = 1;

template <class Fn> void parallel_range(int64_t n, Fn fn) {
    int nt = g_threads > 1 ? g_threads : 1;
    if (nt == 1 || n < 1024) {
        fn((int64_t)0, n, 0);
        return;
    }
    std::vector<std::thread> th;
    int64_t chunk = (n + nt - 1) / nt;
    for (int t = 0; t < nt; ++t) {
        int64_t b = t * chunk, e = std::min(n, b + chunk);
        if (b >= e) break;
        th.emplace_back([=, &fn]() { fn(b, e, t); });
    }
    for (auto& t : th) t.join();
}

template <class T> inline void atomic_add(T* addr, T val) {
    typedef typename std::conditional<sizeof(T) == 8, uint64_t, uint32_t>::type U;
    U* ua = reinterpret_cast<U*>(addr);
    U old = __atomic_load_n(ua, __ATOMIC_RELAXED);
    for (;;) {
        T cur;
        std::memcpy(&cur, &old, sizeof(T));
        T nv = cur + val;
        U nu;
        std::memcpy(&nu, &nv, sizeof(T));
        if (__atomic_compare_exchange_n(ua, &old, nu, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) return;
    }
}

// ---------------------------------------------------------------- 3x3 algebra
template <class T> inline void mm(const T A[9], const T B[9], T C[9]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}
template <class T> inline void mmT(const T A[9], const T B[9], T C[9]) {  // A B^T
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            C[3 * i + j] = A[3 * i] * B[3 * j] + A[3 * i + 1] * B[3 * j + 1] + A[3 * i + 2] * B[3 * j + 2];
}
template <class T> inline void mTm(const T A[9], const T B[9], T C[9]) {  // A^T B
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            C[3 * i + j] = A[i] * B[j] + A[3 + i] * B[3 + j] + A[6 + i] * B[6 + j];
}
template <class T> inline T det3(const T A[9]) {
    return A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
           A[2] * (A[3] * A[7] - A[4] * A[6]);
}
// inverse transpose: A^{-T}
template <class T> inline void invT3(const T A[9], T R[9]) {
    T d = det3(A);
    T id = T(1) / d;
    // cofactor matrix / det = A^{-T}
    R[0] = (A[4] * A[8] - A[5] * A[7]) * id;
    R[1] = (A[5] * A[6] - A[3] * A[8]) * id;
    R[2] = (A[3] * A[7] - A[4] * A[6]) * id;
    R[3] = (A[2] * A[7] - A[1] * A[8]) * id;
    R[4] = (A[0] * A[8] - A[2] * A[6]) * id;
    R[5] = (A[1] * A[6] - A[0] * A[7]) * id;
    R[6] = (A[1] * A[5] - A[2] * A[4]) * id;
    R[7] = (A[2] * A[3] - A[0] * A[5]) * id;
    R[8] = (A[0] * A[4] - A[1] * A[3]) * id;
}

// Symmetric 3x3 eigen-decomposition by cyclic Jacobi rotations.
// A = V diag(w) V^T, V columns are eigenvectors.
template <class T> void sym_eig3(const T Ain[9], T w[3], T V[9]) {
    T A[9];
    std::memcpy(A, Ain, sizeof(A));
    for (int i = 0; i < 9; ++i) V[i] = (i % 4 == 0) ? T(1) : T(0);
    const T eps = std::is_same<T, double>::value ? T(1e-30) : T(1e-20);
    for (int sweep = 0; sweep < 64; ++sweep) {
        T off = A[1] * A[1] + A[2] * A[2] + A[5] * A[5];
        T dia = A[0] * A[0] + A[4] * A[4] + A[8] * A[8];
        if (off <= eps * dia || off == T(0)) break;
        for (int pq = 0; pq < 3; ++pq) {
            int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
            T apq = A[3 * p + q];
            if (apq == T(0)) continue;
            T theta = (A[3 * q + q] - A[3 * p + p]) / (T(2) * apq);
            T t = (theta >= 0 ? T(1) : T(-1)) / (std::fabs(theta) + std::sqrt(theta * theta + T(1)));
            T c = T(1) / std::sqrt(t * t + T(1)), s = t * c;
            T P[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
            P[3 * p + p] = c;
            P[3 * q + q] = c;
            P[3 * p + q] = s;
            P[3 * q + p] = -s;
            T tmp[9], A2[9], V2[9];
            mm(A, P, tmp);
            mTm(P, tmp, A2);
            std::memcpy(A, A2, sizeof(A));
            mm(V, P, V2);
            std::memcpy(V, V2, sizeof(A));
        }
    }
    w[0] = A[0];
    w[1] = A[4];
    w[2] = A[8];
}

// Polar decomposition F = R S from the eigen-decomposition of F^T F.
template <class T> void polar3(const T F[9], T R[9], T S[9]) {
    T FtF[9], w[3], V[9];
    mTm(F, F, FtF);
    sym_eig3(FtF, w, V);
    T sq[3], isq[3];
    for (int i = 0; i < 3; ++i) {
        T l = w[i] > T(0) ? w[i] : T(0);
        sq[i] = std::sqrt(l);
        isq[i] = sq[i] > T(0) ? T(1) / sq[i] : T(0);
    }
    T Sinv[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            S[3 * i + j] = V[3 * i] * sq[0] * V[3 * j] + V[3 * i + 1] * sq[1] * V[3 * j + 1] +
                           V[3 * i + 2] * sq[2] * V[3 * j + 2];
            Sinv[3 * i + j] = V[3 * i] * isq[0] * V[3 * j] + V[3 * i + 1] * isq[1] * V[3 * j + 1] +
                              V[3 * i + 2] * isq[2] * V[3 * j + 2];
        }
    mm(F, Sinv, R);
}

template <class T> struct Mat {
    int model;
    T E, nu, mu, lam, dmu_dE, dlam_dE, yield, visc;
};
template <class T> Mat<T> make_mat(const oracle_material& m) {
    Mat<T> r;
    r.model = m.model;
    r.E = T(m.E);
    r.nu = T(m.nu);
    T nu = r.nu;
    r.mu = r.E / (T(2) * (T(1) + nu));
    r.lam = r.E * nu / ((T(1) + nu) * (T(1) - T(2) * nu));
    r.dmu_dE = T(1) / (T(2) * (T(1) + nu));
    r.dlam_dE = nu / ((T(1) + nu) * (T(1) - T(2) * nu));
    r.yield = T(m.yield_stress);
    r.visc = T(m.viscosity);
    return r;
}

// Kirchhoff stress tau = P F^T.
template <class T> void kirchhoff(const T F[9], const Mat<T>& mt, T tau[9]) {
    T J = det3(F);
    if (mt.model == ORACLE_FIXED_COROTATED) {
        T R[9], S[9], D[9];
        polar3(F, R, S);
        for (int i = 0; i < 9; ++i) D[i] = F[i] - R[i];
        mmT(D, F, tau);
        for (int i = 0; i < 9; ++i) tau[i] *= T(2) * mt.mu;
        T t = mt.lam * (J - T(1)) * J;
        tau[0] += t;
        tau[4] += t;
        tau[8] += t;
    } else if (mt.model == ORACLE_NEO_HOOKEAN || mt.model == ORACLE_VON_MISES) {
        T B[9];
        mmT(F, F, B);
        T t = mt.lam * std::log(J);
        for (int i = 0; i < 9; ++i) tau[i] = mt.mu * (B[i] - ((i % 4 == 0) ? T(1) : T(0)));
        tau[0] += t;
        tau[4] += t;
        tau[8] += t;
        if (mt.model == ORACLE_VON_MISES) {
            // von Mises return mapping of src/material_point_method.h:375-402 on the
            // Cauchy stress sigma = tau / J: above the yield stress Y the
            // deviatoric part is scaled by Y / vm(sigma).  vm(tau) = J vm(sigma).
            const T p = (tau[0] + tau[4] + tau[8]) / T(3);
            T dev[9], ss = T(0);
            for (int i = 0; i < 9; ++i) {
                dev[i] = tau[i] - ((i % 4 == 0) ? p : T(0));
                ss += dev[i] * dev[i];
            }
            const T vm = std::sqrt(T(1.5) * ss);
            if (vm > J * mt.yield) {
                const T sc = J * mt.yield / vm;
                for (int i = 0; i < 9; ++i) tau[i] = ((i % 4 == 0) ? p : T(0)) + sc * dev[i];
            }
        }
    } else {  // EOS fluid, K = E
        T t = mt.E * J * (J - T(1));
        for (int i = 0; i < 9; ++i) tau[i] = (i % 4 == 0) ? t : T(0);
    }
}

// Adjoint of the Kirchhoff stress: gF += d<taubar, tau>/dF, returns d/dE.
template <class T> T kirchhoff_adj(const T F[9], const Mat<T>& mt, const T tb[9], T gF[9]) {
    T J = det3(F);
    T FiT[9];
    invT3(F, FiT);
    if (mt.model == ORACLE_VON_MISES) {
        // tau = p I + s dev(e), s = J Y / vm(e), above the yield stress (e the
        // neo-Hookean predictor, p = tr(e)/3, vm = sqrt(3/2 |dev e|^2)):
        //   <tb, dtau> = <tb_e, de> + s <tb, dev e> dJ / J,
        //   tb_e = tr(tb)/3 I + s dev(tb) - s <tb, dev e> / |dev e|^2 dev e
        T e[9];
        Mat<T> nh = mt;
        nh.model = ORACLE_NEO_HOOKEAN;
        kirchhoff(F, nh, e);
        const T pe = (e[0] + e[4] + e[8]) / T(3);
        T d[9], ss = T(0);
        for (int i = 0; i < 9; ++i) {
            d[i] = e[i] - ((i % 4 == 0) ? pe : T(0));
            ss += d[i] * d[i];
        }
        const T vm = std::sqrt(T(1.5) * ss);
        if (!(vm > J * mt.yield)) return kirchhoff_adj(F, nh, tb, gF);
        const T sc = J * mt.yield / vm;
        const T pt = (tb[0] + tb[4] + tb[8]) / T(3);
        T tbd = T(0);
        for (int i = 0; i < 9; ++i) tbd += tb[i] * d[i];
        T tbe[9];
        for (int i = 0; i < 9; ++i)
            tbe[i] = ((i % 4 == 0) ? pt : T(0)) + sc * (tb[i] - ((i % 4 == 0) ? pt : T(0))) - sc * tbd / ss * d[i];
        for (int i = 0; i < 9; ++i) gF[i] += sc * tbd * FiT[i];  // (s <tb, d> / J) dJ/dF, dJ/dF = J F^-T
        return kirchhoff_adj(F, nh, tbe, gF);
    }
    T trt = tb[0] + tb[4] + tb[8];
    if (mt.model == ORACLE_FIXED_COROTATED) {
        T R[9], S[9];
        polar3(F, R, S);
        T tbF[9], tbTFR[9], D[9];
        mm(tb, F, tbF);
        for (int i = 0; i < 9; ++i) D[i] = F[i] - R[i];
        mTm(tb, D, tbTFR);
        for (int i = 0; i < 9; ++i) gF[i] += T(2) * mt.mu * (tbF[i] + tbTFR[i]);
        // polar adjoint: Rbar = -2 mu tb F
        T Rb[9];
        for (int i = 0; i < 9; ++i) Rb[i] = -T(2) * mt.mu * tbF[i];
        T RtRb[9];
        mTm(R, Rb, RtRb);
        // y = axial(RtRb - RtRb^T)
        T y[3] = {RtRb[7] - RtRb[5], RtRb[2] - RtRb[6], RtRb[3] - RtRb[1]};
        T Ss[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) Ss[3 * i + j] = T(0.5) * (S[3 * i + j] + S[3 * j + i]);
        T trS = Ss[0] + Ss[4] + Ss[8];
        T G[9];
        for (int i = 0; i < 9; ++i) G[i] = -Ss[i] + ((i % 4 == 0) ? trS : T(0));
        T GiT[9];
        invT3(G, GiT);  // G symmetric -> G^{-T} = G^{-1}
        T z[3];
        for (int i = 0; i < 3; ++i) z[i] = GiT[3 * i] * y[0] + GiT[3 * i + 1] * y[1] + GiT[3 * i + 2] * y[2];
        T Z[9] = {0, -z[2], z[1], z[2], 0, -z[0], -z[1], z[0], 0};
        T RZ[9];
        mm(R, Z, RZ);
        for (int i = 0; i < 9; ++i) gF[i] += RZ[i];
        T c = mt.lam * (T(2) * J - T(1)) * trt * J;
        for (int i = 0; i < 9; ++i) gF[i] += c * FiT[i];
        T tmu[9];
        mmT(D, F, tmu);
        T dmu = 0;
        for (int i = 0; i < 9; ++i) dmu += tb[i] * T(2) * tmu[i];
        T dlam = trt * (J - T(1)) * J;
        return dmu * mt.dmu_dE + dlam * mt.dlam_dE;
    } else if (mt.model == ORACLE_NEO_HOOKEAN) {
        T a[9], b[9];
        mm(tb, F, a);
        mTm(tb, F, b);
        for (int i = 0; i < 9; ++i) gF[i] += mt.mu * (a[i] + b[i]) + mt.lam * trt * FiT[i];
        T B[9];
        mmT(F, F, B);
        T dmu = 0;
        for (int i = 0; i < 9; ++i) dmu += tb[i] * (B[i] - ((i % 4 == 0) ? T(1) : T(0)));
        T dlam = trt * std::log(J);
        return dmu * mt.dmu_dE + dlam * mt.dlam_dE;
    } else {
        T c = mt.E * (T(2) * J - T(1)) * trt * J;
        for (int i = 0; i < 9; ++i) gF[i] += c * FiT[i];
        return trt * J * (J - T(1));
    }
}

// ------------------------------------------------------------ shape functions
// Reference quadratic B-spline, src/material_point_method.h:288-293.
template <class T> inline T ref_quadratic(T x) {
    T abs_x = x < T{0} ? -x : x;
    if (abs_x >= T{1.5}) return T{0};
    if (abs_x < T{0.5}) return T{0.75} - x * x;
    return T{0.5} * (T{1.5} - abs_x) * (T{1.5} - abs_x);
}

// MLS weights for f in [0.5, 1.5): N0, N1, N2 and derivatives d/df.
template <class T> inline void mls_w(T f, T w[3], T dw[3]) {
    T a = T(1.5) - f, b = f - T(1), c = f - T(0.5);
    w[0] = T(0.5) * a * a;
    w[1] = T(0.75) - b * b;
    w[2] = T(0.5) * c * c;
    dw[0] = -a;
    dw[1] = T(-2) * b;
    dw[2] = c;
}

struct Grid {
    int n[3];
    int64_t nodes;
    int64_t idx(int i, int j, int k) const { return ((int64_t)k * n[1] + j) * n[0] + i; }
};

template <class T> struct State {
    std::vector<T> x, v, C, F;
};

// Stencil origin of one coordinate in float (matches the CUDA key kernel and
// the float REF_COMPAT oracle).
// MLS: u = (x - o) * inv_dx with inv_dx = 1/dx rounded to float;
// REF_COMPAT: u = (x - o) / dx as src/material_point_method.h:522-529.
inline int stencil_origin_f(float xa, float oa, float dx, int n, int physics) {
    const float inv_dx = 1.0f / dx;
    float u = physics == ORACLE_MLS ? (xa - oa) * inv_dx : (xa - oa) / dx;
    float s;
    if (physics == ORACLE_MLS)
        s = std::floor(u - 0.5f);
    else
        s = std::floor(u) - 1.0f;
    if (!(s == s)) s = 0.f;
    if (s < 0.f) s = 0.f;
    float hi = (float)(n - 3);
    if (s > hi) s = hi;
    return (int)s;
}

// ----------------------------------------------------------- REF_COMPAT step
// Literal restatement of MPMSolver<T,64>::step (material_point_method.h:479-666),
// serial, same float operations in the same order.
template <class T>
void ref_step(const oracle_scene& sc, Grid& g, State<T>& st, const std::vector<T>& m, int64_t n,
              std::vector<T>& gm, std::vector<T>& gp, std::vector<T>& gv) {
    const T o[3] = {T(sc.origin[0]), T(sc.origin[1]), T(sc.origin[2])};
    const T cs = T(sc.dx);
    const T dt = T(sc.dt);
    const T grav[3] = {T(sc.gravity[0]), T(sc.gravity[1]), T(sc.gravity[2])};
    std::fill(gm.begin(), gm.end(), T(0));
    std::fill(gp.begin(), gp.end(), T(0));
    std::fill(gv.begin(), gv.end(), T(0));
    // particleToGrid (:515-570)
    for (int64_t p = 0; p < n; ++p) {
        const T* pos = &st.x[3 * p];
        const T* vel = &st.v[3 * p];
        T mass = m[p];
        int bi = (int)std::floor((pos[0] - o[0]) / cs);
        int bj = (int)std::floor((pos[1] - o[1]) / cs);
        int bk = (int)std::floor((pos[2] - o[2]) / cs);
        T fx = (pos[0] - o[0]) / cs - bi;
        T fy = (pos[1] - o[1]) / cs - bj;
        T fz = (pos[2] - o[2]) / cs - bk;
        for (int di = -1; di < 2; ++di)
            for (int dj = -1; dj < 2; ++dj)
                for (int dk = -1; dk < 2; ++dk) {
                    int gi = bi + di, gj = bj + dj, gk = bk + dk;
                    if (gi < 0 || gi >= g.n[0] || gj < 0 || gj >= g.n[1] || gk < 0 || gk >= g.n[2]) continue;
                    T wx = ref_quadratic<T>(fx - di);
                    T wy = ref_quadratic<T>(fy - dj);
                    T wz = ref_quadratic<T>(fz - dk);
                    T weight = wx * wy * wz;
                    if (weight > T{1e-10}) {
                        int64_t ni = g.idx(gi, gj, gk);
                        gm[ni] += weight * mass;
                        T m0 = gp[3 * ni] + weight * mass * vel[0];
                        T m1 = gp[3 * ni + 1] + weight * mass * vel[1];
                        T m2 = gp[3 * ni + 2] + weight * mass * vel[2];
                        gp[3 * ni] = m0;
                        gp[3 * ni + 1] = m1;
                        gp[3 * ni + 2] = m2;
                    }
                }
    }
    // updateGridMomentum (:572-585) and calculateGridVelocity (:587-597)
    for (int64_t i = 0; i < g.nodes; ++i) {
        if (gm[i] > T{1e-10}) {
            T a0 = gp[3 * i] + gm[i] * grav[0] * dt;
            T a1 = gp[3 * i + 1] + gm[i] * grav[1] * dt;
            T a2 = gp[3 * i + 2] + gm[i] * grav[2] * dt;
            gp[3 * i] = a0;
            gp[3 * i + 1] = a1;
            gp[3 * i + 2] = a2;
        }
    }
    for (int64_t i = 0; i < g.nodes; ++i) {
        if (gm[i] > T{1e-10}) {
            gv[3 * i] = gp[3 * i] / gm[i];
            gv[3 * i + 1] = gp[3 * i + 1] / gm[i];
            gv[3 * i + 2] = gp[3 * i + 2] / gm[i];
        }
    }
    // gridToParticle (:599-649)
    for (int64_t p = 0; p < n; ++p) {
        const T* pos = &st.x[3 * p];
        T nv[3] = {0, 0, 0};
        int bi = (int)std::floor((pos[0] - o[0]) / cs);
        int bj = (int)std::floor((pos[1] - o[1]) / cs);
        int bk = (int)std::floor((pos[2] - o[2]) / cs);
        T fx = (pos[0] - o[0]) / cs - bi;
        T fy = (pos[1] - o[1]) / cs - bj;
        T fz = (pos[2] - o[2]) / cs - bk;
        for (int di = -1; di < 2; ++di)
            for (int dj = -1; dj < 2; ++dj)
                for (int dk = -1; dk < 2; ++dk) {
                    int gi = bi + di, gj = bj + dj, gk = bk + dk;
                    if (gi < 0 || gi >= g.n[0] || gj < 0 || gj >= g.n[1] || gk < 0 || gk >= g.n[2]) continue;
                    T wx = ref_quadratic<T>(fx - di);
                    T wy = ref_quadratic<T>(fy - dj);
                    T wz = ref_quadratic<T>(fz - dk);
                    T weight = wx * wy * wz;
                    if (weight > T{1e-10}) {
                        int64_t ni = g.idx(gi, gj, gk);
                        T a0 = nv[0] + weight * gv[3 * ni];
                        T a1 = nv[1] + weight * gv[3 * ni + 1];
                        T a2 = nv[2] + weight * gv[3 * ni + 2];
                        nv[0] = a0;
                        nv[1] = a1;
                        nv[2] = a2;
                    }
                }
        st.v[3 * p] = nv[0];
        st.v[3 * p + 1] = nv[1];
        st.v[3 * p + 2] = nv[2];
    }
    // updateParticlePositions (:651-666)
    for (int64_t p = 0; p < n; ++p) {
        T a0 = st.x[3 * p] + st.v[3 * p] * dt;
        T a1 = st.x[3 * p + 1] + st.v[3 * p + 1] * dt;
        T a2 = st.x[3 * p + 2] + st.v[3 * p + 2] * dt;
        st.x[3 * p] = a0;
        st.x[3 * p + 1] = a1;
        st.x[3 * p + 2] = a2;
    }
}

// ------------------------------------------------------------------ MLS step
template <class T> struct Stencil {
    int base[3];
    T f[3];
    T w[3][3], dw[3][3];
};

template <class T> inline void mls_stencil(const oracle_scene& sc, const Grid& g, const T* x, Stencil<T>& s) {
    const T inv_dx = T(1) / T(sc.dx);
    for (int a = 0; a < 3; ++a) {
        T u = (x[a] - T(sc.origin[a])) * inv_dx;
        T b = std::floor(u - T(0.5));
        if (!(b == b)) b = 0;
        if (b < 0) b = 0;
        if (b > T(g.n[a] - 3)) b = T(g.n[a] - 3);
        s.base[a] = (int)b;
        // f clamped to the support: an escaped particle transfers as if at
        // the wall (zero weight derivative there)
        T f = u - b;
        s.f[a] = f < T(0.5) ? T(0.5) : (f > T(1.5) ? T(1.5) : f);
        mls_w(s.f[a], s.w[a], s.dw[a]);
        if (f < T(0.5) || f > T(1.5)) s.dw[a][0] = s.dw[a][1] = s.dw[a][2] = T(0);
    }
}

inline bool in_wall(const oracle_scene& sc, const Grid& g, int a, int idx, int* side) {
    if (idx < sc.bthick) {
        *side = -1;
        return true;
    }
    if (idx >= g.n[a] - sc.bthick) {
        *side = 1;
        return true;
    }
    return false;
}

// grid update for one node; returns v (after BC) and vpre.
template <class T>
inline void mls_grid_node(const oracle_scene& sc, const Grid& g, int i, int j, int k, T m, const T* p, T* vpre, T* v) {
    if (m > T(0)) {
        for (int a = 0; a < 3; ++a) vpre[a] = p[a] / m + T(sc.dt) * T(sc.gravity[a]);
    } else {
        vpre[0] = vpre[1] = vpre[2] = T(0);
    }
    v[0] = vpre[0];
    v[1] = vpre[1];
    v[2] = vpre[2];
    if (sc.boundary == ORACLE_BC_NONE) return;
    int id[3] = {i, j, k};
    for (int a = 0; a < 3; ++a) {
        int side;
        if (!in_wall(sc, g, a, id[a], &side)) continue;
        if (sc.boundary == ORACLE_BC_STICKY) {
            v[0] = v[1] = v[2] = T(0);
        } else if (sc.boundary == ORACLE_BC_SLIP) {
            v[a] = T(0);
        } else {  // separate
            if ((side < 0 && v[a] < T(0)) || (side > 0 && v[a] > T(0))) v[a] = T(0);
        }
    }
}

template <class T> struct Sim {
    oracle_scene sc;
    Grid g;
    std::vector<Mat<T>> mats;
    int64_t n;
    std::vector<T> m, V0;
    std::vector<int> mat;
    std::vector<T> gm, gp, gvpre, gv;
};

template <class T> void mls_p2g(Sim<T>& S, const State<T>& st) {
    const T dx = T(S.sc.dx), D = T(4) / (dx * dx), dt = T(S.sc.dt);
    std::fill(S.gm.begin(), S.gm.end(), T(0));
    std::fill(S.gp.begin(), S.gp.end(), T(0));
    parallel_range(S.n, [&](int64_t pb, int64_t pe, int) {
    for (int64_t p = pb; p < pe; ++p) {
        Stencil<T> s;
        mls_stencil(S.sc, S.g, &st.x[3 * p], s);
        const Mat<T>& mt = S.mats[S.mat[p]];
        T tau[9];
        kirchhoff(&st.F[9 * p], mt, tau);
        if (mt.model == ORACLE_EOS_FLUID && mt.visc > T(0)) {
            // Newtonian viscosity (src/mpm_kernels.cu:131-149): sigma += mu_v (C + C^T)
            // with the APIC C as the velocity gradient; tau = J sigma
            const T* Cp = &st.C[9 * p];
            const T J = det3(&st.F[9 * p]);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) tau[3 * i + j] += J * mt.visc * (Cp[3 * i + j] + Cp[3 * j + i]);
        }
        T A[9];
        for (int i = 0; i < 9; ++i) A[i] = -dt * S.V0[p] * D * tau[i] + S.m[p] * st.C[9 * p + i];
        const T* vp = &st.v[3 * p];
        T mp = S.m[p];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) {
                    T w = s.w[0][i] * s.w[1][j] * s.w[2][k];
                    T d[3] = {(T(i) - s.f[0]) * dx, (T(j) - s.f[1]) * dx, (T(k) - s.f[2]) * dx};
                    int64_t ni = S.g.idx(s.base[0] + i, s.base[1] + j, s.base[2] + k);
                    T cm = w * mp;
                    atomic_add(&S.gm[ni], cm);
                    for (int a = 0; a < 3; ++a) {
                        T c = w * (mp * vp[a] + A[3 * a] * d[0] + A[3 * a + 1] * d[1] + A[3 * a + 2] * d[2]);
                        atomic_add(&S.gp[3 * ni + a], c);
                    }
                }
    }
    });
}

template <class T> void mls_grid(Sim<T>& S) {
    const Grid& g = S.g;
    parallel_range(g.n[2], [&](int64_t kb, int64_t ke, int) {
    for (int k = (int)kb; k < (int)ke; ++k)
        for (int j = 0; j < g.n[1]; ++j)
            for (int i = 0; i < g.n[0]; ++i) {
                int64_t ni = g.idx(i, j, k);
                mls_grid_node(S.sc, g, i, j, k, S.gm[ni], &S.gp[3 * ni], &S.gvpre[3 * ni], &S.gv[3 * ni]);
            }
    });
}

// G2P; also returns the new C (before F update) through Cn when non-null.
template <class T> void mls_g2p(Sim<T>& S, const State<T>& st, State<T>& out) {
    const T dx = T(S.sc.dx), D = T(4) / (dx * dx), dt = T(S.sc.dt);
    parallel_range(S.n, [&](int64_t pb, int64_t pe, int) {
    for (int64_t p = pb; p < pe; ++p) {
        Stencil<T> s;
        mls_stencil(S.sc, S.g, &st.x[3 * p], s);
        T nv[3] = {0, 0, 0}, B[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) {
                    T w = s.w[0][i] * s.w[1][j] * s.w[2][k];
                    T d[3] = {(T(i) - s.f[0]) * dx, (T(j) - s.f[1]) * dx, (T(k) - s.f[2]) * dx};
                    int64_t ni = S.g.idx(s.base[0] + i, s.base[1] + j, s.base[2] + k);
                    const T* gvn = &S.gv[3 * ni];
                    for (int a = 0; a < 3; ++a) {
                        nv[a] += w * gvn[a];
                        for (int b = 0; b < 3; ++b) B[3 * a + b] += w * gvn[a] * d[b];
                    }
                }
        T Cn[9], M[9], Fn[9];
        for (int i = 0; i < 9; ++i) Cn[i] = D * B[i];
        for (int i = 0; i < 9; ++i) M[i] = dt * Cn[i] + ((i % 4 == 0) ? T(1) : T(0));
        mm(M, &st.F[9 * p], Fn);
        if (S.mats[S.mat[p]].model == ORACLE_EOS_FLUID) {
            T J = det3(Fn);
            T c = std::cbrt(J);
            for (int i = 0; i < 9; ++i) Fn[i] = (i % 4 == 0) ? c : T(0);
        }
        for (int a = 0; a < 3; ++a) {
            out.v[3 * p + a] = nv[a];
            out.x[3 * p + a] = st.x[3 * p + a] + dt * nv[a];
        }
        for (int i = 0; i < 9; ++i) {
            out.C[9 * p + i] = Cn[i];
            out.F[9 * p + i] = Fn[i];
        }
    }
    });
}

template <class T> void mls_step(Sim<T>& S, State<T>& st) {
    mls_p2g(S, st);
    mls_grid(S);
    State<T> out = st;
    mls_g2p(S, st, out);
    st = std::move(out);
}

template <class T>
int run_impl(const oracle_scene* sc, const oracle_material* mats, int nmat, int64_t n, double* x, double* v,
             double* C, double* F, const double* m, const double* V0, const int32_t* mat, int steps,
             double* grid_m, double* grid_v) {
    Sim<T> S;
    S.sc = *sc;
    for (int a = 0; a < 3; ++a) {
        if (sc->n[a] < 4) return -2;
        S.g.n[a] = sc->n[a];
    }
    S.g.nodes = (int64_t)sc->n[0] * sc->n[1] * sc->n[2];
    S.n = n;
    for (int i = 0; i < nmat; ++i) S.mats.push_back(make_mat<T>(mats[i]));
    S.m.resize(n);
    S.V0.resize(n);
    S.mat.resize(n);
    State<T> st;
    st.x.resize(3 * n);
    st.v.resize(3 * n);
    st.C.resize(9 * n);
    st.F.resize(9 * n);
    for (int64_t p = 0; p < n; ++p) {
        S.m[p] = T(m[p]);
        S.V0[p] = V0 ? T(V0[p]) : T(0);
        S.mat[p] = mat ? mat[p] : 0;
        if (S.mat[p] < 0 || S.mat[p] >= nmat) return -3;
        for (int a = 0; a < 3; ++a) {
            st.x[3 * p + a] = T(x[3 * p + a]);
            st.v[3 * p + a] = T(v[3 * p + a]);
        }
        for (int i = 0; i < 9; ++i) {
            st.C[9 * p + i] = T(C[9 * p + i]);
            st.F[9 * p + i] = T(F[9 * p + i]);
        }
    }
    S.gm.assign(S.g.nodes, T(0));
    S.gp.assign(3 * S.g.nodes, T(0));
    S.gvpre.assign(3 * S.g.nodes, T(0));
    S.gv.assign(3 * S.g.nodes, T(0));
    for (int s = 0; s < steps; ++s) {
        if (sc->physics == ORACLE_REF_COMPAT)
            ref_step(*sc, S.g, st, S.m, n, S.gm, S.gp, S.gv);
        else
            mls_step(S, st);
    }
    for (int64_t p = 0; p < n; ++p) {
        for (int a = 0; a < 3; ++a) {
            x[3 * p + a] = double(st.x[3 * p + a]);
            v[3 * p + a] = double(st.v[3 * p + a]);
        }
        for (int i = 0; i < 9; ++i) {
            C[9 * p + i] = double(st.C[9 * p + i]);
            F[9 * p + i] = double(st.F[9 * p + i]);
        }
    }
    if (grid_m)
        for (int64_t i = 0; i < S.g.nodes; ++i) grid_m[i] = double(S.gm[i]);
    if (grid_v)
        for (int64_t i = 0; i < 3 * S.g.nodes; ++i) grid_v[i] = double(S.gv[i]);
    return 0;
}

// ------------------------------------------------------------------- adjoint
// Reverse of one MLS step.  st = state at the start of the step, grid arrays
// (gm, gp, gvpre, gv) of that step.  On entry a = adjoint of the step's
// output; on exit a = adjoint of its input.  gE accumulates dL/dE.
void mls_step_adjoint(Sim<double>& S, const State<double>& st, State<double>& a, std::vector<double>& gE) {
    typedef double T;
    const T dx = S.sc.dx, D = T(4) / (dx * dx), dt = S.sc.dt;
    const int64_t n = S.n;
    const Grid& g = S.g;
    // Recompute per-particle C', F'raw and the adjoints through x' = x + dt v'
    // and through the F update.
    std::vector<T> gvt(3 * n), gCt(9 * n), gFraw(9 * n), Cn(9 * n), Fraw(9 * n);
    std::vector<T> gvg(3 * g.nodes, T(0));
    parallel_range(n, [&](int64_t pb, int64_t pe, int) {
    for (int64_t p = pb; p < pe; ++p) {
        Stencil<T> s;
        mls_stencil(S.sc, g, &st.x[3 * p], s);
        T B[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) {
                    T w = s.w[0][i] * s.w[1][j] * s.w[2][k];
                    T d[3] = {(T(i) - s.f[0]) * dx, (T(j) - s.f[1]) * dx, (T(k) - s.f[2]) * dx};
                    int64_t ni = g.idx(s.base[0] + i, s.base[1] + j, s.base[2] + k);
                    for (int aa = 0; aa < 3; ++aa)
                        for (int b = 0; b < 3; ++b) B[3 * aa + b] += w * S.gv[3 * ni + aa] * d[b];
                }
        T M[9];
        for (int i = 0; i < 9; ++i) {
            Cn[9 * p + i] = D * B[i];
            M[i] = dt * Cn[9 * p + i] + ((i % 4 == 0) ? T(1) : T(0));
        }
        mm(M, &st.F[9 * p], &Fraw[9 * p]);
        T gFr[9];
        if (S.mats[S.mat[p]].model == ORACLE_EOS_FLUID) {
            T J = det3(&Fraw[9 * p]);
            T FiT[9];
            invT3(&Fraw[9 * p], FiT);
            T tr = a.F[9 * p] + a.F[9 * p + 4] + a.F[9 * p + 8];
            T c = std::cbrt(J) / T(3) * tr;
            for (int i = 0; i < 9; ++i) gFr[i] = c * FiT[i];
        } else {
            for (int i = 0; i < 9; ++i) gFr[i] = a.F[9 * p + i];
        }
        for (int i = 0; i < 9; ++i) gFraw[9 * p + i] = gFr[i];
        // C' adjoint: incoming + dt * gFraw F^T
        T gFFt[9];
        mmT(gFr, &st.F[9 * p], gFFt);
        for (int i = 0; i < 9; ++i) gCt[9 * p + i] = a.C[9 * p + i] + dt * gFFt[i];
        for (int aa = 0; aa < 3; ++aa) gvt[3 * p + aa] = a.v[3 * p + aa] + dt * a.x[3 * p + aa];
        // scatter grid velocity adjoint
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) {
                    T w = s.w[0][i] * s.w[1][j] * s.w[2][k];
                    T d[3] = {(T(i) - s.f[0]) * dx, (T(j) - s.f[1]) * dx, (T(k) - s.f[2]) * dx};
                    int64_t ni = g.idx(s.base[0] + i, s.base[1] + j, s.base[2] + k);
                    for (int aa = 0; aa < 3; ++aa) {
                        const T* gc = &gCt[9 * p + 3 * aa];
                        T c = w * (gvt[3 * p + aa] + D * (gc[0] * d[0] + gc[1] * d[1] + gc[2] * d[2]));
                        atomic_add(&gvg[3 * ni + aa], c);
                    }
                }
    }
    });
    // grid adjoint: gv -> gvpre (BC mask) -> gp, gm
    std::vector<T> gpn(3 * g.nodes, T(0)), gmn(g.nodes, T(0));
    parallel_range(g.n[2], [&](int64_t kb, int64_t ke, int) {
    for (int k = (int)kb; k < (int)ke; ++k)
        for (int j = 0; j < g.n[1]; ++j)
            for (int i = 0; i < g.n[0]; ++i) {
                int64_t ni = g.idx(i, j, k);
                T m = S.gm[ni];
                if (!(m > T(0))) continue;
                T gvp[3] = {gvg[3 * ni], gvg[3 * ni + 1], gvg[3 * ni + 2]};
                if (S.sc.boundary != ORACLE_BC_NONE) {
                    int id[3] = {i, j, k};
                    const T* vpre = &S.gvpre[3 * ni];
                    T vv[3] = {vpre[0], vpre[1], vpre[2]};
                    bool zero_all = false;
                    bool zero_c[3] = {false, false, false};
                    for (int aa = 0; aa < 3; ++aa) {
                        int side;
                        if (!in_wall(S.sc, g, aa, id[aa], &side)) continue;
                        if (S.sc.boundary == ORACLE_BC_STICKY) {
                            zero_all = true;
                        } else if (S.sc.boundary == ORACLE_BC_SLIP) {
                            zero_c[aa] = true;
                            vv[aa] = 0;
                        } else {
                            if ((side < 0 && vv[aa] < T(0)) || (side > 0 && vv[aa] > T(0))) {
                                zero_c[aa] = true;
                                vv[aa] = 0;
                            }
                        }
                    }
                    for (int aa = 0; aa < 3; ++aa)
                        if (zero_all || zero_c[aa]) gvp[aa] = T(0);
                }
                T pm[3];
                for (int aa = 0; aa < 3; ++aa) pm[aa] = S.gp[3 * ni + aa] / m;
                for (int aa = 0; aa < 3; ++aa) gpn[3 * ni + aa] = gvp[aa] / m;
                gmn[ni] = -(gvp[0] * pm[0] + gvp[1] * pm[1] + gvp[2] * pm[2]) / m;
            }
    });
    // per-particle gather
    const int nmat = (int)S.mats.size();
    std::vector<T> gEt((size_t)nmat * (g_threads > 1 ? g_threads : 1), T(0));
    parallel_range(n, [&](int64_t pb, int64_t pe, int tid) {
        T* gEl = &gEt[(size_t)nmat * tid];
        for (int64_t p = pb; p < pe; ++p) {
            Stencil<T> s;
            mls_stencil(S.sc, g, &st.x[3 * p], s);
            const Mat<T>& mt = S.mats[S.mat[p]];
            T tau[9];
            kirchhoff(&st.F[9 * p], mt, tau);
            const bool viscous = mt.model == ORACLE_EOS_FLUID && mt.visc > T(0);
            if (viscous) {  // as mls_p2g: tau += J mu_v (C + C^T)
                const T* Cp = &st.C[9 * p];
                const T J = det3(&st.F[9 * p]);
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) tau[3 * i + j] += J * mt.visc * (Cp[3 * i + j] + Cp[3 * j + i]);
            }
            T A[9];
            const T mp = S.m[p];
            for (int i = 0; i < 9; ++i) A[i] = -dt * S.V0[p] * D * tau[i] + mp * st.C[9 * p + i];
            const T* vp = &st.v[3 * p];
            const T* gc = &gCt[9 * p];
            T gx[3] = {a.x[3 * p], a.x[3 * p + 1], a.x[3 * p + 2]};
            T gvp[3] = {0, 0, 0}, Ab[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    for (int k = 0; k < 3; ++k) {
                        int o[3] = {i, j, k};
                        T w = s.w[0][i] * s.w[1][j] * s.w[2][k];
                        T d[3] = {(T(i) - s.f[0]) * dx, (T(j) - s.f[1]) * dx, (T(k) - s.f[2]) * dx};
                        int64_t ni = g.idx(s.base[0] + i, s.base[1] + j, s.base[2] + k);
                        const T* vi = &S.gv[3 * ni];
                        const T* gpi = &gpn[3 * ni];
                        T gmi = gmn[ni];
                        // weight adjoint
                        T Cd[3];
                        for (int aa = 0; aa < 3; ++aa) Cd[aa] = gc[3 * aa] * d[0] + gc[3 * aa + 1] * d[1] + gc[3 * aa + 2] * d[2];
                        T Ad[3];
                        for (int aa = 0; aa < 3; ++aa) Ad[aa] = A[3 * aa] * d[0] + A[3 * aa + 1] * d[1] + A[3 * aa + 2] * d[2];
                        T wb = gmi * mp;
                        for (int aa = 0; aa < 3; ++aa)
                            wb += gvt[3 * p + aa] * vi[aa] + D * vi[aa] * Cd[aa] + gpi[aa] * (mp * vp[aa] + Ad[aa]);
                        // dw/dx
                        for (int aa = 0; aa < 3; ++aa) {
                            T dwa = s.dw[aa][o[aa]];
                            for (int bb = 0; bb < 3; ++bb)
                                if (bb != aa) dwa *= s.w[bb][o[bb]];
                            gx[aa] += wb * dwa / dx;
                        }
                        // explicit d = x_i - x_p terms
                        for (int aa = 0; aa < 3; ++aa) {
                            // -D w C'^T v_i  and  -w A^T gp_i
                            T t1 = gc[aa] * vi[0] + gc[3 + aa] * vi[1] + gc[6 + aa] * vi[2];
                            T t2 = A[aa] * gpi[0] + A[3 + aa] * gpi[1] + A[6 + aa] * gpi[2];
                            gx[aa] -= w * (D * t1 + t2);
                        }
                        for (int aa = 0; aa < 3; ++aa) {
                            gvp[aa] += w * mp * gpi[aa];
                            for (int bb = 0; bb < 3; ++bb) Ab[3 * aa + bb] += w * gpi[aa] * d[bb];
                        }
                    }
            T gF[9];
            // F' = (I + dt C') F  ->  gF = (I + dt C')^T gFraw
            T M[9];
            for (int i = 0; i < 9; ++i) M[i] = dt * Cn[9 * p + i] + ((i % 4 == 0) ? T(1) : T(0));
            mTm(M, &gFraw[9 * p], gF);
            T tb[9];
            for (int i = 0; i < 9; ++i) tb[i] = -dt * S.V0[p] * D * Ab[i];
            gEl[S.mat[p]] += kirchhoff_adj(&st.F[9 * p], mt, tb, gF);
            T gCv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            if (viscous) {
                // tau_v = J mu_v (C + C^T): d/dC = J mu_v (tb + tb^T),
                // d/dF = mu_v <tb, C + C^T> dJ/dF with dJ/dF = J F^-T
                const T* Fp = &st.F[9 * p];
                const T* Cp = &st.C[9 * p];
                const T J = det3(Fp);
                T FiT[9];
                invT3(Fp, FiT);
                T tc = T(0);
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        gCv[3 * i + j] = J * mt.visc * (tb[3 * i + j] + tb[3 * j + i]);
                        tc += tb[3 * i + j] * (Cp[3 * i + j] + Cp[3 * j + i]);
                    }
                for (int i = 0; i < 9; ++i) gF[i] += mt.visc * tc * J * FiT[i];
            }
            for (int aa = 0; aa < 3; ++aa) {
                a.x[3 * p + aa] = gx[aa];
                a.v[3 * p + aa] = gvp[aa];
            }
            for (int i = 0; i < 9; ++i) {
                a.C[9 * p + i] = mp * Ab[i] + gCv[i];
                a.F[9 * p + i] = gF[i];
            }
        }
    });
    for (size_t t = 0; t < gEt.size(); ++t) gE[t % nmat] += gEt[t];
}

}  // namespace

extern "C" int oracle_run(int prec, const oracle_scene* s, const oracle_material* mats, int nmat, int64_t n,
                          double* x, double* v, double* C, double* F, const double* m, const double* V0,
                          const int32_t* mat, int steps, int nthreads, double* grid_m, double* grid_v) {
    if (!s || !mats || nmat < 1 || n < 0 || steps < 0) return -1;
    g_threads = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
    if (prec == 64) return run_impl<double>(s, mats, nmat, n, x, v, C, F, m, V0, mat, steps, grid_m, grid_v);
    if (prec == 32) return run_impl<float>(s, mats, nmat, n, x, v, C, F, m, V0, mat, steps, grid_m, grid_v);
    return -1;
}

extern "C" int oracle_keys(const oracle_scene* s, int64_t n, const float* x, uint32_t cell_base, uint32_t* keys) {
    if (!s) return -1;
    int nt[3];
    for (int a = 0; a < 3; ++a) nt[a] = ((s->n[a] - 3) >> 2) + 1;
    float o[3] = {(float)s->origin[0], (float)s->origin[1], (float)s->origin[2]};
    float dx = (float)s->dx;
    for (int64_t p = 0; p < n; ++p) {
        int c[3];
        for (int a = 0; a < 3; ++a) c[a] = stencil_origin_f(x[3 * p + a], o[a], dx, s->n[a], s->physics);
        uint32_t tile = (uint32_t)(((c[2] >> 2) * nt[1] + (c[1] >> 2)) * nt[0] + (c[0] >> 2));
        uint32_t local = (uint32_t)((c[2] & 3) * 16 + (c[1] & 3) * 4 + (c[0] & 3));
        keys[p] = cell_base + tile * 64u + local;
    }
    return 0;
}

extern "C" int oracle_stable_sort(int64_t n, const uint32_t* keys, const uint32_t* vals, uint32_t* out_keys,
                                  uint32_t* out_vals) {
    std::vector<int64_t> idx(n);
    for (int64_t i = 0; i < n; ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) { return keys[a] < keys[b]; });
    for (int64_t i = 0; i < n; ++i) {
        out_keys[i] = keys[idx[i]];
        out_vals[i] = vals ? vals[idx[i]] : (uint32_t)idx[i];
    }
    return 0;
}

extern "C" int oracle_adjoint(const oracle_scene* sc, const oracle_material* mats, int nmat, int64_t n,
                              const double* x, const double* v, const double* C, const double* F,
                              const double* m, const double* V0, const int32_t* mat, int steps, int nthreads,
                              double* gx, double* gv, double* gC, double* gF, double* gE) {
    if (!sc || sc->physics != ORACLE_MLS || nmat < 1 || n < 0 || steps < 0) return -1;
    g_threads = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
    Sim<double> S;
    S.sc = *sc;
    for (int a = 0; a < 3; ++a) S.g.n[a] = sc->n[a];
    S.g.nodes = (int64_t)sc->n[0] * sc->n[1] * sc->n[2];
    S.n = n;
    for (int i = 0; i < nmat; ++i) S.mats.push_back(make_mat<double>(mats[i]));
    S.m.assign(m, m + n);
    S.V0.assign(V0, V0 + n);
    S.mat.resize(n);
    for (int64_t p = 0; p < n; ++p) {
        S.mat[p] = mat ? mat[p] : 0;
        if (S.mat[p] < 0 || S.mat[p] >= nmat) return -3;
    }
    S.gm.assign(S.g.nodes, 0);
    S.gp.assign(3 * S.g.nodes, 0);
    S.gvpre.assign(3 * S.g.nodes, 0);
    S.gv.assign(3 * S.g.nodes, 0);
    // States are kept every K steps and each segment is recomputed from its
    // checkpoint before its reverse, so host memory stays at about
    // (steps / K + K) states instead of steps + 1.
    const int K = std::max(1, (int)std::ceil(std::sqrt((double)std::max(steps, 1))));
    const int nseg = (steps + K - 1) / K;
    std::vector<State<double>> ck(std::max(nseg, 1));
    ck[0].x.assign(x, x + 3 * n);
    ck[0].v.assign(v, v + 3 * n);
    ck[0].C.assign(C, C + 9 * n);
    ck[0].F.assign(F, F + 9 * n);
    {
        State<double> cur = ck[0];
        for (int s = 0; s < steps; ++s) {
            if (s % K == 0) ck[s / K] = cur;
            mls_step(S, cur);
        }
    }
    State<double> a;
    a.x.assign(gx, gx + 3 * n);
    a.v.assign(gv, gv + 3 * n);
    a.C.assign(gC, gC + 9 * n);
    a.F.assign(gF, gF + 9 * n);
    std::vector<double> gEv(nmat, 0.0);
    std::vector<State<double>> hist(K);
    for (int seg = nseg - 1; seg >= 0; --seg) {
        const int s0 = seg * K, len = std::min(K, steps - s0);
        hist[0] = ck[seg];
        for (int j = 1; j < len; ++j) {
            hist[j] = hist[j - 1];
            mls_step(S, hist[j]);
        }
        for (int j = len - 1; j >= 0; --j) {
            // rebuild the grid of step s0 + j
            mls_p2g(S, hist[j]);
            mls_grid(S);
            mls_step_adjoint(S, hist[j], a, gEv);
        }
    }
    std::memcpy(gx, a.x.data(), sizeof(double) * 3 * n);
    std::memcpy(gv, a.v.data(), sizeof(double) * 3 * n);
    std::memcpy(gC, a.C.data(), sizeof(double) * 9 * n);
    std::memcpy(gF, a.F.data(), sizeof(double) * 9 * n);
    for (int i = 0; i < nmat; ++i) gE[i] = gEv[i];
    return 0;
}

// ------------------------------------------------------------ consumers
// SPH-MPM contact coupling, restating SPHMPMCouplingSystem::findCouplingPairs
// (src/sph_mpm_coupling.h:453-485: every (SPH, MPM) pair closer than the
// coupling radius, SPH index outer, MPM index inner), computeCouplingForces
// (:487-545: normal spring k (r - d) plus damping c (dv . n) along
// n = (x_mpm - x_sph) / d, friction -mu k (r - d) along the tangential
// velocity, skipped when d < 1e-6; the fluid force, minus the solid force,
// added to the SPH particle when two-way) and getTotalCouplingEnergy
// (:563-575: sum of k (r - d)^2 / 2), in float and in the same order, so that
// it matches the reference's own class bit for bit.
extern "C" int oracle_sph_coupling(int64_t n_sph, const float* sph_x, const float* sph_v, int64_t n_mpm,
                                   const float* mpm_x, const float* mpm_v, float k, float c, float mu, float r,
                                   int two_way, float* sph_force, float* mpm_force, int64_t* n_pairs,
                                   float* energy) {
    int64_t pairs = 0;
    float e = 0.f;
    for (int64_t i = 0; i < 3 * n_mpm; ++i) mpm_force[i] = 0.f;
    for (int64_t s = 0; s < n_sph; ++s) {
        const float* y = &sph_x[3 * s];
        const float* vy = &sph_v[3 * s];
        float fs[3] = {0.f, 0.f, 0.f};
        for (int64_t p = 0; p < n_mpm; ++p) {
            const float rv[3] = {mpm_x[3 * p] - y[0], mpm_x[3 * p + 1] - y[1], mpm_x[3 * p + 2] - y[2]};
            const float d = std::sqrt(rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2]);
            if (!(d < r)) continue;
            ++pairs;
            const float pen = r - d;
            e += 0.5f * k * pen * pen;
            if (d < 1e-6f) continue;
            const float inv = 1.f / d;
            const float n[3] = {rv[0] * inv, rv[1] * inv, rv[2] * inv};
            const float dv[3] = {mpm_v[3 * p] - vy[0], mpm_v[3 * p + 1] - vy[1], mpm_v[3 * p + 2] - vy[2]};
            const float fn = k * pen;
            const float vn = dv[0] * n[0] + dv[1] * n[1] + dv[2] * n[2];
            const float fd = c * vn;
            float solid[3];
            for (int a = 0; a < 3; ++a) solid[a] = n[a] * (fn + fd);
            const float tv[3] = {dv[0] - n[0] * vn, dv[1] - n[1] * vn, dv[2] - n[2] * vn};
            const float ts = std::sqrt(tv[0] * tv[0] + tv[1] * tv[1] + tv[2] * tv[2]);
            if (ts > 1e-6f) {
                const float it = 1.f / ts;
                const float fm = mu * fn;
                for (int a = 0; a < 3; ++a) solid[a] = solid[a] + (tv[a] * it) * (-fm);
            }
            for (int a = 0; a < 3; ++a) {
                mpm_force[3 * p + a] += solid[a];
                if (two_way) fs[a] += solid[a] * -1.f;
            }
        }
        for (int a = 0; a < 3; ++a) sph_force[3 * s + a] = fs[a];
    }
    *n_pairs = pairs;
    *energy = e;
    return 0;
}

// Kinetic energy of particle sets, restating the energy monitor of
// FSISimulationManager (computeTotalEnergy, src/fsi_coupling.h:837-858):
// sum over particles of m |v|^2 / 2, here per material id (FP64).
extern "C" int oracle_kinetic_energy(int64_t n, const double* v, const double* m, const int32_t* mat, int nmat,
                                     double* per_material) {
    for (int i = 0; i < nmat; ++i) per_material[i] = 0.0;
    for (int64_t p = 0; p < n; ++p) {
        const int id = mat ? mat[p] : 0;
        if (id < 0 || id >= nmat) return -3;
        per_material[id] += 0.5 * m[p] * (v[3 * p] * v[3 * p] + v[3 * p + 1] * v[3 * p + 1] + v[3 * p + 2] * v[3 * p + 2]);
    }
    return 0;
}
