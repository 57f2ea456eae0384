/*
 * oracle.h -- C interface of the CPU oracle for the MLS-MPM step.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product path (physgrad_b200/,
 * include/) links, loads or calls this library.  It is the checker that the
 * CUDA kernels are compared against in tests/, in __graft_entry__.smoke() and
 * in the cpu_baseline leg of bench.py.
 *
 * What it restates (reference file:line, paths inside pedroscortes/physgrad):
 *   - REF_COMPAT physics: the CPU solver physgrad::mpm::MPMSolver<T,64>::step()
 *     in src/material_point_method.h:479-500 (P2G :515-570, grid momentum
 *     :572-585, grid velocity :587-597, G2P :599-649, positions :651-666), the
 *     quadratic B-spline MPMShapeFunctions::quadratic at :288-293, grid index
 *     MPMGrid::getNodeIndex at :249-253.  The float instance performs the same
 *     float operations in the same order, so that it can be checked bit for
 *     bit against the reference compiled from its own sources (oracle/_ref).
 *   - MLS physics (not present in the reference, which has no APIC, no
 *     fixed-corotated model and no walls): MLS-MPM of Hu et al., SIGGRAPH
 *     2018, with the APIC affine matrix of Jiang et al. 2015, the
 *     fixed-corotated energy of Stomakhin et al. 2012, the compressible
 *     neo-Hookean law in the Kirchhoff form of the Cauchy stress stated at
 *     src/mpm_kernels.cu:97-128 (sigma = mu/J (B - I) + lambda/J ln J I), a
 *     weakly compressible EOS fluid p = -K (J - 1) where K is carried in the
 *     youngs_modulus field as src/mpm_data_structures.h:87-94 does for
 *     FLUID, the F update (I + dt C) F of src/mpm_kernels.cu:384-397 and the
 *     grid update order of src/mpm_kernels.cu:511-544.  ELASTOPLASTIC
 *     (ORACLE_VON_MISES): the neo-Hookean predictor with the von Mises return
 *     mapping of src/material_point_method.h:375-402 (deviatoric Cauchy stress
 *     scaled down to the yield stress; stateless, as there).  FLUID viscosity:
 *     the Newtonian stress 2 mu_v sym(grad v) of src/mpm_kernels.cu:131-149
 *     with the APIC C as grad v, added to the EOS pressure (forward only).
 *   - The cell-key definition and a stable sort (std::stable_sort) that the
 *     GPU radix sort must reproduce bit for bit.
 *   - The reverse-mode adjoint of the MLS step (FP64), used to check the
 *     GPU adjoint coordinate by coordinate; it is itself checked against
 *     central finite differences in tests/.
 *
 * Parity pin: the REF_COMPAT float instance is pinned against the
 * reference's own CPU solver built from its sources (oracle/_ref) and the
 * golden fixtures in tests/golden/ produced from it.  The MLS physics has no
 * counterpart in the reference: "parity unpinned" for MLS, and for gradients
 * (the reference's MPM adjoint, src/differentiable_mpm.h:871-876, records an
 * empty backward and returns zeros).
 */
#ifndef PGMPM_ORACLE_H
#define PGMPM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_MLS = 0, ORACLE_REF_COMPAT = 1 };
enum { ORACLE_BC_NONE = 0, ORACLE_BC_STICKY = 1, ORACLE_BC_SLIP = 2, ORACLE_BC_SEPARATE = 3 };
enum { ORACLE_FIXED_COROTATED = 0, ORACLE_NEO_HOOKEAN = 1, ORACLE_EOS_FLUID = 2, ORACLE_VON_MISES = 3 };

typedef struct {
    int32_t n[3];        /* grid nodes per axis */
    int32_t physics;     /* ORACLE_MLS / ORACLE_REF_COMPAT */
    int32_t boundary;    /* ORACLE_BC_* (MLS only) */
    int32_t bthick;      /* wall thickness in nodes */
    int32_t pad0, pad1;
    double dx;
    double origin[3];
    double dt;
    double gravity[3];
} oracle_scene;

typedef struct {
    int32_t model;       /* ORACLE_FIXED_COROTATED / NEO_HOOKEAN / EOS_FLUID / VON_MISES */
    int32_t pad;
    double E;            /* Young's modulus, or bulk modulus K for EOS_FLUID */
    double nu;
    double yield_stress; /* VON_MISES: von Mises yield stress of the Cauchy stress */
    double viscosity;    /* EOS_FLUID: dynamic viscosity (0: inviscid) */
} oracle_material;

/* Advance `steps` steps.  x,v: [n][3]; C,F: [n][9] row-major; m,V0: [n];
 * mat: [n] material index (NULL = all 0).  prec = 64 (double) or 32 (float
 * mirror).  grid_m [nodes] / grid_v [nodes][3] (may be NULL): grid mass and
 * velocity of the last step, linear index k*nx*ny + j*nx + i.  Returns 0 or a
 * negative error code. */
int oracle_run(int prec, const oracle_scene* s, const oracle_material* mats, int nmat,
               int64_t n, double* x, double* v, double* C, double* F,
               const double* m, const double* V0, const int32_t* mat,
               int steps, int nthreads, double* grid_m, double* grid_v);

/* Cell keys of float positions x [n][3]: the stencil origin s per axis
 * (MLS: floor((x-o)/dx - 0.5), REF_COMPAT: floor((x-o)/dx) - 1, both in
 * float and clamped to [0, n-3]), tile-major: key = cell_base +
 * tile_linear*64 + (sz&3)*16 + (sy&3)*4 + (sx&3). */
int oracle_keys(const oracle_scene* s, int64_t n, const float* x, uint32_t cell_base, uint32_t* keys);

/* Stable sort of (key, value) pairs by key (std::stable_sort). */
int oracle_stable_sort(int64_t n, const uint32_t* keys, const uint32_t* vals,
                       uint32_t* out_keys, uint32_t* out_vals);

/* Reverse-mode adjoint of `steps` MLS steps (FP64).  Inputs as oracle_run
 * (state is not modified).  gx,gv [n][3], gC,gF [n][9]: on entry the adjoint
 * of the final state, on exit the adjoint of the initial state.  gE [nmat]:
 * on exit dL/dE per material (dL/dK for EOS_FLUID). */
int oracle_adjoint(const oracle_scene* s, const oracle_material* mats, int nmat,
                   int64_t n, const double* x, const double* v, const double* C, const double* F,
                   const double* m, const double* V0, const int32_t* mat, int steps, int nthreads,
                   double* gx, double* gv, double* gC, double* gF, double* gE);

#ifdef __cplusplus
}
#endif
#endif
