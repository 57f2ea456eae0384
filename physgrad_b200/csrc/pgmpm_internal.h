// pgmpm_internal.h -- declarations shared by the CUDA translation units of
// libpgmpm.so.  Not installed; the public surface is include/pgmpm.h.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "pgmpm_device.cuh"

namespace pgmpm {

// counters[] layout.  Words [0, CNT_RESET) are cleared every step:
// active node tiles, occupied cell tiles, active node count (u64), the
// work cursors of the tile kernels, and the occupied cell tiles per size
// class (CNT_BUCKETS classes, largest first).  CNT_FLAGS (sticky error
// flags) is cleared only by pgmpm_check_status.
constexpr int CNT_BUCKETS = 8;
enum {
    CNT_TILES = 0,
    CNT_CTILES = 1,
    CNT_ACTIVE = 2,
    CNT_P2G_CURSOR = 4,
    CNT_G2P_CURSOR = 5,
    CNT_BUCKET = 6,
    CNT_RESET = CNT_BUCKET + CNT_BUCKETS,
    CNT_FLAGS = CNT_RESET,
    CNT_STAMP = CNT_RESET + 1,  // sparse grids: step counter; a node tile is active when its flag equals it
    CNT_WORDS = 16
};
static_assert(CNT_STAMP < CNT_WORDS, "counter layout");

// Everything a step kernel needs, passed by value.
struct View {
    int64_t N;
    int S, M;
    const SceneDev* scenes;
    const MatDev* mats;
    float4* q;                 // 6 planes of N float4 (state at the start of the step)
    float4* q_out;             // where G2P writes the new state (== q in place; MLS only otherwise)
    float4* pay;               // MLS P2G payload of the state in q (4 planes), read by P2G
    float4* pay_out;           // payload of the state G2P writes (null: G2P does not write one)
    int write_vc;              // MLS G2P stores v and C (planes 3-5); 0 between the steps of one
                               // call, where the next step reads them only through the payload
    const float2* mV;          // (mass, V0)
    const int32_t* mat;        // material id (null when M == 1)
    uint32_t* keys;            // cell key per particle (physical order), input of the next sort
    uint32_t* resort;          // MLS G2P replaying recorded steps: V.keys holds the recorded next
                               // keys; G2P overwrites only those that differ and then sets *resort
                               // (the next step must sort again).  Null: G2P writes every key.
    const uint32_t* skeys;     // sorted keys
    const uint32_t* order;     // sorted position -> physical particle
    float4* grid_mp;           // (m, p) accumulator
    float4* grid_v;            // (v, m) after the grid update
    float4* grid_vpre;         // optional: (v before walls, m), recorded for the adjoint
    uint32_t* tile_flags;      // node tile active flags (per global node tile)
    uint32_t* tile_list;       // active node tiles
    uint32_t* ctile_list;      // occupied cell tiles (global cell tile ids)
    const uint32_t* ptile_list;  // the same tiles, largest first (null: use ctile_list)
    uint2* ctile_range;        // per global cell tile: [begin, end) in sorted order
    const uint2* cell_range;   // per global cell: [begin, end) in sorted order (null: search skeys)
    uint32_t* counters;        // see CNT_*
    int total_ct, total_nt;
    SparseTiles sp;            // sparse grid (sp.cap == 0: dense; tile ids are then slots)
};

// P2G variants: 0 = (cell, z-slice) register accumulation with a staged
// payload, 1 = per-particle shared-memory atomics over fixed chunks,
// 2 = one thread per cell, 108 register accumulators, no staging,
// 3 = variant 2 with a cell's accumulators split over two lanes (MLS
// forward; the REF physics and the adjoint scatter run variant 2).
// G2P variant 2 = direct gather in physical particle order (default).
// G2P variants: 0 = node tile staged in shared memory, 1 = direct gather.
struct Tuning {
    int p2g_block = 192;   // variant 0 uses exactly 192 threads (64 cells x 3 z-slices)
    int ppt = 1024;        // variant 1: particles per chunk; variant 0: sub-chunk staged at once is fixed
    int g2p_block = 128;   // 64..512 swept: 64 and 128 equal, 192..512 up to 2.5% slower
    int grid_block = 256;
    int p2g_variant = 2;
    int g2p_variant = 2;
    int tile_blocks_per_sm = 3;  // persistent P2G tile kernel: blocks per SM
    int g2p_tiles_per_sm = 2;    // persistent G2P tile kernel: blocks per SM (256 threads)
    int cell_blocks_per_sm = 6;  // persistent P2G thread-per-cell kernel (variant 2): blocks per SM
    int pair_blocks_per_sm = 5;  // persistent P2G two-threads-per-cell kernel (variant 3): blocks per SM
    int step_sort = 0;           // per-step sort: 0 = bin sort (counting sorts by tile, then cell), 1 = radix sort
    int g2p2g_blocks_per_sm = 4; // fused kernel (P2G variant 5): 4 (255 registers) or 6 (168, some spilled)
};
// P2G variant 5 = variant 4's P2G, fused with the previous step's G2P when
// steps follow one another (launch_g2p2g).

// What one recorded step launches.  MLS with the fused G2P -> P2G kernel
// (P2G variant 5) chains steps: a step's G2P2G does the next step's P2G.
enum StepKind {
    STEP_SPLIT = 0,    // sort, P2G, grid update, G2P (which writes the next payload)
    STEP_FUSED_FIRST,  // sort, P2G, grid update, G2P2G
    STEP_FUSED,        // sort, grid update, G2P2G (P2G done by the previous step's G2P2G)
    STEP_FUSED_LAST,   // sort, grid update, G2P (nothing left pending in grid_mp)
    STEP_KINDS
};

// pgmpm_sort.cu
constexpr int RADIX_TILE = 2048;  // keys per block of the sort kernels
constexpr int RADIX_MAX_DIGITS = 256;
// u32 words of histogram scratch the sort needs for n pairs
constexpr int64_t radix_scratch_words_for(int64_t n) {
    return ((n + RADIX_TILE - 1) / RADIX_TILE) * RADIX_MAX_DIGITS + RADIX_MAX_DIGITS;
}
int64_t radix_sort_scratch_words(int64_t n);
int radix_passes(int key_bits);
cudaError_t radix_sort_pairs(const uint32_t* kin, const uint32_t* vin, uint32_t* ka, uint32_t* va, uint32_t* kb,
                             uint32_t* vb, uint32_t* scratch, int64_t n, int key_bits, int* which,
                             cudaStream_t st);

// Per-step bin sort (pgmpm_sort.cu): keys_in (physical order) -> out_k /
// out_v sorted by key, plus the occupied cell tiles, their ranges, the
// active node tiles and their flags (View fields) and, when cell_range is
// set, every cell's [begin, end) in the sorted order of the occupied tiles.
// ccount and tcount must be zero on entry and are left zero.
struct BinSortBufs {
    const uint32_t* keys_in;
    uint32_t* ccount;      // total_ct * 64 + 1 words (cells + overflow bin), zero between steps
    uint32_t* coff;        // total_ct * 64 words
    uint32_t* tcount;      // total_ct + 1 words, zero between steps
    uint32_t* toff;        // total_ct + 1 words
    uint32_t* bsum;        // bin_sort_scan_blocks(total_ct) words
    uint32_t* slot;        // N words
    uint32_t *out_k, *out_v;  // N words each
    uint2* cell_range;     // total_ct * 64, or null
    uint32_t* ptile_list;  // total_ct: occupied tiles by size class, largest first (null: not built)
    uint32_t* tile_rank;   // total_ct: class and rank of each ctile_list entry (scratch, with ptile_list)
};
int64_t bin_sort_scan_blocks(int total_ct);
cudaError_t bin_sort_step(const View& V, const BinSortBufs& B, int num_sms, cudaStream_t st);

// pgmpm_kernels.cu
struct PhysFlags {
    int physics;     // PHYS_MLS / PHYS_REF (same for every scene)
    bool multi_mat;  // per-particle material ids
    bool has_fluid;  // some material uses the EOS model
    bool has_plastic;  // some material is ELASTOPLASTIC (von Mises)
};
cudaError_t launch_keys(const View& V, const PhysFlags& pf, cudaStream_t st);
cudaError_t launch_payload(const View& V, const PhysFlags& pf, cudaStream_t st);
cudaError_t launch_mark(const View& V, cudaStream_t st);
cudaError_t launch_p2g(const View& V, const PhysFlags& pf, const Tuning& t, int num_sms, cudaStream_t st);
cudaError_t launch_grid(const View& V, const PhysFlags& pf, const Tuning& t, int num_sms, cudaStream_t st);
cudaError_t launch_g2p(const View& V, const PhysFlags& pf, const Tuning& t, int num_sms, cudaStream_t st);
// Fused G2P of this step and P2G of the next (MLS with the bin sort's cell
// table): writes the new state and keys and accumulates the next step's
// (m, p) into V.grid_mp; takes work from the G2P cursor.
cudaError_t launch_g2p2g(const View& V, const PhysFlags& pf, const Tuning& t, int num_sms, cudaStream_t st);
cudaError_t launch_pack(const View& V, const float* x, const float* v, const float* C, const float* F,
                        const float* m, const float* V0, const int32_t* mat, const uint32_t* order,
                        uint32_t* user_of_phys, uint32_t* phys_of_user, float2* mV_out, int32_t* mat_out,
                        cudaStream_t st);
// phys_of_user: upload index -> physical slot (written by launch_pack)
cudaError_t launch_unpack(const View& V, const uint32_t* phys_of_user, float* x, float* v, float* C, float* F,
                          cudaStream_t st);
// ORs the error flags of `slots` counter blocks (stride CNT_WORDS) into
// live[CNT_FLAGS] and clears them.
cudaError_t launch_merge_flags(uint32_t* slots_counters, int slots, uint32_t* live, cudaStream_t st);
cudaError_t launch_grid_download(const View& V, int scene, const SceneDev& sc, float* mass, float* vel,
                                 cudaStream_t st);

// Reverse pass of one MLS step (pgmpm_adjoint.cu, and the scatter in
// pgmpm_kernels.cu).  V describes the step as it ran (V.q = state before the
// step, order / tiles / grid_v / grid_vpre of the step); V.grid_mp is the
// scatter target for dL/dv_i.
struct AdjView {
    // adjoint of the particle state after the step, overwritten with the
    // adjoint of the state before it (physical order, same plane packing)
    float4* g;                 // 6 planes
    const float4* q_next;      // state after the step (C' for the F update and the fluid reset)
    float4* grid_gv;           // (0, dL/dv_i) scatter target, zeroed by the grid adjoint
    float4* grid_gpm;          // (dL/dp_i, dL/dm_i) per node
    float* gE;                 // [M] dL/dE accumulators
};
cudaError_t launch_adj_scatter(const View& V, const AdjView& A, const PhysFlags& pf, const Tuning& t, int num_sms,
                               cudaStream_t st);
cudaError_t launch_adj_grid(const View& V, const AdjView& A, const Tuning& t, int num_sms, cudaStream_t st);
cudaError_t launch_adj_gather(const View& V, const AdjView& A, const PhysFlags& pf, const Tuning& t,
                              cudaStream_t st);
cudaError_t launch_state_to_planes(const float* x, const float* v, const float* C, const float* F,
                                   const uint32_t* user_of_phys, float4* g, int64_t N, cudaStream_t st);
// reverse of one REF_COMPAT step (pgmpm_ref_adjoint.cu); particle arrays in
// the caller's order, G: one float4 per grid node, zeroed by the caller
cudaError_t launch_ref_adjoint(const View& V, const float* x, const float* v, const float* m, const float* gx,
                               const float* gv, float4* G, float* gx_in, float* gv_in, float* gm_in, float* ggrav,
                               int num_sms, cudaStream_t st);
cudaError_t launch_planes_to_state(const float4* g, const uint32_t* phys_of_user, float* x, float* v, float* C,
                                   float* F, int64_t N, cudaStream_t st);

}  // namespace pgmpm
