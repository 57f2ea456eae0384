// pgmpm_solver_impl.h -- the solver handle behind pgmpm_solver and the step
// recorder, shared by the C-ABI translation units (pgmpm_capi.cu,
// pgmpm_diff.cu).  Not installed.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/pgmpm.h"
#include "pgmpm_internal.h"

namespace pgmpm {

// Records an error message for pgmpm_last_error() and returns code.
int fail(int code, const char* fmt, ...);

#define CK(expr)                                                                                             \
    do {                                                                                                     \
        cudaError_t e_ = (expr);                                                                             \
        if (e_ != cudaSuccess)                                                                               \
            return ::pgmpm::fail(e_ == cudaErrorMemoryAllocation ? PGMPM_ERR_OOM : PGMPM_ERR_CUDA,           \
                                 "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__);       \
    } while (0)

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    cudaError_t alloc(size_t b) {
        release();
        if (b == 0) b = 16;
        cudaError_t e = cudaMalloc(&p, b);
        if (e == cudaSuccess) bytes = b;
        return e;
    }
    cudaError_t ensure(size_t b) { return bytes >= b ? cudaSuccess : alloc(b); }
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

inline int bits_for(uint64_t v) {
    int b = 0;
    while ((1ull << b) < v) ++b;
    return b < 1 ? 1 : b;
}

// Buffers one step reads and writes.  The live solver uses its own; the
// reverse pass replays steps into per-step tape slots.
struct StepBufs {
    float4* q;             // state at the start of the step (read by P2G and G2P)
    float4* q_out;         // state G2P writes (== q for the live solver)
    float4* pay;           // MLS P2G payload of q, rewritten by G2P for q_out (null for REF physics)
    uint32_t* keys_in;     // keys sorted by this step
    uint32_t* keys_out;    // keys G2P writes for the next step (may equal keys_in)
    uint32_t *ka, *va, *kb, *vb;  // sort ping-pong; result in (ka, va) if which == 0 else (kb, vb)
    int which;
    float4* grid_v;
    float4* grid_vpre;     // may be null
    uint32_t* tile_flags;
    uint32_t* tile_list;
    uint32_t* ctile_list;
    uint2* ctile_range;
    uint2* cell_range;     // per-cell ranges written by the bin sort (null: not kept)
    uint32_t* ptile_list;  // occupied tiles largest first, built by the bin sort (null: not kept)
    uint32_t* counters;
    // Replay of a recorded step (bin sort only): the sort's outputs above are
    // the forward's, valid while keys_in equals the forward's keys.  The step
    // runs its sort only when *resort is set (a conditional graph node; the
    // step must be captured), and its G2P compares the new keys with the
    // recorded ones in keys_out and sets *resort when one differs.
    uint32_t* resort = nullptr;
    int sort_mode = 0;  // 0: sort keys_in; 1: keep the recorded sort; 2: keep it unless *resort
};

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int d) {
        cudaGetDevice(&prev);
        if (prev != d) cudaSetDevice(d);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

inline cudaStream_t ST(void* s) { return reinterpret_cast<cudaStream_t>(s); }

int material_to_dev(const pgmpm_material& m, MatDev& d);

}  // namespace pgmpm

struct pgmpm_solver_s {
    int device = 0;
    int num_sms = 148;
    int S = 0, M = 0;
    int64_t N = 0;
    std::vector<pgmpm_scene_desc> desc;
    std::vector<pgmpm::SceneDev> scenes;
    std::vector<pgmpm_material> mats_h;
    std::vector<int64_t> counts;
    pgmpm::PhysFlags pf{};
    int total_ct = 0, total_nt = 0;
    int key_bits = 1;
    int sort_which = 0;
    pgmpm::Tuning tune;
    bool use_graph = true;
    bool profiling = false;
    bool uploaded = false;

    // device buffers
    pgmpm::DevBuf d_scenes, d_mats, q, pay, mV, mat, user_of_phys, phys_of_user, keys, ka, va, kb, vb, sort_scratch;
    pgmpm::DevBuf grid_mp, grid_v, grid_vpre, tile_flags, tile_list, ctile_list, ctile_range, counters, staging;
    pgmpm::DevBuf bs_ccount, bs_coff, bs_tcount, bs_toff, bs_bsum, bs_slot, cell_range;  // per-step bin sort
    pgmpm::DevBuf ptile_list, tile_rank;  // largest-first occupied tile list (bin sort)
    // sparse grid (sp_cap > 0): tile pool hash (slot codes) and the per-tile
    // node-tile slots; total_ct == total_nt == sp_cap
    pgmpm::DevBuf sp_code, sp_nbr, sp_box, sp_rev;
    uint32_t sp_cap = 0;
    int sp_shift = 0;
    // consumers (pgmpm_coupling.cu): particle x and v, host staging, the
    // candidate hash grid and lists, the pair count and energy sums
    pgmpm::DevBuf cpl_xv, cpl_stage, cpl_off, cpl_idx, cpl_acc, cpl_mf;
    pgmpm_hashgrid cpl_grid = nullptr;
    float cpl_cell = 0.f;
    int64_t cpl_cap = 0;
    uint32_t* h_counters = nullptr;  // pinned

    // fused G2P -> P2G (p2g_variant 5): true while grid_mp holds the P2G of
    // the live state, done by the last step's G2P2G (the payload buffer is
    // then stale).  Cleared by pgmpm::unprime.
    bool primed = false;

    // graphs, one per step kind and [0] the call's last step / [1] a step
    // that another step of the same call follows (v, C not stored)
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t step_exec[pgmpm::STEP_KINDS][2] = {};
    cudaGraph_t step_graph[pgmpm::STEP_KINDS][2] = {};
    cudaEvent_t ev[6] = {};

    // metrics
    pgmpm_metrics met{};

    // differentiation (pgmpm_forward_checkpointed / pgmpm_backward)
    int ck_steps = 0, ck_every = 0, ck_count = 0;
    bool ck_valid = false;
    pgmpm::DevBuf ck_q, ck_keys;         // checkpoints: states (6N float4) + keys (N u32)
    int tape_slots = 0;                  // allocated tape depth (steps per segment)
    int tape_sets = 0;                   // 2 with the bin sort: a segment is replayed into one
                                         // set while the previous one is reversed from the other
    pgmpm::DevBuf tape_q, tape_keys;     // per set: (slots + 1) states and keys
    pgmpm::DevBuf tape_pay;              // payload of the replayed state (one, reused by every slot)
    pgmpm::DevBuf tape_sk, tape_ord;     // per set: slots x N sorted keys / order
    pgmpm::DevBuf tape_gv, tape_gvpre;   // per set: slots x nodes float4
    pgmpm::DevBuf tape_flags, tape_tiles, tape_ctiles, tape_crange, tape_counters;
    pgmpm::DevBuf tape_cells, tape_ptile;  // per slot: cell ranges and largest-first tile list (bin sort)
    bool tape_has_last = false;           // the tape holds the forward's last segment (no replay needed)
    bool tape_has_prev = false;           // set 1 holds the forward's second-to-last segment
    // captured tape work, each for one segment length: [0] replay + reverse
    // of a segment (set 0), [1] forward of a segment into set 0, [2], [3]
    // reverse of set 0 / 1, [4], [5] replay into set 0 / 1, [6] forward of a
    // segment into set 1
    static constexpr int kTapeGraphs = 7;
    cudaGraphExec_t tape_exec[kTapeGraphs] = {};
    int tape_exec_len[kTapeGraphs] = {-1, -1, -1, -1, -1, -1, -1};
    // Recorded forward (the bin sort, split steps): the per-step sort outputs
    // of the tape (tape_sk .. tape_ptile) hold one slot per forward step,
    // rec_keys the keys of every state, so that a replay keeps the forward's
    // sort.  Its graphs are per segment: (kind, length, first step) -> graph,
    // kind as tape_exec plus [7], a recorded live segment of the forward.
    int rec_mode = 1;           // pgmpm_set_sort_record: 0 off, 1 on, 2 on with replays that always sort
    int tape_rec = 0;           // forward steps the per-step arrays hold (0: slots only)
    bool ck_rec = false;        // the valid checkpointed forward was recorded
    pgmpm::DevBuf rec_keys;     // (tape_rec + 1) x N
    pgmpm::DevBuf rec_resort;   // one flag per tape set (a replayed key changed)
    std::map<std::tuple<int, int, int>, cudaGraphExec_t> seg_exec;
    cudaStream_t side_stream = nullptr;  // the replay that overlaps a segment's reverse
    cudaStream_t body_stream = nullptr;  // captures the bodies of conditional graph nodes
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    pgmpm::DevBuf adj_g, adj_grid_gv, adj_grid_gpm, adj_gE, adj_stage;

    pgmpm::StepBufs live_bufs() const {
        pgmpm::StepBufs b;
        b.q = q.as<float4>();
        b.q_out = q.as<float4>();
        b.pay = pf.physics == pgmpm::PHYS_MLS ? pay.as<float4>() : nullptr;
        b.keys_in = keys.as<uint32_t>();
        b.keys_out = keys.as<uint32_t>();
        b.ka = ka.as<uint32_t>();
        b.va = va.as<uint32_t>();
        b.kb = kb.as<uint32_t>();
        b.vb = vb.as<uint32_t>();
        b.which = sort_which;
        b.grid_v = grid_v.as<float4>();
        b.grid_vpre = nullptr;
        b.tile_flags = tile_flags.as<uint32_t>();
        b.tile_list = tile_list.as<uint32_t>();
        b.ctile_list = ctile_list.as<uint32_t>();
        b.ctile_range = ctile_range.as<uint2>();
        b.cell_range = cell_range.as<uint2>();
        b.ptile_list = ptile_list.as<uint32_t>();
        b.counters = counters.as<uint32_t>();
        return b;
    }

    pgmpm::View view_for(const pgmpm::StepBufs& b) const {
        pgmpm::View V;
        V.N = N;
        V.S = S;
        V.M = M;
        V.scenes = d_scenes.as<pgmpm::SceneDev>();
        V.mats = d_mats.as<pgmpm::MatDev>();
        V.q = b.q;
        V.q_out = b.q_out;
        V.pay = b.pay;
        V.pay_out = b.pay;
        V.write_vc = 1;
        V.mV = mV.as<float2>();
        V.mat = pf.multi_mat ? mat.as<int32_t>() : nullptr;
        V.keys = b.keys_out;
        V.resort = b.resort;
        V.skeys = b.which ? b.kb : b.ka;
        V.order = b.which ? b.vb : b.va;
        V.grid_mp = grid_mp.as<float4>();
        V.grid_v = b.grid_v;
        V.grid_vpre = b.grid_vpre;
        V.tile_flags = b.tile_flags;
        V.tile_list = b.tile_list;
        V.ctile_list = b.ctile_list;
        V.ctile_range = b.ctile_range;
        V.cell_range = tune.step_sort == 0 ? b.cell_range : nullptr;
        V.ptile_list = tune.step_sort == 0 ? b.ptile_list : nullptr;
        V.counters = b.counters;
        V.total_ct = total_ct;
        V.total_nt = total_nt;
        V.sp.code = sp_code.as<uint32_t>();
        V.sp.nbr = sp_nbr.as<uint4>();
        V.sp.box = sp_box.as<float4>();
        V.sp.rev = sp_rev.as<uint2>();
        V.sp.cap = sp_cap;
        V.sp.shift = sp_shift;
        return V;
    }

    pgmpm::View view() const { return view_for(live_bufs()); }

    void drop_tape_graphs() {
        for (int i = 0; i < kTapeGraphs; ++i) {
            if (tape_exec[i]) cudaGraphExecDestroy(tape_exec[i]);
            tape_exec[i] = nullptr;
            tape_exec_len[i] = -1;
        }
        for (auto& kv : seg_exec)
            if (kv.second) cudaGraphExecDestroy(kv.second);
        seg_exec.clear();
    }

    void drop_graph() {
        for (int k = 0; k < pgmpm::STEP_KINDS; ++k)
            for (int m = 0; m < 2; ++m) {
                if (step_exec[k][m]) cudaGraphExecDestroy(step_exec[k][m]);
                if (step_graph[k][m]) cudaGraphDestroy(step_graph[k][m]);
                step_exec[k][m] = nullptr;
                step_graph[k][m] = nullptr;
            }
        drop_tape_graphs();
    }

    // the live steps run the fused G2P -> P2G kernel
    bool fused() const {
        return pf.physics == pgmpm::PHYS_MLS && tune.p2g_variant == 5 && tune.step_sort == 0 && N > 0 && !sp_cap;
    }

    ~pgmpm_solver_s() {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        drop_graph();
        if (cpl_grid) pgmpm_hashgrid_destroy(cpl_grid);
        if (cap_stream) cudaStreamDestroy(cap_stream);
        if (side_stream) cudaStreamDestroy(side_stream);
        if (body_stream) cudaStreamDestroy(body_stream);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (h_counters) cudaFreeHost(h_counters);
        cudaSetDevice(prev);
    }
};

namespace pgmpm {
// Recompute the live MLS payload from the live state (after an upload, a
// material change or a state restore).
int refresh_payload(pgmpm_solver s, cudaStream_t st);
// Allocate the bin sort's buffers (8 bytes per cell, counters cleared).
int alloc_bin_sort(pgmpm_solver s);
// Enqueue one step of kind `kind` on `st` using buffers `b` (events
// ev[0..4] when timed).  write_vc = false lets an MLS step leave v and C
// (state planes 3-5) unwritten when the next step follows in the same call:
// that step reads them only through the payload (or the fused kernel does
// not read them), and the call's last step writes them.
int record_step(pgmpm_solver s, const StepBufs& b, cudaStream_t st, bool timed, bool write_vc = true,
                StepKind kind = STEP_SPLIT);
// The kind of step k of n consecutive steps that start from a state whose
// P2G is (primed) or is not already in grid_mp; drain: the last step leaves
// nothing pending (G2P instead of G2P2G).
StepKind step_kind(pgmpm_solver s, int k, int n, bool primed, bool drain);
// Drops the pending P2G of the fused path (grid_mp cleared, payload
// recomputed from the state), so that the next step starts with its own P2G.
int unprime(pgmpm_solver s, cudaStream_t st);
// Run n steps of the live state (graph, eager or profiled).
int run_steps(pgmpm_solver s, int n_steps, cudaStream_t st);
}  // namespace pgmpm
