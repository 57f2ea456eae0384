// pgmpm_diff.cu -- checkpointed differentiation of the MLS-MPM step
// (pgmpm_forward_checkpointed / pgmpm_backward) and the reference-shaped
// launcher launch_mpm_timestep_forward.
//
// Forward: the state (6 planes + keys) is copied to a checkpoint every k
// steps (CheckpointStrategy::UNIFORM of src/differentiable_mpm.h:66); the
// last segment runs straight into the tape.  Backward, segment by segment
// from the last: the segment is replayed from its checkpoint into per-step
// tape slots (state j and j+1, keys, the sort's order, tile lists, cell
// ranges, grid v and v before the walls) using the same step kernels pointed
// at the tape -- skipped for the segment the forward left in the tape --
// then the three reverse kernels run for each step from the last to the
// first.  Tape depth = k steps.  With the bin sort the tape has two sets of
// k slots: segment s - 1 is replayed into one set on a side stream while
// segment s is reversed from the other, both latency-bound and at low
// occupancy.  With the radix step sort (whose ping-pong buffers the replay
// shares) a segment's replay and reverse run in turn.  Each piece is one
// CUDA graph (captured once per segment length; checkpoint copies outside).
//
// Sort record (bin sort, split steps, when it fits): the forward also keeps
// every step's sort outputs and every state's keys, indexed by forward step,
// so a replay keeps the forward's sorts.  Its first step always can (the
// checkpoint is the forward's state bit for bit); a later step sorts again
// through a conditional graph node only when the previous replayed G2P wrote
// a key that differs from the recorded one.  These graphs are per segment.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "pgmpm_solver_impl.h"

using namespace pgmpm;

namespace {

size_t nodes_of(pgmpm_solver s) { return (size_t)s->total_nt * 64; }

// Bytes one forward step adds to the record: sorted keys, order and the next
// keys per particle, node-tile flags and list, cell-tile list and ranges,
// cell ranges and the largest-first list, counters.
size_t rec_step_bytes(pgmpm_solver s) {
    const size_t N = (size_t)std::max<int64_t>(s->N, 1);
    const size_t ct = std::max<size_t>((size_t)s->total_ct, 1);
    return 12 * N + 8 * (size_t)s->total_nt + ct * (4 + 8 + 8 * 64 + 4) + 4 * CNT_WORDS;
}

// The tape: `slots` steps per set (states, keys, grid), and per-step sort
// outputs for max(slots x sets, rec) steps (rec > 0: the recorded forward's
// steps, indexed by forward step).
int ensure_tape(pgmpm_solver s, int slots, int rec = 0) {
    const int sets = s->bs_ccount.p ? 2 : 1;  // the overlapped backward needs the bin sort
    if (s->tape_slots >= slots && s->tape_sets == sets && s->tape_q.p && s->tape_rec >= rec) return PGMPM_OK;
    const size_t N = (size_t)std::max<int64_t>(s->N, 1);
    const size_t nodes = nodes_of(s);
    const size_t gs = (size_t)slots * sets;           // grid slots over all sets
    const size_t ss = std::max(gs, (size_t)rec);      // per-step sort slots
    s->tape_slots = 0;
    s->tape_sets = 0;
    s->tape_rec = 0;
    s->tape_has_last = false;
    s->tape_has_prev = false;
    s->ck_rec = false;      // the record goes with the old tape (the checkpoints stay)
    s->drop_tape_graphs();  // they hold the old tape's addresses
    CK(s->tape_q.alloc(sizeof(float4) * 6 * N * (slots + 1) * sets));
    CK(s->tape_keys.alloc(sizeof(uint32_t) * N * (slots + 1) * sets));
    if (s->pf.physics == PHYS_MLS) CK(s->tape_pay.alloc(sizeof(float4) * 4 * N));
    CK(s->tape_sk.alloc(sizeof(uint32_t) * N * ss));
    CK(s->tape_ord.alloc(sizeof(uint32_t) * N * ss));
    CK(s->tape_gv.alloc(sizeof(float4) * nodes * gs));
    CK(s->tape_gvpre.alloc(sizeof(float4) * nodes * gs));
    CK(s->tape_flags.alloc(sizeof(uint32_t) * (size_t)s->total_nt * ss));
    CK(s->tape_tiles.alloc(sizeof(uint32_t) * (size_t)s->total_nt * ss));
    CK(s->tape_ctiles.alloc(sizeof(uint32_t) * (size_t)s->total_ct * ss));
    CK(s->tape_crange.alloc(sizeof(uint2) * (size_t)s->total_ct * ss));
    CK(s->tape_counters.alloc(sizeof(uint32_t) * CNT_WORDS * ss));
    CK(cudaMemset(s->tape_counters.p, 0, s->tape_counters.bytes));
    if (s->bs_ccount.p) {  // the bin sort is available: per-slot cell tables
        CK(s->tape_cells.alloc(sizeof(uint2) * 64 * std::max<size_t>((size_t)s->total_ct, 1) * ss));
        CK(s->tape_ptile.alloc(sizeof(uint32_t) * std::max<size_t>((size_t)s->total_ct, 1) * ss));
    }
    if (rec) {
        CK(s->rec_keys.alloc(sizeof(uint32_t) * N * ((size_t)rec + 1)));
        // [0], [1]: a replayed key changed (per tape set); [2]: replayed steps
        // that sorted again, kept across tapes
        if (!s->rec_resort.p) {
            CK(s->rec_resort.alloc(sizeof(uint32_t) * 4));
            CK(cudaMemset(s->rec_resort.p, 0, s->rec_resort.bytes));
        }
        CK(cudaMemset(s->rec_resort.p, 0, 2 * sizeof(uint32_t)));
    } else {
        s->rec_keys.release();
    }
    s->tape_slots = slots;
    s->tape_sets = sets;
    s->tape_rec = rec;
    return PGMPM_OK;
}

// Points the sort outputs and counters of b at per-step slot js.
void set_sort_slot(pgmpm_solver s, StepBufs& b, size_t js) {
    const size_t N = (size_t)std::max<int64_t>(s->N, 1);
    uint32_t* sk = s->tape_sk.as<uint32_t>() + N * js;
    uint32_t* so = s->tape_ord.as<uint32_t>() + N * js;
    // the sort's last pass must land in the slot: pair a when which == 0
    b.which = s->sort_which;
    if (b.which == 0) {
        b.ka = sk;
        b.va = so;
        b.kb = s->kb.as<uint32_t>();
        b.vb = s->vb.as<uint32_t>();
    } else {
        b.ka = s->ka.as<uint32_t>();
        b.va = s->va.as<uint32_t>();
        b.kb = sk;
        b.vb = so;
    }
    b.tile_flags = s->tape_flags.as<uint32_t>() + (size_t)s->total_nt * js;
    b.tile_list = s->tape_tiles.as<uint32_t>() + (size_t)s->total_nt * js;
    b.ctile_list = s->tape_ctiles.as<uint32_t>() + (size_t)s->total_ct * js;
    b.ctile_range = s->tape_crange.as<uint2>() + (size_t)s->total_ct * js;
    const size_t ct = std::max<size_t>((size_t)s->total_ct, 1);
    b.cell_range = s->tape_cells.p ? s->tape_cells.as<uint2>() + ct * 64 * js : nullptr;
    b.ptile_list = s->tape_ptile.p ? s->tape_ptile.as<uint32_t>() + ct * js : nullptr;
    b.counters = s->tape_counters.as<uint32_t>() + CNT_WORDS * js;
}

// Buffers of slot j of tape set t: the step from state j to state j+1.
// States of set t are t (slots + 1) + j; grid data of slot j is slot
// t slots + j.  Without a record (g < 0) the sort outputs and keys are the
// slot's too; with one, they are those of forward step g (keys g and g + 1).
StepBufs tape_bufs(pgmpm_solver s, int j, int t = 0, int g = -1) {
    const size_t N = (size_t)std::max<int64_t>(s->N, 1);
    const size_t nodes = nodes_of(s);
    const size_t qs = (size_t)t * (s->tape_slots + 1) + j;  // state j of set t
    const size_t jg = (size_t)t * s->tape_slots + j;        // grid slot of set t
    StepBufs b;
    b.q = s->tape_q.as<float4>() + 6 * N * qs;
    b.q_out = s->tape_q.as<float4>() + 6 * N * (qs + 1);
    b.pay = s->pf.physics == PHYS_MLS ? s->tape_pay.as<float4>() : nullptr;
    if (g >= 0) {
        b.keys_in = s->rec_keys.as<uint32_t>() + N * (size_t)g;
        b.keys_out = s->rec_keys.as<uint32_t>() + N * ((size_t)g + 1);
    } else {
        b.keys_in = s->tape_keys.as<uint32_t>() + N * qs;
        b.keys_out = s->tape_keys.as<uint32_t>() + N * (qs + 1);
    }
    set_sort_slot(s, b, g >= 0 ? (size_t)g : jg);
    b.grid_v = s->tape_gv.as<float4>() + nodes * jg;
    b.grid_vpre = s->tape_gvpre.as<float4>() + nodes * jg;
    return b;
}

// Runs body(stream) under capture on the solver's capture stream and keeps
// the instantiated graph: in tape_exec[kind] (tagged with len) when base < 0,
// else in seg_exec under (kind, len, base).  ex receives the graph.
template <class Body>
int tape_graph(pgmpm_solver s, int kind, int len, int base, cudaGraphExec_t& ex, Body&& body) {
    cudaGraphExec_t* slot;
    if (base >= 0 && s->seg_exec.size() >= 4096) s->drop_tape_graphs();  // bound the per-segment cache
    if (base < 0) {
        if (s->tape_exec[kind] && s->tape_exec_len[kind] != len) {
            cudaGraphExecDestroy(s->tape_exec[kind]);
            s->tape_exec[kind] = nullptr;
            s->tape_exec_len[kind] = -1;
        }
        slot = &s->tape_exec[kind];
    } else {
        slot = &s->seg_exec[std::make_tuple(kind, len, base)];
    }
    if (*slot) {
        ex = *slot;
        return PGMPM_OK;
    }
    CK(cudaStreamBeginCapture(s->cap_stream, cudaStreamCaptureModeThreadLocal));
    int rc = body(s->cap_stream);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->cap_stream, &g);
    if (rc != PGMPM_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    CK(e);
    e = cudaGraphInstantiate(slot, g, 0);
    cudaGraphDestroy(g);
    CK(e);
    if (base < 0) s->tape_exec_len[kind] = len;
    ex = *slot;
    return PGMPM_OK;
}

// Forward of slots 0..len-1 of tape set t (state 0 and its payload in place,
// grid_mp clear).  With the fused kernel each slot's G2P2G does the next
// slot's P2G; the last slot runs the split G2P, so nothing is left pending
// in grid_mp and the payload buffer holds the final state's payload.
// g0 >= 0: the slots are forward steps g0.. of the record; replay: they were
// recorded already, so each step keeps its recorded sort (the first always,
// the others unless the previous step's G2P changed a key).
int record_tape_forward(pgmpm_solver s, int len, cudaStream_t st, int t = 0, int g0 = -1, bool replay = false) {
    for (int j = 0; j < len; ++j) {
        StepBufs b = tape_bufs(s, j, t, g0 < 0 ? -1 : g0 + j);
        if (replay && g0 >= 0) {
            b.resort = s->rec_resort.as<uint32_t>() + t;
            b.sort_mode = j == 0 ? 1 : 2;
        }
        int rc = record_step(s, b, st, false, true, step_kind(s, j, len, false, true));
        if (rc) return rc;
    }
    return PGMPM_OK;
}

// Reverse kernels of slots len-1 .. 0 of tape set t.
int record_tape_reverse(pgmpm_solver s, const AdjView& A0, int len, cudaStream_t st, int t = 0, int g0 = -1) {
    AdjView A = A0;
    for (int j = len - 1; j >= 0; --j) {
        StepBufs b = tape_bufs(s, j, t, g0 < 0 ? -1 : g0 + j);
        View V = s->view_for(b);
        V.grid_mp = A.grid_gv;  // scatter target of the G2P reverse
        A.q_next = b.q_out;
        // the slot's P2G work cursor is zero: the grid update of the slot's
        // forward step cleared it after P2G (and a previous reverse's grid
        // adjoint after its scatter)
        CK(launch_adj_scatter(V, A, s->pf, s->tune, s->num_sms, st));
        CK(launch_adj_grid(V, A, s->tune, s->num_sms, st));
        CK(launch_adj_gather(V, A, s->pf, s->tune, st));
    }
    return PGMPM_OK;
}

// Steps g0 .. g0 + len - 1 of a recorded forward on the live state: each
// step's sort writes its slot of the record and its G2P the next state's
// keys; the segment's last step stores v and C (the checkpoint that follows
// copies the whole state).
int run_recorded(pgmpm_solver s, int g0, int len, cudaStream_t st) {
    cudaGraphExec_t ex = nullptr;
    int rc = tape_graph(s, 7, len, g0, ex, [&](cudaStream_t c) -> int {
        for (int j = 0; j < len; ++j) {
            StepBufs b = s->live_bufs();
            const size_t N = (size_t)std::max<int64_t>(s->N, 1);
            b.keys_in = s->rec_keys.as<uint32_t>() + N * (size_t)(g0 + j);
            b.keys_out = s->rec_keys.as<uint32_t>() + N * (size_t)(g0 + j + 1);
            set_sort_slot(s, b, (size_t)(g0 + j));
            int r = record_step(s, b, c, false, j + 1 == len, STEP_SPLIT);
            if (r) return r;
        }
        CK(launch_merge_flags(s->tape_counters.as<uint32_t>() + (size_t)CNT_WORDS * g0, len,
                              s->counters.as<uint32_t>(), c));
        return PGMPM_OK;
    });
    if (rc) return rc;
    CK(cudaGraphLaunch(ex, st));
    s->met.total_steps += len;
    return PGMPM_OK;
}

// Backward over all segments with two tape sets: while segment seg is
// reversed from set `cur` on st, segment seg - 1 is replayed into the other
// set on the side stream (it starts after everything before it on st, so the
// set's previous reverse is done; st waits for it before the next reverse).
// The replay uses the payload buffer, the bin sort's scratch and the P2G
// accumulator, which no reverse kernel touches.
int backward_overlapped(pgmpm_solver s, const AdjView& A, cudaStream_t st) {
    const size_t Nz = (size_t)std::max<int64_t>(s->N, 1);
    const int k = s->ck_every;
    if (!s->side_stream) CK(cudaStreamCreateWithFlags(&s->side_stream, cudaStreamNonBlocking));
    if (!s->ev_fork) CK(cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming));
    if (!s->ev_join) CK(cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming));
    cudaStream_t side = s->side_stream;
    auto seg_len = [&](int seg) { return std::min(k, s->ck_steps - seg * k); };
    // with a recorded forward, segment seg's steps are forward steps
    // seg k .. and keep their recorded sorts (graphs per segment).  Kernel
    // variants changed to the fused step since the forward: replay every
    // segment with its own sorts (the tape's segments hold the record's).
    const bool rec = s->ck_rec && !s->fused();
    if (s->ck_rec && !rec) {
        s->tape_has_last = false;
        s->tape_has_prev = false;
        s->ck_rec = false;
    }
    auto replay = [&](int seg, int t, cudaStream_t cs) -> int {
        const int len = seg_len(seg);
        const int g0 = rec ? seg * k : -1;
        const StepBufs b0 = tape_bufs(s, 0, t, g0);
        CK(cudaMemcpyAsync(b0.q, s->ck_q.as<float4>() + 6 * Nz * seg, sizeof(float4) * 6 * Nz,
                           cudaMemcpyDeviceToDevice, cs));
        CK(cudaMemcpyAsync(b0.keys_in, s->ck_keys.as<uint32_t>() + Nz * seg, sizeof(uint32_t) * Nz,
                           cudaMemcpyDeviceToDevice, cs));
        cudaGraphExec_t ex = nullptr;
        int rc = tape_graph(s, 4 + t, len, g0, ex, [&](cudaStream_t c) -> int {
            if (rec) CK(cudaMemsetAsync(s->rec_resort.as<uint32_t>() + t, 0, sizeof(uint32_t), c));
            CK(launch_payload(s->view_for(b0), s->pf, c));
            return record_tape_forward(s, len, c, t, g0, true);
        });
        if (rc) return rc;
        CK(cudaGraphLaunch(ex, cs));
        return PGMPM_OK;
    };
    auto reverse = [&](int seg, int t, cudaStream_t cs) -> int {
        const int len = seg_len(seg);
        const int g0 = rec ? seg * k : -1;
        cudaGraphExec_t ex = nullptr;
        int rc = tape_graph(s, 2 + t, len, g0, ex,
                            [&](cudaStream_t c) { return record_tape_reverse(s, A, len, c, t, g0); });
        if (rc) return rc;
        CK(cudaGraphLaunch(ex, cs));
        return PGMPM_OK;
    };
    const int last = s->ck_count - 1;
    int rc = PGMPM_OK;
    if (!s->tape_has_last) {  // the forward did not leave the last segment in set 0
        rc = replay(last, 0, st);
        if (rc) return rc;
    }
    s->tape_has_last = false;  // the replays below overwrite it
    // the forward left the second-to-last segment in set 1: no replay of it
    const bool have_prev = s->tape_has_prev && last > 0;
    s->tape_has_prev = false;
    int cur = 0;
    for (int seg = last; seg >= 0; --seg) {
        const bool fork = seg > 0 && !(have_prev && seg == last);
        if (fork) {
            CK(cudaEventRecord(s->ev_fork, st));
            CK(cudaStreamWaitEvent(side, s->ev_fork, 0));
            rc = replay(seg - 1, 1 - cur, side);
            if (rc) return rc;
        }
        rc = reverse(seg, cur, st);
        if (rc) return rc;
        if (fork) {
            CK(cudaEventRecord(s->ev_join, side));
            CK(cudaStreamWaitEvent(st, s->ev_join, 0));
        }
        cur = 1 - cur;
    }
    return PGMPM_OK;
}

// The adjoint covers every material model (the von Mises cap and the fluid
// viscosity included, kirchhoff_adjoint / add_viscous_adjoint).
int check_differentiable(pgmpm_solver) { return PGMPM_OK; }

}  // namespace

extern "C" {

int pgmpm_forward_checkpointed(pgmpm_solver s, int32_t n_steps, int32_t checkpoint_every, void* stream) {
    if (!s || n_steps < 1 || checkpoint_every < 1) return fail(PGMPM_ERR_ARG, "need n_steps >= 1, checkpoint_every >= 1");
    if (s->pf.physics != PHYS_MLS) return fail(PGMPM_ERR_UNSUPPORTED, "differentiation needs PGMPM_PHYSICS_MLS");
    if (s->sp_cap) return fail(PGMPM_ERR_UNSUPPORTED, "differentiation needs a dense grid");
    if (!s->uploaded) return fail(PGMPM_ERR_STATE, "no particles uploaded");
    if (int rc0 = check_differentiable(s)) return rc0;
    DeviceGuard dg(s->device);
    cudaStream_t st = ST(stream);
    const int k = std::min(checkpoint_every, n_steps);
    const int nseg = (n_steps + k - 1) / k;
    const size_t N = (size_t)std::max<int64_t>(s->N, 1);
    CK(s->ck_q.ensure(sizeof(float4) * 6 * N * nseg));
    CK(s->ck_keys.ensure(sizeof(uint32_t) * N * nseg));
    // Record the forward (every step's sort and keys) when the steps are
    // split bin-sorted steps and the tape with the record is modest: at most
    // 1/16 of the device's memory, with a quarter of it still free after it
    // (other solvers of the process keep room for their tapes).  The
    // backward's replays then keep the forward's sorts.  Otherwise (or when
    // its allocation fails) the tape is the plain one and the replays sort.
    int rec = 0;
    if (s->rec_mode && s->tune.step_sort == 0 && s->bs_ccount.p && !s->fused() && s->N > 0) {
        size_t fr = 0, tot = 0;
        const size_t tape = (size_t)2 * (k + 1) * N * (96 + 4) + 64 * N + (size_t)2 * k * nodes_of(s) * 32;
        const size_t need = tape + rec_step_bytes(s) * (size_t)n_steps;
        if (s->tape_rec >= n_steps && s->tape_slots >= k)
            rec = n_steps;
        else if (cudaMemGetInfo(&fr, &tot) == cudaSuccess && need <= tot / 16 && fr >= need + tot / 4)
            rec = n_steps;
    }
    int rc = ensure_tape(s, k, rec);
    if (rc == PGMPM_ERR_OOM && rec) {
        cudaGetLastError();  // clear the failed allocation
        rec = 0;
        rc = ensure_tape(s, k, 0);
    }
    if (rc) return rc;
    s->ck_valid = false;
    s->ck_rec = false;
    s->tape_has_last = false;
    s->tape_has_prev = false;
    rc = unprime(s, st);  // checkpoints and replays start from the state alone
    if (rc) return rc;
    // Runs a segment in the slots of tape set t, so that the backward does
    // not replay it, then hands the final state back to the live buffers
    // (the tape starts from the state and its payload, with grid_mp clear).
    // g0 >= 0: the recorded forward's steps g0 .. (the record's keys g0 are
    // the state's already)
    auto run_in_tape = [&](int len, int t, int g0) -> int {
        int r = unprime(s, st);
        if (r) return r;
        const StepBufs first = tape_bufs(s, 0, t, g0);
        CK(cudaMemcpyAsync(first.q, s->q.p, sizeof(float4) * 6 * N, cudaMemcpyDeviceToDevice, st));
        if (g0 < 0)
            CK(cudaMemcpyAsync(first.keys_in, s->keys.p, sizeof(uint32_t) * N, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(s->tape_pay.p, s->pay.p, sizeof(float4) * 4 * N, cudaMemcpyDeviceToDevice, st));
        const int kind = t == 0 ? 1 : 6;
        cudaGraphExec_t ex = nullptr;
        r = tape_graph(s, kind, len, g0, ex, [&](cudaStream_t cs) { return record_tape_forward(s, len, cs, t, g0); });
        if (r) return r;
        CK(cudaGraphLaunch(ex, st));
        const StepBufs last = tape_bufs(s, len - 1, t, g0);
        CK(cudaMemcpyAsync(s->q.p, last.q_out, sizeof(float4) * 6 * N, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(s->keys.p, last.keys_out, sizeof(uint32_t) * N, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(s->pay.p, s->tape_pay.p, sizeof(float4) * 4 * N, cudaMemcpyDeviceToDevice, st));
        // what a live step leaves for pgmpm_download_grid and the metrics
        CK(cudaMemcpyAsync(s->grid_v.p, last.grid_v, sizeof(float4) * nodes_of(s), cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(s->tile_flags.p, last.tile_flags, sizeof(uint32_t) * (size_t)s->total_nt,
                           cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(s->counters.as<uint32_t>() + CNT_ACTIVE, last.counters + CNT_ACTIVE, 2 * sizeof(uint32_t),
                           cudaMemcpyDeviceToDevice, st));
        CK(launch_merge_flags(s->tape_counters.as<uint32_t>() + (size_t)CNT_WORDS * (g0 >= 0 ? g0 : s->tape_slots * t),
                              len, s->counters.as<uint32_t>(), st));
        s->met.total_steps += len;
        return PGMPM_OK;
    };
    // with two tape sets (the overlapped backward) the second-to-last
    // segment runs in set 1 as well, so the backward replays one segment less
    const bool prev_in_tape = s->tape_sets == 2 && s->tune.step_sort == 0 && nseg >= 2;
    // recorded: the live keys stay as they are until the last segment; the
    // steps read and write the record's
    uint32_t* rk = rec ? s->rec_keys.as<uint32_t>() : nullptr;
    if (rec) CK(cudaMemcpyAsync(rk, s->keys.p, sizeof(uint32_t) * N, cudaMemcpyDeviceToDevice, st));
    for (int seg = 0; seg < nseg; ++seg) {
        CK(cudaMemcpyAsync(s->ck_q.as<float4>() + 6 * N * seg, s->q.p, sizeof(float4) * 6 * N,
                           cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(s->ck_keys.as<uint32_t>() + N * seg, rec ? rk + N * (size_t)seg * k : s->keys.as<uint32_t>(),
                           sizeof(uint32_t) * N, cudaMemcpyDeviceToDevice, st));
        const int len = std::min(k, n_steps - seg * k);
        if (s->N == 0 || seg + 2 < nseg || (seg + 2 == nseg && !prev_in_tape)) {
            rc = rec ? run_recorded(s, seg * k, len, st) : run_steps(s, len, st);
            if (rc) return rc;
            continue;
        }
        const int t = seg + 1 == nseg ? 0 : 1;
        rc = run_in_tape(len, t, rec ? seg * k : -1);
        if (rc) return rc;
        if (t == 0)
            s->tape_has_last = true;
        else
            s->tape_has_prev = true;
    }
    s->ck_steps = n_steps;
    s->ck_every = k;
    s->ck_count = nseg;
    s->ck_valid = true;
    s->ck_rec = rec > 0;
    return PGMPM_OK;
}

int pgmpm_backward(pgmpm_solver s, const float* gx_out, const float* gv_out, const float* gC_out, const float* gF_out,
                   float* gx_in, float* gv_in, float* gC_in, float* gF_in, float* gE, int32_t ptr_kind, void* stream) {
    if (!s) return fail(PGMPM_ERR_ARG, "null solver");
    if (!s->ck_valid) return fail(PGMPM_ERR_STATE, "call pgmpm_forward_checkpointed first");
    if (int rc0 = check_differentiable(s)) return rc0;
    if (ptr_kind != PGMPM_PTR_HOST && ptr_kind != PGMPM_PTR_DEVICE) return fail(PGMPM_ERR_ARG, "bad ptr_kind");
    DeviceGuard dg(s->device);
    cudaStream_t st = ST(stream);
    const int64_t N = s->N;
    const size_t Nz = (size_t)std::max<int64_t>(N, 1);
    const int M = s->M;
    int rc = ensure_tape(s, s->ck_every);
    if (rc) return rc;
    // the replays accumulate their P2G in grid_mp: drop a pending fused P2G
    // of the live state (recomputed by its next step)
    rc = unprime(s, st);
    if (rc) return rc;
    CK(s->adj_g.ensure(sizeof(float4) * 6 * Nz));
    CK(s->adj_grid_gv.ensure(sizeof(float4) * nodes_of(s)));
    CK(s->adj_grid_gpm.ensure(sizeof(float4) * nodes_of(s)));
    CK(s->adj_gE.ensure(sizeof(float) * M));
    CK(cudaMemsetAsync(s->adj_grid_gv.p, 0, s->adj_grid_gv.bytes, st));
    CK(cudaMemsetAsync(s->adj_gE.p, 0, sizeof(float) * M, st));
    // output adjoint (upload order) -> physical planes
    const float *dx = gx_out, *dv = gv_out, *dC = gC_out, *dF = gF_out;
    if (ptr_kind == PGMPM_PTR_HOST && N > 0) {
        CK(s->adj_stage.ensure(sizeof(float) * 24 * Nz));
        float* b = s->adj_stage.as<float>();
        float *sx = b, *sv = b + 3 * N, *sC = b + 6 * N, *sF = b + 15 * N;
        if (gx_out) CK(cudaMemcpyAsync(sx, gx_out, sizeof(float) * 3 * N, cudaMemcpyHostToDevice, st));
        if (gv_out) CK(cudaMemcpyAsync(sv, gv_out, sizeof(float) * 3 * N, cudaMemcpyHostToDevice, st));
        if (gC_out) CK(cudaMemcpyAsync(sC, gC_out, sizeof(float) * 9 * N, cudaMemcpyHostToDevice, st));
        if (gF_out) CK(cudaMemcpyAsync(sF, gF_out, sizeof(float) * 9 * N, cudaMemcpyHostToDevice, st));
        dx = gx_out ? sx : nullptr;
        dv = gv_out ? sv : nullptr;
        dC = gC_out ? sC : nullptr;
        dF = gF_out ? sF : nullptr;
    }
    CK(launch_state_to_planes(dx, dv, dC, dF, s->user_of_phys.as<uint32_t>(), s->adj_g.as<float4>(), N, st));
    AdjView A;
    A.g = s->adj_g.as<float4>();
    A.grid_gv = s->adj_grid_gv.as<float4>();
    A.grid_gpm = s->adj_grid_gpm.as<float4>();
    A.gE = s->adj_gE.as<float>();
    const int k = s->ck_every;
    const bool overlapped = s->tape_sets == 2 && s->tune.step_sort == 0;
    if (s->ck_rec && !overlapped) {
        // the step sort changed to the radix sort since a recorded forward:
        // the tape's segments hold the record's sorts, which the one-set
        // path does not index, so every segment is replayed with its sorts
        s->tape_has_last = false;
        s->tape_has_prev = false;
        s->ck_rec = false;
    }
    if (overlapped && N > 0) {
        rc = backward_overlapped(s, A, st);
        if (rc) return rc;
    }
    for (int seg = s->ck_count - 1; seg >= 0 && N > 0 && !overlapped; --seg) {
        const int len = std::min(k, s->ck_steps - seg * k);
        if (seg == s->ck_count - 1 && s->tape_has_last) {
            // the forward left this segment in the tape
            cudaGraphExec_t ex = nullptr;
            rc = tape_graph(s, 2, len, -1, ex, [&](cudaStream_t cs) { return record_tape_reverse(s, A, len, cs); });
            if (rc) return rc;
            CK(cudaGraphLaunch(ex, st));
            s->tape_has_last = false;  // the replays below overwrite it
            continue;
        }
        s->tape_has_last = false;
        CK(cudaMemcpyAsync(s->tape_q.p, s->ck_q.as<float4>() + 6 * Nz * seg, sizeof(float4) * 6 * Nz,
                           cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(s->tape_keys.p, s->ck_keys.as<uint32_t>() + Nz * seg, sizeof(uint32_t) * Nz,
                           cudaMemcpyDeviceToDevice, st));
        cudaGraphExec_t ex = nullptr;
        rc = tape_graph(s, 0, len, -1, ex, [&](cudaStream_t cs) -> int {
            CK(launch_payload(s->view_for(tape_bufs(s, 0)), s->pf, cs));
            int r = record_tape_forward(s, len, cs);
            if (r) return r;
            return record_tape_reverse(s, A, len, cs);
        });
        if (rc) return rc;
        CK(cudaGraphLaunch(ex, st));
    }
    CK(launch_merge_flags(s->tape_counters.as<uint32_t>(), std::max(s->tape_slots * s->tape_sets, s->tape_rec),
                          s->counters.as<uint32_t>(), st));
    // physical planes -> caller's arrays (upload order)
    if (ptr_kind == PGMPM_PTR_DEVICE) {
        CK(launch_planes_to_state(A.g, s->phys_of_user.as<uint32_t>(), gx_in, gv_in, gC_in, gF_in, N, st));
        if (gE) CK(cudaMemcpyAsync(gE, A.gE, sizeof(float) * M, cudaMemcpyDeviceToDevice, st));
        return PGMPM_OK;
    }
    CK(s->adj_stage.ensure(sizeof(float) * 24 * Nz));
    float* b = s->adj_stage.as<float>();
    float *sx = b, *sv = b + 3 * N, *sC = b + 6 * N, *sF = b + 15 * N;
    CK(launch_planes_to_state(A.g, s->phys_of_user.as<uint32_t>(), gx_in ? sx : nullptr, gv_in ? sv : nullptr,
                              gC_in ? sC : nullptr, gF_in ? sF : nullptr, N, st));
    if (gx_in && N) CK(cudaMemcpyAsync(gx_in, sx, sizeof(float) * 3 * N, cudaMemcpyDeviceToHost, st));
    if (gv_in && N) CK(cudaMemcpyAsync(gv_in, sv, sizeof(float) * 3 * N, cudaMemcpyDeviceToHost, st));
    if (gC_in && N) CK(cudaMemcpyAsync(gC_in, sC, sizeof(float) * 9 * N, cudaMemcpyDeviceToHost, st));
    if (gF_in && N) CK(cudaMemcpyAsync(gF_in, sF, sizeof(float) * 9 * N, cudaMemcpyDeviceToHost, st));
    if (gE) CK(cudaMemcpyAsync(gE, A.gE, sizeof(float) * M, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return PGMPM_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------
// launch_mpm_timestep_forward: src/pytorch_autograd.cu:371-382 shape.
// One REF_COMPAT step on the unit cube with a grid_resolution^3 grid.  A
// solver per (device, particle count, resolution) is kept for the process so
// repeated calls reuse their device buffers.
namespace {
struct LaunchEntry {
    pgmpm_solver s = nullptr;
    pgmpm::DevBuf masses;  // the last forward's masses: the backward's signature carries none
};
std::mutex g_launch_mu;
std::map<std::tuple<int, int, int>, LaunchEntry> g_launch_solvers;

// per-call dt into the scene table (the dt word only: gravity arrives as a
// device pointer and is copied there by the forward)
bool launch_set_dt(pgmpm_solver s, float dt, cudaStream_t st, const char* who) {
    if (s->scenes[0].dt == dt) return true;
    s->scenes[0].dt = dt;
    if (cudaMemcpyAsync(&s->d_scenes.as<SceneDev>()[0].dt, &s->scenes[0].dt, sizeof(float), cudaMemcpyHostToDevice,
                        st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        fail(PGMPM_ERR_CUDA, "%s: dt update failed", who);
        return false;
    }
    return true;
}
}  // namespace

extern "C" void launch_mpm_timestep_forward(float* positions, float* velocities, const float* masses,
                                            int num_particles, int grid_resolution, float dt, const float* gravity,
                                            void* stream) {
    if (num_particles < 0 || grid_resolution < 4 || !(dt > 0.f) || (num_particles > 0 && (!positions || !velocities || !masses))) {
        fail(PGMPM_ERR_ARG, "launch_mpm_timestep_forward: invalid arguments");
        return;
    }
    if (num_particles == 0) return;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaStream_t st = ST(stream);
    pgmpm_solver s = nullptr;
    LaunchEntry* entry = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_launch_mu);
        auto key = std::make_tuple(dev, num_particles, grid_resolution);
        auto it = g_launch_solvers.find(key);
        if (it == g_launch_solvers.end()) {
            pgmpm_scene_desc d{};
            d.n[0] = d.n[1] = d.n[2] = grid_resolution;
            d.physics = PGMPM_PHYSICS_REF_COMPAT;
            d.boundary = PGMPM_BC_NONE;
            d.dx = 1.0f / (float)grid_resolution;
            d.dt = dt;
            const int64_t cnt = num_particles;
            pgmpm_material mat{PGMPM_MAT_ELASTIC, PGMPM_MODEL_FIXED_COROTATED, 1e6f, 0.3f, 1000.f};
            if (pgmpm_create(&d, 1, &cnt, &mat, 1, dev, &s) != PGMPM_OK) return;
            entry = &g_launch_solvers[key];
            entry->s = s;
        } else {
            entry = &it->second;
            s = entry->s;
        }
    }
    // per-call dt and gravity (device pointer) into the scene table
    if (!launch_set_dt(s, dt, st, "launch_mpm_timestep_forward")) return;
    if (gravity) {
        if (cudaMemcpyAsync(&s->d_scenes.as<SceneDev>()[0].gravity[0], gravity, 3 * sizeof(float),
                            cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
            fail(PGMPM_ERR_CUDA, "launch_mpm_timestep_forward: gravity copy failed");
            return;
        }
    }
    std::vector<float> ones;  // volumes are not used by the REF_COMPAT physics
    if (pgmpm_upload(s, positions, velocities, nullptr, nullptr, masses, nullptr, nullptr, PGMPM_PTR_DEVICE, stream))
        return;
    if (pgmpm_step(s, 1, stream)) return;
    if (pgmpm_download(s, positions, velocities, nullptr, nullptr, PGMPM_PTR_DEVICE, stream)) return;
    // kept for launch_mpm_timestep_backward
    if (entry->masses.ensure(sizeof(float) * (size_t)num_particles) != cudaSuccess ||
        cudaMemcpyAsync(entry->masses.p, masses, sizeof(float) * (size_t)num_particles, cudaMemcpyDeviceToDevice,
                        st) != cudaSuccess)
        fail(PGMPM_ERR_CUDA, "launch_mpm_timestep_forward: keeping the masses failed");
}

// launch_mpm_timestep_backward: src/pytorch_autograd.cu:384-402 shape.  The
// reverse of the step launch_mpm_timestep_forward runs, from that step's
// inputs (saved_positions, saved_velocities); masses and gravity are those of
// the last forward call with the same device, particle count and resolution.
// The forward step is recomputed (its grid is the linearisation point), then
// the three reverse kernels of pgmpm_ref_adjoint.cu run.  grad_gravity is
// added to, as the reference's kernel does (zero it first); grad_masses may
// be NULL.
extern "C" void launch_mpm_timestep_backward(const float* grad_positions, const float* grad_velocities,
                                             float* grad_input_positions, float* grad_input_velocities,
                                             float* grad_masses, float* grad_gravity, const float* saved_positions,
                                             const float* saved_velocities, int num_particles, int grid_resolution,
                                             float dt, void* stream) {
    if (num_particles < 0 || grid_resolution < 4 || !(dt > 0.f) ||
        (num_particles > 0 && (!grad_positions || !grad_velocities || !grad_input_positions ||
                               !grad_input_velocities || !saved_positions || !saved_velocities))) {
        fail(PGMPM_ERR_ARG, "launch_mpm_timestep_backward: invalid arguments");
        return;
    }
    if (num_particles == 0) return;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaStream_t st = ST(stream);
    pgmpm_solver s = nullptr;
    const float* masses = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_launch_mu);
        auto it = g_launch_solvers.find(std::make_tuple(dev, num_particles, grid_resolution));
        if (it == g_launch_solvers.end() || !it->second.masses.p) {
            fail(PGMPM_ERR_STATE,
                 "launch_mpm_timestep_backward: no launch_mpm_timestep_forward call with this device, particle "
                 "count and resolution");
            return;
        }
        s = it->second.s;
        masses = it->second.masses.as<float>();
    }
    if (!launch_set_dt(s, dt, st, "launch_mpm_timestep_backward")) return;
    if (pgmpm_upload(s, saved_positions, saved_velocities, nullptr, nullptr, masses, nullptr, nullptr,
                     PGMPM_PTR_DEVICE, stream))
        return;
    if (pgmpm_step(s, 1, stream)) return;
    const size_t gbytes = sizeof(float4) * nodes_of(s);
    if (s->adj_grid_gv.ensure(gbytes) != cudaSuccess || cudaMemsetAsync(s->adj_grid_gv.p, 0, gbytes, st) != cudaSuccess) {
        fail(PGMPM_ERR_CUDA, "launch_mpm_timestep_backward: grid adjoint buffer");
        return;
    }
    if (launch_ref_adjoint(s->view(), saved_positions, saved_velocities, masses, grad_positions, grad_velocities,
                           s->adj_grid_gv.as<float4>(), grad_input_positions, grad_input_velocities, grad_masses,
                           grad_gravity, s->num_sms, st) != cudaSuccess)
        fail(PGMPM_ERR_CUDA, "launch_mpm_timestep_backward: %s", cudaGetErrorString(cudaGetLastError()));
}
