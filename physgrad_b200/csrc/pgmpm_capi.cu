// pgmpm_capi.cu -- the C-ABI of include/pgmpm.h: solver handle, device
// memory, step driver (CUDA graph per step), metrics and autotuner.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/pgmpm.h"
#include "pgmpm_internal.h"

#include "pgmpm_solver_impl.h"

using namespace pgmpm;

namespace {
thread_local std::string g_err;
}  // namespace

// Sets the message returned by pgmpm_last_error() (shared with the other
// translation units of the library) and returns code.
int pgmpm_set_error(int code, const char* msg) {
    g_err = msg ? msg : "";
    return code;
}

namespace pgmpm {

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int material_to_dev(const pgmpm_material& m, MatDev& d) {
    int model;
    if (m.type == PGMPM_MAT_FLUID) {
        if (m.model != PGMPM_MODEL_EOS_FLUID)
            return fail(PGMPM_ERR_UNSUPPORTED, "FLUID material requires PGMPM_MODEL_EOS_FLUID");
        if (!(m.viscosity >= 0.f) || !std::isfinite(m.viscosity))
            return fail(PGMPM_ERR_ARG, "FLUID viscosity must be finite and >= 0");
        model = MODEL_EOS;
    } else if (m.type == PGMPM_MAT_ELASTIC || m.type == PGMPM_MAT_JELLY) {
        if (m.model != PGMPM_MODEL_FIXED_COROTATED && m.model != PGMPM_MODEL_NEO_HOOKEAN)
            return fail(PGMPM_ERR_UNSUPPORTED, "elastic material requires FIXED_COROTATED or NEO_HOOKEAN");
        model = m.model == PGMPM_MODEL_FIXED_COROTATED ? MODEL_FCR : MODEL_NH;
    } else if (m.type == PGMPM_MAT_ELASTOPLASTIC) {
        if (!(m.yield_stress > 0.f) || !std::isfinite(m.yield_stress))
            return fail(PGMPM_ERR_ARG, "ELASTOPLASTIC yield_stress must be finite and > 0");
        model = MODEL_VM;
    } else {
        return fail(PGMPM_ERR_UNSUPPORTED, "material type %d (SAND/SNOW) has no implementation", m.type);
    }
    if (!(m.youngs_modulus >= 0.f) || !std::isfinite(m.youngs_modulus))
        return fail(PGMPM_ERR_ARG, "invalid youngs_modulus");
    const double E = m.youngs_modulus, nu = m.poisson_ratio;
    if (model != MODEL_EOS && !(nu > -1.0 && nu < 0.5))
        return fail(PGMPM_ERR_ARG, "poisson_ratio must be in (-1, 0.5)");
    std::memset(&d, 0, sizeof(d));
    d.model = model;
    d.yield = model == MODEL_VM ? m.yield_stress : 0.f;
    d.visc = model == MODEL_EOS ? m.viscosity : 0.f;
    d.E = (float)E;
    if (d.model != MODEL_EOS) {
        d.mu = (float)(E / (2.0 * (1.0 + nu)));
        d.lam = (float)(E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)));
        d.dmu_dE = (float)(1.0 / (2.0 * (1.0 + nu)));
        d.dlam_dE = (float)(nu / ((1.0 + nu) * (1.0 - 2.0 * nu)));
    }
    return PGMPM_OK;
}

int alloc_bin_sort(pgmpm_solver s) {
    if (s->bs_ccount.p) return PGMPM_OK;
    const size_t ct = (size_t)s->total_ct;
    CK(s->bs_ccount.alloc(sizeof(uint32_t) * (ct * 64 + 1)));
    CK(s->bs_coff.alloc(sizeof(uint32_t) * ct * 64));
    CK(s->bs_tcount.alloc(sizeof(uint32_t) * (ct + 1)));
    CK(s->bs_toff.alloc(sizeof(uint32_t) * (ct + 1)));
    CK(s->bs_bsum.alloc(sizeof(uint32_t) * (size_t)bin_sort_scan_blocks((int)ct)));
    CK(s->bs_slot.alloc(sizeof(uint32_t) * (size_t)std::max<int64_t>(s->N, 1)));
    CK(s->cell_range.alloc(sizeof(uint2) * 64 * std::max<size_t>(ct, 1)));
    CK(s->ptile_list.alloc(sizeof(uint32_t) * std::max<size_t>(ct, 1)));
    CK(s->tile_rank.alloc(sizeof(uint32_t) * std::max<size_t>(ct, 1)));
    // the counters start at zero and every sort leaves them zero
    CK(cudaMemset(s->bs_ccount.p, 0, s->bs_ccount.bytes));
    CK(cudaMemset(s->bs_tcount.p, 0, s->bs_tcount.bytes));
    return PGMPM_OK;
}

int refresh_payload(pgmpm_solver s, cudaStream_t st) {
    if (s->N == 0 || s->pf.physics != PHYS_MLS) return PGMPM_OK;
    CK(launch_payload(s->view(), s->pf, st));
    return PGMPM_OK;
}

// Sets the condition of a conditional graph node from *flag (or to 1 when
// always), clears the flag and counts the steps that sort again in *count
// (one thread).
__global__ void k_resort_cond(cudaGraphConditionalHandle h, uint32_t* flag, uint32_t* count, int always) {
    const uint32_t f = *flag | (always ? 1u : 0u);
    *flag = 0u;
    if (f) *count += 1u;
    cudaGraphSetConditional(h, f ? 1u : 0u);
}

// Under stream capture on st: the bin sort as the body of an IF node whose
// condition k_resort_cond takes from *flag, so that a replayed step sorts
// only when its G2P found a key that differs from the recorded one.
int conditional_sort(pgmpm_solver s, const View& V, const BinSortBufs& B, uint32_t* flag, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    CK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, nullptr, nullptr));
    if (cs != cudaStreamCaptureStatusActive || !g)
        return fail(PGMPM_ERR_STATE, "internal: a conditional sort needs a stream capture");
    if (!s->body_stream) CK(cudaStreamCreateWithFlags(&s->body_stream, cudaStreamNonBlocking));
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
    k_resort_cond<<<1, 1, 0, st>>>(h, flag, s->rec_resort.as<uint32_t>() + 2, s->rec_mode == 2 ? 1 : 0);
    CK(cudaGetLastError());
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    CK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeIf;
    np.conditional.size = 1;
    cudaGraphNode_t cn = nullptr;
    CK(cudaGraphAddNode(&cn, g, deps, nd, &np));
    CK(cudaStreamUpdateCaptureDependencies(st, &cn, 1, cudaStreamSetCaptureDependencies));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    CK(cudaStreamBeginCaptureToGraph(s->body_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    const cudaError_t e = bin_sort_step(V, B, s->num_sms, s->body_stream);
    cudaGraph_t out = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(s->body_stream, &out);
    CK(e);
    CK(e2);
    return PGMPM_OK;
}

int record_step(pgmpm_solver s, const StepBufs& b, cudaStream_t st, bool timed, bool write_vc, StepKind kind) {
    if (s->N == 0) {  // nothing to move; keep the timing events consistent
        if (timed)
            for (int i = 0; i < 5; ++i) CK(cudaEventRecord(s->ev[i], st));
        return PGMPM_OK;
    }
    if (kind != STEP_SPLIT && !(s->pf.physics == PHYS_MLS && s->tune.step_sort == 0))
        return fail(PGMPM_ERR_STATE, "internal: fused step without the bin sort");
    if (b.sort_mode != 0 && (s->tune.step_sort != 0 || kind != STEP_SPLIT || (b.sort_mode == 2 && !b.resort)))
        return fail(PGMPM_ERR_STATE, "internal: a recorded sort needs the bin sort and split steps");
    View V = s->view_for(b);
    // P2G variant 1 builds its payload from the state's v and C
    V.write_vc = write_vc || s->pf.physics != PHYS_MLS || s->tune.p2g_variant == 1 ? 1 : 0;
    // per-step resets: tile counts, active node count, work cursors, and the
    // active node tile flags.  The bin sort's first kernel clears the
    // counters and the sort writes every flag itself, so a bin-sorted step
    // has no memset node.
    if (s->tune.step_sort != 0) {
        CK(cudaMemsetAsync(b.tile_flags, 0, sizeof(uint32_t) * (size_t)s->total_nt, st));
        CK(cudaMemsetAsync(b.counters, 0, sizeof(uint32_t) * CNT_RESET, st));
    }
    if (timed) CK(cudaEventRecord(s->ev[0], st));
    if (s->tune.step_sort == 0) {
        BinSortBufs B;
        B.keys_in = b.keys_in;
        B.ccount = s->bs_ccount.as<uint32_t>();
        B.coff = s->bs_coff.as<uint32_t>();
        B.tcount = s->bs_tcount.as<uint32_t>();
        B.toff = s->bs_toff.as<uint32_t>();
        B.bsum = s->bs_bsum.as<uint32_t>();
        B.slot = s->bs_slot.as<uint32_t>();
        B.out_k = b.which ? b.kb : b.ka;  // where the step's readers look (View::skeys / order)
        B.out_v = b.which ? b.vb : b.va;
        B.cell_range = b.cell_range;
        B.ptile_list = b.ptile_list;
        B.tile_rank = s->tile_rank.as<uint32_t>();
        if (b.sort_mode == 0) {
            CK(bin_sort_step(V, B, s->num_sms, st));
        } else if (b.sort_mode == 2) {
            int rc = conditional_sort(s, V, B, b.resort, st);
            if (rc) return rc;
        }
    } else {
        int which = 0;
        CK(radix_sort_pairs(b.keys_in, nullptr, b.ka, b.va, b.kb, b.vb, s->sort_scratch.as<uint32_t>(), s->N,
                            s->key_bits, &which, st));
        if (which != b.which) return fail(PGMPM_ERR_STATE, "internal: sort buffer parity changed");
        CK(launch_mark(V, st));
    }
    if (timed) CK(cudaEventRecord(s->ev[1], st));
    // a fused step's P2G was done by the previous step's G2P2G
    if (kind == STEP_SPLIT || kind == STEP_FUSED_FIRST) CK(launch_p2g(V, s->pf, s->tune, s->num_sms, st));
    if (timed) CK(cudaEventRecord(s->ev[2], st));
    CK(launch_grid(V, s->pf, s->tune, s->num_sms, st));
    if (timed) CK(cudaEventRecord(s->ev[3], st));
    if (kind == STEP_FUSED_FIRST || kind == STEP_FUSED) {
        V.pay_out = nullptr;  // the payload stays in the SM; the buffer goes stale
        CK(launch_g2p2g(V, s->pf, s->tune, s->num_sms, st));
    } else {
        CK(launch_g2p(V, s->pf, s->tune, s->num_sms, st));
    }
    if (timed) CK(cudaEventRecord(s->ev[4], st));
    return PGMPM_OK;
}

StepKind step_kind(pgmpm_solver s, int k, int n, bool primed, bool drain) {
    if (!s->fused()) return STEP_SPLIT;
    const bool first = k == 0 && !primed;
    if (drain && k + 1 == n) return first ? STEP_SPLIT : STEP_FUSED_LAST;
    return first ? STEP_FUSED_FIRST : STEP_FUSED;
}

int unprime(pgmpm_solver s, cudaStream_t st) {
    if (!s->primed) return PGMPM_OK;
    s->primed = false;
    CK(cudaMemsetAsync(s->grid_mp.p, 0, s->grid_mp.bytes, st));
    return refresh_payload(s, st);
}

}  // namespace pgmpm

namespace {

// The step graph of one kind (mid = false: the call's last step; mid = true:
// a step that another step of the same call follows, v and C not stored).
int build_graph(pgmpm_solver s, StepKind kind, bool mid) {
    cudaGraph_t& graph = s->step_graph[kind][mid ? 1 : 0];
    cudaGraphExec_t& exec = s->step_exec[kind][mid ? 1 : 0];
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    CK(cudaStreamBeginCapture(s->cap_stream, cudaStreamCaptureModeThreadLocal));
    int rc = record_step(s, s->live_bufs(), s->cap_stream, false, !mid, kind);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->cap_stream, &g);
    if (rc != PGMPM_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    CK(e);
    graph = g;
    CK(cudaGraphInstantiate(&exec, g, 0));
    return PGMPM_OK;
}

}  // namespace

namespace pgmpm {
// Live steps.  With the fused kernel a call leaves the next step's P2G in
// grid_mp (s->primed), so a following call continues without a P2G of its
// own; anything that changes the state or its parameters unprimes first.
int run_steps(pgmpm_solver s, int n_steps, cudaStream_t st) {
    if (!s->uploaded) return fail(PGMPM_ERR_STATE, "no particles uploaded");
    if (!s->fused()) {
        int rc = unprime(s, st);
        if (rc) return rc;
    }
    for (int k = 0; k < n_steps; ++k) {
        const StepKind kind = step_kind(s, k, n_steps, s->primed, false);
        if (s->profiling) {
            int rc = record_step(s, s->live_bufs(), st, true, true, kind);
            if (rc) return rc;
            CK(cudaEventSynchronize(s->ev[4]));
            float a, b, c, d;
            CK(cudaEventElapsedTime(&a, s->ev[0], s->ev[1]));
            CK(cudaEventElapsedTime(&b, s->ev[1], s->ev[2]));
            CK(cudaEventElapsedTime(&c, s->ev[2], s->ev[3]));
            CK(cudaEventElapsedTime(&d, s->ev[3], s->ev[4]));
            s->met.sort_ms = a;
            s->met.p2g_ms = b;
            s->met.grid_ms = c;
            s->met.g2p_ms = d;
            s->met.last_step_ms = a + b + c + d;
            s->met.average_step_ms =
                (s->met.average_step_ms * s->met.total_steps + s->met.last_step_ms) / (s->met.total_steps + 1);
            s->met.particle_steps_per_s = s->met.average_step_ms > 0 ? s->N / (s->met.average_step_ms * 1e-3) : 0;
        } else if (s->use_graph) {
            const bool mid = k + 1 < n_steps;
            if (!s->step_exec[kind][mid ? 1 : 0]) {
                int rc = build_graph(s, kind, mid);
                if (rc) return rc;
            }
            CK(cudaGraphLaunch(s->step_exec[kind][mid ? 1 : 0], st));
        } else {
            int rc = record_step(s, s->live_bufs(), st, false, k + 1 == n_steps, kind);
            if (rc) return rc;
        }
        if (kind == STEP_FUSED_FIRST || kind == STEP_FUSED) s->primed = true;
        s->met.total_steps++;
    }
    return PGMPM_OK;
}

}  // namespace pgmpm

// ============================================================== C-ABI
extern "C" {

const char* pgmpm_last_error(void) { return g_err.c_str(); }
void pgmpm_clear_error(void) { g_err.clear(); }
int pgmpm_abi_version(void) { return PGMPM_ABI_VERSION; }

int pgmpm_create(const pgmpm_scene_desc* scenes, int32_t n_scenes, const int64_t* particle_counts,
                 const pgmpm_material* materials, int32_t n_materials, int32_t device, pgmpm_solver* out) {
    return pgmpm_create_ex(scenes, n_scenes, particle_counts, materials, n_materials, device, nullptr, out);
}

int pgmpm_create_ex(const pgmpm_scene_desc* scenes, int32_t n_scenes, const int64_t* particle_counts,
                    const pgmpm_material* materials, int32_t n_materials, int32_t device,
                    const pgmpm_create_options* options, pgmpm_solver* out) {
    if (!out) return fail(PGMPM_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!scenes || n_scenes < 1 || !particle_counts) return fail(PGMPM_ERR_ARG, "need >= 1 scene and counts");
    if (!materials || n_materials < 1) return fail(PGMPM_ERR_ARG, "need >= 1 material");
    const bool sparse = options && options->sparse_grid;
    if (sparse) {
        if (n_scenes != 1 || scenes[0].physics != PGMPM_PHYSICS_MLS)
            return fail(PGMPM_ERR_UNSUPPORTED, "sparse grids: one scene with PGMPM_PHYSICS_MLS");
        if (options->max_tiles < 0) return fail(PGMPM_ERR_ARG, "max_tiles must be >= 0");
        for (int a = 0; a < 3; ++a)
            if (scenes[0].n[a] > 4 * ((1 << 10) - 2) + 3)
                return fail(PGMPM_ERR_ARG, "sparse grids: at most %d nodes per axis", 4 * ((1 << 10) - 2) + 3);
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
        return fail(PGMPM_ERR_CUDA, "no CUDA device available");
    if (device < 0 || device >= ndev) return fail(PGMPM_ERR_ARG, "device %d out of range", device);
    DeviceGuard dg(device);
    auto s = new pgmpm_solver_s();
    s->device = device;
    cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, device);
    s->S = n_scenes;
    s->M = n_materials;
    s->desc.assign(scenes, scenes + n_scenes);
    s->counts.assign(particle_counts, particle_counts + n_scenes);
    s->mats_h.assign(materials, materials + n_materials);
    int64_t N = 0;
    int64_t ct_base = 0, nt_base = 0;
    const int physics = scenes[0].physics;
    for (int i = 0; i < n_scenes; ++i) {
        const pgmpm_scene_desc& d = scenes[i];
        if (d.physics != PGMPM_PHYSICS_MLS && d.physics != PGMPM_PHYSICS_REF_COMPAT) {
            delete s;
            return fail(PGMPM_ERR_ARG, "scene %d: unknown physics %d", i, d.physics);
        }
        if (d.physics != physics) {
            delete s;
            return fail(PGMPM_ERR_ARG, "all scenes of one solver must use the same physics");
        }
        if (d.n[0] < 4 || d.n[1] < 4 || d.n[2] < 4 || !(d.dx > 0.f) || !(d.dt > 0.f) || particle_counts[i] < 0) {
            delete s;
            return fail(PGMPM_ERR_ARG, "scene %d: need n >= 4 per axis, dx > 0, dt > 0, count >= 0", i);
        }
        if (d.boundary < PGMPM_BC_NONE || d.boundary > PGMPM_BC_SEPARATE || d.boundary_thickness < 0) {
            delete s;
            return fail(PGMPM_ERR_ARG, "scene %d: invalid boundary", i);
        }
        SceneDev sd;
        std::memset(&sd, 0, sizeof(sd));
        for (int a = 0; a < 3; ++a) {
            sd.n[a] = d.n[a];
            sd.ct[a] = ((d.n[a] - 3) >> 2) + 1;
            sd.nt[a] = sd.ct[a] + 1;
            sd.origin[a] = d.origin[a];
            sd.gravity[a] = d.gravity[a];
        }
        sd.ct_base = (int)ct_base;
        sd.nt_base = (int)nt_base;
        ct_base += (int64_t)sd.ct[0] * sd.ct[1] * sd.ct[2];
        nt_base += (int64_t)sd.nt[0] * sd.nt[1] * sd.nt[2];
        sd.physics = d.physics == PGMPM_PHYSICS_MLS ? PHYS_MLS : PHYS_REF;
        sd.boundary = d.physics == PGMPM_PHYSICS_MLS ? d.boundary : BC_NONE;
        sd.bthick = d.boundary_thickness;
        sd.p_begin = (int)N;
        N += particle_counts[i];
        sd.p_end = (int)std::min<int64_t>(N, 0x7FFFFFFF);
        sd.dx = d.dx;
        sd.D = 4.f / (d.dx * d.dx);
        sd.inv_dx = 1.0f / d.dx;
        sd.dt = d.dt;
        s->scenes.push_back(sd);
        if (!sparse && (ct_base * 64 > 0xFFFFFFFFll || nt_base * 64 >= 0x7FFFFFFFll)) {
            delete s;
            return fail(PGMPM_ERR_ARG, "grids too large for 32-bit cell keys (a sparse grid stores only touched tiles)");
        }
    }
    if (N >= 0x7FFFFFFF) {
        delete s;
        return fail(PGMPM_ERR_ARG, "too many particles (max 2^31-2)");
    }
    s->N = N;
    if (sparse) {
        // the tile pool: a power of two of at least twice the tiles asked for
        // (the hash stays at most half full), one slot per cell / node tile
        const int64_t want = options->max_tiles > 0 ? options->max_tiles : std::max<int64_t>(4096, N / 128);
        int64_t cap = 1;
        while (cap < 2 * want) cap <<= 1;
        if (cap > ((int64_t)1 << 25)) {
            delete s;
            return fail(PGMPM_ERR_ARG, "sparse grids: max_tiles %lld above 2^24", (long long)want);
        }
        ct_base = nt_base = cap;
        s->sp_cap = (uint32_t)cap;
        int lg = 0;
        while ((1ll << lg) < cap) ++lg;
        s->sp_shift = 32 - lg;
    }
    s->total_ct = (int)ct_base;
    s->total_nt = (int)nt_base;
    s->key_bits = bits_for((uint64_t)ct_base * 64);
    s->pf.physics = physics == PGMPM_PHYSICS_MLS ? PHYS_MLS : PHYS_REF;
    s->pf.multi_mat = n_materials > 1;
    s->pf.has_fluid = false;
    s->pf.has_plastic = false;
    std::vector<MatDev> md(n_materials);
    for (int i = 0; i < n_materials; ++i) {
        int rc = material_to_dev(materials[i], md[i]);
        if (rc) {
            delete s;
            return rc;
        }
        if (md[i].model == MODEL_EOS) s->pf.has_fluid = true;
        if (md[i].model == MODEL_VM) s->pf.has_plastic = true;
    }
    int sw = 0;
    {
        int passes = radix_passes(s->key_bits);
        sw = (passes - 1) & 1;
    }
    s->sort_which = sw;
    const size_t n4 = sizeof(uint32_t) * (size_t)std::max<int64_t>(N, 1);
    cudaError_t e = cudaSuccess;
#define AL(buf, bytes)                                         \
    if (e == cudaSuccess) e = (buf).alloc(bytes);
    AL(s->d_scenes, sizeof(SceneDev) * n_scenes);
    AL(s->d_mats, sizeof(MatDev) * n_materials);
    AL(s->q, sizeof(float4) * 6 * (size_t)std::max<int64_t>(N, 1));
    if (s->pf.physics == PHYS_MLS) AL(s->pay, sizeof(float4) * 4 * (size_t)std::max<int64_t>(N, 1));
    AL(s->mV, sizeof(float2) * (size_t)std::max<int64_t>(N, 1));
    if (s->pf.multi_mat) AL(s->mat, n4);
    AL(s->user_of_phys, n4);
    AL(s->phys_of_user, n4);
    AL(s->keys, n4);
    AL(s->ka, n4);
    AL(s->va, n4);
    AL(s->kb, n4);
    AL(s->vb, n4);
    AL(s->sort_scratch, sizeof(uint32_t) * (size_t)radix_sort_scratch_words(std::max<int64_t>(N, 1)));
    AL(s->grid_mp, sizeof(float4) * 64 * (size_t)nt_base);
    AL(s->grid_v, sizeof(float4) * 64 * (size_t)nt_base);
    AL(s->tile_flags, sizeof(uint32_t) * (size_t)nt_base);
    AL(s->tile_list, sizeof(uint32_t) * (size_t)nt_base);
    AL(s->ctile_list, sizeof(uint32_t) * (size_t)ct_base);
    AL(s->ctile_range, sizeof(uint2) * (size_t)ct_base);
    AL(s->counters, sizeof(uint32_t) * CNT_WORDS);
    if (sparse) {
        AL(s->sp_code, sizeof(uint32_t) * (size_t)s->sp_cap);
        AL(s->sp_nbr, sizeof(uint4) * 2 * (size_t)s->sp_cap);
        AL(s->sp_box, sizeof(float4) * 216 * (size_t)s->sp_cap);
        AL(s->sp_rev, sizeof(uint2) * 8 * (size_t)s->sp_cap);
    }
#undef AL
    // the bin sort keeps 8 bytes per cell: default for grids with at most ~8
    // cells per particle, the radix sort (O(N) per pass) for sparser ones
    s->tune.step_sort = sparse || (int64_t)ct_base * 64 <= 8 * std::max<int64_t>(N, 1) + (1 << 20) ? 0 : 1;
    // P2G (MLS): balanced particle runs over the bin sort's cell table;
    // without it, two lanes per cell pays off when the occupied tiles
    // outnumber the resident blocks (many particles), one lane otherwise
    s->tune.p2g_variant = s->pf.physics != PHYS_MLS ? 2
                          : s->tune.step_sort == 0  ? 4
                          : N >= (int64_t)1 << 20   ? 3
                                                    : 2;
    if (e == cudaSuccess && s->tune.step_sort == 0 && alloc_bin_sort(s) != PGMPM_OK) e = cudaErrorMemoryAllocation;
    if (e == cudaSuccess) e = cudaMemcpy(s->d_scenes.p, s->scenes.data(), sizeof(SceneDev) * n_scenes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->d_mats.p, md.data(), sizeof(MatDev) * n_materials, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(s->grid_mp.p, 0, s->grid_mp.bytes);
    if (e == cudaSuccess) e = cudaMemset(s->grid_v.p, 0, s->grid_v.bytes);
    if (e == cudaSuccess) e = cudaMemset(s->tile_flags.p, 0, s->tile_flags.bytes);
    if (e == cudaSuccess) e = cudaMemset(s->counters.p, 0, s->counters.bytes);
    if (e == cudaSuccess && sparse) e = cudaMemset(s->sp_code.p, 0xFF, s->sp_code.bytes);  // every slot free
    if (e == cudaSuccess && sparse) e = cudaMemset(s->sp_nbr.p, 0, s->sp_nbr.bytes);
    if (e == cudaSuccess && sparse) e = cudaMemset(s->sp_box.p, 0, s->sp_box.bytes);
    if (e == cudaSuccess && sparse) e = cudaMemset(s->sp_rev.p, 0, s->sp_rev.bytes);  // stamp 0: no step yet
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->cap_stream, cudaStreamNonBlocking);
    for (int i = 0; i < 6 && e == cudaSuccess; ++i) e = cudaEventCreate(&s->ev[i]);
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_counters, sizeof(uint32_t) * CNT_WORDS);
    if (e != cudaSuccess) {
        delete s;
        return fail(e == cudaErrorMemoryAllocation ? PGMPM_ERR_OOM : PGMPM_ERR_CUDA, "create: %s",
                    cudaGetErrorString(e));
    }
    s->met.num_particles = N;
    *out = s;
    return PGMPM_OK;
}

int pgmpm_destroy(pgmpm_solver s) {
    if (!s) return PGMPM_OK;
    {
        DeviceGuard dg(s->device);
        cudaDeviceSynchronize();
    }
    delete s;
    return PGMPM_OK;
}

int pgmpm_set_materials(pgmpm_solver s, const pgmpm_material* materials, int32_t n_materials) {
    if (!s || !materials || n_materials != s->M) return fail(PGMPM_ERR_ARG, "material count must match create()");
    DeviceGuard dg(s->device);
    std::vector<MatDev> md(n_materials);
    bool fluid = false, plastic = false;
    for (int i = 0; i < n_materials; ++i) {
        int rc = material_to_dev(materials[i], md[i]);
        if (rc) return rc;
        fluid |= md[i].model == MODEL_EOS;
        plastic |= md[i].model == MODEL_VM;
    }
    if (fluid != s->pf.has_fluid || plastic != s->pf.has_plastic) {  // kernels are chosen by these
        s->pf.has_fluid = fluid;
        s->pf.has_plastic = plastic;
        s->drop_graph();
    }
    // ordered with prior work on the legacy stream; graphs read the table at run time
    CK(cudaMemcpy(s->d_mats.p, md.data(), sizeof(MatDev) * n_materials, cudaMemcpyHostToDevice));
    s->mats_h.assign(materials, materials + n_materials);
    s->ck_valid = false;  // a replay would run with the new table
    if (s->uploaded) {
        // the payload (and a pending fused P2G) hold the stress of the old
        // material table
        CK(cudaDeviceSynchronize());
        if (s->primed) {
            s->primed = false;
            CK(cudaMemsetAsync(s->grid_mp.p, 0, s->grid_mp.bytes, s->cap_stream));
        }
        int rc = refresh_payload(s, s->cap_stream);
        if (rc) return rc;
        CK(cudaStreamSynchronize(s->cap_stream));
    }
    return PGMPM_OK;
}

int pgmpm_set_scene_params(pgmpm_solver s, int32_t scene, float dt, const float* gravity) {
    if (!s) return fail(PGMPM_ERR_ARG, "null solver");
    if (scene < 0 || scene >= s->S) return fail(PGMPM_ERR_ARG, "scene %d out of range [0, %d)", scene, s->S);
    if (!(dt > 0.f) || !std::isfinite(dt)) return fail(PGMPM_ERR_ARG, "dt must be positive and finite");
    if (gravity)
        for (int a = 0; a < 3; ++a)
            if (!std::isfinite(gravity[a])) return fail(PGMPM_ERR_ARG, "gravity must be finite");
    SceneDev& sd = s->scenes[scene];
    bool same = sd.dt == dt;
    if (gravity)
        for (int a = 0; a < 3; ++a) same = same && sd.gravity[a] == gravity[a];
    if (same) return PGMPM_OK;
    DeviceGuard dg(s->device);
    sd.dt = dt;
    s->desc[scene].dt = dt;
    if (gravity)
        for (int a = 0; a < 3; ++a) sd.gravity[a] = s->desc[scene].gravity[a] = gravity[a];
    // kernels and captured graphs read the scene table from device memory
    CK(cudaMemcpy(s->d_scenes.as<SceneDev>() + scene, &sd, sizeof(SceneDev), cudaMemcpyHostToDevice));
    s->ck_valid = false;  // a replay would run with the new dt / gravity
    if (s->uploaded && s->pf.physics == PHYS_MLS) {
        // the payload (and a pending fused P2G) hold -dt V0 D tau of the old dt
        CK(cudaDeviceSynchronize());
        if (s->primed) {
            s->primed = false;
            CK(cudaMemsetAsync(s->grid_mp.p, 0, s->grid_mp.bytes, s->cap_stream));
        }
        int rc = refresh_payload(s, s->cap_stream);
        if (rc) return rc;
        CK(cudaStreamSynchronize(s->cap_stream));
    }
    return PGMPM_OK;
}

int pgmpm_upload(pgmpm_solver s, const float* x, const float* v, const float* C, const float* F, const float* m,
                 const float* V0, const int32_t* mat, int32_t ptr_kind, void* stream) {
    if (!s) return fail(PGMPM_ERR_ARG, "null solver");
    if (s->N > 0 && (!x || !m)) return fail(PGMPM_ERR_ARG, "x and m are required");
    DeviceGuard dg(s->device);
    cudaStream_t st = ST(stream);
    const int64_t N = s->N;
    const float *dx_ = x, *dv = v, *dC = C, *dF = F, *dm = m, *dV0 = V0;
    const int32_t* dmat = mat;
    if (ptr_kind == PGMPM_PTR_HOST && N > 0) {
        const size_t fl = 3 + 3 + 9 + 9 + 1 + 1;
        CK(s->staging.ensure(sizeof(float) * fl * N + sizeof(int32_t) * N));
        float* b = s->staging.as<float>();
        float* sx = b;
        float* sv = sx + 3 * N;
        float* sC = sv + 3 * N;
        float* sF = sC + 9 * N;
        float* sm = sF + 9 * N;
        float* sV = sm + N;
        int32_t* smat = reinterpret_cast<int32_t*>(sV + N);
        CK(cudaMemcpyAsync(sx, x, sizeof(float) * 3 * N, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(sm, m, sizeof(float) * N, cudaMemcpyHostToDevice, st));
        dx_ = sx;
        dm = sm;
        dv = v ? sv : nullptr;
        dC = C ? sC : nullptr;
        dF = F ? sF : nullptr;
        dV0 = V0 ? sV : nullptr;
        dmat = mat ? smat : nullptr;
        if (v) CK(cudaMemcpyAsync(sv, v, sizeof(float) * 3 * N, cudaMemcpyHostToDevice, st));
        if (C) CK(cudaMemcpyAsync(sC, C, sizeof(float) * 9 * N, cudaMemcpyHostToDevice, st));
        if (F) CK(cudaMemcpyAsync(sF, F, sizeof(float) * 9 * N, cudaMemcpyHostToDevice, st));
        if (V0) CK(cudaMemcpyAsync(sV, V0, sizeof(float) * N, cudaMemcpyHostToDevice, st));
        if (mat) CK(cudaMemcpyAsync(smat, mat, sizeof(int32_t) * N, cudaMemcpyHostToDevice, st));
    } else if (ptr_kind != PGMPM_PTR_DEVICE && ptr_kind != PGMPM_PTR_HOST) {
        return fail(PGMPM_ERR_ARG, "ptr_kind must be PGMPM_PTR_HOST or PGMPM_PTR_DEVICE");
    }
    if (mat && s->M == 1) dmat = nullptr;
    if (s->primed) {  // the pending P2G is the old state's
        s->primed = false;
        CK(cudaMemsetAsync(s->grid_mp.p, 0, s->grid_mp.bytes, st));
    }
    if (N > 0) {
        View V = s->view();
        // 1. identity pack (user order) to compute the keys
        CK(cudaMemsetAsync(s->keys.p, 0, sizeof(uint32_t) * N, st));
        // order = identity: use va as a temporary iota through the sort of all-zero keys
        int w0 = 0;
        CK(radix_sort_pairs(s->keys.as<uint32_t>(), nullptr, s->ka.as<uint32_t>(), s->va.as<uint32_t>(),
                            s->kb.as<uint32_t>(), s->vb.as<uint32_t>(), s->sort_scratch.as<uint32_t>(), N, 1, &w0,
                            st));
        const uint32_t* iota = w0 ? s->vb.as<uint32_t>() : s->va.as<uint32_t>();
        CK(launch_pack(V, dx_, dv, dC, dF, dm, dV0, dmat, iota, s->user_of_phys.as<uint32_t>(), s->phys_of_user.as<uint32_t>(), s->mV.as<float2>(),
                       s->pf.multi_mat ? s->mat.as<int32_t>() : nullptr, st));
        // 2. keys of the user-order positions, stable sort -> physical order
        CK(launch_keys(V, s->pf, st));
        int which = 0;
        CK(radix_sort_pairs(s->keys.as<uint32_t>(), nullptr, s->ka.as<uint32_t>(), s->va.as<uint32_t>(),
                            s->kb.as<uint32_t>(), s->vb.as<uint32_t>(), s->sort_scratch.as<uint32_t>(), N,
                            s->key_bits, &which, st));
        const uint32_t* ord = which ? s->vb.as<uint32_t>() : s->va.as<uint32_t>();
        const uint32_t* sk = which ? s->kb.as<uint32_t>() : s->ka.as<uint32_t>();
        // 3. pack in sorted order; the sorted keys are the keys of the physical order
        CK(launch_pack(V, dx_, dv, dC, dF, dm, dV0, dmat, ord, s->user_of_phys.as<uint32_t>(), s->phys_of_user.as<uint32_t>(), s->mV.as<float2>(),
                       s->pf.multi_mat ? s->mat.as<int32_t>() : nullptr, st));
        CK(cudaMemcpyAsync(s->keys.p, sk, sizeof(uint32_t) * N, cudaMemcpyDeviceToDevice, st));
        int rc = refresh_payload(s, st);
        if (rc) return rc;
    }
    s->uploaded = true;
    return PGMPM_OK;
}

int pgmpm_download(pgmpm_solver s, float* x, float* v, float* C, float* F, int32_t ptr_kind, void* stream) {
    if (!s) return fail(PGMPM_ERR_ARG, "null solver");
    if (!s->uploaded) return fail(PGMPM_ERR_STATE, "no particles uploaded");
    DeviceGuard dg(s->device);
    cudaStream_t st = ST(stream);
    const int64_t N = s->N;
    if (N == 0) return PGMPM_OK;
    View V = s->view();
    if (ptr_kind == PGMPM_PTR_DEVICE) {
        CK(launch_unpack(V, s->phys_of_user.as<uint32_t>(), x, v, C, F, st));
        return PGMPM_OK;
    }
    if (ptr_kind != PGMPM_PTR_HOST) return fail(PGMPM_ERR_ARG, "bad ptr_kind");
    CK(s->staging.ensure(sizeof(float) * 26 * N + sizeof(int32_t) * N));
    float* sx = s->staging.as<float>();
    float* sv = sx + 3 * N;
    float* sC = sv + 3 * N;
    float* sF = sC + 9 * N;
    CK(launch_unpack(V, s->phys_of_user.as<uint32_t>(), x ? sx : nullptr, v ? sv : nullptr, C ? sC : nullptr,
                     F ? sF : nullptr, st));
    if (x) CK(cudaMemcpyAsync(x, sx, sizeof(float) * 3 * N, cudaMemcpyDeviceToHost, st));
    if (v) CK(cudaMemcpyAsync(v, sv, sizeof(float) * 3 * N, cudaMemcpyDeviceToHost, st));
    if (C) CK(cudaMemcpyAsync(C, sC, sizeof(float) * 9 * N, cudaMemcpyDeviceToHost, st));
    if (F) CK(cudaMemcpyAsync(F, sF, sizeof(float) * 9 * N, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return PGMPM_OK;
}

int pgmpm_vtk_write_particles(const char* path, int64_t n, const float* x, const float* v, const float* F,
                              const int32_t* mat, double time) {
    if (!path || n < 0 || (n > 0 && !x)) return fail(PGMPM_ERR_ARG, "vtk: need a path and positions");
    if (n > ((int64_t)1 << 30)) return fail(PGMPM_ERR_ARG, "vtk: more than 2^30 particles (legacy VTK uses int32)");
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(PGMPM_ERR_ARG, "vtk: cannot open %s for writing", path);
    // the legacy binary format is big-endian
    std::vector<unsigned char> buf;
    auto put = [&](uint32_t w) {
        buf.push_back((unsigned char)(w >> 24));
        buf.push_back((unsigned char)(w >> 16));
        buf.push_back((unsigned char)(w >> 8));
        buf.push_back((unsigned char)w);
    };
    auto putf = [&](float a) {
        uint32_t w;
        std::memcpy(&w, &a, 4);
        put(w);
    };
    auto text = [&](const char* fmt, auto... a) {
        char line[256];
        const int k = std::snprintf(line, sizeof(line), fmt, a...);
        buf.insert(buf.end(), line, line + k);
    };
    const long long nn = (long long)n;
    buf.reserve((size_t)n * 36 + 512);
    text("# vtk DataFile Version 3.0\nphysgrad_b200 MPM particles, t = %.9g\nBINARY\nDATASET POLYDATA\n", time);
    text("POINTS %lld float\n", nn);
    for (int64_t i = 0; i < 3 * n; ++i) putf(x[i]);
    text("\nVERTICES %lld %lld\n", nn, 2 * nn);
    for (int64_t i = 0; i < n; ++i) {
        put(1u);
        put((uint32_t)i);
    }
    text("\nPOINT_DATA %lld\n", nn);
    if (v) {
        text("VECTORS velocity float\n");
        for (int64_t i = 0; i < 3 * n; ++i) putf(v[i]);
        text("\n");
    }
    if (F) {
        text("SCALARS J float 1\nLOOKUP_TABLE default\n");
        for (int64_t i = 0; i < n; ++i) {
            const float* a = F + 9 * i;
            putf(a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                 a[2] * (a[3] * a[7] - a[4] * a[6]));
        }
        text("\n");
    }
    if (mat) {
        text("SCALARS material int 1\nLOOKUP_TABLE default\n");
        for (int64_t i = 0; i < n; ++i) put((uint32_t)mat[i]);
        text("\n");
    }
    const bool ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
    const bool closed = std::fclose(f) == 0;
    if (!ok || !closed) return fail(PGMPM_ERR_ARG, "vtk: writing %s failed", path);
    return PGMPM_OK;
}

int pgmpm_write_vtk(pgmpm_solver s, const char* path, double time, void* stream) {
    if (!s) return fail(PGMPM_ERR_ARG, "null solver");
    if (!s->uploaded) return fail(PGMPM_ERR_STATE, "no particles uploaded");
    const int64_t N = s->N;
    std::vector<float> x(3 * N), v(3 * N), F(9 * N);
    int rc = pgmpm_download(s, x.data(), v.data(), nullptr, F.data(), PGMPM_PTR_HOST, stream);
    if (rc) return rc;
    std::vector<int32_t> mat;
    if (s->pf.multi_mat && N > 0) {  // physical order on the device -> upload order
        DeviceGuard dg(s->device);
        std::vector<int32_t> mp(N);
        std::vector<uint32_t> u(N);
        CK(cudaMemcpy(mp.data(), s->mat.p, sizeof(int32_t) * N, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(u.data(), s->user_of_phys.p, sizeof(uint32_t) * N, cudaMemcpyDeviceToHost));
        mat.assign(N, 0);
        for (int64_t i = 0; i < N; ++i)
            if (u[i] < (uint64_t)N) mat[u[i]] = mp[i];
    }
    return pgmpm_vtk_write_particles(path, N, x.data(), v.data(), F.data(), mat.empty() ? nullptr : mat.data(), time);
}

int pgmpm_download_grid(pgmpm_solver s, int32_t scene, float* mass, float* velocity, int32_t ptr_kind,
                        void* stream) {
    if (!s || scene < 0 || scene >= s->S) return fail(PGMPM_ERR_ARG, "bad solver or scene");
    DeviceGuard dg(s->device);
    cudaStream_t st = ST(stream);
    const SceneDev& sc = s->scenes[scene];
    const int64_t nodes = (int64_t)sc.n[0] * sc.n[1] * sc.n[2];
    View V = s->view();
    if (ptr_kind == PGMPM_PTR_DEVICE) {
        CK(launch_grid_download(V, scene, sc, mass, velocity, st));
        return PGMPM_OK;
    }
    DevBuf tmp;
    CK(tmp.alloc(sizeof(float) * 4 * nodes));
    float* dm = tmp.as<float>();
    float* dv = dm + nodes;
    CK(launch_grid_download(V, scene, sc, dm, dv, st));
    if (mass) CK(cudaMemcpyAsync(mass, dm, sizeof(float) * nodes, cudaMemcpyDeviceToHost, st));
    if (velocity) CK(cudaMemcpyAsync(velocity, dv, sizeof(float) * 3 * nodes, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return PGMPM_OK;
}

int pgmpm_step(pgmpm_solver s, int32_t n_steps, void* stream) {
    if (!s || n_steps < 0) return fail(PGMPM_ERR_ARG, "bad arguments");
    DeviceGuard dg(s->device);
    return run_steps(s, n_steps, ST(stream));
}

int pgmpm_advance_host(pgmpm_solver s, const float* x_in, const float* v_in, const float* C_in, const float* F_in,
                       const float* m, const float* V0, const int32_t* mat, int32_t n_steps, float* x_out,
                       float* v_out, float* C_out, float* F_out, void* stream) {
    int rc = pgmpm_upload(s, x_in, v_in, C_in, F_in, m, V0, mat, PGMPM_PTR_HOST, stream);
    if (rc) return rc;
    rc = pgmpm_step(s, n_steps, stream);
    if (rc) return rc;
    return pgmpm_download(s, x_out, v_out, C_out, F_out, PGMPM_PTR_HOST, stream);
}

int pgmpm_check_status(pgmpm_solver s, uint32_t* flags, void* stream) {
    if (!s || !flags) return fail(PGMPM_ERR_ARG, "bad arguments");
    DeviceGuard dg(s->device);
    cudaStream_t st = ST(stream);
    CK(cudaMemcpyAsync(s->h_counters, s->counters.p, sizeof(uint32_t) * CNT_WORDS, cudaMemcpyDeviceToHost, st));
    CK(cudaMemsetAsync(s->counters.as<uint32_t>() + CNT_FLAGS, 0, sizeof(uint32_t), st));
    CK(cudaStreamSynchronize(st));
    *flags = s->h_counters[CNT_FLAGS];
    uint64_t act;
    std::memcpy(&act, &s->h_counters[CNT_ACTIVE], sizeof(act));
    s->met.active_nodes = (int64_t)act;
    return PGMPM_OK;
}

int pgmpm_set_tuning(pgmpm_solver s, int32_t p2g_block, int32_t ppt, int32_t g2p_block, int32_t use_graph) {
    if (!s) return fail(PGMPM_ERR_ARG, "null solver");
    auto okb = [](int b) { return b == 0 || (b >= 64 && b <= 512 && b % 64 == 0); };
    if (!okb(p2g_block) || !okb(g2p_block)) return fail(PGMPM_ERR_ARG, "block sizes must be 64..512, multiple of 64");
    if (ppt != 0 && (ppt < 32 || ppt > (1 << 20))) return fail(PGMPM_ERR_ARG, "ppt must be in [32, 2^20]");
    if (p2g_block) s->tune.p2g_block = p2g_block;
    if (ppt) s->tune.ppt = ppt;
    if (g2p_block) s->tune.g2p_block = g2p_block;
    if (use_graph >= 0) s->use_graph = use_graph != 0;
    s->drop_graph();
    return PGMPM_OK;
}

int pgmpm_set_kernel_variants(pgmpm_solver s, int32_t p2g_variant, int32_t g2p_variant, int32_t p2g_tiles_per_sm,
                              int32_t g2p_tiles_per_sm) {
    if (!s) return fail(PGMPM_ERR_ARG, "null solver");
    if (p2g_variant > 5 || g2p_variant > 2 || p2g_tiles_per_sm > 16 || g2p_tiles_per_sm > 16)
        return fail(PGMPM_ERR_ARG, "p2g_variant 0..5, g2p_variant 0..2; blocks per SM at most 16");
    if (s->sp_cap && ((p2g_variant >= 0 && p2g_variant != 4) || (g2p_variant >= 0 && g2p_variant != 2)))
        return fail(PGMPM_ERR_UNSUPPORTED, "sparse grids run P2G variant 4 and G2P variant 2 only");
    if (p2g_variant == 5 && p2g_tiles_per_sm > 0 && p2g_tiles_per_sm != 4 && p2g_tiles_per_sm != 6)
        return fail(PGMPM_ERR_ARG, "p2g_variant 5 runs 4 or 6 blocks per SM");
    if (p2g_variant >= 0) s->tune.p2g_variant = p2g_variant;
    if (g2p_variant >= 0) s->tune.g2p_variant = g2p_variant;
    if (p2g_tiles_per_sm > 0) {
        if (s->tune.p2g_variant == 5)
            s->tune.g2p2g_blocks_per_sm = p2g_tiles_per_sm;
        else if (s->tune.p2g_variant == 2)
            s->tune.cell_blocks_per_sm = p2g_tiles_per_sm;
        else if (s->tune.p2g_variant >= 3)
            s->tune.pair_blocks_per_sm = std::min(p2g_tiles_per_sm, 5);
        else
            s->tune.tile_blocks_per_sm = p2g_tiles_per_sm;
    }
    if (g2p_tiles_per_sm > 0) s->tune.g2p_tiles_per_sm = g2p_tiles_per_sm;
    s->drop_graph();
    return PGMPM_OK;
}

int pgmpm_set_sort_record(pgmpm_solver s, int32_t on) {
    if (!s) return fail(PGMPM_ERR_ARG, "null solver");
    if (on < 0 || on > 2) return fail(PGMPM_ERR_ARG, "on must be 0, 1 or 2");
    s->rec_mode = on;  // from the next pgmpm_forward_checkpointed on
    s->drop_tape_graphs();
    return PGMPM_OK;
}

int pgmpm_get_replay_resorts(pgmpm_solver s, int64_t* steps) {
    if (!s || !steps) return fail(PGMPM_ERR_ARG, "null argument");
    *steps = 0;
    if (!s->rec_resort.p) return PGMPM_OK;
    DeviceGuard dg(s->device);
    uint32_t c = 0;
    CK(cudaMemcpy(&c, s->rec_resort.as<uint32_t>() + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    *steps = c;
    return PGMPM_OK;
}

int pgmpm_set_step_sort(pgmpm_solver s, int32_t kind) {
    if (!s) return fail(PGMPM_ERR_ARG, "null solver");
    if (kind != PGMPM_SORT_BINS && kind != PGMPM_SORT_RADIX)
        return fail(PGMPM_ERR_ARG, "kind must be PGMPM_SORT_BINS or PGMPM_SORT_RADIX");
    if (s->sp_cap && kind != PGMPM_SORT_BINS) return fail(PGMPM_ERR_UNSUPPORTED, "sparse grids use the bin sort");
    if (kind == PGMPM_SORT_BINS) {
        DeviceGuard dg(s->device);
        int rc = alloc_bin_sort(s);
        if (rc) return rc;
    }
    s->tune.step_sort = kind;
    s->drop_graph();
    return PGMPM_OK;
}

int pgmpm_set_profiling(pgmpm_solver s, int32_t profile) {
    if (!s) return fail(PGMPM_ERR_ARG, "null solver");
    s->profiling = profile != 0;
    return PGMPM_OK;
}

int pgmpm_get_metrics(pgmpm_solver s, pgmpm_metrics* out) {
    if (!s || !out) return fail(PGMPM_ERR_ARG, "bad arguments");
    s->met.p2g_block = s->tune.p2g_block;
    s->met.p2g_ppt = s->tune.ppt;
    s->met.g2p_block = s->tune.g2p_block;
    s->met.graph_enabled = s->use_graph ? 1 : 0;
    s->met.p2g_variant = s->tune.p2g_variant;
    s->met.g2p_variant = s->tune.g2p_variant;
    s->met.p2g_tiles_per_sm = s->tune.p2g_variant == 5   ? s->tune.g2p2g_blocks_per_sm
                              : s->tune.p2g_variant == 2 ? s->tune.cell_blocks_per_sm
                              : s->tune.p2g_variant >= 3 ? s->tune.pair_blocks_per_sm
                                                         : s->tune.tile_blocks_per_sm;
    s->met.g2p_tiles_per_sm = s->tune.g2p_tiles_per_sm;
    *out = s->met;
    return PGMPM_OK;
}

int pgmpm_autotune(pgmpm_solver s, int32_t reps, void* stream) {
    if (!s) return fail(PGMPM_ERR_ARG, "null solver");
    if (!s->uploaded) return fail(PGMPM_ERR_STATE, "upload particles before autotuning");
    if (s->N == 0 || s->sp_cap) return PGMPM_OK;  // sparse grids have one kernel set
    DeviceGuard dg(s->device);
    cudaStream_t st = ST(stream);
    if (reps < 1) reps = 3;
    int rc0 = unprime(s, st);  // the trials run split steps from the payload
    if (rc0) return rc0;
    // save state (planes + keys) and restore after the trials
    DevBuf save;
    const size_t qb = sizeof(float4) * 6 * (size_t)s->N;
    CK(save.alloc(qb + sizeof(uint32_t) * s->N));
    CK(cudaMemcpyAsync(save.p, s->q.p, qb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(save.as<char>() + qb, s->keys.p, sizeof(uint32_t) * s->N, cudaMemcpyDeviceToDevice, st));
    const Tuning keep = s->tune;
    const bool keep_graph = s->use_graph, keep_prof = s->profiling;
    s->use_graph = false;
    s->profiling = false;
    // candidates: the tile kernels at several resident blocks per SM, and the
    // chunked / direct variants over (block size, particles per chunk)
    struct Cand {
        int variant, block, ppt, tiles_per_sm;
    };
    const Cand p2g_c[] = {{4, 128, 0, 4}, {4, 128, 0, 5}, {3, 128, 0, 4}, {3, 128, 0, 5}, {2, 64, 0, 4}, {2, 64, 0, 6}, {2, 64, 0, 8},
                          {0, 192, 0, 2}, {0, 192, 0, 3}, {1, 256, 512, 0}, {1, 256, 1024, 0}};
    const Cand g2p_c[] = {{2, 128, 0, 0}, {2, 256, 0, 0}, {2, 512, 0, 0}, {0, 256, 0, 2},
                          {1, 128, 0, 0}, {1, 256, 0, 0}};
    Tuning best = keep;
    float best_p2g = 1e30f, best_g2p = 1e30f;
    View V = s->view();
    auto time_it = [&](auto&& fn, int cursor, float& ms) -> int {
        CK(cudaEventRecord(s->ev[0], st));
        for (int r = 0; r < reps; ++r) {
            CK(cudaMemsetAsync(s->counters.as<uint32_t>() + cursor, 0, sizeof(uint32_t), st));
            CK(fn());
        }
        CK(cudaEventRecord(s->ev[1], st));
        CK(cudaEventSynchronize(s->ev[1]));
        CK(cudaEventElapsedTime(&ms, s->ev[0], s->ev[1]));
        return PGMPM_OK;
    };
    // one real step so the sorted order, tile lists and grid velocity exist
    int rc = record_step(s, s->live_bufs(), st, false);
    if (rc) return rc;
    for (const Cand& c : p2g_c) {
        Tuning t = keep;
        t.p2g_variant = c.variant;
        if (c.variant == 0) {
            t.tile_blocks_per_sm = c.tiles_per_sm;
        } else if (c.variant == 2) {
            t.cell_blocks_per_sm = c.tiles_per_sm;
        } else if (c.variant >= 3) {
            t.pair_blocks_per_sm = c.tiles_per_sm;
        } else {
            t.p2g_block = c.block;
            t.ppt = c.ppt;
        }
        float ms = 0.f;
        rc = time_it([&]() { return launch_p2g(V, s->pf, t, s->num_sms, st); }, CNT_P2G_CURSOR, ms);
        if (rc) return rc;
        if (ms < best_p2g) {
            best_p2g = ms;
            best.p2g_variant = t.p2g_variant;
            best.tile_blocks_per_sm = t.tile_blocks_per_sm;
            best.cell_blocks_per_sm = t.cell_blocks_per_sm;
            best.pair_blocks_per_sm = t.pair_blocks_per_sm;
            best.p2g_block = t.p2g_block;
            best.ppt = t.ppt;
        }
    }
    for (const Cand& c : g2p_c) {
        Tuning t = best;
        t.g2p_variant = c.variant;
        t.g2p_block = c.block;
        if (c.variant == 0) t.g2p_tiles_per_sm = c.tiles_per_sm;
        float ms = 0.f;
        rc = time_it([&]() { return launch_g2p(V, s->pf, t, s->num_sms, st); }, CNT_G2P_CURSOR, ms);
        if (rc) return rc;
        if (ms < best_g2p) {
            best_g2p = ms;
            best.g2p_variant = t.g2p_variant;
            best.g2p_block = t.g2p_block;
            best.g2p_tiles_per_sm = t.g2p_tiles_per_sm;
        }
    }
    // the fused path runs variant 4's P2G for the first step of a chain
    if (keep.p2g_variant == 5 && best.p2g_variant == 4) {
        best.p2g_variant = 5;
        best.g2p2g_blocks_per_sm = keep.g2p2g_blocks_per_sm;
    }
    // restore: state, keys, clean accumulator grid
    CK(cudaMemcpyAsync(s->q.p, save.p, qb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s->keys.p, save.as<char>() + qb, sizeof(uint32_t) * s->N, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemsetAsync(s->grid_mp.p, 0, s->grid_mp.bytes, st));
    rc = refresh_payload(s, st);
    if (rc) return rc;
    CK(cudaStreamSynchronize(st));
    s->tune = best;
    s->use_graph = keep_graph;
    s->profiling = keep_prof;
    s->drop_graph();
    return PGMPM_OK;
}

int pgmpm_get_array(pgmpm_solver s, int32_t which, uint32_t* out, int32_t ptr_kind, void* stream) {
    if (!s || !out) return fail(PGMPM_ERR_ARG, "bad arguments");
    DeviceGuard dg(s->device);
    const void* src = nullptr;
    switch (which) {
        case PGMPM_ARRAY_USER_INDEX: src = s->user_of_phys.p; break;
        case PGMPM_ARRAY_KEYS: src = s->keys.p; break;
        case PGMPM_ARRAY_SORTED_KEYS: src = s->sort_which ? s->kb.p : s->ka.p; break;
        case PGMPM_ARRAY_SORTED_ORDER: src = s->sort_which ? s->vb.p : s->va.p; break;
        default: return fail(PGMPM_ERR_ARG, "unknown array %d", which);
    }
    if (s->N == 0) return PGMPM_OK;
    cudaStream_t st = ST(stream);
    CK(cudaMemcpyAsync(out, src, sizeof(uint32_t) * s->N,
                       ptr_kind == PGMPM_PTR_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return PGMPM_OK;
}

int pgmpm_radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out, uint32_t* vals_out,
                           int64_t n, int32_t key_bits, void* stream) {
    if (n < 0 || (n > 0 && (!keys_in || !keys_out || !vals_out)) || key_bits < 1 || key_bits > 32)
        return fail(PGMPM_ERR_ARG, "bad arguments");
    if (n == 0) return PGMPM_OK;
    cudaStream_t st = ST(stream);
    DevBuf a, b, sc;
    CK(a.alloc(sizeof(uint32_t) * 2 * n));
    CK(b.alloc(sizeof(uint32_t) * 2 * n));
    CK(sc.alloc(sizeof(uint32_t) * radix_sort_scratch_words(n)));
    int which = 0;
    uint32_t* ka = a.as<uint32_t>();
    uint32_t* kb = b.as<uint32_t>();
    CK(radix_sort_pairs(keys_in, vals_in, ka, ka + n, kb, kb + n, sc.as<uint32_t>(), n, key_bits, &which, st));
    const uint32_t* rk = which ? kb : ka;
    CK(cudaMemcpyAsync(keys_out, rk, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(vals_out, rk + n, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
    CK(cudaStreamSynchronize(st));
    return PGMPM_OK;
}

}  // extern "C"
