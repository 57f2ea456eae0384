// pgmpm_hashgrid.cu -- spatial hash grid for particle neighbourhoods on the
// GPU: the structure of physgrad::sparse::SpatialHashGrid<float, uint32_t>
// (src/sparse_data_structures.h:44-296; used by the FSI coupling,
// src/fsi_coupling.h:72), with its build and neighbour query as kernels.
//
//   cell id    morton(c) % total_cells, c = the cell coordinates of a point,
//              truncated to uint32 and clamped to the resolution (the
//              reference's getCellID, :143-151, Morton code :121-131)
//   build      per-cell counts (a histogram of the cell ids), starts (their
//              exclusive scan) and a stable sort of (cell id, particle index)
//              pairs (the existing LSD radix sort): the reference's count /
//              exclusive scan / stable fill (:155-190) give the same arrays
//   neighbours for a query point, every particle stored in the cells of the
//              (2 ceil(r / cell) + 1)^3 block around its cell, in the
//              reference's order (x outer, z inner; a cell's particles by
//              index), with no distance test -- as getNeighbors (:206-240),
//              which computes radius^2 but does not use it.  Two passes: a
//              count (thread per query), a scan into offsets, then the fill
//              (8 lanes per query, so each list is written contiguously).
//
// Float arithmetic is IEEE single (no contraction), so cell ids match the
// reference's host code bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "pgmpm_solver_impl.h"

using namespace pgmpm;

struct pgmpm_hashgrid_s {
    int device = 0;
    float cell = 0.f;
    float dmin[3] = {0.f, 0.f, 0.f};
    uint32_t res[3] = {0, 0, 0};
    uint32_t total = 0;
    int key_bits = 1;
    int64_t max_particles = 0;
    int64_t n = 0;  // particles of the last build
    bool built = false;
    DevBuf counts, starts;          // per cell
    DevBuf cell_ids;                // per particle: cell id (particle order)
    DevBuf ka, va, kb, vb, scratch, pos_stage;  // sort buffers; va keeps the sorted particle indices
    DevBuf qcount, qstage, qout_stage, scan_tmp, stats;  // query scratch, kept between calls
};

namespace {

constexpr int HG_T = 256;

struct HGDev {
    float cell, dmin[3];
    uint32_t res[3], total;
    unsigned long long total_m;  // 2^64 / total + 1 (mod 2^64), for hg_mod
};

// a % total by direct computation of the remainder (Lemire, Kaser and Kurz,
// "Faster remainder by direct computation", 2019): for 32-bit a and d and
// M = floor(2^64 / d) + 1, a mod d = floor(((M a) mod 2^64) d / 2^64).
__device__ __forceinline__ uint32_t hg_mod(uint32_t a, const HGDev& G) {
    return (uint32_t)__umul64hi(G.total_m * (unsigned long long)a, (unsigned long long)G.total);
}

// src/sparse_data_structures.h:121-128: bit interleave in uint32 arithmetic
__device__ __forceinline__ uint32_t hg_expand(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
__device__ __forceinline__ uint32_t hg_morton(uint32_t x, uint32_t y, uint32_t z) {
    return hg_expand(x) | (hg_expand(y) << 1) | (hg_expand(z) << 2);
}
// (x - min) / cell in IEEE single, truncated toward zero to a 64-bit integer
// and reduced mod 2^32: the host's float -> uint32 conversion
__device__ __forceinline__ uint32_t hg_coord(float x, float mn, float cell) {
    return (uint32_t)(unsigned long long)__float2ll_rz(__fdiv_rn(__fsub_rn(x, mn), cell));
}

// cell id per particle, and the per-cell counts (one atomic per particle:
// input order is arbitrary, so a warp's particles rarely share a cell and
// aggregating them over the warp cost more than it saved)
__global__ void k_hg_cells(HGDev G, const float* __restrict__ pos, int64_t n, uint32_t* __restrict__ cell_ids,
                           uint32_t* __restrict__ counts) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t c[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) c[a] = min(hg_coord(pos[3 * i + a], G.dmin[a], G.cell), G.res[a] - 1u);
    const uint32_t id = hg_mod(hg_morton(c[0], c[1], c[2]), G);
    cell_ids[i] = id;
    atomicAdd(&counts[id], 1u);
}

// Fill pass, HG_FG lanes per query: they take the block's cells in the
// reference's order (linear index t = (dx (2s+1) + dy) (2s+1) + dz), HG_FG at
// a time, give each cell its place by a scan over the lanes and copy the
// cell's particles, so a query's list is written into one contiguous stretch
// by its lanes together.
// (dx, dy, dz) of cell t of the block, packed 10 bits each, for the block's
// cells in shared memory when there are at most HG_TAB of them
constexpr int HG_TAB = 1024;
__device__ __forceinline__ uint32_t hg_offsets(uint32_t t, uint32_t w) {
    return (t % w) << 20 | ((t / w) % w) << 10 | (t / (w * w));
}
__device__ __forceinline__ void hg_fill_table(uint32_t* tab, uint32_t ncell, uint32_t w) {
    if (ncell <= (uint32_t)HG_TAB)
        for (uint32_t t = threadIdx.x; t < ncell; t += blockDim.x) tab[t] = hg_offsets(t, w);
    __syncthreads();
}
__device__ __forceinline__ bool hg_cell_of(const HGDev& G, const uint32_t c[3], uint32_t src, uint32_t w,
                                           uint32_t ncell, const uint32_t* tab, uint32_t t, uint32_t& id) {
    const uint32_t o = ncell <= (uint32_t)HG_TAB ? tab[t] : hg_offsets(t, w);
    const uint32_t dx = o & 1023u, dy = (o >> 10) & 1023u, dz = o >> 20;
    const uint32_t gx = c[0] + dx - src, gy = c[1] + dy - src, gz = c[2] + dz - src;  // wrap: below 0 fails
    if (gx >= G.res[0] || gy >= G.res[1] || gz >= G.res[2]) return false;
    id = hg_mod(hg_morton(gx, gy, gz), G);
    return true;
}

// Count pass, one thread per query: the block's cells in nested loops (the
// reference's order does not matter for a sum)
__global__ void k_hg_qcount(HGDev G, const float* __restrict__ q, int64_t nq, uint32_t src,
                            const uint32_t* __restrict__ counts, uint32_t* __restrict__ qcount) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nq) return;
    uint32_t c[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) c[a] = hg_coord(q[3 * i + a], G.dmin[a], G.cell);
    uint32_t k = 0;
    for (uint32_t dx = 0; dx <= 2 * src; ++dx) {
        const uint32_t gx = c[0] + dx - src;  // uint32 wrap: below 0 fails the range test
        if (gx >= G.res[0]) continue;
        for (uint32_t dy = 0; dy <= 2 * src; ++dy) {
            const uint32_t gy = c[1] + dy - src;
            if (gy >= G.res[1]) continue;
            for (uint32_t dz = 0; dz <= 2 * src; ++dz) {
                const uint32_t gz = c[2] + dz - src;
                if (gz >= G.res[2]) continue;
                k += counts[hg_mod(hg_morton(gx, gy, gz), G)];
            }
        }
    }
    qcount[i] = k;
}

constexpr int HG_FG = 8;  // lanes per query in the fill (4 queries per warp; 4 lanes and 32 were slower)
__global__ void k_hg_qfill(HGDev G, const float* __restrict__ q, int64_t nq, uint32_t src,
                           const uint32_t* __restrict__ counts, const uint32_t* __restrict__ starts,
                           const uint32_t* __restrict__ sorted_index, const int64_t* __restrict__ offsets,
                           uint32_t* __restrict__ out) {
    __shared__ uint32_t tab[HG_TAB];
    const uint32_t w = 2 * src + 1, ncell = w * w * w;
    hg_fill_table(tab, ncell, w);
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / HG_FG;
    const int lane = threadIdx.x & 31, sub = lane % HG_FG;
    const uint32_t gmask = ((1u << HG_FG) - 1u) << (lane - sub);  // this query's lanes
    if (i >= nq) return;  // a query's lanes leave together
    uint32_t c[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) c[a] = hg_coord(q[3 * i + a], G.dmin[a], G.cell);
    int64_t o = offsets[i];
    for (uint32_t t0 = 0; t0 < ncell; t0 += HG_FG) {
        const uint32_t t = t0 + sub;
        uint32_t id = 0, k = 0, s0 = 0;
        if (t < ncell && hg_cell_of(G, c, src, w, ncell, tab, t, id)) {
            k = counts[id];
            s0 = starts[id];
        }
        uint32_t x = k;  // inclusive scan of the counts over the query's lanes
#pragma unroll
        for (int d = 1; d < HG_FG; d <<= 1) {
            const uint32_t y = __shfl_up_sync(gmask, x, d, HG_FG);
            if (sub >= d) x += y;
        }
        const uint32_t kmax = __reduce_max_sync(gmask, k);
        if (kmax < 2 * HG_FG) {
            // short cells: each lane copies its own cell's entries
            const int64_t base = o + (x - k);
            for (uint32_t j = 0; j < k; ++j) out[base + j] = sorted_index[s0 + j];
        } else {
            // long cells: the query's lanes copy each cell together, so the
            // list is written (and the sorted index read) in runs
#pragma unroll 1
            for (int m = 0; m < HG_FG; ++m) {
                const uint32_t km = __shfl_sync(gmask, k, m, HG_FG);
                const uint32_t sm = __shfl_sync(gmask, s0, m, HG_FG);
                const int64_t bm = o + (__shfl_sync(gmask, x, m, HG_FG) - km);
                for (uint32_t j = (uint32_t)sub; j < km; j += HG_FG) out[bm + j] = sorted_index[sm + j];
            }
        }
        o += __shfl_sync(gmask, x, HG_FG - 1, HG_FG);
    }
}

// Exclusive scan of n uint32 counts into int64 offsets[0..n] (offsets[n] =
// total): per-block sums, one block scanning the sums, then each block's
// scan plus its carry.
constexpr int SCAN_T = 1024;
__device__ __forceinline__ int64_t block_incl_scan(int64_t x, int64_t* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int64_t w = lane < SCAN_T / 32 ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= o) w += y;
        }
        sh[lane] = w;
    }
    __syncthreads();
    const int64_t r = x + (warp ? sh[warp - 1] : 0);
    __syncthreads();
    return r;
}
__global__ void __launch_bounds__(SCAN_T) k_scan_sums(const uint32_t* __restrict__ in, int64_t n,
                                                      int64_t* __restrict__ bsum) {
    __shared__ int64_t sh[32];
    const int64_t i = (int64_t)blockIdx.x * SCAN_T + threadIdx.x;
    const int64_t r = block_incl_scan(i < n ? in[i] : 0, sh);
    if (threadIdx.x == SCAN_T - 1) bsum[blockIdx.x] = r;
}
__global__ void __launch_bounds__(SCAN_T) k_scan_carry(int64_t* __restrict__ bsum, int64_t nb) {
    __shared__ int64_t sh[32];
    __shared__ int64_t s_tot;
    int64_t carry = 0;
    for (int64_t b0 = 0; b0 < nb; b0 += SCAN_T) {
        const int64_t i = b0 + threadIdx.x;
        const int64_t v = i < nb ? bsum[i] : 0;
        const int64_t r = block_incl_scan(v, sh);
        if (i < nb) bsum[i] = carry + r - v;  // exclusive, over all blocks so far
        if (threadIdx.x == SCAN_T - 1) s_tot = r;
        __syncthreads();
        carry += s_tot;
        __syncthreads();
    }
}
// OutT: int64 query offsets (with the total in out[n]) or uint32 cell starts
template <class OutT, bool TOTAL>
__global__ void __launch_bounds__(SCAN_T) k_scan_apply(const uint32_t* __restrict__ in, int64_t n,
                                                       const int64_t* __restrict__ bsum, OutT* __restrict__ out) {
    __shared__ int64_t sh[32];
    const int64_t i = (int64_t)blockIdx.x * SCAN_T + threadIdx.x;
    const int64_t v = i < n ? in[i] : 0;
    const int64_t r = block_incl_scan(v, sh);
    if (i < n) out[i] = (OutT)(bsum[blockIdx.x] + r - v);
    if (TOTAL && i == n - 1) out[n] = (OutT)(bsum[blockIdx.x] + r);
}

__global__ void k_hg_stats(const uint32_t* __restrict__ counts, uint32_t total,
                           unsigned long long* __restrict__ st) {  // occupied, max, particles
    uint32_t occ = 0, mx = 0;
    unsigned long long sum = 0;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < total; c += gridDim.x * blockDim.x) {
        const uint32_t k = counts[c];
        occ += k > 0;
        mx = max(mx, k);
        sum += k;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        occ += __shfl_down_sync(0xFFFFFFFFu, occ, o);
        mx = max(mx, __shfl_down_sync(0xFFFFFFFFu, mx, o));
        sum += __shfl_down_sync(0xFFFFFFFFu, sum, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&st[0], (unsigned long long)occ);
        atomicMax(&st[1], (unsigned long long)mx);
        atomicAdd(&st[2], sum);
    }
}

HGDev dev_of(const pgmpm_hashgrid_s* g) {
    HGDev d;
    d.cell = g->cell;
    for (int a = 0; a < 3; ++a) {
        d.dmin[a] = g->dmin[a];
        d.res[a] = g->res[a];
    }
    d.total = g->total;
    d.total_m = ~0ull / g->total + 1ull;  // wraps to 0 for total = 1, where every remainder is 0
    return d;
}

int blocks_of(int64_t n, int t) { return (int)std::max<int64_t>(1, (n + t - 1) / t); }

// copies nfloat floats from host (or takes the device pointer) into stage
const float* staged(DevBuf& stage, const float* p, int64_t nfloat, int32_t kind, cudaStream_t st, int& rc) {
    rc = PGMPM_OK;
    if (kind == PGMPM_PTR_DEVICE) return p;
    if (stage.ensure(sizeof(float) * std::max<int64_t>(nfloat, 1)) != cudaSuccess) {
        rc = fail(PGMPM_ERR_OOM, "hashgrid: staging allocation failed");
        return nullptr;
    }
    if (nfloat && cudaMemcpyAsync(stage.p, p, sizeof(float) * nfloat, cudaMemcpyHostToDevice, st) != cudaSuccess) {
        rc = fail(PGMPM_ERR_CUDA, "hashgrid: host copy failed");
        return nullptr;
    }
    return stage.as<float>();
}

}  // namespace

extern "C" {

int pgmpm_hashgrid_create(float cell_size, const float* domain_min, const float* domain_max, int64_t max_particles,
                          int32_t device, pgmpm_hashgrid* out) {
    if (!out || !domain_min || !domain_max) return fail(PGMPM_ERR_ARG, "hashgrid: null argument");
    *out = nullptr;
    if (!(cell_size > 0.f) || !std::isfinite(cell_size) || max_particles < 0 || max_particles > 0xFFFFFFFFll)
        return fail(PGMPM_ERR_ARG, "hashgrid: cell_size > 0 and 0 <= max_particles < 2^32 required");
    auto* g = new pgmpm_hashgrid_s();
    g->device = device;
    g->cell = cell_size;
    uint64_t total = 1;
    for (int a = 0; a < 3; ++a) {
        g->dmin[a] = domain_min[a];
        const float r = std::ceil((domain_max[a] - domain_min[a]) / cell_size);  // single precision, as the host class
        if (!(r >= 1.f) || !(r < 4294967296.f)) {
            delete g;
            return fail(PGMPM_ERR_ARG, "hashgrid: each axis needs 1 .. 2^32-1 cells");
        }
        g->res[a] = (uint32_t)r;
        total *= g->res[a];
    }
    if (total > 0xFFFFFFFFull) {
        delete g;
        return fail(PGMPM_ERR_ARG, "hashgrid: more than 2^32 - 1 cells");
    }
    g->total = (uint32_t)total;
    g->key_bits = std::max(1, bits_for(total));
    g->max_particles = max_particles;
    DeviceGuard dg(device);
    const size_t n = (size_t)std::max<int64_t>(max_particles, 1);
    cudaError_t e = g->counts.alloc(sizeof(uint32_t) * total);
    if (e == cudaSuccess) e = g->starts.alloc(sizeof(uint32_t) * total);
    if (e == cudaSuccess) e = g->cell_ids.alloc(sizeof(uint32_t) * n);
    if (e == cudaSuccess) e = g->ka.alloc(sizeof(uint32_t) * n);
    if (e == cudaSuccess) e = g->va.alloc(sizeof(uint32_t) * n);
    if (e == cudaSuccess) e = g->kb.alloc(sizeof(uint32_t) * n);
    if (e == cudaSuccess) e = g->vb.alloc(sizeof(uint32_t) * n);
    if (e == cudaSuccess) e = g->scratch.alloc(sizeof(uint32_t) * radix_sort_scratch_words((int64_t)n));
    if (e == cudaSuccess) e = g->stats.alloc(sizeof(unsigned long long) * 3);
    if (e != cudaSuccess) {
        delete g;
        return fail(e == cudaErrorMemoryAllocation ? PGMPM_ERR_OOM : PGMPM_ERR_CUDA, "hashgrid: %s",
                    cudaGetErrorString(e));
    }
    *out = g;
    return PGMPM_OK;
}

int pgmpm_hashgrid_destroy(pgmpm_hashgrid g) {
    if (!g) return PGMPM_OK;
    DeviceGuard dg(g->device);
    delete g;
    return PGMPM_OK;
}

int pgmpm_hashgrid_build(pgmpm_hashgrid g, const float* positions, int64_t n, int32_t ptr_kind, void* stream) {
    if (!g || n < 0 || (n > 0 && !positions)) return fail(PGMPM_ERR_ARG, "hashgrid: bad arguments");
    if (n > g->max_particles) return fail(PGMPM_ERR_ARG, "hashgrid: more particles than max_particles");
    if (ptr_kind != PGMPM_PTR_HOST && ptr_kind != PGMPM_PTR_DEVICE) return fail(PGMPM_ERR_ARG, "bad ptr_kind");
    DeviceGuard dg(g->device);
    cudaStream_t st = ST(stream);
    int rc;
    const float* pos = staged(g->pos_stage, positions, 3 * n, ptr_kind, st, rc);
    if (rc) return rc;
    const HGDev G = dev_of(g);
    uint32_t* ids = g->cell_ids.as<uint32_t>();
    uint32_t* counts = g->counts.as<uint32_t>();
    const uint32_t* sorted_index = nullptr;
    // per-cell counts (histogram of the cell ids), starts = their exclusive scan
    CK(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * g->total, st));
    if (n > 0) {
        k_hg_cells<<<blocks_of(n, HG_T), HG_T, 0, st>>>(G, pos, n, ids, counts);
        CK(cudaGetLastError());
    }
    const int64_t nb = ((int64_t)g->total + SCAN_T - 1) / SCAN_T;
    CK(g->scan_tmp.ensure(sizeof(int64_t) * nb));
    int64_t* bsum = g->scan_tmp.as<int64_t>();
    k_scan_sums<<<(int)nb, SCAN_T, 0, st>>>(counts, g->total, bsum);
    k_scan_carry<<<1, SCAN_T, 0, st>>>(bsum, nb);
    k_scan_apply<uint32_t, false><<<(int)nb, SCAN_T, 0, st>>>(counts, g->total, bsum, g->starts.as<uint32_t>());
    CK(cudaGetLastError());
    // particles ordered by cell, by index within a cell (stable sort)
    if (n > 0) {
        int which = 0;
        CK(radix_sort_pairs(ids, nullptr, g->ka.as<uint32_t>(), g->va.as<uint32_t>(), g->kb.as<uint32_t>(),
                            g->vb.as<uint32_t>(), g->scratch.as<uint32_t>(), n, g->key_bits, &which, st));
        sorted_index = which ? g->vb.as<uint32_t>() : g->va.as<uint32_t>();
    }
    // keep the sorted indices where queries read them
    if (n > 0 && sorted_index != g->va.as<uint32_t>())
        CK(cudaMemcpyAsync(g->va.p, sorted_index, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
    g->n = n;
    g->built = true;
    return PGMPM_OK;
}

int pgmpm_hashgrid_get_table(pgmpm_hashgrid g, uint32_t* counts, uint32_t* starts, uint32_t* particle_indices,
                             uint32_t* cell_ids, int32_t ptr_kind, void* stream) {
    if (!g || !g->built) return fail(PGMPM_ERR_STATE, "hashgrid: build first");
    if (ptr_kind != PGMPM_PTR_HOST && ptr_kind != PGMPM_PTR_DEVICE) return fail(PGMPM_ERR_ARG, "bad ptr_kind");
    DeviceGuard dg(g->device);
    cudaStream_t st = ST(stream);
    const cudaMemcpyKind k = ptr_kind == PGMPM_PTR_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (counts) CK(cudaMemcpyAsync(counts, g->counts.p, sizeof(uint32_t) * g->total, k, st));
    if (starts) CK(cudaMemcpyAsync(starts, g->starts.p, sizeof(uint32_t) * g->total, k, st));
    if (particle_indices && g->n) CK(cudaMemcpyAsync(particle_indices, g->va.p, sizeof(uint32_t) * g->n, k, st));
    if (cell_ids && g->n) CK(cudaMemcpyAsync(cell_ids, g->cell_ids.p, sizeof(uint32_t) * g->n, k, st));
    if (ptr_kind == PGMPM_PTR_HOST) CK(cudaStreamSynchronize(st));
    return PGMPM_OK;
}

int pgmpm_hashgrid_neighbors(pgmpm_hashgrid g, const float* queries, int64_t nq, float radius, int64_t* offsets,
                             uint32_t* indices, int64_t capacity, int64_t* total, int32_t ptr_kind, void* stream) {
    if (!g || !g->built) return fail(PGMPM_ERR_STATE, "hashgrid: build first");
    if (nq < 0 || (nq > 0 && !queries) || !offsets || !total || capacity < 0 || !(radius >= 0.f) ||
        !std::isfinite(radius))
        return fail(PGMPM_ERR_ARG, "hashgrid: bad query arguments");
    if (ptr_kind != PGMPM_PTR_HOST && ptr_kind != PGMPM_PTR_DEVICE) return fail(PGMPM_ERR_ARG, "bad ptr_kind");
    const float sr = std::ceil(radius / g->cell);  // single precision, as the host class
    // (2 src + 1)^3 cells per query must count in uint32
    if (!(sr < 512.f)) return fail(PGMPM_ERR_ARG, "hashgrid: radius spans more than 511 cells");
    const uint32_t src = (uint32_t)sr;
    DeviceGuard dg(g->device);
    cudaStream_t st = ST(stream);
    int rc;
    const float* q = staged(g->qstage, queries, 3 * nq, ptr_kind, st, rc);
    if (rc) return rc;
    const HGDev G = dev_of(g);
    CK(g->qcount.ensure(sizeof(uint32_t) * std::max<int64_t>(nq, 1)));
    const int64_t nb = std::max<int64_t>(1, (nq + SCAN_T - 1) / SCAN_T);
    // scan_tmp: block sums, then the offsets when the caller's are on the host
    const size_t off_bytes = sizeof(int64_t) * (size_t)(nq + 1);
    CK(g->scan_tmp.ensure(sizeof(int64_t) * nb + (ptr_kind == PGMPM_PTR_HOST ? off_bytes : 0)));
    int64_t* bsum = g->scan_tmp.as<int64_t>();
    int64_t* doff = ptr_kind == PGMPM_PTR_HOST ? bsum + nb : offsets;
    if (nq > 0) {
        k_hg_qcount<<<blocks_of(nq, HG_T), HG_T, 0, st>>>(G, q, nq, src, g->counts.as<uint32_t>(),
                                                          g->qcount.as<uint32_t>());
        k_scan_sums<<<(int)nb, SCAN_T, 0, st>>>(g->qcount.as<uint32_t>(), nq, bsum);
        k_scan_carry<<<1, SCAN_T, 0, st>>>(bsum, nb);
        k_scan_apply<int64_t, true><<<(int)nb, SCAN_T, 0, st>>>(g->qcount.as<uint32_t>(), nq, bsum, doff);
        CK(cudaGetLastError());
    } else {
        CK(cudaMemsetAsync(doff, 0, sizeof(int64_t), st));
    }
    int64_t tot = 0;
    CK(cudaMemcpyAsync(&tot, doff + nq, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    *total = tot;
    if (ptr_kind == PGMPM_PTR_HOST) CK(cudaMemcpyAsync(offsets, doff, off_bytes, cudaMemcpyDeviceToHost, st));
    if (indices && tot <= capacity && tot > 0) {
        uint32_t* dout = indices;
        if (ptr_kind == PGMPM_PTR_HOST) {
            CK(g->qout_stage.ensure(sizeof(uint32_t) * tot));
            dout = g->qout_stage.as<uint32_t>();
        }
        k_hg_qfill<<<blocks_of(nq * HG_FG, HG_T), HG_T, 0, st>>>(G, q, nq, src, g->counts.as<uint32_t>(),
                                                              g->starts.as<uint32_t>(), g->va.as<uint32_t>(), doff,
                                                              dout);
        CK(cudaGetLastError());
        if (ptr_kind == PGMPM_PTR_HOST)
            CK(cudaMemcpyAsync(indices, dout, sizeof(uint32_t) * tot, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    } else if (ptr_kind == PGMPM_PTR_HOST) {
        CK(cudaStreamSynchronize(st));
    }
    return PGMPM_OK;
}

int pgmpm_hashgrid_stats(pgmpm_hashgrid g, pgmpm_hashgrid_info* out) {
    if (!g || !out) return fail(PGMPM_ERR_ARG, "hashgrid: null argument");
    DeviceGuard dg(g->device);
    unsigned long long h[3] = {0, 0, 0};  // before a build: no particles
    if (g->built) {
        CK(cudaMemset(g->stats.p, 0, sizeof(h)));
        k_hg_stats<<<std::min(blocks_of(g->total, HG_T), 148 * 8), HG_T>>>(g->counts.as<uint32_t>(), g->total,
                                                                          g->stats.as<unsigned long long>());
        CK(cudaGetLastError());
        CK(cudaMemcpy(h, g->stats.p, sizeof(h), cudaMemcpyDeviceToHost));
    }
    std::memset(out, 0, sizeof(*out));
    out->occupied_cells = (uint32_t)h[0];
    out->max_particles_per_cell = (uint32_t)h[1];
    out->average_particles_per_cell = (float)h[2] / (float)std::max<unsigned long long>(1, h[0]);
    out->load_factor = (float)h[0] / (float)g->total;
    // the host class's accounting: two words per cell and two per particle slot
    const double bytes = 2.0 * 4.0 * g->total + 2.0 * 4.0 * (double)g->max_particles;
    out->memory_usage_mb = (float)(bytes / (1024.0 * 1024.0));
    out->total_cells = g->total;
    for (int a = 0; a < 3; ++a) out->resolution[a] = g->res[a];
    return PGMPM_OK;
}

}  // extern "C"
