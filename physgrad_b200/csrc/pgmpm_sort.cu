// pgmpm_sort.cu -- stable LSD radix sort of (u32 key, u32 value) pairs.
//
// Each pass sorts by one digit of `bits` (<= 8) bits with three kernels:
//   rs_hist     per-block digit histogram of a 2048-key tile (warp-aggregated
//               shared atomics), written digit-major hist[d][block]
//   rs_scan     one block per digit: exclusive scan of its row over blocks,
//               row totals to totals[d]
//   rs_scatter  block-local stable rank (per-warp ranking with match_any,
//               warp prefix per digit), keys staged in shared memory in
//               block-sorted order, then written out so that consecutive
//               threads store consecutive positions of a digit run.
// Stability: inside a block, warps own contiguous 256-key ranges processed
// in order, lanes in order; across blocks, the digit-major exclusive scan
// orders blocks.  The result is therefore identical to a stable CPU sort.
// Scratch: hist (digits x blocks u32), totals (256 u32), and ping-pong
// (key, value) buffers of n pairs, provided by the caller.
#include "pgmpm_internal.h"

namespace pgmpm {

namespace {
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ITEMS = 8;  // keys per thread per tile
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_MAXD = 256;
static_assert(RS_TILE == RADIX_TILE && RS_MAXD == RADIX_MAX_DIGITS, "scratch sizing must match the kernels");

__global__ void __launch_bounds__(RS_THREADS) rs_hist(const uint32_t* __restrict__ keys, int64_t n, int shift,
                                                      int bits, uint32_t* __restrict__ hist, int nblocks) {
    // warp-private histograms with native integer shared atomics, summed at the end
    __shared__ uint32_t cnt[RS_WARPS][RS_MAXD];
    const int nd = 1 << bits;
    const uint32_t mask = (uint32_t)nd - 1u;
    for (int d = threadIdx.x; d < RS_WARPS * RS_MAXD; d += RS_THREADS) (&cnt[0][0])[d] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t base = (int64_t)blockIdx.x * RS_TILE + warp * (32 * RS_ITEMS);
    uint32_t k[RS_ITEMS];
#pragma unroll
    for (int r = 0; r < RS_ITEMS; ++r) {
        const int64_t i = base + r * 32 + lane;
        k[r] = i < n ? __ldg(keys + i) : 0u;
    }
#pragma unroll
    for (int r = 0; r < RS_ITEMS; ++r) {
        const int64_t i = base + r * 32 + lane;
        if (i < n) atomicAdd(&cnt[warp][(k[r] >> shift) & mask], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < nd; d += RS_THREADS) {
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < RS_WARPS; ++w) s += cnt[w][d];
        hist[(int64_t)d * nblocks + blockIdx.x] = s;
    }
}

// Lanes of the warp holding the same digit as this lane (bits <= 8), built
// from one ballot per digit bit; only lanes with `ok` participate.
__device__ __forceinline__ uint32_t digit_peers(uint32_t d, int bits, bool ok) {
    uint32_t peers = __ballot_sync(0xFFFFFFFFu, ok);
    if (!ok) peers = ~peers;
    for (int b = 0; b < bits; ++b) {
        const bool bit = (d >> b) & 1u;
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, bit);
        peers &= bit ? bal : ~bal;
    }
    return peers;
}

// Block-wide exclusive scan of one value per thread (blockDim.x <= 1024).
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* sh, uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nw ? sh[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= o) w += y;
        }
        sh[lane] = w;  // inclusive warp totals
    }
    __syncthreads();
    const uint32_t before = warp > 0 ? sh[warp - 1] : 0u;
    total = sh[nw - 1];
    __syncthreads();
    return before + x - v;
}

__global__ void __launch_bounds__(1024) rs_scan(uint32_t* __restrict__ hist, int nblocks,
                                                uint32_t* __restrict__ totals) {
    __shared__ uint32_t sh[32];
    uint32_t* row = hist + (int64_t)blockIdx.x * nblocks;
    uint32_t carry = 0;
    for (int b0 = 0; b0 < nblocks; b0 += blockDim.x) {
        const int b = b0 + threadIdx.x;
        const uint32_t v = b < nblocks ? row[b] : 0u;
        uint32_t tot;
        const uint32_t ex = block_excl_scan(v, sh, tot);
        if (b < nblocks) row[b] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

__global__ void __launch_bounds__(RS_THREADS) rs_scatter(const uint32_t* __restrict__ kin,
                                                         const uint32_t* __restrict__ vin,
                                                         uint32_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                         int64_t n, int shift, int bits,
                                                         const uint32_t* __restrict__ hist, int nblocks,
                                                         const uint32_t* __restrict__ totals) {
    __shared__ uint32_t wcnt[RS_WARPS][RS_MAXD];
    __shared__ uint32_t boff[RS_MAXD];   // block-local exclusive digit offsets
    __shared__ uint32_t goff[RS_MAXD];   // global position of this block's first key of digit d
    __shared__ uint32_t skey[RS_TILE];
    __shared__ uint32_t sval[RS_TILE];
    __shared__ uint32_t sh[32];
    const int nd = 1 << bits;
    const uint32_t mask = (uint32_t)nd - 1u;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < RS_WARPS * RS_MAXD; d += RS_THREADS) (&wcnt[0][0])[d] = 0;
    // global digit prefix (exclusive scan of totals) + this block's row offset
    {
        const uint32_t t = threadIdx.x < nd ? totals[threadIdx.x] : 0u;
        uint32_t tot;
        const uint32_t ex = block_excl_scan(t, sh, tot);
        if (threadIdx.x < nd) goff[threadIdx.x] = ex + hist[(int64_t)threadIdx.x * nblocks + blockIdx.x];
    }
    __syncthreads();
    const int64_t tile0 = (int64_t)blockIdx.x * RS_TILE;
    const int64_t base = tile0 + warp * (32 * RS_ITEMS);
    uint32_t k[RS_ITEMS], v[RS_ITEMS], rk[RS_ITEMS];
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < RS_ITEMS; ++r) {
        const int64_t i = base + r * 32 + lane;
        const bool ok = i < n;
        k[r] = ok ? kin[i] : 0xFFFFFFFFu;
        v[r] = ok ? (vin ? vin[i] : (uint32_t)i) : 0u;
        const uint32_t d = ok ? ((k[r] >> shift) & mask) : 0u;
        const uint32_t peers = digit_peers(d, bits, ok);
        uint32_t c = 0u;
        if (ok) c = wcnt[warp][d];
        rk[r] = c + (uint32_t)__popc(peers & lt);
        __syncwarp();
        if (ok && lane == __ffs(peers) - 1) wcnt[warp][d] = c + (uint32_t)__popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive prefix over warps, and block total
    uint32_t mytot = 0u;
    if (threadIdx.x < nd) {
        uint32_t run = 0u;
#pragma unroll
        for (int w = 0; w < RS_WARPS; ++w) {
            const uint32_t c = wcnt[w][threadIdx.x];
            wcnt[w][threadIdx.x] = run;
            run += c;
        }
        mytot = run;
    }
    {
        uint32_t tot;
        const uint32_t ex = block_excl_scan(mytot, sh, tot);
        if (threadIdx.x < nd) boff[threadIdx.x] = ex;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_ITEMS; ++r) {
        const int64_t i = base + r * 32 + lane;
        if (i < n) {
            const uint32_t d = (k[r] >> shift) & mask;
            const uint32_t lp = boff[d] + wcnt[warp][d] + rk[r];
            if (lp < (uint32_t)RS_TILE) {
                skey[lp] = k[r];
                sval[lp] = v[r];
            }
        }
    }
    __syncthreads();
    const int cnt = (int)min((int64_t)RS_TILE, n - tile0);
    for (int j = threadIdx.x; j < cnt; j += RS_THREADS) {
        const uint32_t kk = skey[j];
        const uint32_t d = (kk >> shift) & mask;
        const uint32_t pos = goff[d] + (uint32_t)j - boff[d];
        if ((int64_t)pos < n) {
            kout[pos] = kk;
            vout[pos] = sval[j];
        }
    }
}

// --------------------------------------------------- per-step bin sort
// The MPM step groups particles by cell with a counting sort over the cells
// (key = cell tile << 6 | cell in tile) instead of a full radix sort:
//   bs_count     clears the step's counters (words [0, CNT_RESET));
//                particles per cell and per cell tile, and each particle's
//                slot in its cell.  Lanes holding equal keys in a run (the
//                physical order stays close to cell order) share one atomic:
//                the run's first lane adds the run length.  8 keys per thread
//                with their loads and atomics issued back to back.
//   bs_reduce / bs_down
//                exclusive scan of the tile counts (block totals, then each
//                block adds the totals before it; on grids of up to 64 Ki
//                cell tiles bs_down sums the counts before its range itself
//                and bs_reduce is not launched); bs_down also emits each
//                occupied tile (sorted range, entry in the occupied-tile
//                list, rank in its size class).
//   bs_finish    (a) one warp per occupied tile: scan of its 64 cell counts
//                -> every cell's first sorted position and range, clearing
//                the cell and tile counters, and the tile's slot in the
//                largest-first list P2G takes work from (the last tiles a
//                persistent P2G block picks up are then small ones, which
//                shortens the kernel's tail); (b) one thread per node tile:
//                active iff one of the 8 cell tiles around it is occupied.
//   bs_scatter   particle -> cell offset + slot.
// The counters are left zero for the next step by their readers, so a step
// costs O(N + occupied cells + tiles) with no clearing pass.  Keys come out
// sorted; particles that share a cell in atomic-arrival order, which the
// step does not rely on.
constexpr int BS_T = 256;
constexpr int BS_ITEMS = 8;                 // keys per thread in bs_count / bs_scatter
constexpr int BS_TILE = BS_T * BS_ITEMS;    // keys per block
constexpr int BS_SCAN = 1024;               // tile counts per scan block
// up to this many scan blocks (64 Ki cell tiles, a 256^3 grid) bs_down sums
// the counts before its range directly, without bs_reduce: the last block
// reads at most 63 Ki words from L2
constexpr int BS_DIRECT_BLOCKS = 64;

// Run structure of `bin` over a warp: first lane of this lane's run and one
// past its last lane.  A run is a maximal stretch of consecutive lanes with
// the same bin and the same ok.
__device__ __forceinline__ void bs_run(uint32_t bin, bool ok, int lane, int& start, int& end) {
    const uint32_t prev = __shfl_up_sync(0xFFFFFFFFu, bin, 1);
    const uint32_t okp = __shfl_up_sync(0xFFFFFFFFu, (uint32_t)ok, 1);
    const bool head = lane == 0 || bin != prev || (uint32_t)ok != okp;
    const uint32_t heads = __ballot_sync(0xFFFFFFFFu, head);
    const uint32_t upto = lane == 31 ? 0xFFFFFFFFu : ((2u << lane) - 1u);  // lanes <= this one
    start = 31 - __clz(heads & upto);
    const uint32_t after = heads & ~upto;
    end = after ? __ffs(after) - 1 : 32;
}

__global__ void __launch_bounds__(BS_T) bs_count(const uint32_t* __restrict__ keys, int64_t n, uint32_t ncells,
                                                 uint32_t* __restrict__ ccount, uint32_t* __restrict__ tcount,
                                                 uint32_t* __restrict__ slot, uint32_t* __restrict__ counters) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // the step's per-step counters start at zero: this is the step's first
    // kernel and it reads none of them (the step recording issues no memset)
    if (blockIdx.x == 0 && threadIdx.x < CNT_RESET) counters[threadIdx.x] = 0u;
    // a new step stamp (sparse grids mark active node tiles with it)
    if (blockIdx.x == 0 && threadIdx.x == 0) counters[CNT_STAMP] += 1u;
    const int64_t base = (int64_t)blockIdx.x * BS_TILE + warp * (32 * BS_ITEMS);
    uint32_t k[BS_ITEMS], cb[BS_ITEMS];
    int st[BS_ITEMS];
    bool bad = false;
#pragma unroll
    for (int r = 0; r < BS_ITEMS; ++r) {
        const int64_t i = base + r * 32 + lane;
        k[r] = i < n ? keys[i] : 0u;
        if (i < n && k[r] >= ncells) {  // out-of-range key: overflow bin after the last cell
            bad = true;
            k[r] = ncells;
        }
    }
#pragma unroll
    for (int r = 0; r < BS_ITEMS; ++r) {
        const bool ok = base + r * 32 + lane < n;
        int e, ts, te;
        bs_run(k[r], ok, lane, st[r], e);
        bs_run(k[r] >> 6, ok, lane, ts, te);
        cb[r] = 0u;
        if (ok && lane == st[r]) cb[r] = atomicAdd(&ccount[k[r]], (uint32_t)(e - st[r]));
        if (ok && lane == ts) atomicAdd(&tcount[k[r] >> 6], (uint32_t)(te - ts));
    }
#pragma unroll
    for (int r = 0; r < BS_ITEMS; ++r) {
        const int64_t i = base + r * 32 + lane;
        const uint32_t b = __shfl_sync(0xFFFFFFFFu, cb[r], st[r]);
        if (i < n) slot[i] = b + (uint32_t)(lane - st[r]);
    }
    if (bad) atomicOr(&counters[CNT_FLAGS], FLAG_TILE_RANGE);
}

__global__ void __launch_bounds__(BS_SCAN) bs_reduce(const uint32_t* __restrict__ tcount, int64_t n,
                                                     uint32_t* __restrict__ bsum) {
    __shared__ uint32_t sh[32];
    const int64_t i = (int64_t)blockIdx.x * BS_SCAN + threadIdx.x;
    uint32_t tot;
    block_excl_scan(i < n ? tcount[i] : 0u, sh, tot);
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

// Warp-aggregated append of `item` (lanes with want) to list / counter;
// returns the slot written (meaningful where want).
__device__ __forceinline__ uint32_t bs_append(uint32_t* list, uint32_t* counter, bool want, uint32_t item,
                                              int lane) {
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, want);
    if (!m) return 0u;
    const int leader = __ffs(m) - 1;
    uint32_t b = 0;
    if (lane == leader) b = atomicAdd(counter, (uint32_t)__popc(m));
    b = __shfl_sync(0xFFFFFFFFu, b, leader);
    const uint32_t slot = b + __popc(m & ((1u << lane) - 1u));
    if (want) list[slot] = item;
    return slot;
}

// Size class of an occupied tile, 0 = largest (>= 1024 particles) ...
// CNT_BUCKETS - 1 = smallest (< 16).
__device__ __forceinline__ int bs_class(uint32_t count) {
    const int lg = 31 - __clz(count);  // count >= 1
    return min(CNT_BUCKETS - 1, max(0, 10 - lg));
}

// bsum: the per-block totals of bs_reduce, or null when the blocks are few
// (BS_DIRECT_BLOCKS): each block then sums the tile counts before its own
// range itself, and the step has no bs_reduce launch.  The tile counts are
// left for bs_finish to clear, since later blocks read earlier blocks' range.
__global__ void __launch_bounds__(BS_SCAN) bs_down(View V, const uint32_t* __restrict__ tcount, int64_t n,
                                                   const uint32_t* __restrict__ bsum, uint32_t* __restrict__ toff,
                                                   uint32_t* __restrict__ ccount_overflow,
                                                   uint32_t* __restrict__ tile_rank) {
    __shared__ uint32_t sh[32];
    const int lane = threadIdx.x & 31;
    // this block's first position: the tile totals of the blocks before it
    uint32_t part = 0u;
    if (bsum) {
        for (uint32_t b = threadIdx.x; b < blockIdx.x; b += BS_SCAN) part += bsum[b];
    } else {
        const int64_t end = (int64_t)blockIdx.x * BS_SCAN;
        for (int64_t i = threadIdx.x; i < end; i += BS_SCAN) part += tcount[i];
    }
    uint32_t base;
    block_excl_scan(part, sh, base);
    const int64_t t = (int64_t)blockIdx.x * BS_SCAN + threadIdx.x;
    const uint32_t c = t < n ? tcount[t] : 0u;
    uint32_t tot;
    const uint32_t ex = block_excl_scan(c, sh, tot) + base;
    if (t < n) toff[t] = ex;
    if (t == n - 1) *ccount_overflow = 0u;
    const bool occ = t < (int64_t)V.total_ct && c > 0u;  // not the overflow bin
    if (occ) V.ctile_range[t] = make_uint2(ex, ex + c);
    const uint32_t w = bs_append(V.ctile_list, &V.counters[CNT_CTILES], occ, (uint32_t)t, lane);
    if (tile_rank) {
        // rank inside the tile's size class (lanes of one class share an atomic)
        const uint32_t cls = occ ? (uint32_t)bs_class(c) : (uint32_t)(CNT_BUCKETS + lane);
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, cls);
        const int leader = __ffs(peers) - 1;
        uint32_t b = 0;
        if (occ && lane == leader) b = atomicAdd(&V.counters[CNT_BUCKET + cls], (uint32_t)__popc(peers));
        b = __shfl_sync(0xFFFFFFFFu, b, leader);
        if (occ) tile_rank[w] = (cls << 28) | (b + (uint32_t)__popc(peers & ((1u << lane) - 1u)));
    }
}

// Blocks [0, cell_blocks): (a), the rest: (b).  See the overview above.
// (a) also clears the tile counts bs_count wrote (the occupied tiles' and
// the overflow bin's, the only non-zero ones) for the next step.
__global__ void __launch_bounds__(BS_T) bs_finish(View V, uint32_t* __restrict__ ccount,
                                                  uint32_t* __restrict__ tcount,
                                                  const uint32_t* __restrict__ toff, uint32_t* __restrict__ coff,
                                                  uint2* __restrict__ cell_range, const uint32_t* __restrict__ tile_rank,
                                                  uint32_t* __restrict__ ptile_list, int cell_blocks) {
    const int lane = threadIdx.x & 31;
    if ((int)blockIdx.x < cell_blocks) {
        if (blockIdx.x == 0 && threadIdx.x == 0) tcount[V.total_ct] = 0u;
        const uint32_t ntiles = V.counters[CNT_CTILES];
        const uint32_t nwarps = (uint32_t)cell_blocks * (BS_T / 32);
        // first slot of each size class in the largest-first list
        uint32_t cls_off = 0u;
        if (ptile_list) {
            const uint32_t cnt = lane < CNT_BUCKETS ? V.counters[CNT_BUCKET + lane] : 0u;
            uint32_t x = cnt;
#pragma unroll
            for (int o = 1; o < CNT_BUCKETS; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
                if (lane >= o) x += y;
            }
            cls_off = x - cnt;
        }
        for (uint32_t w = (blockIdx.x * BS_T + threadIdx.x) >> 5; w < ntiles; w += nwarps) {
            const uint32_t t = V.ctile_list[w];
            if (lane == 0) tcount[t] = 0u;
            if (ptile_list) {
                const uint32_t tr = tile_rank[w];
                const uint32_t off = __shfl_sync(0xFFFFFFFFu, cls_off, (int)(tr >> 28));
                if (lane == 0) ptile_list[off + (tr & 0x0FFFFFFFu)] = t;
            }
            uint2* cc2 = reinterpret_cast<uint2*>(ccount + (size_t)t * 64) + lane;
            const uint2 cc = *cc2;
            *cc2 = make_uint2(0u, 0u);  // left clear for the next step
            uint32_t x = cc.x + cc.y;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
                if (lane >= o) x += y;
            }
            const uint32_t e = toff[t] + x - cc.x - cc.y;  // first position of cell 2*lane
            reinterpret_cast<uint2*>(coff + (size_t)t * 64)[lane] = make_uint2(e, e + cc.x);
            if (cell_range) {
                cell_range[(size_t)t * 64 + 2 * lane] = make_uint2(e, e + cc.x);
                cell_range[(size_t)t * 64 + 2 * lane + 1] = make_uint2(e + cc.x, e + cc.x + cc.y);
            }
            if (V.sp.cap) {
                // sparse grid: lanes 0..7 find (or claim) the slots of the 8
                // node tiles the cell tile's stencils reach, list them for the
                // tile, and mark them active for this step (the first marker
                // appends the tile to the active list)
                uint32_t nslot = SP_NONE;
                uint32_t f = 0;
                if (lane < 8) {
                    int tx, ty, tz;
                    sp_decode(V.sp.code[t], tx, ty, tz);
                    nslot = sp_find_or_insert(V.sp, sp_code(tx + (lane & 1), ty + ((lane >> 1) & 1), tz + (lane >> 2)),
                                              f);
                    reinterpret_cast<uint32_t*>(V.sp.nbr + 2 * (size_t)t)[lane] = nslot == SP_NONE ? 0u : nslot;
                }
                if (f) atomicOr(&V.counters[CNT_FLAGS], f);
                const uint32_t stamp = V.counters[CNT_STAMP];
                // node tile nslot lies at offset `lane` of this tile's box (one
                // writer per (node tile, offset): t = nslot - offset)
                if (lane < 8 && nslot != SP_NONE) V.sp.rev[8 * (size_t)nslot + lane] = make_uint2(t, stamp);
                const bool fresh = lane < 8 && nslot != SP_NONE && atomicExch(&V.tile_flags[nslot], stamp) != stamp;
                bs_append(V.tile_list, &V.counters[CNT_TILES], fresh, nslot, lane);
            }
        }
        return;
    }
    const int64_t nt = (int64_t)(blockIdx.x - cell_blocks) * BS_T + threadIdx.x;
    bool act = false;
    if (nt < V.total_nt) {
        const int s = V.S == 1 ? 0 : scene_of_node_tile(V.scenes, V.S, (int)nt);
        const SceneDev& sc = V.scenes[s];
        const int l = (int)nt - sc.nt_base;
        const int x = l % sc.nt[0], y = (l / sc.nt[0]) % sc.nt[1], z = l / (sc.nt[0] * sc.nt[1]);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int cx = x - (k & 1), cy = y - ((k >> 1) & 1), cz = z - (k >> 2);
            if (cx < 0 || cy < 0 || cz < 0 || cx >= sc.ct[0] || cy >= sc.ct[1] || cz >= sc.ct[2]) continue;
            const int ct = sc.ct_base + (cz * sc.ct[1] + cy) * sc.ct[0] + cx;
            act |= toff[ct + 1] > toff[ct];
        }
        V.tile_flags[nt] = act ? 1u : 0u;
    }
    bs_append(V.tile_list, &V.counters[CNT_TILES], act, (uint32_t)nt, lane);
}

__global__ void __launch_bounds__(BS_T) bs_scatter(const uint32_t* __restrict__ keys, int64_t n, uint32_t ncells,
                                                   const uint32_t* __restrict__ slot,
                                                   const uint32_t* __restrict__ coff,
                                                   const uint32_t* __restrict__ toff_overflow,
                                                   uint32_t* __restrict__ ok_, uint32_t* __restrict__ ov) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t base = (int64_t)blockIdx.x * BS_TILE + warp * (32 * BS_ITEMS);
    uint32_t k[BS_ITEMS], sl[BS_ITEMS], pos[BS_ITEMS];
#pragma unroll
    for (int r = 0; r < BS_ITEMS; ++r) {
        const int64_t i = base + r * 32 + lane;
        k[r] = i < n ? keys[i] : 0u;
        sl[r] = i < n ? slot[i] : 0u;
    }
#pragma unroll
    for (int r = 0; r < BS_ITEMS; ++r) pos[r] = (k[r] < ncells ? coff[k[r]] : *toff_overflow) + sl[r];
#pragma unroll
    for (int r = 0; r < BS_ITEMS; ++r) {
        const int64_t i = base + r * 32 + lane;
        if (i < n && (int64_t)pos[r] < n) {
            ok_[pos[r]] = k[r];
            ov[pos[r]] = (uint32_t)i;
        }
    }
}
}  // namespace

int64_t bin_sort_scan_blocks(int total_ct) { return ((int64_t)total_ct + 1 + BS_SCAN - 1) / BS_SCAN; }

cudaError_t bin_sort_step(const View& V, const BinSortBufs& B, int num_sms, cudaStream_t st) {
    const int64_t n = V.N;
    if (n <= 0) return cudaSuccess;
    const uint32_t ncells = (uint32_t)V.total_ct * 64u;
    const int64_t ntb = (int64_t)V.total_ct + 1;  // tiles + overflow bin
    const int nb = (int)bin_sort_scan_blocks(V.total_ct);
    const int gk = (int)((n + BS_TILE - 1) / BS_TILE);
    bs_count<<<gk, BS_T, 0, st>>>(B.keys_in, n, ncells, B.ccount, B.tcount, B.slot, V.counters);
    const bool direct = nb <= BS_DIRECT_BLOCKS;
    if (!direct) bs_reduce<<<nb, BS_SCAN, 0, st>>>(B.tcount, ntb, B.bsum);
    bs_down<<<nb, BS_SCAN, 0, st>>>(V, B.tcount, ntb, direct ? nullptr : B.bsum, B.toff, B.ccount + ncells,
                                    B.ptile_list ? B.tile_rank : nullptr);
    const int cell_blocks = num_sms * 2;
    // sparse grids mark their node tiles from the occupied cell tiles
    const int node_blocks = V.sp.cap ? 0 : (V.total_nt + BS_T - 1) / BS_T;
    bs_finish<<<cell_blocks + node_blocks, BS_T, 0, st>>>(V, B.ccount, B.tcount, B.toff, B.coff, B.cell_range,
                                                           B.tile_rank, B.ptile_list, cell_blocks);
    bs_scatter<<<gk, BS_T, 0, st>>>(B.keys_in, n, ncells, B.slot, B.coff, B.toff + V.total_ct, B.out_k, B.out_v);
    return cudaGetLastError();
}

int64_t radix_sort_scratch_words(int64_t n) { return radix_scratch_words_for(n); }

int radix_passes(int key_bits) { return key_bits <= 0 ? 0 : (key_bits + 7) / 8; }

// Sorts (kin, vin) by the low key_bits bits.  Buffers: (ka, va), (kb, vb)
// ping-pong targets of n words each; scratch of radix_sort_scratch_words(n)
// u32.  Returns which buffer pair holds the result (0 = a, 1 = b) through
// *which.  vin may be null (values = index).  No allocation, no sync.
cudaError_t radix_sort_pairs(const uint32_t* kin, const uint32_t* vin, uint32_t* ka, uint32_t* va, uint32_t* kb,
                             uint32_t* vb, uint32_t* scratch, int64_t n, int key_bits, int* which,
                             cudaStream_t st) {
    *which = 0;
    if (n <= 0) return cudaSuccess;
    const int passes = radix_passes(key_bits < 1 ? 1 : key_bits);
    const int bits = (key_bits + passes - 1) / passes;
    const int nb = (int)((n + RS_TILE - 1) / RS_TILE);
    uint32_t* hist = scratch;
    uint32_t* totals = scratch + (int64_t)nb * RS_MAXD;
    const uint32_t* ck = kin;
    const uint32_t* cv = vin;
    int shift = 0;
    for (int p = 0; p < passes; ++p) {
        uint32_t* ok = (p & 1) ? kb : ka;
        uint32_t* ov = (p & 1) ? vb : va;
        const int b = min(bits, key_bits - shift) > 0 ? min(bits, key_bits - shift) : 1;
        rs_hist<<<nb, RS_THREADS, 0, st>>>(ck, n, shift, b, hist, nb);
        rs_scan<<<1 << b, 1024, 0, st>>>(hist, nb, totals);
        rs_scatter<<<nb, RS_THREADS, 0, st>>>(ck, cv, ok, ov, n, shift, b, hist, nb, totals);
        ck = ok;
        cv = ov;
        shift += b;
        *which = p & 1;
    }
    return cudaGetLastError();
}

}  // namespace pgmpm
