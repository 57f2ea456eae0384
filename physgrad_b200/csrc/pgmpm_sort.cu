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
// The MPM step groups particles by cell without a full radix sort: the key
// is (cell tile << 6 | cell in tile), and both levels are counting sorts.
//   bs_count     one pass over the keys: particles per cell tile (warp-
//                aggregated atomics, match.any on the tile) and each
//                particle's slot inside its tile.
//   bs_reduce / bs_top / bs_down
//                exclusive scan of the tile counts (reduce, scan of block
//                sums, scan + offsets).  bs_down also emits every occupied
//                tile: its sorted range, its entry in the occupied-tile list
//                and the marks of the 8 node tiles it touches.
//   bs_scatter   particle -> tile offset + slot (tile-grouped order).
//   bs_cells     per occupied tile: 64-bin counting sort by cell into the
//                final (key, particle) arrays, and every cell's range.
// O(N + tiles) traffic.  Keys come out sorted; the order of particles that
// share a cell depends on atomic arrival, which the step does not rely on.
constexpr int BS_T = 256;
constexpr int BS_SCAN = 1024;  // tile counts per scan block

__global__ void __launch_bounds__(BS_T) bs_count(const uint32_t* __restrict__ keys, int64_t n, uint32_t total_ct,
                                                 uint32_t* __restrict__ tcount, uint32_t* __restrict__ slot,
                                                 uint32_t* __restrict__ counters) {
    const int lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    const int64_t stride = (int64_t)gridDim.x * BS_T;
    uint32_t bad = 0;
    // whole warps iterate together (match.any needs every lane)
    for (int64_t base = (int64_t)blockIdx.x * BS_T + (threadIdx.x & ~31); base < n; base += stride) {
        const int64_t i = base + lane;
        const bool ok = i < n;
        uint32_t t = 0xFFFFFFFFu;
        if (ok) {
            t = keys[i] >> 6;
            if (t >= total_ct) {  // out-of-range key: overflow bin after the last tile
                bad = 1;
                t = total_ct;
            }
        }
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, t);
        const int leader = __ffs(peers) - 1;
        uint32_t b = 0;
        if (ok && lane == leader) b = atomicAdd(&tcount[t], (uint32_t)__popc(peers));
        b = __shfl_sync(0xFFFFFFFFu, b, leader);
        if (ok) slot[i] = b + (uint32_t)__popc(peers & lt);
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

__global__ void __launch_bounds__(BS_SCAN) bs_top(uint32_t* __restrict__ bsum, int nb) {
    __shared__ uint32_t sh[32];
    uint32_t carry = 0;
    for (int b0 = 0; b0 < nb; b0 += BS_SCAN) {
        const int b = b0 + threadIdx.x;
        const uint32_t v = b < nb ? bsum[b] : 0u;
        uint32_t tot;
        const uint32_t ex = block_excl_scan(v, sh, tot);
        if (b < nb) bsum[b] = carry + ex;
        carry += tot;
    }
}

__global__ void __launch_bounds__(BS_SCAN) bs_down(View V, const uint32_t* __restrict__ tcount, int64_t n,
                                                   const uint32_t* __restrict__ bsum, uint32_t* __restrict__ toff) {
    __shared__ uint32_t sh[32];
    const int64_t t = (int64_t)blockIdx.x * BS_SCAN + threadIdx.x;
    const uint32_t c = t < n ? tcount[t] : 0u;
    uint32_t tot;
    const uint32_t ex = block_excl_scan(c, sh, tot) + bsum[blockIdx.x];
    if (t >= n) return;
    toff[t] = ex;
    if (c == 0 || t >= V.total_ct) return;  // empty, or the overflow bin
    V.ctile_range[t] = make_uint2(ex, ex + c);
    V.ctile_list[atomicAdd(&V.counters[CNT_CTILES], 1u)] = (uint32_t)t;
    const int s = V.S == 1 ? 0 : scene_of_cell_tile(V.scenes, V.S, (int)t);
    const SceneDev& sc = V.scenes[s];
    const int lt = (int)t - sc.ct_base;
    const int tx = lt % sc.ct[0], ty = (lt / sc.ct[0]) % sc.ct[1], tz = lt / (sc.ct[0] * sc.ct[1]);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int nx = tx + (k & 1), ny = ty + ((k >> 1) & 1), nz = tz + (k >> 2);
        const uint32_t nt = (uint32_t)(sc.nt_base + (nz * sc.nt[1] + ny) * sc.nt[0] + nx);
        if (atomicExch(&V.tile_flags[nt], 1u) == 0u) V.tile_list[atomicAdd(&V.counters[CNT_TILES], 1u)] = nt;
    }
}

__global__ void __launch_bounds__(BS_T) bs_scatter(const uint32_t* __restrict__ keys, int64_t n, uint32_t total_ct,
                                                   const uint32_t* __restrict__ slot,
                                                   const uint32_t* __restrict__ toff, uint32_t* __restrict__ tk,
                                                   uint32_t* __restrict__ tv) {
    const int64_t stride = (int64_t)gridDim.x * BS_T;
    for (int64_t i = (int64_t)blockIdx.x * BS_T + threadIdx.x; i < n; i += stride) {
        const uint32_t key = keys[i];
        const uint32_t t = min(key >> 6, total_ct);
        const uint32_t pos = toff[t] + slot[i];
        if ((int64_t)pos < n) {
            tk[pos] = key;
            tv[pos] = (uint32_t)i;
        }
    }
}

__global__ void __launch_bounds__(BS_T) bs_cells(View V, const uint32_t* __restrict__ tk,
                                                 const uint32_t* __restrict__ tv, uint32_t* __restrict__ ok_,
                                                 uint32_t* __restrict__ ov, uint2* __restrict__ cell_range) {
    __shared__ uint32_t s_cnt[64];
    __shared__ uint32_t s_off[64];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t ntiles = V.counters[CNT_CTILES];
    for (uint32_t w = blockIdx.x; w < ntiles; w += gridDim.x) {
        const uint32_t ct = V.ctile_list[w];
        const uint2 rg = V.ctile_range[ct];
        if (threadIdx.x < 64) s_cnt[threadIdx.x] = 0u;
        __syncthreads();
        for (uint32_t b = rg.x + warp * 32; b < rg.y; b += BS_T) {
            const uint32_t i = b + lane;
            const bool ok = i < rg.y;
            const uint32_t c = ok ? (tk[i] & 63u) : 64u + lane;
            const uint32_t peers = __match_any_sync(0xFFFFFFFFu, c);
            if (ok && lane == __ffs(peers) - 1) atomicAdd(&s_cnt[c], (uint32_t)__popc(peers));
        }
        __syncthreads();
        if (warp == 0) {
            const uint32_t a = s_cnt[2 * lane], b = s_cnt[2 * lane + 1];
            uint32_t x = a + b;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
                if (lane >= o) x += y;
            }
            const uint32_t e = x - a - b;  // exclusive prefix of cell 2*lane
            s_off[2 * lane] = e;
            s_off[2 * lane + 1] = e + a;
            if (cell_range) {
                cell_range[(size_t)ct * 64 + 2 * lane] = make_uint2(rg.x + e, rg.x + e + a);
                cell_range[(size_t)ct * 64 + 2 * lane + 1] = make_uint2(rg.x + e + a, rg.x + e + a + b);
            }
        }
        __syncthreads();
        for (uint32_t b = rg.x + warp * 32; b < rg.y; b += BS_T) {
            const uint32_t i = b + lane;
            const bool ok = i < rg.y;
            const uint32_t key = ok ? tk[i] : 0u;
            const uint32_t c = ok ? (key & 63u) : 64u + lane;
            const uint32_t peers = __match_any_sync(0xFFFFFFFFu, c);
            const int leader = __ffs(peers) - 1;
            uint32_t base = 0;
            if (ok && lane == leader) base = atomicAdd(&s_off[c], (uint32_t)__popc(peers));
            base = __shfl_sync(0xFFFFFFFFu, base, leader);
            if (ok) {
                const uint32_t pos = rg.x + base + (uint32_t)__popc(peers & lt);
                if (pos < rg.y) {
                    ok_[pos] = key;
                    ov[pos] = tv[i];
                }
            }
        }
        __syncthreads();
    }
}
}  // namespace

int64_t bin_sort_scan_blocks(int total_ct) { return ((int64_t)total_ct + 1 + BS_SCAN - 1) / BS_SCAN; }

cudaError_t bin_sort_step(const View& V, const BinSortBufs& B, int num_sms, cudaStream_t st) {
    const int64_t n = V.N;
    if (n <= 0) return cudaSuccess;
    const int64_t nbins = (int64_t)V.total_ct + 1;  // + overflow bin
    const int nb = (int)bin_sort_scan_blocks(V.total_ct);
    cudaError_t e = cudaMemsetAsync(B.tcount, 0, sizeof(uint32_t) * nbins, st);
    if (e != cudaSuccess) return e;
    const int64_t g64 = (n + BS_T - 1) / BS_T;
    const int g = (int)(g64 < (int64_t)num_sms * 8 ? g64 : (int64_t)num_sms * 8);
    bs_count<<<g, BS_T, 0, st>>>(B.keys_in, n, (uint32_t)V.total_ct, B.tcount, B.slot, V.counters);
    bs_reduce<<<nb, BS_SCAN, 0, st>>>(B.tcount, nbins, B.bsum);
    bs_top<<<1, BS_SCAN, 0, st>>>(B.bsum, nb);
    bs_down<<<nb, BS_SCAN, 0, st>>>(V, B.tcount, nbins, B.bsum, B.toff);
    bs_scatter<<<g, BS_T, 0, st>>>(B.keys_in, n, (uint32_t)V.total_ct, B.slot, B.toff, B.tmp_k, B.tmp_v);
    bs_cells<<<num_sms * 8, BS_T, 0, st>>>(V, B.tmp_k, B.tmp_v, B.out_k, B.out_v, B.cell_range);
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
