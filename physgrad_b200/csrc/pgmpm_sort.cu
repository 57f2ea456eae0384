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
}  // namespace

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
