// Stable LSD radix sort of 32-bit cell keys with 32-bit payloads.
//
// The reference bins particles into x-slabs for its OpenMP scatter
// (GATHER_SCATTER::Prepare_Scatter, Hybrid_Methods/Iterators/GATHER_SCATTER.cpp:
// 33-87); here particles are sorted by (block, cell) key every substep so a
// CTA can own a block of cells.  Only the low `bits` bits take part, in
// digits of up to 8 bits.
//
// One kernel counts every digit place's global histogram up front; then one
// kernel per digit place does the whole pass (the single-pass "onesweep"
// scheme of Adinets & Merrill, 2022):
//   * tiles are numbered in the order CTAs start (atomic ticket), so a tile
//     only ever waits on tiles that are already running;
//   * each tile ranks its keys stably (warp __match_any_sync + popc, warp by
//     warp in index order), publishes its per-digit counts, and looks back
//     over earlier tiles' published counts / inclusive prefixes (decoupled
//     look-back) to find where its keys go;
//   * keys are staged in shared memory in digit order and runs of equal
//     digits are written to consecutive global addresses.
// Status words carry an epoch (bumped on the device by the histogram kernel),
// so nothing needs clearing between sorts and the sort replays inside a CUDA
// graph.  Every spin-wait is bounded: past the limit the kernel sets an error
// flag and moves on instead of hanging.
// The result is bit-identical to a CPU stable sort on the same keys.
#pragma once
#include <cuda/atomic>
#include <cuda_runtime.h>

#include <cstdint>

namespace mpm_sort {

constexpr int kThreads = 256;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;   // 4096 keys per tile
// Small sorts (up to kSmallSortMax keys) use 1024-key tiles: four times the
// CTAs, so a sort of a few hundred thousand keys still spreads over the SMs.
constexpr int kSmallItems = 4;
constexpr int kSmallTile = kThreads * kSmallItems;
constexpr int64_t kSmallSortMax = 1 << 21;
constexpr int kRadix = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxPasses = 4;
constexpr uint32_t kSpinLimit = 1u << 22;
// Status words keep the epoch in their top 30 bits; the epoch counter itself
// is a 32-bit word, so it is compared modulo 2^30 on both sides.
constexpr uint32_t kEpochMask = (1u << 30) - 1u;

constexpr uint64_t kFlagAggregate = 1;
constexpr uint64_t kFlagInclusive = 2;

// global scratch layout (in 32-bit words)
//   [0, 1024)                   digit histograms, kMaxPasses x 256
//   [1024, 1028)                tile tickets per pass
//   [1028]                      epoch
//   then (8-byte aligned)       status words, kMaxPasses x tiles x 256 (uint64)
constexpr int kHistWords = kMaxPasses * kRadix;
constexpr int kTicketOff = kHistWords;
constexpr int kEpochOff = kTicketOff + kMaxPasses;
constexpr int kStatusOff = kEpochOff + 4;     // keep 16-byte alignment

__host__ __device__ constexpr int64_t tiles_for(int64_t n, int tile = kTile) { return (n + tile - 1) / tile; }
// Scratch for any sort of up to n keys, whichever tile size it picks.
inline int64_t scratch_words(int64_t n)
{
    int64_t t = tiles_for(n > 0 ? n : 1);
    int64_t small = tiles_for(n < kSmallSortMax ? (n > 0 ? n : 1) : kSmallSortMax, kSmallTile);
    return kStatusOff + 2 * (int64_t)kMaxPasses * (t > small ? t : small) * kRadix;
}

__device__ __forceinline__ int passes_for(int bits) { return (bits + 7) / 8; }
__device__ __forceinline__ uint32_t digit_mask(int bits, int pass)
{
    int w = bits - 8 * pass;
    return w >= 8 ? 255u : ((1u << w) - 1u);
}

// Global histograms of every digit place; also resets the tile tickets and
// bumps the epoch (block 0, thread 0).  `scratch` histograms must be zero.
__global__ void __launch_bounds__(kThreads) k_upfront_hist(const uint32_t* __restrict__ keys, int64_t n, int bits,
    uint32_t* __restrict__ scratch)
{
    __shared__ uint32_t cnt[kMaxPasses][kRadix];
    const int passes = passes_for(bits);
    for(int i = threadIdx.x; i < kMaxPasses * kRadix; i += kThreads) (&cnt[0][0])[i] = 0;
    __syncthreads();
    // keys arrive nearly sorted (last substep's order), so the lanes of a warp
    // mostly share their high digits: one atomic per distinct digit per warp
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * kThreads;
    const int64_t end = (n + 31) & ~(int64_t)31;   // whole warps stay in the loop
    for(int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < end; i += stride) {
        const bool ok = i < n;
        const uint32_t k = ok ? keys[i] : 0u;
        for(int p = 0; p < passes; p++) {
            const uint32_t dg = ok ? (k >> (8 * p)) & digit_mask(bits, p) : 256u;
            const uint32_t peers = __match_any_sync(0xffffffffu, dg);
            if(ok && (__ffs(peers) - 1) == lane) atomicAdd(&cnt[p][dg], (uint32_t)__popc(peers));
        }
    }
    __syncthreads();
    for(int i = threadIdx.x; i < passes * kRadix; i += kThreads) {
        uint32_t c = (&cnt[0][0])[i];
        if(c) atomicAdd(&scratch[i], c);
    }
    if(blockIdx.x == 0 && threadIdx.x == 0) {
        for(int p = 0; p < kMaxPasses; p++) scratch[kTicketOff + p] = 0;
        scratch[kEpochOff] += 1;
    }
}

// Pieces for callers that build the histograms themselves while they write
// the keys (radix_sort(..., have_hist = true)).
//
// Count `key` into the shared histograms `cnt[kMaxPasses][kRadix]`: one
// atomic per distinct digit among the converged lanes that call it.
__device__ __forceinline__ void hist_add(uint32_t (*cnt)[kRadix], uint32_t key, int bits)
{
    const int passes = passes_for(bits);
    const int lane = threadIdx.x & 31;
    const unsigned active = __activemask();
    for(int p = 0; p < passes; p++) {
        const uint32_t dg = (key >> (8 * p)) & digit_mask(bits, p);
        const uint32_t peers = __match_any_sync(active, dg);
        if((__ffs(peers) - 1) == lane) atomicAdd(&cnt[p][dg], (uint32_t)__popc(peers));
    }
}

// Count the lowest digit only (the caller accounts for the others).
__device__ __forceinline__ void hist_add_low(uint32_t (*cnt)[kRadix], uint32_t key, int bits)
{
    const int lane = threadIdx.x & 31;
    const unsigned active = __activemask();
    const uint32_t dg = key & digit_mask(bits, 0);
    const uint32_t peers = __match_any_sync(active, dg);
    if((__ffs(peers) - 1) == lane) atomicAdd(&cnt[0][dg], (uint32_t)__popc(peers));
}

// Add `count` keys that share `key`'s digits of passes 1 and up.
__device__ __forceinline__ void hist_add_high(uint32_t (*cnt)[kRadix], uint32_t key, uint32_t count, int bits)
{
    for(int p = 1; p < passes_for(bits); p++) atomicAdd(&cnt[p][(key >> (8 * p)) & digit_mask(bits, p)], count);
}

// Add `count` sentinel keys (all bits set) to the global histograms.
__device__ __forceinline__ void hist_add_sentinels(uint32_t* scratch, uint32_t count, int bits)
{
    if(!count) return;
    for(int p = 0; p < passes_for(bits); p++) atomicAdd(&scratch[p * kRadix + digit_mask(bits, p)], count);
}

// After a sort has run: clear the histograms for the next one, reset the tile
// tickets and start a new epoch (one CTA; nothing else may touch the scratch).
__device__ __forceinline__ void hist_reset(uint32_t* scratch)
{
    for(int i = threadIdx.x; i < kHistWords; i += blockDim.x) scratch[i] = 0;
    if(threadIdx.x == 0) {
        for(int p = 0; p < kMaxPasses; p++) scratch[kTicketOff + p] = 0;
        scratch[kEpochOff] += 1;
    }
}

__device__ inline uint32_t block_exclusive_scan(uint32_t v, uint32_t* smem, uint32_t& total)
{
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for(int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if(lane >= o) x += y;
    }
    if(lane == 31) smem[warp] = x;
    __syncthreads();
    if(warp == 0) {
        uint32_t s = lane < (int)(blockDim.x >> 5) ? smem[lane] : 0;
#pragma unroll
        for(int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if(lane >= o) s += y;
        }
        smem[lane] = s;
    }
    __syncthreads();
    uint32_t warp_prefix = warp ? smem[warp - 1] : 0;
    total = smem[(blockDim.x >> 5) - 1];
    __syncthreads();
    return warp_prefix + x - v;
}

template<int ITEMS> struct PassSmem {
    uint32_t wcnt[kWarps][kRadix];
    uint32_t dstart[kRadix];
    uint32_t gbase[kRadix];
    uint32_t skey[kThreads * ITEMS];
    uint32_t sval[kThreads * ITEMS];
    uint32_t scan_tmp[32];
    uint32_t tile;
};

// One digit place over tiles of kThreads * ITEMS keys.  vals_in == nullptr
// means payload = index.
template<int ITEMS>
__global__ void __launch_bounds__(kThreads) k_onesweep(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
    uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, int64_t n, int bits, int pass, int64_t tiles,
    uint32_t* __restrict__ scratch, unsigned* __restrict__ err_flags, unsigned timeout_flag, uint32_t spin_limit)
{
    constexpr int kItems = ITEMS, kTile = kThreads * ITEMS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PassSmem<ITEMS>& S = *reinterpret_cast<PassSmem<ITEMS>*>(smem_raw);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int shift = 8 * pass;
    const uint32_t mask = digit_mask(bits, pass);
    for(int i = threadIdx.x; i < kWarps * kRadix; i += kThreads) (&S.wcnt[0][0])[i] = 0;
    if(threadIdx.x == 0) S.tile = atomicAdd(&scratch[kTicketOff + pass], 1u);
    __syncthreads();
    const uint32_t tile = S.tile;
    const uint64_t epoch = scratch[kEpochOff] & kEpochMask;
    uint64_t* status = reinterpret_cast<uint64_t*>(scratch + kStatusOff) + (int64_t)pass * tiles * kRadix;

    const int64_t base = (int64_t)tile * kTile;
    uint32_t key[kItems], rank[kItems];
    const uint32_t lt = (1u << lane) - 1u;
    const int64_t wbase = base + warp * (32 * kItems) + lane;
    // all loads first, so the 16 keys of a thread are in flight together
#pragma unroll
    for(int k = 0; k < kItems; k++) {
        int64_t idx = wbase + k * 32;
        key[k] = idx < n ? keys_in[idx] : 0u;
    }
#pragma unroll
    for(int k = 0; k < kItems; k++) {
        bool ok = wbase + k * 32 < n;
        uint32_t dg = ok ? (key[k] >> shift) & mask : 256u;
        uint32_t peers = __match_any_sync(0xffffffffu, dg);
        uint32_t r = 0;
        if(ok) r = S.wcnt[warp][dg] + __popc(peers & lt);
        __syncwarp();
        if(ok && (31 - __clz(peers)) == lane) S.wcnt[warp][dg] += __popc(peers);
        __syncwarp();
        rank[k] = r;
    }
    __syncthreads();
    // thread d owns digit d: exclusive over warps, tile total
    const int d = threadIdx.x;
    uint32_t tot = 0;
    {
        uint32_t off = 0;
        for(int w = 0; w < kWarps; w++) { uint32_t c = S.wcnt[w][d]; S.wcnt[w][d] = off; off += c; }
        tot = off;
    }
    // publish and look back (decoupled look-back, one digit per thread)
    cuda::atomic_ref<uint64_t, cuda::thread_scope_device> mine(status[(int64_t)tile * kRadix + d]);
    uint32_t excl = 0;
    if(tile == 0) {
        mine.store((epoch << 34) | (kFlagInclusive << 32) | tot, cuda::memory_order_relaxed);
    } else {
        mine.store((epoch << 34) | (kFlagAggregate << 32) | tot, cuda::memory_order_relaxed);
        // Read kWindow predecessors at once: when every tile starts together,
        // tile k walks about k/2 tiles back before it meets an inclusive
        // prefix, so the walk's latency, not its work, is what costs.  Tile 0
        // is always inclusive, so the walk stops at j = 0 at the latest.
        constexpr int kWindow = 8;
        int64_t j = (int64_t)tile - 1;
        uint32_t spins = 0;
        bool done = false;
        while(!done) {
            uint64_t w[kWindow];
#pragma unroll
            for(int u = 0; u < kWindow; u++) {
                w[u] = 0;
                if(j - u >= 0) {
                    cuda::atomic_ref<uint64_t, cuda::thread_scope_device> other(status[(j - u) * kRadix + d]);
                    w[u] = other.load(cuda::memory_order_relaxed);
                }
            }
            int adv = 0;
            bool stop = false;
#pragma unroll
            for(int u = 0; u < kWindow; u++) {
                if(stop || j - u < 0) break;
                const uint64_t flag = (w[u] >> 34) == epoch ? (w[u] >> 32) & 3u : 0u;
                if(flag == 0) { stop = true; break; }     // not published yet: poll again from here
                excl += (uint32_t)w[u];
                adv++;
                if(flag == kFlagInclusive) { done = true; stop = true; }
            }
            if(done) break;
            if(adv == 0 && ++spins > spin_limit) { atomicOr(err_flags, timeout_flag); break; }
            j -= adv;
        }
        mine.store((epoch << 34) | (kFlagInclusive << 32) | (excl + tot), cuda::memory_order_relaxed);
    }
    // global start of digit d: exclusive scan of the upfront histogram
    uint32_t gtotal;
    uint32_t gex = block_exclusive_scan(scratch[pass * kRadix + d], S.scan_tmp, gtotal);
    S.gbase[d] = gex + excl;
    uint32_t total;
    uint32_t ex = block_exclusive_scan(tot, S.scan_tmp, total);
    S.dstart[d] = ex;
    __syncthreads();
#pragma unroll
    for(int k = 0; k < kItems; k++) {
        if(wbase + k * 32 < n) {
            uint32_t dg = (key[k] >> shift) & mask;
            uint32_t pos = S.dstart[dg] + S.wcnt[warp][dg] + rank[k];
            S.skey[pos] = key[k];
            S.sval[pos] = (uint32_t)(warp * (32 * kItems) + k * 32 + lane);   // tile-local index
        }
    }
    __syncthreads();
    const int64_t tile_n = n - base < kTile ? n - base : kTile;
    for(int i = threadIdx.x; i < tile_n; i += kThreads) {
        uint32_t k0 = S.skey[i];
        uint32_t dg = (k0 >> shift) & mask;
        int64_t pos = (int64_t)S.gbase[dg] + (i - S.dstart[dg]);
        int64_t src = base + S.sval[i];
        keys_out[pos] = k0;
        vals_out[pos] = vals_in ? vals_in[src] : (uint32_t)src;
    }
}

template<int ITEMS> inline size_t pass_smem() { return sizeof(PassSmem<ITEMS>); }

inline cudaError_t prepare()
{
    cudaError_t e = cudaFuncSetAttribute(k_onesweep<kItems>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pass_smem<kItems>());
    if(e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_onesweep<kSmallItems>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)pass_smem<kSmallItems>());
}

// Sorts keys[0..n) by their low `bits` bits (1..32).  keys is read only;
// the result lands in (keys_out, vals_out), which must not alias keys;
// (keys_alt, vals_alt) are ping-pong buffers.  scratch = scratch_words(n)
// words whose epoch region persists between sorts.  n < 2^30.
// `small_tiles` allows 1024-key tiles for n <= kSmallSortMax.  `have_hist`:
// the caller built the histograms of `keys` in the scratch (hist_add), reset
// the tickets and started a new epoch after the previous sort (hist_reset).
inline cudaError_t radix_sort(const uint32_t* keys, uint32_t* keys_out, uint32_t* vals_out, uint32_t* keys_alt,
    uint32_t* vals_alt, int64_t n, int bits, uint32_t* scratch, unsigned* err_flags, unsigned timeout_flag,
    int hist_blocks, cudaStream_t st, bool small_tiles = true, bool have_hist = false)
{
    if(n == 0) return cudaSuccess;
    int passes = (bits + 7) / 8;
    const bool small = small_tiles && n <= kSmallSortMax;
    int64_t tiles = small ? tiles_for(n, kSmallTile) : tiles_for(n);
    if(!have_hist) {
        cudaError_t e = cudaMemsetAsync(scratch, 0, kHistWords * sizeof(uint32_t), st);
        if(e != cudaSuccess) return e;
        int hb = (int)((n + kThreads * 4 - 1) / (kThreads * 4));
        if(hb > hist_blocks) hb = hist_blocks;
        if(hb < 1) hb = 1;
        k_upfront_hist<<<hb, kThreads, 0, st>>>(keys, n, bits, scratch);
    }
    // ping-pong so that the last pass writes (keys_out, vals_out)
    const uint32_t* kin = keys;
    const uint32_t* vin = nullptr;
    for(int p = 0; p < passes; p++) {
        bool last_to_out = ((passes - 1 - p) % 2) == 0;
        uint32_t* ko = last_to_out ? keys_out : keys_alt;
        uint32_t* vo = last_to_out ? vals_out : vals_alt;
        if(small)
            k_onesweep<kSmallItems><<<(unsigned)tiles, kThreads, pass_smem<kSmallItems>(), st>>>(
                kin, vin, ko, vo, n, bits, p, tiles, scratch, err_flags, timeout_flag, kSpinLimit);
        else
            k_onesweep<kItems><<<(unsigned)tiles, kThreads, pass_smem<kItems>(), st>>>(
                kin, vin, ko, vo, n, bits, p, tiles, scratch, err_flags, timeout_flag, kSpinLimit);
        kin = ko;
        vin = vo;
    }
    return cudaGetLastError();
}

}  // namespace mpm_sort
