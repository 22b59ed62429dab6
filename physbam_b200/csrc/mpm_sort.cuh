// Stable LSD radix sort of 32-bit cell keys with 32-bit payloads.
//
// The reference bins particles into x-slabs for its OpenMP scatter
// (GATHER_SCATTER::Prepare_Scatter, Hybrid_Methods/Iterators/GATHER_SCATTER.cpp:
// 33-87); here particles are sorted by (block, cell) key every substep so a
// CTA can own a block of cells.  Only the low `bits` bits take part, in 8-bit
// digits.  Per digit place:
//   1. every tile counts its digits (digit-major table [digit][tile]);
//   2. the table is exclusive-scanned (3 kernels);
//   3. each tile ranks its keys stably (warp __match_any_sync + popc, warp
//      by warp in index order), stages them in shared memory in digit order
//      and writes runs of equal digits to consecutive global addresses.
// The result is bit-identical to a CPU stable sort on the same keys.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace mpm_sort {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;   // 2048 keys per tile
constexpr int kRadix = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxPasses = 4;
constexpr int kScanChunk = 4096;

__host__ __device__ inline int64_t tiles_for(int64_t n) { return (n + kTile - 1) / kTile; }

// hist[digit][tile] for one digit place, on the keys in their current order.
__global__ void __launch_bounds__(kThreads) k_hist(const uint32_t* __restrict__ keys, int64_t n, int shift,
    int64_t tiles, uint32_t* __restrict__ hist)
{
    __shared__ uint32_t cnt[kRadix];
    for(int i = threadIdx.x; i < kRadix; i += kThreads) cnt[i] = 0;
    __syncthreads();
    int64_t base = (int64_t)blockIdx.x * kTile;
    for(int k = 0; k < kItems; k++) {
        int64_t idx = base + k * kThreads + threadIdx.x;
        if(idx < n) atomicAdd(&cnt[(keys[idx] >> shift) & 255u], 1u);
    }
    __syncthreads();
    for(int i = threadIdx.x; i < kRadix; i += kThreads) hist[(int64_t)i * tiles + blockIdx.x] = cnt[i];
}

// --- exclusive scan of a uint32 array (per-chunk reduce, scan of partials, downsweep)
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

__global__ void __launch_bounds__(kThreads) k_scan_reduce(const uint32_t* __restrict__ in, int64_t len, uint32_t* __restrict__ part)
{
    __shared__ uint32_t red[kWarps];
    int64_t base = (int64_t)blockIdx.x * kScanChunk;
    uint32_t s = 0;
    for(int i = threadIdx.x; i < kScanChunk; i += kThreads) {
        int64_t j = base + i;
        if(j < len) s += in[j];
    }
#pragma unroll
    for(int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if(threadIdx.x == 0) {
        uint32_t t = 0;
        for(int w = 0; w < kWarps; w++) t += red[w];
        part[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(kThreads) k_scan_partials(uint32_t* part, int64_t nparts)
{
    __shared__ uint32_t smem[32];
    uint32_t carry = 0;
    for(int64_t base = 0; base < nparts; base += kThreads) {
        int64_t j = base + threadIdx.x;
        uint32_t v = j < nparts ? part[j] : 0, total;
        uint32_t ex = block_exclusive_scan(v, smem, total);
        if(j < nparts) part[j] = carry + ex;
        carry += total;
    }
}

__global__ void __launch_bounds__(kThreads) k_scan_down(uint32_t* __restrict__ data, int64_t len, const uint32_t* __restrict__ part)
{
    __shared__ uint32_t smem[32];
    int64_t base = (int64_t)blockIdx.x * kScanChunk;
    uint32_t carry = part[blockIdx.x];
    constexpr int per = kScanChunk / kThreads;   // 16 consecutive items per thread
    uint32_t v[per], s = 0;
    int64_t j0 = base + (int64_t)threadIdx.x * per;
#pragma unroll
    for(int i = 0; i < per; i++) { v[i] = j0 + i < len ? data[j0 + i] : 0; s += v[i]; }
    uint32_t total;
    uint32_t ex = block_exclusive_scan(s, smem, total);
    uint32_t run = carry + ex;
#pragma unroll
    for(int i = 0; i < per; i++) {
        if(j0 + i < len) data[j0 + i] = run;
        run += v[i];
    }
}

// One digit place: stable rank + scatter.  vals_in == nullptr means payload = index.
__global__ void __launch_bounds__(kThreads) k_scatter(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
    uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, int64_t n, int shift, int64_t tiles,
    const uint32_t* __restrict__ offsets)
{
    __shared__ uint32_t wcnt[kWarps][kRadix];
    __shared__ uint32_t dstart[kRadix];
    __shared__ uint32_t skey[kTile];
    __shared__ uint32_t sval[kTile];
    __shared__ uint32_t scan_tmp[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for(int i = threadIdx.x; i < kWarps * kRadix; i += kThreads) (&wcnt[0][0])[i] = 0;
    __syncthreads();

    const int64_t base = (int64_t)blockIdx.x * kTile;
    uint32_t key[kItems], val[kItems], rank[kItems];
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for(int k = 0; k < kItems; k++) {
        int64_t idx = base + warp * (32 * kItems) + k * 32 + lane;
        bool ok = idx < n;
        key[k] = ok ? keys_in[idx] : 0xffffffffu;
        val[k] = ok ? (vals_in ? vals_in[idx] : (uint32_t)idx) : 0u;
        uint32_t dg = ok ? (key[k] >> shift) & 255u : 256u;
        uint32_t peers = __match_any_sync(0xffffffffu, dg);
        uint32_t r = 0;
        if(ok) r = wcnt[warp][dg] + __popc(peers & lt);
        __syncwarp();
        if(ok && (31 - __clz(peers)) == lane) wcnt[warp][dg] += __popc(peers);
        __syncwarp();
        rank[k] = r;
    }
    __syncthreads();
    // per digit: exclusive over warps, tile total; then exclusive over digits
    uint32_t tot = 0;
    for(int dg = threadIdx.x; dg < kRadix; dg += kThreads) {
        uint32_t off = 0;
        for(int w = 0; w < kWarps; w++) { uint32_t c = wcnt[w][dg]; wcnt[w][dg] = off; off += c; }
        tot = off;
    }
    uint32_t total;
    uint32_t ex = block_exclusive_scan(tot, scan_tmp, total);
    if(threadIdx.x < kRadix) dstart[threadIdx.x] = ex;
    __syncthreads();
#pragma unroll
    for(int k = 0; k < kItems; k++) {
        int64_t idx = base + warp * (32 * kItems) + k * 32 + lane;
        if(idx < n) {
            uint32_t dg = (key[k] >> shift) & 255u;
            uint32_t pos = dstart[dg] + wcnt[warp][dg] + rank[k];
            skey[pos] = key[k];
            sval[pos] = val[k];
        }
    }
    __syncthreads();
    int64_t tile_n = n - base < kTile ? n - base : kTile;
    for(int i = threadIdx.x; i < tile_n; i += kThreads) {
        uint32_t k0 = skey[i];
        uint32_t dg = (k0 >> shift) & 255u;
        int64_t pos = (int64_t)offsets[(int64_t)dg * tiles + blockIdx.x] + (i - dstart[dg]);
        keys_out[pos] = k0;
        vals_out[pos] = sval[i];
    }
}

// Scratch: hist = 256*tiles words, part = ceil(256*tiles/chunk) words.
inline int64_t hist_words(int64_t n) { return (int64_t)kRadix * tiles_for(n); }
inline int64_t part_words(int64_t n) { return (kRadix * tiles_for(n) + kScanChunk - 1) / kScanChunk + 1; }

// Sorts keys[0..n) by their low `bits` bits.  On return *keys_out / *vals_out
// point at whichever buffers hold the result (keys/keys_alt, vals/vals_alt).
inline cudaError_t radix_sort(uint32_t* keys, uint32_t* keys_alt, uint32_t* vals, uint32_t* vals_alt,
    int64_t n, int bits, uint32_t* hist, uint32_t* part, cudaStream_t st,
    uint32_t** keys_out, uint32_t** vals_out)
{
    int passes = (bits + 7) / 8;
    if(passes > kMaxPasses) passes = kMaxPasses;
    if(passes < 1) passes = 1;
    int64_t tiles = tiles_for(n);
    *keys_out = keys;
    *vals_out = nullptr;
    if(n == 0) return cudaSuccess;
    int64_t len = (int64_t)kRadix * tiles;
    int64_t chunks = (len + kScanChunk - 1) / kScanChunk;
    uint32_t *kin = keys, *vin = nullptr, *kout = keys_alt, *vout = vals_alt;
    for(int p = 0; p < passes; p++) {
        uint32_t* h = hist;
        k_hist<<<(unsigned)tiles, kThreads, 0, st>>>(kin, n, 8 * p, tiles, h);
        k_scan_reduce<<<(unsigned)chunks, kThreads, 0, st>>>(h, len, part);
        k_scan_partials<<<1, kThreads, 0, st>>>(part, chunks);
        k_scan_down<<<(unsigned)chunks, kThreads, 0, st>>>(h, len, part);
        k_scatter<<<(unsigned)tiles, kThreads, 0, st>>>(kin, vin, kout, vout, n, 8 * p, tiles, h);
        // ping-pong: keys <-> keys_alt, vals_alt <-> vals
        kin = kout;
        vin = vout;
        kout = (kout == keys_alt) ? keys : keys_alt;
        vout = (vout == vals_alt) ? vals : vals_alt;
    }
    *keys_out = kin;
    *vals_out = vin;
    return cudaGetLastError();
}

}  // namespace mpm_sort
