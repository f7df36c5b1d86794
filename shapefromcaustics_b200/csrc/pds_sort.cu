// Stable LSD radix sort of 32-bit keys with a 32-bit index payload, for sm_100a, exposed as
// pds_sort_u32. (The splatting plan bins photons with a counting sort by bucket, pds_plan.cu;
// this sort serves callers that need the stable order of arbitrary keys.) The permutation
// equals a CPU stable sort bit for bit, so every pass is stable:
//   upsweep    per 2048-key block digit counts (warp-aggregated shared atomics), block-major
//   col scan   column-wise exclusive scan of the [blocks][radix] count matrix in three
//              coalesced kernels (group partials, one-CTA top scan with digit bases, group
//              down-sweep), yielding each block's first output slot per digit
//   downsweep  stable rank inside the block (warp-striped order: warp w owns a contiguous
//              256-key range, ranked per 32-key step with __match_any_sync), the block's
//              keys staged in shared memory in digit order, then each digit's run written
//              contiguously (coalesced stores instead of one scattered store per key)
// Digits are at most 8 bits; the number of passes is ceil(key_bits / 8) with the bits spread
// evenly, so a 9-bit key space costs two 5/4-bit passes and a 16-bit one two 8-bit passes.
#include <cstdint>
#include <cuda_runtime.h>

#include "pds_internal.h"

namespace pds {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kIpt = 8;                        // keys per thread
constexpr int kTileKeys = kThreads * kIpt;     // keys per sort block
constexpr int kGroup = 64;                     // sort blocks per column-scan group

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__global__ __launch_bounds__(kThreads) void sort_upsweep(const uint32_t* __restrict__ keys,
                                                         int64_t n, int shift, int bits,
                                                         uint32_t* __restrict__ hist) {
    __shared__ uint32_t cnt[256];
    const int radix = 1 << bits;
    const uint32_t mask = uint32_t(radix - 1);
    for (int d = threadIdx.x; d < radix; d += kThreads) cnt[d] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t base = int64_t(blockIdx.x) * kTileKeys;
#pragma unroll 4
    for (int j = 0; j < kIpt; ++j) {
        const int64_t i = base + int64_t(j) * kThreads + threadIdx.x;
        const bool valid = i < n;
        const uint32_t d = valid ? (__ldg(keys + i) >> shift) & mask : 0xFFFFFFFFu;
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        if (valid && lane == __ffs(peers) - 1) atomicAdd(&cnt[d], uint32_t(__popc(peers)));
    }
    __syncthreads();
    for (int d = threadIdx.x; d < radix; d += kThreads)
        hist[int64_t(blockIdx.x) * radix + d] = cnt[d];
}

__global__ __launch_bounds__(kThreads) void sort_col_partials(const uint32_t* __restrict__ hist,
                                                              int64_t nblocks, int radix,
                                                              uint32_t* __restrict__ part) {
    const int d = threadIdx.x;
    if (d >= radix) return;
    const int64_t b0 = int64_t(blockIdx.x) * kGroup;
    const int64_t b1 = min(b0 + kGroup, nblocks);
    uint32_t s = 0;
    for (int64_t b = b0; b < b1; ++b) s += hist[b * radix + d];
    part[int64_t(blockIdx.x) * radix + d] = s;
}

__global__ __launch_bounds__(kThreads) void sort_col_top(uint32_t* __restrict__ part,
                                                         int64_t ngroups, int radix) {
    __shared__ uint32_t tot[kThreads];
    const int d = threadIdx.x;
    uint32_t run = 0;
    if (d < radix) {
        for (int64_t g = 0; g < ngroups; ++g) {
            const uint32_t t = part[g * radix + d];
            part[g * radix + d] = run;
            run += t;
        }
    }
    tot[d] = d < radix ? run : 0u;
    __syncthreads();
    // exclusive scan of the digit totals (Hillis-Steele over 256 entries)
    for (int off = 1; off < kThreads; off <<= 1) {
        const uint32_t v = d >= off ? tot[d - off] : 0u;
        __syncthreads();
        tot[d] += v;
        __syncthreads();
    }
    const uint32_t base = d > 0 ? tot[d - 1] : 0u;
    if (d < radix)
        for (int64_t g = 0; g < ngroups; ++g) part[g * radix + d] += base;
}

__global__ __launch_bounds__(kThreads) void sort_col_down(uint32_t* __restrict__ hist,
                                                          int64_t nblocks, int radix,
                                                          const uint32_t* __restrict__ part) {
    const int d = threadIdx.x;
    if (d >= radix) return;
    const int64_t b0 = int64_t(blockIdx.x) * kGroup;
    const int64_t b1 = min(b0 + kGroup, nblocks);
    uint32_t run = part[int64_t(blockIdx.x) * radix + d];
    for (int64_t b = b0; b < b1; ++b) {
        const uint32_t t = hist[b * radix + d];
        hist[b * radix + d] = run;
        run += t;
    }
}

__global__ __launch_bounds__(kThreads) void sort_downsweep(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, int64_t n,
    int shift, int bits, const uint32_t* __restrict__ hist, uint32_t* __restrict__ keys_out,
    uint32_t* __restrict__ vals_out) {
    __shared__ uint32_t wcnt[kWarps][256];
    __shared__ uint32_t boff[256];
    __shared__ uint32_t dstart[256];
    __shared__ uint32_t skey[kTileKeys];
    __shared__ uint32_t sval[kTileKeys];
    const int radix = 1 << bits;
    const uint32_t mask = uint32_t(radix - 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int k = threadIdx.x; k < kWarps * 256; k += kThreads) (&wcnt[0][0])[k] = 0;
    for (int d = threadIdx.x; d < radix; d += kThreads)
        boff[d] = hist[int64_t(blockIdx.x) * radix + d];
    __syncthreads();

    const int64_t block0 = int64_t(blockIdx.x) * kTileKeys;
    const int64_t base = block0 + int64_t(warp) * (32 * kIpt);
    const uint32_t lt = lanemask_lt();
    uint32_t k[kIpt], v[kIpt], rank[kIpt];
#pragma unroll
    for (int j = 0; j < kIpt; ++j) {
        const int64_t i = base + j * 32 + lane;
        const bool valid = i < n;
        k[j] = valid ? __ldg(keys_in + i) : 0xFFFFFFFFu;
        v[j] = valid ? (vals_in ? __ldg(vals_in + i) : uint32_t(i)) : 0u;
        const uint32_t d = valid ? (k[j] >> shift) & mask : 0xFFFFFFFFu;
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        uint32_t prior = 0;
        if (valid) prior = wcnt[warp][d];
        rank[j] = prior + __popc(peers & lt);
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) wcnt[warp][d] = prior + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive offsets of the warps, and the block's total
    uint32_t total = 0;
    if (threadIdx.x < radix) {
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t t = wcnt[w][threadIdx.x];
            wcnt[w][threadIdx.x] = total;
            total += t;
        }
    }
    // exclusive scan of the block's digit totals (Hillis-Steele over 256 entries)
    dstart[threadIdx.x] = total;
    __syncthreads();
    for (int off = 1; off < kThreads; off <<= 1) {
        const uint32_t add = threadIdx.x >= off ? dstart[threadIdx.x - off] : 0u;
        __syncthreads();
        dstart[threadIdx.x] += add;
        __syncthreads();
    }
    const uint32_t incl = dstart[threadIdx.x];
    __syncthreads();
    dstart[threadIdx.x] = incl - total;
    __syncthreads();
    // stage the block's keys in digit order, then write each digit's run contiguously
#pragma unroll
    for (int j = 0; j < kIpt; ++j) {
        const int64_t i = base + j * 32 + lane;
        if (i < n) {
            const uint32_t d = (k[j] >> shift) & mask;
            const uint32_t spos = dstart[d] + wcnt[warp][d] + rank[j];
            skey[spos] = k[j];
            sval[spos] = v[j];
        }
    }
    __syncthreads();
    const int count = int(min(int64_t(kTileKeys), n - block0));
    for (int t = threadIdx.x; t < count; t += kThreads) {
        const uint32_t key = skey[t];
        const uint32_t d = (key >> shift) & mask;
        const uint32_t pos = boff[d] + (uint32_t(t) - dstart[d]);
        keys_out[pos] = key;
        vals_out[pos] = sval[t];
    }
}

}  // namespace

int sort_passes(int key_bits) { return key_bits <= 0 ? 0 : (key_bits + 7) / 8; }

size_t sort_aux_bytes(int64_t n) {
    const int64_t nb = (n + kTileKeys - 1) / kTileKeys;
    const int64_t ng = (nb + kGroup - 1) / kGroup;
    return align_up(size_t(nb > 0 ? nb : 1) * 256 * sizeof(uint32_t), 256) +
           align_up(size_t(ng > 0 ? ng : 1) * 256 * sizeof(uint32_t), 256);
}

cudaError_t radix_sort(const uint32_t* keys_in, uint32_t* k0, uint32_t* k1, uint32_t* v0,
                       uint32_t* v1, int64_t n, int key_bits, void* aux, cudaStream_t st,
                       uint32_t** keys_out, uint32_t** vals_out) {
    const int passes = sort_passes(key_bits);
    *keys_out = nullptr;
    *vals_out = nullptr;
    if (n <= 0) return cudaSuccess;
    const int64_t nb = (n + kTileKeys - 1) / kTileKeys;
    const int64_t ng = (nb + kGroup - 1) / kGroup;
    uint32_t* hist = static_cast<uint32_t*>(aux);
    uint32_t* part = reinterpret_cast<uint32_t*>(static_cast<char*>(aux) +
                                                 align_up(size_t(nb) * 256 * sizeof(uint32_t), 256));
    const uint32_t* kin = keys_in;
    const uint32_t* vin = nullptr;
    uint32_t* kb[2] = {k0, k1};
    uint32_t* vb[2] = {v0, v1};
    if (passes == 0) {
        // a single key value: the identity permutation
        cudaError_t e = cudaMemcpyAsync(k0, keys_in, size_t(n) * 4, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return e;
        iota_u32(v0, n, st);
        *keys_out = k0;
        *vals_out = v0;
        return cudaGetLastError();
    }
    int shift = 0;
    for (int p = 0; p < passes; ++p) {
        const int bits = key_bits / passes + (p < key_bits % passes ? 1 : 0);
        const int radix = 1 << bits;
        sort_upsweep<<<unsigned(nb), kThreads, 0, st>>>(kin, n, shift, bits, hist);
        sort_col_partials<<<unsigned(ng), kThreads, 0, st>>>(hist, nb, radix, part);
        sort_col_top<<<1, kThreads, 0, st>>>(part, ng, radix);
        sort_col_down<<<unsigned(ng), kThreads, 0, st>>>(hist, nb, radix, part);
        sort_downsweep<<<unsigned(nb), kThreads, 0, st>>>(kin, vin, n, shift, bits, hist,
                                                           kb[p & 1], vb[p & 1]);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        kin = kb[p & 1];
        vin = vb[p & 1];
        shift += bits;
    }
    *keys_out = kb[(passes - 1) & 1];
    *vals_out = vb[(passes - 1) & 1];
    return cudaSuccess;
}

}  // namespace pds
