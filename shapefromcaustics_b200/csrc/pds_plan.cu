// Photon binning of the splatting plan, for sm_100a.
//
// Reference: PyOptix/kernel/photon_differentials.cu:76-89 (the footprint each photon's
// threads recompute in both kernels). Here every photon is binned once per plan, by a
// counting sort over its bucket (simulation, channel, screen tile of the centre pixel,
// footprint class) in two passes over the photon inputs:
//
//   count pass       (coalesced SoA reads) the exact integer footprint and the bucket of every
//                    photon; each CTA takes a contiguous photon range (one or two simulations)
//                    and counts its buckets in a shared-memory histogram over the window of
//                    buckets (up to 32768) that starts at its first photon's simulation; the
//                    histogram is added into the global counts and kept per CTA. Photons wider
//                    than the apron go to the wide list.
//   bucket scan      exclusive scan of the bucket counts (three parallel kernels), giving each
//                    bucket its first sorted position; a copy serves as the place pass's
//                    cursors.
//   place pass       the same CTA ranges: each CTA reserves its share of every bucket with one
//                    atomic on the bucket's cursor, hands positions out from shared memory,
//                    re-bins its photons and writes each one's 32-byte record at its position
//                    (one whole sector), keeping the position per photon (coalesced) for the
//                    backward's gradient spread.
//   chunk_tile       the tile holding the first photon of every tile-kernel work chunk.
//
// Nothing per photon is kept between the passes but the inverse map of wide and untouched
// photons: the place pass recomputes the keys from the inputs (40 bytes a photon read twice)
// instead of writing and reading back keys and photon-order records. Global atomics are per
// CTA and bucket rather than per photon (buckets outside a CTA's window, possible for
// simulations with more buckets than the window, take one global atomic per photon). Photons
// of one bucket land in an arbitrary order; every photon's result is independent of it
// (forward sums are reassociated, as the reference's atomics also do).
#include <cstdint>
#include <cuda_runtime.h>

#include "pds_device.cuh"
#include "pds_internal.h"
#include "pds_splat.h"

namespace pds {

namespace {

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Few large CTAs: the histogram flush and the cursor reservations cost one global atomic per
// CTA and touched bucket, so fewer, larger CTAs make fewer of them. A CTA of 768 threads gives
// each thread the registers to hold the next photon's inputs while it bins the current one
// (measured 3% faster than 1024 threads with one photon in flight).
constexpr int kPlanKernelThreads = 768;
// CTAs of a plan pass at most (each keeps its window histogram between the passes)
constexpr int64_t kPlanMaxCtas = 512;
// buckets of a CTA's shared histogram (128 KB: a 2048^2 image's buckets at 5 class bits; the
// SM keeps about 100 KB of L1 cache for the streamed loads)
constexpr int kMaxWindow = 32768;

// First bucket of the simulation owning photon i.
__device__ __forceinline__ uint32_t window_base(const SimTable& st, int64_t i, int cb) {
    return uint32_t(load_sim(st, find_sim_of_photon(st, i)).tile_base) << cb;
}

__device__ __forceinline__ void zero_window(uint32_t* hist, int window) {
    for (int j = threadIdx.x; j < window; j += blockDim.x) hist[j] = 0u;
}

// The bucket of one photon (key_invalid, key_big, or (tile << cb) | class), for the tile path
// its box radius max(rx, ry) in rmax, and when PLACE its 32-byte record. Both passes run it on
// the same inputs, so they agree on every key.
template <bool PLACE>
__device__ __forceinline__ uint32_t bin_photon(const PlanArgs& a, const pds_sim& sim, double s2w,
                                               double s2h, int64_t ch, float x, float y,
                                               float rad, float e, float m00, float m01,
                                               float m10, float m11, Rec& r, int& rmax) {
    const int T = a.cfg.tile, A = a.cfg.apron, cb = a.cfg.class_bits;
    const uint32_t cls_max = (1u << cb) - 1u;
    if (!(ch >= 0 && ch < sim.channels)) return a.key_invalid;
    const Footprint f = make_footprint(x, y, rad, sim.height, sim.width, a.mpr);
    int32_t x0, x1, y0, y1;
    if (!clip_box(f, sim.height, sim.width, x0, x1, y0, y1)) return a.key_invalid;
    if (f.rx > A || f.ry > A) return a.key_big;
    rmax = max(f.rx, f.ry);
    const int pcx = min(max(f.px_c, 0), sim.width - 1);
    const int pcy = min(max(f.py_c, 0), sim.height - 1);
    // the tile edge is a power of two (16, 32 or 64, checked by the configuration), so the
    // tile of a (non-negative) centre pixel is a shift, not an integer division
    const int tsh = __ffs(T) - 1;
    const int tx = pcx >> tsh, ty = pcy >> tsh;
    const uint32_t tile = uint32_t(sim.tile_base) +
                          uint32_t((int32_t(ch) * sim.tiles_y + ty) * sim.tiles_x + tx);
    const float dy0 = corner_offset_step(f.py_c, s2h, y);
    uint32_t cls = min(uint32_t(max(f.rx, f.ry)), cls_max);
    if (cb == kRowClassBits) {
        // the row walk's classes: rows and row width inside the box
        cls = f.ellipse_all ? plan_row_class(m00, m01, m10, m11, dy0, sim.width, sim.height, f.rx,
                                             x0 - f.px_c, x1 - f.px_c, y0 - f.py_c, y1 - f.py_c)
                            : cls_max;
    } else if (a.cfg.band) {
        // photons of a warp then have similar band areas (trip counts): classes of 1/k octave
        // of the area, k = 1, 2, 3 for up to 3, 4 and 5 class bits
        const float dx0 = corner_offset_step(f.px_c, s2w, x);
        const float sy = float(s2h);  // 2 / H, the division done once per simulation
        const Band bd = make_band(m00, m01, m10, m11, dx0, dy0, sy, 0.5f * float(sim.width),
                                  0.5f * float(sim.height), float(f.rx) + 1.f);
        int area = (2 * f.rx + 1) * (2 * f.ry + 1);
        if (bd.on && f.ellipse_all)
            area = min(area, (min(bd.ky1, f.ry) - max(bd.ky0, -f.ry) + 1) * bd.bw);
        // floor(k log2 area) = floor(log2 area^k), exactly
        const int k = cb <= 3 ? 1 : cb - 2;
        const uint64_t a1 = uint64_t(max(area, 1));
        const uint64_t ak = k == 1 ? a1 : (k == 2 ? a1 * a1 : a1 * a1 * a1);
        const int lg = 63 - __clzll(ak);
        cls = min(uint32_t(max(lg - k, 0)), cls_max);
    }
    if (PLACE) {
        const uint32_t flags = (f.ellipse_all ? kFlagEllipseAll : 0u) | (e > 0.f ? 0u : kFlagFwdSkip);
        r.dx0 = corner_offset_step(f.px_c, s2w, x);
        r.dy0 = dy0;
        r.m00 = m00;
        r.m01 = m01;
        r.m10 = m10;
        r.m11 = m11;
        r.e = e;
        r.packed = pack_rec(f.px_c - (tx * T - A), f.py_c - (ty * T - A), f.rx, f.ry, flags);
    }
    return (tile << cb) | cls;
}

// One pass of the plan over a CTA's contiguous photon range (coalesced SoA reads; each thread
// loads its next photon's inputs while it bins the current one).
//   count (PLACE = false): every photon's bucket into the CTA's shared histogram window (global
//       atomics for buckets outside it), the histogram added into the global counts and kept
//       per CTA in cta_hist; wide photons appended to the wide list; the inverse map of wide
//       and untouched photons.
//   place (PLACE = true, after the scan): the CTA reserves its share of every window bucket
//       with one atomic on the bucket's cursor (from its kept histogram), re-bins its photons,
//       builds each tile-path photon's record and writes it at its sorted position (one whole
//       32-byte sector), keeping the position in the inverse map.
template <bool PLACE>
__global__ __launch_bounds__(kPlanKernelThreads) void plan_pass_kernel(PlanArgs a) {
    extern __shared__ uint32_t hist[];  // a.window buckets
    const int64_t n = a.ph.n;
    const int lane = threadIdx.x & 31;
    const int64_t r0 = int64_t(blockIdx.x) * a.range, r1 = min(r0 + a.range, n);
    const uint32_t kb0 = window_base(a.sims, r0, a.cfg.class_bits);
    const int64_t wend = min(int64_t(a.window), int64_t(a.key_big) - int64_t(kb0));
    uint32_t* mine = a.cta_hist + int64_t(blockIdx.x) * a.window;
    if (PLACE) {
        // hist[j] becomes the CTA's first position in window bucket j
        for (int j = threadIdx.x; j < a.window; j += blockDim.x) {
            const uint32_t c = j < wend ? mine[j] : 0u;
            hist[j] = c ? atomicAdd(a.cursor + kb0 + j, c) : 0u;
        }
    } else {
        zero_window(hist, a.window);
    }
    __syncthreads();
    uint32_t c_tile = 0, c_inv = 0;
    const int64_t* __restrict__ cp = a.ph.cp;
    const float* __restrict__ X = a.ph.X;
    const float* __restrict__ R = a.ph.R;
    const float* __restrict__ E = a.ph.E;
    const float* __restrict__ M = a.ph.M;
    // The thread's simulation is followed along its photons (contiguous per simulation) rather
    // than searched per photon: one table load when a simulation boundary is crossed.
    int sidx = find_sim_of_photon(a.sims, min(r0 + int64_t(threadIdx.x), n - 1));
    pds_sim sim = load_sim(a.sims, sidx);
    int64_t next_begin = sim_end(a.sims, sidx);
    // the pixel pitch in normalised coordinates (2 / W, 2 / H) of the thread's simulation,
    // kept across photons by the count pass (24% faster on 2^23 photons); the place pass, one
    // spilled register short, divides per photon instead (8% faster that way)
    double s2w = 0.0, s2h = 0.0;
    if (!PLACE) {
        s2w = corner_step(sim.width);
        s2h = corner_step(sim.height);
    }
    // whole warps step together (the wide list's ballot needs every lane)
    int64_t nch = 0;
    float nx = 0.f, ny = 0.f, nrad = 0.f, ne = 0.f, n00 = 0.f, n01 = 0.f, n10 = 0.f, n11 = 0.f;
    {
        const int64_t i = r0 + threadIdx.x;
        if (i < r1) {
            nch = __ldg(cp + i); nx = __ldg(X + i); ny = __ldg(X + n + i); nrad = __ldg(R + i);
            n00 = __ldg(M + i); n01 = __ldg(M + n + i);
            n10 = __ldg(M + 3 * n + i); n11 = __ldg(M + 4 * n + i);
            if (PLACE) ne = __ldg(E + i);
        }
    }
    for (int64_t base = r0; base < r1; base += blockDim.x) {
        const int64_t i = base + threadIdx.x;
        const bool valid = i < r1;
        const int64_t ch = nch;
        const float x = nx, y = ny, rad = nrad, e = ne, m00 = n00, m01 = n01, m10 = n10,
                    m11 = n11;
        {
            const int64_t j = i + blockDim.x;
            if (j < r1) {
                nch = __ldg(cp + j); nx = __ldg(X + j); ny = __ldg(X + n + j);
                nrad = __ldg(R + j); n00 = __ldg(M + j);
                n01 = __ldg(M + n + j); n10 = __ldg(M + 3 * n + j); n11 = __ldg(M + 4 * n + j);
                if (PLACE) ne = __ldg(E + j);
            }
        }
        uint32_t key = a.key_invalid;
        int rmax = 0;
        Rec r;
        if (valid) {
            while (i >= next_begin) {  // at most the table's length in all
                ++sidx;
                sim = load_sim(a.sims, sidx);
                next_begin = sim_end(a.sims, sidx);
                if (!PLACE) {
                    s2w = corner_step(sim.width);
                    s2h = corner_step(sim.height);
                }
            }
            key = bin_photon<PLACE>(a, sim, PLACE ? corner_step(sim.width) : s2w,
                                    PLACE ? corner_step(sim.height) : s2h, ch, x, y, rad, e,
                                    m00, m01, m10, m11, r, rmax);
        }
        const bool tile_path = key < a.key_big;
        if (PLACE) {
            if (tile_path) {
                const uint32_t j = key - kb0;
                const uint32_t pos = j < uint32_t(a.window) ? atomicAdd(hist + j, 1u)
                                                           : atomicAdd(a.cursor + key, 1u);
                // both passes bin with the same code on the same inputs, so every position is
                // below the tile-path count; the guard keeps a mismatch inside the arrays
                if (pos < uint32_t(n)) {
                    a.srecs[pos] = r;
                    a.inv[i] = pos;
                }
            }
            continue;
        }
        const bool wide = key == a.key_big;
        c_tile += tile_path;
        c_inv += valid && key == a.key_invalid;
        if (valid && key == a.key_invalid) a.inv[i] = kInvalidPos;
        if (tile_path) {
            const uint32_t j = key - kb0;
            if (j < uint32_t(a.window)) atomicAdd(hist + j, 1u);
            else atomicAdd(a.counts + key, 1u);
            // the tile's largest box radius (the backward stages only the tile's pixels within
            // it): an atomic only where the photon's radius exceeds the value seen (a stale,
            // lower value only costs a redundant atomic; the value only grows)
            uint32_t* tr = a.tile_r + (key >> a.cfg.class_bits);
            if (uint32_t(rmax) > *tr) atomicMax(tr, uint32_t(rmax));
        }
        // wide photons: appended to the wide list (one atomic per warp)
        const uint32_t wm = __ballot_sync(0xFFFFFFFFu, wide);
        if (wm) {
            uint32_t wbase = 0;
            if (lane == __ffs(wm) - 1) wbase = atomicAdd(a.counters + 1, uint32_t(__popc(wm)));
            wbase = __shfl_sync(0xFFFFFFFFu, wbase, __ffs(wm) - 1);
            if (wide) {
                const uint32_t k = wbase + __popc(wm & lanemask_lt());
                a.wide[k] = uint32_t(i);
                a.inv[i] = kWideBit | k;
            }
        }
    }
    if (PLACE) return;
    // block totals -> the tile-path and untouched counters; the window -> the bucket counts
    // and this CTA's kept histogram
    __shared__ uint32_t red[2];
    if (threadIdx.x < 2) red[threadIdx.x] = 0;
    __syncthreads();
    for (int j = threadIdx.x; j < wend; j += blockDim.x) {
        const uint32_t c = hist[j];
        mine[j] = c;
        if (c) atomicAdd(a.counts + kb0 + j, c);
    }
    c_tile = __reduce_add_sync(0xFFFFFFFFu, c_tile);
    c_inv = __reduce_add_sync(0xFFFFFFFFu, c_inv);
    if (lane == 0) {
        atomicAdd(&red[0], c_tile);
        atomicAdd(&red[1], c_inv);
    }
    __syncthreads();
    if (threadIdx.x == 0 && red[0]) atomicAdd(a.counters + 0, red[0]);
    if (threadIdx.x == 1 && red[1]) atomicAdd(a.counters + 2, red[1]);
}

// ------------------------------------------------------------------ bucket scan --------
// Exclusive scan of counts[0, nb) into start[0, nb] (start[nb] = the total) and cursor[0, nb):
// per-CTA sums of kScanItems buckets, one CTA scanning those sums, then each CTA's rescan.

constexpr int kScanThreads = 256;
constexpr int kScanPer = 16;
constexpr int kScanItems = kScanThreads * kScanPer;

// Exclusive scan of one value per thread over the CTA; *total gets the CTA's sum.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t wsum[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kScanThreads / 32 ? wsum[lane] : 0u;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, off);
            if (lane >= off) w += y;
        }
        if (lane < kScanThreads / 32) wsum[lane] = w;
    }
    __syncthreads();
    const uint32_t before = warp > 0 ? wsum[warp - 1] : 0u;
    *total = wsum[kScanThreads / 32 - 1];
    __syncthreads();
    return before + x - v;
}

__global__ __launch_bounds__(kScanThreads) void bucket_reduce(const uint32_t* __restrict__ counts,
                                                              int64_t nb,
                                                              uint32_t* __restrict__ part) {
    const int64_t b0 = int64_t(blockIdx.x) * kScanItems;
    uint32_t s = 0;
    for (int k = threadIdx.x; k < kScanItems; k += kScanThreads) {
        const int64_t j = b0 + k;
        if (j < nb) s += __ldg(counts + j);
    }
    uint32_t total;
    block_exclusive_scan(s, &total);
    if (threadIdx.x == 0) part[blockIdx.x] = total;
}

__global__ __launch_bounds__(kScanThreads) void bucket_top(uint32_t* __restrict__ part,
                                                           int64_t np, uint32_t* __restrict__ start,
                                                           int64_t nb) {
    uint32_t carry = 0;
    for (int64_t b = 0; b < np; b += kScanThreads) {
        const int64_t j = b + threadIdx.x;
        const uint32_t v = j < np ? part[j] : 0u;
        uint32_t total;
        const uint32_t ex = block_exclusive_scan(v, &total);
        if (j < np) part[j] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) start[nb] = carry;
}

__global__ __launch_bounds__(kScanThreads) void bucket_down(const uint32_t* __restrict__ counts,
                                                            int64_t nb,
                                                            const uint32_t* __restrict__ part,
                                                            uint32_t* __restrict__ start,
                                                            uint32_t* __restrict__ cursor) {
    // thread t owns buckets [b0 + t * kScanPer, + kScanPer)
    const int64_t b0 = int64_t(blockIdx.x) * kScanItems + int64_t(threadIdx.x) * kScanPer;
    uint32_t v[kScanPer];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        v[k] = b0 + k < nb ? __ldg(counts + b0 + k) : 0u;
        s += v[k];
    }
    uint32_t total;
    uint32_t run = part[blockIdx.x] + block_exclusive_scan(s, &total);
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        if (b0 + k < nb) {
            start[b0 + k] = run;
            cursor[b0 + k] = run;
        }
        run += v[k];
    }
}

// Tile of the first photon of every work chunk: the last tile whose bucket range starts at or
// before the chunk's first position (empty tiles start where their successor does).
__global__ __launch_bounds__(256) void chunk_tile_kernel(ScanArgs a) {
    const int64_t n_tile = min(int64_t(a.counters[0]), a.n);
    const int64_t nchunks = (n_tile + a.chunk - 1) / a.chunk;
    for (int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; c < nchunks;
         c += int64_t(gridDim.x) * blockDim.x) {
        const uint32_t p = uint32_t(c * a.chunk);
        int64_t lo = 0, hi = a.n_tiles - 1;
        while (lo < hi) {
            const int64_t mid = (lo + hi + 1) >> 1;
            if (__ldg(a.start + (mid << a.cb)) <= p) lo = mid; else hi = mid - 1;
        }
        a.chunk_tile[c] = uint32_t(lo);
    }
}

// The plan's binning per photon: its bucket (from its sorted position and the bucket starts)
// and its slot (sorted position, wide-list index, or kInvalidPos).
__global__ __launch_bounds__(256) void plan_export_kernel(const uint32_t* __restrict__ inv,
                                                          const uint32_t* __restrict__ start,
                                                          int64_t nb, uint32_t key_big,
                                                          uint32_t key_invalid, int64_t n,
                                                          uint32_t* bucket, uint32_t* slot) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x) {
        const uint32_t v = inv[i];
        uint32_t b;
        if (v == kInvalidPos) {
            b = key_invalid;
        } else if (v & kWideBit) {
            b = key_big;
        } else {
            // the last bucket whose first position is at or before v (empty buckets start
            // where their successor does, so this is v's own bucket)
            int64_t lo = 0, hi = nb - 1;
            while (lo < hi) {
                const int64_t mid = (lo + hi + 1) >> 1;
                if (start[mid] <= v) lo = mid; else hi = mid - 1;
            }
            b = uint32_t(lo);
        }
        bucket[i] = b;
        slot[i] = v == kInvalidPos ? kInvalidPos : (v & ~kWideBit);
    }
}

int num_sms() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

unsigned capped_blocks(int64_t items, int per_sm) {
    const int64_t blocks = (items + 255) / 256;
    const int64_t cap = int64_t(num_sms()) * per_sm;
    return unsigned(blocks < 1 ? 1 : (blocks < cap ? blocks : cap));
}

}  // namespace

int64_t bucket_scan_parts(int64_t nb) { return (nb + kScanItems - 1) / kScanItems; }

template <typename K>
cudaError_t window_smem(K kernel, int32_t window) {
    const size_t smem = size_t(window) * 4;
    if (smem <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
}

// Window and photons per CTA of the two plan passes: the window holds a simulation's buckets
// where it can (at most kMaxWindow); as many CTAs per SM as the window's shared memory allows
// (the kernels' shared-memory limit is raised first, or the occupancy query would see a kernel
// that cannot launch), at most kPlanMaxCtas in all (the size of the kept histograms), and the
// photons are split evenly over one wave of them (at least 8192 a CTA, so the window's clear
// and flush are amortised).
void plan_shape(int64_t n, int64_t nb, int32_t* window, int64_t* range) {
    const int64_t w = nb < kMaxWindow ? nb : kMaxWindow;
    *window = int32_t(w > 0 ? w : 1);
    const size_t smem = size_t(*window) * 4;
    int per_sm = 1;
    if (window_smem(plan_pass_kernel<false>, *window) != cudaSuccess ||
        window_smem(plan_pass_kernel<true>, *window) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, plan_pass_kernel<false>,
                                                      kPlanKernelThreads, smem) != cudaSuccess)
        per_sm = 1;
    if (per_sm < 1) per_sm = 1;
    int64_t ctas = int64_t(num_sms()) * per_sm;
    if (ctas > kPlanMaxCtas) ctas = kPlanMaxCtas;
    int64_t r = (n + ctas - 1) / ctas;
    r = (r + kPlanKernelThreads - 1) / kPlanKernelThreads * kPlanKernelThreads;
    *range = r < 8192 ? 8192 : r;
}

int64_t plan_hist_entries(int64_t n, int64_t nb) {
    const int64_t w = nb < kMaxWindow ? (nb > 0 ? nb : 1) : kMaxWindow;
    const int64_t by_n = (n + 8191) / 8192;
    return (by_n < kPlanMaxCtas ? (by_n > 0 ? by_n : 1) : kPlanMaxCtas) * w;
}

template <bool PLACE>
cudaError_t launch_pass(const PlanArgs& a, cudaStream_t st) {
    if (a.ph.n <= 0) return cudaSuccess;
    cudaError_t e = window_smem(plan_pass_kernel<PLACE>, a.window);
    if (e != cudaSuccess) return e;
    plan_pass_kernel<PLACE><<<unsigned((a.ph.n + a.range - 1) / a.range), kPlanKernelThreads,
                              size_t(a.window) * 4, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_plan_count(const PlanArgs& a, cudaStream_t st) { return launch_pass<false>(a, st); }

cudaError_t launch_plan_place(const PlanArgs& a, cudaStream_t st) { return launch_pass<true>(a, st); }

cudaError_t launch_plan_export(const uint32_t* inv, const uint32_t* start, int64_t nb,
                               uint32_t key_big, uint32_t key_invalid, int64_t n,
                               uint32_t* bucket, uint32_t* slot, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    plan_export_kernel<<<capped_blocks(n, 8), 256, 0, st>>>(inv, start, nb, key_big, key_invalid,
                                                            n, bucket, slot);
    return cudaGetLastError();
}

cudaError_t launch_bucket_scan(const ScanArgs& a, cudaStream_t st) {
    const int64_t np = bucket_scan_parts(a.nb);
    bucket_reduce<<<unsigned(np), kScanThreads, 0, st>>>(a.counts, a.nb, a.part);
    bucket_top<<<1, kScanThreads, 0, st>>>(a.part, np, a.start, a.nb);
    bucket_down<<<unsigned(np), kScanThreads, 0, st>>>(a.counts, a.nb, a.part, a.start,
                                                       a.cursor);
    return cudaGetLastError();
}

cudaError_t launch_chunk_tiles(const ScanArgs& a, cudaStream_t st) {
    if (a.n <= 0) return cudaSuccess;
    chunk_tile_kernel<<<capped_blocks((a.n + a.chunk - 1) / a.chunk, 4), 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace pds
