// extern "C" entry points of libpds_b200.so (declared in include/pds_b200.h).
//
// This layer validates arguments the way the reference's binding does
// (PyOptix/PhotonDifferentialSplattig.cpp:14-22: matching photon counts, 2-row positions,
// 2x3 matrices, one channel row), lays the workspace out, and enqueues
//   plan:     counter and bucket-count reset, plan count pass, bucket scan, plan place pass,
//             chunk_tile_kernel
//   forward:  output reset, fwd_tiles_kernel, tail_fwd_kernel
//   backward: bwd_tiles_kernel, tail_bwd_kernel, grad_scatter_kernel
// on the caller's stream. It allocates nothing and never synchronises. Failures return a
// PDS_ERR_* code and leave a message for pds_last_error() (the reference raises through
// TORCH_CHECK and does not check its launches, photon_differentials.cu:125, :234).
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "pds_internal.h"
#include "pds_splat.h"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* where) {
    g_err = std::string(where) + ": " + cudaGetErrorString(e);
    return PDS_ERR_CUDA;
}

struct Resolved {
    pds::Cfg cfg;
    int64_t n_buckets;
    uint32_t key_big, key_invalid;
};

int resolve_cfg(const pds_config* in, pds_config& out) {
    out.tile = (in && in->tile) ? in->tile : 64;
    out.chunk = (in && in->chunk) ? in->chunk : 2048;
    out.class_bits = (in && in->class_bits) ? in->class_bits : 5;
    if (out.class_bits == -1) out.class_bits = 0;
    out.apron_max = (in && in->apron_max) ? in->apron_max : 32;
    out.walk = (in && in->walk) ? in->walk : 3;
    out.min_blocks = (in && in->min_blocks) ? in->min_blocks : 3;
    out.coop_radius = (in && in->coop_radius) ? in->coop_radius : -1;
    if (out.coop_radius < -1 || out.coop_radius > 63)
        return fail(PDS_ERR_INVALID_ARGUMENT, "pds_config.coop_radius must be -1 or in [1, 63]");
    if (out.min_blocks < 2 || out.min_blocks > 4)
        return fail(PDS_ERR_INVALID_ARGUMENT, "pds_config.min_blocks must be 2, 3 or 4");
    if (out.walk < 1 || out.walk > 4)
        return fail(PDS_ERR_INVALID_ARGUMENT,
                    "pds_config.walk must be 1 (box), 2 (support spans), 3 (support band) or "
                    "4 (band rows padded per warp)");
    if (out.tile != 16 && out.tile != 32 && out.tile != 64)
        return fail(PDS_ERR_INVALID_ARGUMENT, "pds_config.tile must be 16, 32 or 64");
    if (out.chunk < 256 || out.chunk > (1 << 20) || out.chunk % 256 != 0)
        return fail(PDS_ERR_INVALID_ARGUMENT,
                    "pds_config.chunk must be a multiple of 256 in [256, 1048576]");
    if (out.class_bits < 0 || out.class_bits > 6)
        return fail(PDS_ERR_INVALID_ARGUMENT, "pds_config.class_bits must be -1 or in [1, 6]");
    if (out.apron_max < 1 || out.apron_max > 63 || out.tile + 2 * out.apron_max > 255)
        return fail(PDS_ERR_INVALID_ARGUMENT,
                    "pds_config.apron_max must be in [1, 63] with tile + 2*apron_max <= 255");
    return PDS_OK;
}

// Photons per tile-kernel work chunk: the configured chunk, lowered for small photon counts
// so that every resident CTA of the tile kernels (3 per SM) gets about four chunks; at least
// 256 photons (one CTA-wide batch).
int32_t effective_chunk(int32_t chunk, int64_t n) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        sms = 148;
    const int64_t target = (n + int64_t(sms) * 12 - 1) / (int64_t(sms) * 12);
    const int64_t c = (target + 255) / 256 * 256;
    return int32_t(c < 256 ? 256 : (c < chunk ? c : chunk));
}

int resolve(const pds_config* in, int32_t mpr, int64_t n_tiles, int64_t n, Resolved& r) {
    pds_config c;
    int rc = resolve_cfg(in, c);
    if (rc) return rc;
    if (n_tiles < 1 || n_tiles >= (int64_t(1) << 30))
        return fail(PDS_ERR_UNSUPPORTED, "tile count outside [1, 2^30)");
    const uint64_t inv = uint64_t(n_tiles + 1) << c.class_bits;
    if (inv >= (uint64_t(1) << 32))
        return fail(PDS_ERR_UNSUPPORTED, "sort key space exceeds 32 bits; lower class_bits");
    r.cfg.tile = c.tile;
    r.cfg.chunk = effective_chunk(c.chunk, n);
    r.cfg.class_bits = c.class_bits;
    r.cfg.apron = mpr < 0 ? 0 : (mpr < c.apron_max ? mpr : c.apron_max);
    // odd pitch: the rows of one column of the accumulator fall in different banks
    r.cfg.sw = (c.tile + 2 * r.cfg.apron) | 1;
    // the row walk sends photons without a band to the support-span walk
    r.cfg.spans = (c.walk == 2 || c.walk == 4) ? 1 : 0;
    r.cfg.band = c.walk == 3 ? 1 : 0;
    r.cfg.rows = c.walk == 4 ? 1 : 0;
    // default: the forward at 3 CTAs an SM (room for its record staging buffers), the
    // backward at 4 (measured best for each); an explicit min_blocks sets both
    r.cfg.min_blocks = c.min_blocks;
    r.cfg.min_blocks_bwd = (in && in->min_blocks) ? c.min_blocks : 4;
    r.cfg.coop_r = c.coop_radius > 0 ? c.coop_radius : 0;
    r.n_buckets = n_tiles << c.class_bits;
    r.key_big = uint32_t(r.n_buckets);
    r.key_invalid = uint32_t(inv);
    return PDS_OK;
}

// The plan's workspace: the inverse map, the wide list, the records in sorted order, the
// bucket counts, starts and cursors, each plan CTA's window histogram (kept from the count pass
// for the place pass), the chunks' tiles, each tile's largest box radius (sized by the bucket
// count, which bounds the tile count), and the backward's gradient records (stage, 32 bytes a
// photon).
struct Layout {
    size_t counters, inv, wide, stage, srecs, counts, start, cursor, part, cta_hist, chunk_tile,
        tile_r, total;
};

// Photon count n, bucket count nb (tiles << class bits).
Layout make_layout(int64_t n, int64_t nb) {
    Layout L;
    const size_t nn = size_t(n > 0 ? n : 1);
    const size_t nbb = size_t(nb > 0 ? nb : 1);
    size_t off = 0;
    L.counters = off; off += 256;
    L.inv = off; off += pds::align_up(nn * 4, 256);
    L.wide = off; off += pds::align_up(nn * 4, 256);
    L.stage = off; off += pds::align_up(nn * sizeof(pds::GradRec), 256);
    L.srecs = off; off += pds::align_up(nn * sizeof(pds::Rec), 256);
    L.counts = off; off += pds::align_up(nbb * 4, 256);
    L.start = off; off += pds::align_up((nbb + 1) * 4, 256);
    L.cursor = off; off += pds::align_up(nbb * 4, 256);
    L.part = off; off += pds::align_up(size_t(pds::bucket_scan_parts(int64_t(nbb))) * 4, 256);
    L.cta_hist = off;
    off += pds::align_up(size_t(pds::plan_hist_entries(int64_t(nn), int64_t(nbb))) * 4, 256);
    L.chunk_tile = off; off += pds::align_up((nn / 256 + 2) * 4, 256);  // chunks >= 256
    L.tile_r = off; off += pds::align_up(nbb * 4, 256);
    L.total = off;
    return L;
}

struct Bufs {
    uint32_t* counters;
    uint32_t *inv, *wide, *counts, *start, *cursor, *part, *cta_hist, *chunk_tile, *tile_r;
    pds::Rec* srecs;
    pds::GradRec* stage;
};

Bufs bufs(void* ws, const Layout& L) {
    char* b = static_cast<char*>(ws);
    Bufs r;
    r.counters = reinterpret_cast<uint32_t*>(b + L.counters);
    r.inv = reinterpret_cast<uint32_t*>(b + L.inv);
    r.wide = reinterpret_cast<uint32_t*>(b + L.wide);
    r.counts = reinterpret_cast<uint32_t*>(b + L.counts);
    r.start = reinterpret_cast<uint32_t*>(b + L.start);
    r.cursor = reinterpret_cast<uint32_t*>(b + L.cursor);
    r.part = reinterpret_cast<uint32_t*>(b + L.part);
    r.cta_hist = reinterpret_cast<uint32_t*>(b + L.cta_hist);
    r.chunk_tile = reinterpret_cast<uint32_t*>(b + L.chunk_tile);
    r.tile_r = reinterpret_cast<uint32_t*>(b + L.tile_r);
    r.srecs = reinterpret_cast<pds::Rec*>(b + L.srecs);
    r.stage = reinterpret_cast<pds::GradRec*>(b + L.stage);
    return r;
}

// Bucket count of a configuration over n_tiles tiles (0 when the configuration is invalid;
// the entry points report that).
int64_t bucket_count(const pds_config* cfg, int64_t n_tiles) {
    pds_config c;
    if (resolve_cfg(cfg, c) != PDS_OK || n_tiles < 1 || n_tiles >= (int64_t(1) << 30)) return 0;
    return n_tiles << c.class_bits;
}

int check_photons(const float* E, const float* X, const float* M, const int64_t* cp,
                  const float* R, int64_t n) {
    if (n < 0) return fail(PDS_ERR_INVALID_ARGUMENT, "negative photon count");
    if (n >= int64_t(0x7FFFFFFFll))
        return fail(PDS_ERR_UNSUPPORTED, "photon count must be below 2^31 - 1");
    if (n > 0 && (!E || !X || !M || !cp || !R))
        return fail(PDS_ERR_INVALID_ARGUMENT, "null photon array");
    return PDS_OK;
}

int check_ws(void* ws, size_t have, size_t need) {
    if (!ws) return fail(PDS_ERR_WORKSPACE, "workspace is null");
    if (reinterpret_cast<uintptr_t>(ws) % 256 != 0)
        return fail(PDS_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    if (have < need)
        return fail(PDS_ERR_WORKSPACE, "workspace too small: need " + std::to_string(need) +
                                           " bytes, got " + std::to_string(have));
    return PDS_OK;
}

int check_image(int64_t C, int64_t H, int64_t W) {
    if (C < 1 || H < 1 || W < 1)
        return fail(PDS_ERR_INVALID_ARGUMENT, "output_size entries must be positive");
    if (H > 65535 || W > 65535)
        return fail(PDS_ERR_UNSUPPORTED, "image height and width must be at most 65535");
    if (C > 65535) return fail(PDS_ERR_UNSUPPORTED, "at most 65535 channels");
    return PDS_OK;
}

pds_sim single_sim(int64_t n, int64_t C, int64_t H, int64_t W, int tile) {
    pds_sim s;
    std::memset(&s, 0, sizeof(s));
    s.photon_begin = 0;
    s.n_photons = n;
    s.image_offset = 0;
    s.channels = int32_t(C);
    s.height = int32_t(H);
    s.width = int32_t(W);
    s.tiles_x = int32_t((W + tile - 1) / tile);
    s.tiles_y = int32_t((H + tile - 1) / tile);
    s.tile_base = 0;
    return s;
}

pds::SimTable table_one(const pds_sim& s) {
    pds::SimTable t;
    t.dev = nullptr;
    t.n = 1;
    t.one = s;
    return t;
}

pds::SimTable table_dev(const pds_sim* dev, int32_t n) {
    pds::SimTable t;
    std::memset(&t, 0, sizeof(t));
    t.dev = dev;
    t.n = n;
    return t;
}

// ---- shared implementations -------------------------------------------------------

int plan_impl(const pds::Photons& ph, const pds::SimTable& st, int64_t n_tiles, int32_t mpr,
              const pds_config* cfg, void* ws, size_t ws_bytes, cudaStream_t s) {
    Resolved r;
    int rc = resolve(cfg, mpr, n_tiles, ph.n, r);
    if (rc) return rc;
    const Layout L = make_layout(ph.n, r.n_buckets);
    rc = check_ws(ws, ws_bytes, L.total);
    if (rc) return rc;
    const Bufs b = bufs(ws, L);
    cudaError_t e = cudaMemsetAsync(b.counters, 0, 16, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.counts, 0, size_t(r.n_buckets) * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.tile_r, 0, size_t(n_tiles) * 4, s);
    if (e != cudaSuccess) return cuda_fail(e, "plan: counter reset");
    pds::PlanArgs a;
    a.ph = ph;
    a.sims = st;
    a.mpr = mpr;
    a.cfg = r.cfg;
    a.key_big = r.key_big;
    a.key_invalid = r.key_invalid;
    a.counts = b.counts;
    a.inv = b.inv;
    a.wide = b.wide;
    a.counters = b.counters;
    a.cta_hist = b.cta_hist;
    a.cursor = b.cursor;
    a.srecs = b.srecs;
    a.tile_r = b.tile_r;
    pds::plan_shape(ph.n, r.n_buckets, &a.window, &a.range);
    e = pds::launch_plan_count(a, s);
    if (e != cudaSuccess) return cuda_fail(e, "plan count pass");
    pds::ScanArgs sa;
    sa.counts = b.counts;
    sa.counters = b.counters;
    sa.part = b.part;
    sa.start = b.start;
    sa.cursor = b.cursor;
    sa.chunk_tile = b.chunk_tile;
    sa.n = ph.n;
    sa.nb = r.n_buckets;
    sa.n_tiles = n_tiles;
    sa.chunk = r.cfg.chunk;
    sa.cb = r.cfg.class_bits;
    e = pds::launch_bucket_scan(sa, s);
    if (e != cudaSuccess) return cuda_fail(e, "bucket scan");
    e = pds::launch_plan_place(a, s);
    if (e != cudaSuccess) return cuda_fail(e, "plan place pass");
    e = pds::launch_chunk_tiles(sa, s);
    if (e != cudaSuccess) return cuda_fail(e, "chunk_tile_kernel");
    return PDS_OK;
}

int tile_args(const pds::Photons& ph, const pds::SimTable& st, int64_t n_tiles, int32_t mpr,
              const pds_config* cfg, void* ws, size_t ws_bytes, pds::TileArgs& a) {
    Resolved r;
    int rc = resolve(cfg, mpr, n_tiles, ph.n, r);
    if (rc) return rc;
    const Layout L = make_layout(ph.n, r.n_buckets);
    rc = check_ws(ws, ws_bytes, L.total);
    if (rc) return rc;
    const Bufs b = bufs(ws, L);
    std::memset(&a, 0, sizeof(a));
    a.ph = ph;
    a.sims = st;
    a.mpr = mpr;
    a.cfg = r.cfg;
    a.n_tiles = n_tiles;
    a.srecs = b.srecs;
    a.start = b.start;
    a.chunk_tile = b.chunk_tile;
    a.inv = b.inv;
    a.wide = b.wide;
    a.tile_r = b.tile_r;
    a.stage = b.stage;
    a.counters = b.counters;
    a.queue = b.counters + 4;  // [0..3) plan counters; [4] the tile kernels' work counter
    return PDS_OK;
}

int forward_impl(const pds::Photons& ph, const pds::SimTable& st, int64_t n_tiles,
                 int64_t image_elems, int32_t mpr, float* out, const pds_config* cfg, void* ws,
                 size_t ws_bytes, cudaStream_t s) {
    if (!out) return fail(PDS_ERR_INVALID_ARGUMENT, "null output image");
    pds::TileArgs a;
    int rc = tile_args(ph, st, n_tiles, mpr, cfg, ws, ws_bytes, a);
    if (rc) return rc;
    a.out = out;
    a.image_elems = image_elems;
    cudaError_t e = cudaMemsetAsync(out, 0, size_t(image_elems) * sizeof(float), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.queue, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return cuda_fail(e, "forward: output reset");
    if (ph.n == 0) return PDS_OK;
    e = pds::launch_forward(a, s);
    if (e != cudaSuccess) return cuda_fail(e, "fwd_tiles_kernel");
    return PDS_OK;
}

int backward_impl(const float* grad, const pds::Photons& ph, const pds::SimTable& st,
                  int64_t n_tiles, int64_t image_elems, int32_t mpr, float* gE, float* gX,
                  float* gM, const pds_config* cfg, void* ws, size_t ws_bytes, cudaStream_t s) {
    // all three outputs null: the gradients stay in the workspace as records
    const bool records = !gE && !gX && !gM;
    if (ph.n > 0 && (!grad || (!records && (!gE || !gX || !gM))))
        return fail(PDS_ERR_INVALID_ARGUMENT, "null gradient array");
    pds::TileArgs a;
    int rc = tile_args(ph, st, n_tiles, mpr, cfg, ws, ws_bytes, a);
    if (rc) return rc;
    if (ph.n == 0) return PDS_OK;
    a.grad = grad;
    a.image_elems = image_elems;
    a.gE = gE;
    a.gX = gX;
    a.gM = gM;
    cudaError_t e = cudaMemsetAsync(a.queue, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return cuda_fail(e, "backward: work counter reset");
    e = pds::launch_backward(a, s);
    if (e != cudaSuccess) return cuda_fail(e, "bwd_tiles_kernel");
    return PDS_OK;
}

pds::Photons photons(const float* E, const float* X, const float* M, const int64_t* cp,
                     const float* R, int64_t n) {
    pds::Photons p;
    p.E = E; p.X = X; p.M = M; p.cp = cp; p.R = R; p.n = n;
    return p;
}

int single_tiles(const pds_config* cfg, int64_t C, int64_t H, int64_t W, int64_t* n_tiles,
                 pds_sim* sim, int64_t n) {
    pds_config c;
    int rc = resolve_cfg(cfg, c);
    if (rc) return rc;
    rc = check_image(C, H, W);
    if (rc) return rc;
    *sim = single_sim(n, C, H, W, c.tile);
    *n_tiles = C * int64_t(sim->tiles_x) * sim->tiles_y;
    return PDS_OK;
}

}  // namespace

extern "C" {

const char* pds_last_error(void) { return g_err.c_str(); }

const char* pds_version(void) { return "pds_b200 1.0 (sm_100a)"; }

size_t pds_workspace_bytes(int64_t n, int64_t C, int64_t H, int64_t W, const pds_config* cfg) {
    pds_config c;
    if (resolve_cfg(cfg, c) != PDS_OK || C < 1 || H < 1 || W < 1) return make_layout(n, 1).total;
    const int64_t tiles = C * ((H + c.tile - 1) / c.tile) * ((W + c.tile - 1) / c.tile);
    return make_layout(n, bucket_count(cfg, tiles)).total;
}

size_t pds_batch_workspace_bytes(int64_t n_total, int64_t n_tiles_total, const pds_config* cfg) {
    return make_layout(n_total, bucket_count(cfg, n_tiles_total)).total;
}

int pds_plan_f32(const float* E, const float* X, const float* M, const int64_t* cp,
                 const float* R, int64_t n, int64_t C, int64_t H, int64_t W, int32_t mpr,
                 void* ws, size_t ws_bytes, const pds_config* cfg, void* stream) {
    int rc = check_photons(E, X, M, cp, R, n);
    if (rc) return rc;
    pds_sim sim;
    int64_t nt;
    rc = single_tiles(cfg, C, H, W, &nt, &sim, n);
    if (rc) return rc;
    return plan_impl(photons(E, X, M, cp, R, n), table_one(sim), nt, mpr, cfg, ws, ws_bytes,
                     static_cast<cudaStream_t>(stream));
}

int pds_forward_planned_f32(const float* E, const float* X, const float* M, const int64_t* cp,
                            const float* R, int64_t n, int64_t C, int64_t H, int64_t W,
                            int32_t mpr, float* out, void* ws, size_t ws_bytes,
                            const pds_config* cfg, void* stream) {
    int rc = check_photons(E, X, M, cp, R, n);
    if (rc) return rc;
    pds_sim sim;
    int64_t nt;
    rc = single_tiles(cfg, C, H, W, &nt, &sim, n);
    if (rc) return rc;
    return forward_impl(photons(E, X, M, cp, R, n), table_one(sim), nt, C * H * W, mpr, out,
                        cfg, ws, ws_bytes, static_cast<cudaStream_t>(stream));
}

int pds_backward_planned_f32(const float* G, const float* E, const float* X, const float* M,
                             const int64_t* cp, const float* R, int64_t n, int64_t C, int64_t H,
                             int64_t W, int32_t mpr, float* gE, float* gX, float* gM, void* ws,
                             size_t ws_bytes, const pds_config* cfg, void* stream) {
    int rc = check_photons(E, X, M, cp, R, n);
    if (rc) return rc;
    pds_sim sim;
    int64_t nt;
    rc = single_tiles(cfg, C, H, W, &nt, &sim, n);
    if (rc) return rc;
    return backward_impl(G, photons(E, X, M, cp, R, n), table_one(sim), nt, C * H * W, mpr, gE,
                         gX, gM, cfg, ws, ws_bytes, static_cast<cudaStream_t>(stream));
}

int pds_forward_f32(const float* E, const float* X, const float* M, const int64_t* cp,
                    const float* R, int64_t n, int64_t C, int64_t H, int64_t W, int32_t mpr,
                    float* out, void* ws, size_t ws_bytes, const pds_config* cfg, void* stream) {
    int rc = pds_plan_f32(E, X, M, cp, R, n, C, H, W, mpr, ws, ws_bytes, cfg, stream);
    if (rc) return rc;
    return pds_forward_planned_f32(E, X, M, cp, R, n, C, H, W, mpr, out, ws, ws_bytes, cfg,
                                   stream);
}

int pds_backward_f32(const float* G, const float* E, const float* X, const float* M,
                     const int64_t* cp, const float* R, int64_t n, int64_t C, int64_t H,
                     int64_t W, int32_t mpr, float* gE, float* gX, float* gM, void* ws,
                     size_t ws_bytes, const pds_config* cfg, void* stream) {
    int rc = pds_plan_f32(E, X, M, cp, R, n, C, H, W, mpr, ws, ws_bytes, cfg, stream);
    if (rc) return rc;
    return pds_backward_planned_f32(G, E, X, M, cp, R, n, C, H, W, mpr, gE, gX, gM, ws,
                                    ws_bytes, cfg, stream);
}

// The simulations' image ranges [image_offset, image_offset + C*H*W): each must be identical
// to or disjoint from every other (simulations that share an image are summed into it, as the
// reference's caller sums its simulations); the end of the last range in *elems.
static int check_image_ranges(const pds_sim* sims, int32_t n_sims, int64_t* elems) {
    std::vector<std::pair<int64_t, int64_t>> r;
    r.reserve(size_t(n_sims));
    for (int32_t s = 0; s < n_sims; ++s) {
        const pds_sim& d = sims[s];
        if (d.image_offset < 0) return fail(PDS_ERR_INVALID_ARGUMENT, "negative image_offset");
        const int64_t size = int64_t(d.channels) * d.height * d.width;
        if (d.image_offset > INT64_MAX - size)
            return fail(PDS_ERR_INVALID_ARGUMENT, "image range overflows");
        r.emplace_back(d.image_offset, d.image_offset + size);
    }
    std::sort(r.begin(), r.end());
    int64_t end = 0;
    for (size_t k = 0; k < r.size(); ++k) {
        if (k > 0 && r[k].first < r[k - 1].second && r[k] != r[k - 1])
            return fail(PDS_ERR_INVALID_ARGUMENT,
                        "simulation image ranges overlap without being the same image");
        end = r[k].second > end ? r[k].second : end;
    }
    *elems = end;
    return PDS_OK;
}

int pds_batch_image_elems(const pds_sim* sims, int32_t n_sims, int64_t* image_elems) {
    if (!sims || n_sims < 1 || !image_elems)
        return fail(PDS_ERR_INVALID_ARGUMENT, "pds_batch_image_elems: empty or null table");
    for (int32_t s = 0; s < n_sims; ++s) {
        int rc = check_image(sims[s].channels, sims[s].height, sims[s].width);
        if (rc) return rc;
    }
    return check_image_ranges(sims, n_sims, image_elems);
}

int pds_batch_layout(pds_sim* sims, int32_t n_sims, const pds_config* cfg, int64_t* n_tiles) {
    pds_config c;
    int rc = resolve_cfg(cfg, c);
    if (rc) return rc;
    if (!sims || n_sims < 1 || !n_tiles)
        return fail(PDS_ERR_INVALID_ARGUMENT, "pds_batch_layout: empty or null table");
    int64_t base = 0, next_photon = 0;
    for (int32_t s = 0; s < n_sims; ++s) {
        pds_sim& d = sims[s];
        rc = check_image(d.channels, d.height, d.width);
        if (rc) return rc;
        if (d.n_photons < 0 || d.photon_begin != next_photon)
            return fail(PDS_ERR_INVALID_ARGUMENT,
                        "simulations must cover the photon arrays contiguously and in order");
        next_photon += d.n_photons;
        d.tiles_x = int32_t((d.width + c.tile - 1) / c.tile);
        d.tiles_y = int32_t((d.height + c.tile - 1) / c.tile);
        d.tile_base = int32_t(base);
        base += int64_t(d.channels) * d.tiles_x * d.tiles_y;
        if (base >= (int64_t(1) << 30)) return fail(PDS_ERR_UNSUPPORTED, "too many tiles");
    }
    int64_t elems = 0;
    rc = check_image_ranges(sims, n_sims, &elems);
    if (rc) return rc;
    *n_tiles = base;
    return PDS_OK;
}

int pds_batch_plan_f32(const float* E, const float* X, const float* M, const int64_t* cp,
                       const float* R, int64_t n_total, const pds_sim* sims_dev, int32_t n_sims,
                       int64_t n_tiles, int32_t mpr, void* ws, size_t ws_bytes,
                       const pds_config* cfg, void* stream) {
    int rc = check_photons(E, X, M, cp, R, n_total);
    if (rc) return rc;
    if (!sims_dev || n_sims < 1) return fail(PDS_ERR_INVALID_ARGUMENT, "null simulation table");
    return plan_impl(photons(E, X, M, cp, R, n_total), table_dev(sims_dev, n_sims), n_tiles, mpr,
                     cfg, ws, ws_bytes, static_cast<cudaStream_t>(stream));
}

int pds_batch_forward_planned_f32(const float* E, const float* X, const float* M,
                                  const int64_t* cp, const float* R, int64_t n_total,
                                  const pds_sim* sims_dev, int32_t n_sims, int64_t n_tiles,
                                  int64_t image_elems, int32_t mpr, float* out, void* ws,
                                  size_t ws_bytes, const pds_config* cfg, void* stream) {
    int rc = check_photons(E, X, M, cp, R, n_total);
    if (rc) return rc;
    if (!sims_dev || n_sims < 1) return fail(PDS_ERR_INVALID_ARGUMENT, "null simulation table");
    if (image_elems < 0) return fail(PDS_ERR_INVALID_ARGUMENT, "negative image_elems");
    return forward_impl(photons(E, X, M, cp, R, n_total), table_dev(sims_dev, n_sims), n_tiles,
                        image_elems, mpr, out, cfg, ws, ws_bytes,
                        static_cast<cudaStream_t>(stream));
}

int pds_batch_backward_planned_f32(const float* G, const float* E, const float* X,
                                   const float* M, const int64_t* cp, const float* R,
                                   int64_t n_total, const pds_sim* sims_dev, int32_t n_sims,
                                   int64_t n_tiles, int64_t image_elems, int32_t mpr, float* gE,
                                   float* gX, float* gM, void* ws, size_t ws_bytes,
                                   const pds_config* cfg, void* stream) {
    int rc = check_photons(E, X, M, cp, R, n_total);
    if (rc) return rc;
    if (!sims_dev || n_sims < 1) return fail(PDS_ERR_INVALID_ARGUMENT, "null simulation table");
    if (image_elems < 0) return fail(PDS_ERR_INVALID_ARGUMENT, "negative image_elems");
    return backward_impl(G, photons(E, X, M, cp, R, n_total), table_dev(sims_dev, n_sims),
                         n_tiles, image_elems, mpr, gE, gX, gM, cfg, ws, ws_bytes,
                         static_cast<cudaStream_t>(stream));
}

static int check_plate(const float* h, int32_t rows, int32_t cols, const pds_plate* plate,
                       const float* px, const float* py, const float* flux, int64_t n) {
    if (!plate) return fail(PDS_ERR_INVALID_ARGUMENT, "null plate");
    if (rows < 1 || cols < 1 || !h) return fail(PDS_ERR_INVALID_ARGUMENT, "empty height field");
    if (n < 0) return fail(PDS_ERR_INVALID_ARGUMENT, "negative photon count");
    if (n > 0 && (!px || !py || !flux)) return fail(PDS_ERR_INVALID_ARGUMENT, "null photon array");
    if (!(plate->texel > 0.f) || !(plate->ior > 0.f) || !(plate->receiver_half > 0.f) ||
        !(plate->receiver_distance >= 0.f))
        return fail(PDS_ERR_INVALID_ARGUMENT, "plate parameters must be positive");
    return PDS_OK;
}

int pds_refract_forward_f32(const float* h, int32_t rows, int32_t cols, const pds_plate* plate,
                            const float* px, const float* py, const float* flux,
                            const int64_t* channel, int64_t n, float* Ep, float* xp, float* Mp,
                            int64_t* cp, float* radius, void* stream) {
    int rc = check_plate(h, rows, cols, plate, px, py, flux, n);
    if (rc) return rc;
    if (n > 0 && (!Ep || !xp || !Mp || !cp || !radius))
        return fail(PDS_ERR_INVALID_ARGUMENT, "null output array");
    cudaError_t e = pds::launch_refract(false, h, rows, cols, *plate, nullptr, nullptr, 0, px, py,
                                        flux, channel, n, Ep,
                                        xp, Mp, cp, radius, nullptr, nullptr, nullptr, nullptr,
                                        static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "refract_fwd_kernel");
    return PDS_OK;
}

int pds_refract_backward_f32(const float* h, int32_t rows, int32_t cols, const pds_plate* plate,
                             const float* px, const float* py, const float* flux, int64_t n,
                             const float* gE, const float* gX, const float* gM, float* gh,
                             void* stream) {
    int rc = check_plate(h, rows, cols, plate, px, py, flux, n);
    if (rc) return rc;
    if (n > 0 && (!gE || !gX || !gM || !gh))
        return fail(PDS_ERR_INVALID_ARGUMENT, "null gradient array");
    cudaError_t e = pds::launch_refract(true, h, rows, cols, *plate, nullptr, nullptr, 0, px, py,
                                        flux, nullptr, n,
                                        nullptr, nullptr, nullptr, nullptr, nullptr, gE, gX, gM,
                                        gh, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "refract_bwd_kernel");
    return PDS_OK;
}

int pds_batch_refract_forward_f32(const float* h, int32_t rows, int32_t cols,
                                  const pds_plate* plates_dev, const int64_t* begins_dev,
                                  int32_t n_sims, const float* px, const float* py,
                                  const float* flux, const int64_t* channel, int64_t n,
                                  float* Ep, float* xp, float* Mp, int64_t* cp, float* radius,
                                  void* stream) {
    if (!plates_dev || !begins_dev || n_sims < 1)
        return fail(PDS_ERR_INVALID_ARGUMENT, "null or empty plate table");
    if (rows < 1 || cols < 1 || !h) return fail(PDS_ERR_INVALID_ARGUMENT, "empty height field");
    if (n < 0) return fail(PDS_ERR_INVALID_ARGUMENT, "negative photon count");
    if (n > 0 && (!px || !py || !flux)) return fail(PDS_ERR_INVALID_ARGUMENT, "null photon array");
    if (n > 0 && (!Ep || !xp || !Mp || !cp || !radius))
        return fail(PDS_ERR_INVALID_ARGUMENT, "null output array");
    pds_plate unused;
    std::memset(&unused, 0, sizeof(unused));
    unused.receiver_half = 1.f;
    cudaError_t e = pds::launch_refract(false, h, rows, cols, unused, plates_dev, begins_dev,
                                        n_sims, px, py, flux, channel, n, Ep, xp, Mp, cp, radius,
                                        nullptr, nullptr, nullptr, nullptr,
                                        static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "refract_fwd_kernel (batch)");
    return PDS_OK;
}

int pds_batch_refract_backward_f32(const float* h, int32_t rows, int32_t cols,
                                   const pds_plate* plates_dev, const int64_t* begins_dev,
                                   int32_t n_sims, const float* px, const float* py,
                                   const float* flux, int64_t n, const float* gE, const float* gX,
                                   const float* gM, float* gh, void* stream) {
    if (!plates_dev || !begins_dev || n_sims < 1)
        return fail(PDS_ERR_INVALID_ARGUMENT, "null or empty plate table");
    if (rows < 1 || cols < 1 || !h) return fail(PDS_ERR_INVALID_ARGUMENT, "empty height field");
    if (n < 0) return fail(PDS_ERR_INVALID_ARGUMENT, "negative photon count");
    if (n > 0 && (!px || !py || !flux)) return fail(PDS_ERR_INVALID_ARGUMENT, "null photon array");
    if (n > 0 && (!gE || !gX || !gM || !gh))
        return fail(PDS_ERR_INVALID_ARGUMENT, "null gradient array");
    pds_plate unused;
    std::memset(&unused, 0, sizeof(unused));
    unused.receiver_half = 1.f;
    cudaError_t e = pds::launch_refract(true, h, rows, cols, unused, plates_dev, begins_dev,
                                        n_sims, px, py, flux, nullptr, n, nullptr, nullptr,
                                        nullptr, nullptr, nullptr, gE, gX, gM, gh,
                                        static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "refract_bwd_kernel (batch)");
    return PDS_OK;
}

// The gradient records of a plan in ws (n photons over n_tiles tiles, configuration cfg).
static int plan_records(const void* ws, size_t ws_bytes, int64_t n, int64_t n_tiles,
                        const pds_config* cfg, pds::GradRecords* rec) {
    const int64_t nb = bucket_count(cfg, n_tiles);
    if (nb <= 0) {
        pds_config c;
        int rc = resolve_cfg(cfg, c);
        return rc ? rc : fail(PDS_ERR_UNSUPPORTED, "tile count outside [1, 2^30)");
    }
    const Layout L = make_layout(n, nb);
    int rc = check_ws(const_cast<void*>(ws), ws_bytes, L.total);
    if (rc) return rc;
    const Bufs b = bufs(const_cast<void*>(ws), L);
    rec->inv = b.inv;
    rec->stage = reinterpret_cast<const float*>(b.stage);
    rec->counters = b.counters;
    return PDS_OK;
}

int pds_refract_backward_planned_f32(const float* h, int32_t rows, int32_t cols,
                                     const pds_plate* plate, const float* px, const float* py,
                                     const float* flux, int64_t n, int64_t C, int64_t H,
                                     int64_t W, const void* ws, size_t ws_bytes,
                                     const pds_config* cfg, float* gh, void* stream) {
    int rc = check_plate(h, rows, cols, plate, px, py, flux, n);
    if (rc) return rc;
    if (n > 0 && !gh) return fail(PDS_ERR_INVALID_ARGUMENT, "null gradient array");
    pds_sim sim;
    int64_t nt;
    rc = single_tiles(cfg, C, H, W, &nt, &sim, n);
    if (rc) return rc;
    pds::GradRecords rec;
    rc = plan_records(ws, ws_bytes, n, nt, cfg, &rec);
    if (rc) return rc;
    cudaError_t e = pds::launch_refract(true, h, rows, cols, *plate, nullptr, nullptr, 0, px, py,
                                        flux, nullptr, n, nullptr, nullptr, nullptr, nullptr,
                                        nullptr, nullptr, nullptr, nullptr, gh,
                                        static_cast<cudaStream_t>(stream), &rec);
    if (e != cudaSuccess) return cuda_fail(e, "refract_bwd_kernel (records)");
    return PDS_OK;
}

int pds_batch_refract_backward_planned_f32(const float* h, int32_t rows, int32_t cols,
                                           const pds_plate* plates_dev, const int64_t* begins_dev,
                                           int32_t n_sims, const float* px, const float* py,
                                           const float* flux, int64_t n, int64_t n_tiles,
                                           const void* ws, size_t ws_bytes,
                                           const pds_config* cfg, float* gh, void* stream) {
    if (!plates_dev || !begins_dev || n_sims < 1)
        return fail(PDS_ERR_INVALID_ARGUMENT, "null or empty plate table");
    if (rows < 1 || cols < 1 || !h) return fail(PDS_ERR_INVALID_ARGUMENT, "empty height field");
    if (n < 0) return fail(PDS_ERR_INVALID_ARGUMENT, "negative photon count");
    if (n > 0 && (!px || !py || !flux)) return fail(PDS_ERR_INVALID_ARGUMENT, "null photon array");
    if (n > 0 && !gh) return fail(PDS_ERR_INVALID_ARGUMENT, "null gradient array");
    pds::GradRecords rec;
    int rc = plan_records(ws, ws_bytes, n, n_tiles, cfg, &rec);
    if (rc) return rc;
    pds_plate unused;
    std::memset(&unused, 0, sizeof(unused));
    unused.receiver_half = 1.f;
    cudaError_t e = pds::launch_refract(true, h, rows, cols, unused, plates_dev, begins_dev,
                                        n_sims, px, py, flux, nullptr, n, nullptr, nullptr,
                                        nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, gh,
                                        static_cast<cudaStream_t>(stream), &rec);
    if (e != cudaSuccess) return cuda_fail(e, "refract_bwd_kernel (batch, records)");
    return PDS_OK;
}

static int check_point(const pds_point_light* light, const float* dir, const float* dth,
                       const float* dph, int64_t n) {
    if (!light) return fail(PDS_ERR_INVALID_ARGUMENT, "null light");
    if (n > 0 && (!dir || !dth || !dph))
        return fail(PDS_ERR_INVALID_ARGUMENT, "null photon direction array");
    return PDS_OK;
}

int pds_refract_point_forward_f32(const float* h, int32_t rows, int32_t cols,
                                  const pds_plate* plate, const pds_point_light* light,
                                  const float* dir, const float* dth, const float* dph,
                                  const float* flux, const int64_t* channel, int64_t n, float* Ep,
                                  float* xp, float* Mp, int64_t* cp, float* radius, void* stream) {
    int rc = check_plate(h, rows, cols, plate, dir, dir, flux, n);
    if (rc) return rc;
    rc = check_point(light, dir, dth, dph, n);
    if (rc) return rc;
    if (n > 0 && (!Ep || !xp || !Mp || !cp || !radius))
        return fail(PDS_ERR_INVALID_ARGUMENT, "null output array");
    cudaError_t e = pds::launch_refract_point(false, h, rows, cols, *plate, *light, dir, dth, dph,
                                              flux, channel, n, Ep, xp, Mp, cp, radius, nullptr,
                                              nullptr, nullptr, nullptr,
                                              static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "point_fwd_kernel");
    return PDS_OK;
}

int pds_refract_point_backward_f32(const float* h, int32_t rows, int32_t cols,
                                   const pds_plate* plate, const pds_point_light* light,
                                   const float* dir, const float* dth, const float* dph,
                                   const float* flux, int64_t n, const float* gE, const float* gX,
                                   const float* gM, float* gh, void* stream) {
    int rc = check_plate(h, rows, cols, plate, dir, dir, flux, n);
    if (rc) return rc;
    rc = check_point(light, dir, dth, dph, n);
    if (rc) return rc;
    if (n > 0 && (!gE || !gX || !gM || !gh))
        return fail(PDS_ERR_INVALID_ARGUMENT, "null gradient array");
    cudaError_t e = pds::launch_refract_point(true, h, rows, cols, *plate, *light, dir, dth, dph,
                                              flux, nullptr, n, nullptr, nullptr, nullptr, nullptr,
                                              nullptr, gE, gX, gM, gh,
                                              static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "point_bwd_kernel");
    return PDS_OK;
}

int pds_photon_source_f32(int32_t rows, int32_t cols, int32_t per_texel, float texel,
                          uint64_t seed, uint64_t offset, float* px, float* py, void* stream) {
    if (rows < 1 || cols < 1 || per_texel < 1)
        return fail(PDS_ERR_INVALID_ARGUMENT, "rows, cols and per_texel must be positive");
    const int64_t n = int64_t(rows) * cols * per_texel;
    if (n >= int64_t(0x7FFFFFFFll))
        return fail(PDS_ERR_UNSUPPORTED, "photon count must be below 2^31 - 1");
    if (!(texel > 0.f)) return fail(PDS_ERR_INVALID_ARGUMENT, "texel must be positive");
    if (!px || !py) return fail(PDS_ERR_INVALID_ARGUMENT, "null output array");
    cudaError_t e = pds::launch_source(rows, cols, per_texel, texel, seed, offset, n, px, py,
                                       static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "source_kernel");
    return PDS_OK;
}

int pds_point_light_source_f32(const pds_point_light* light, int64_t n_dir, uint64_t seed,
                               uint64_t offset, const float* coeffs, float* direction,
                               float* dtheta, float* dphi, float* flux, void* stream) {
    if (!light) return fail(PDS_ERR_INVALID_ARGUMENT, "null light");
    if (n_dir < 0) return fail(PDS_ERR_INVALID_ARGUMENT, "negative direction count");
    if (light->simulations < 1 || light->inner < 1 || light->wavelengths < 1)
        return fail(PDS_ERR_INVALID_ARGUMENT,
                    "simulations, inner and wavelengths must be positive");
    if (!(light->xmax > light->xmin) || !(light->ymax > light->ymin))
        return fail(PDS_ERR_INVALID_ARGUMENT, "empty light rectangle");
    if (n_dir * int64_t(light->wavelengths) >= int64_t(0x7FFFFFFFll))
        return fail(PDS_ERR_UNSUPPORTED, "photon count must be below 2^31 - 1");
    if (n_dir > 0 && (!direction || !dtheta || !dphi || !flux))
        return fail(PDS_ERR_INVALID_ARGUMENT, "null output array");
    cudaError_t e = pds::launch_point_light(*light, n_dir, seed, offset, coeffs, direction, dtheta,
                                            dphi, flux, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "point_light_kernel");
    return PDS_OK;
}

size_t pds_landweber_workspace_bytes(int64_t rows, int64_t cols) {
    return pds::landweber_scratch_bytes(rows * cols);
}

int pds_landweber_update_f32(float* d, const float* grad, const float* mask, int64_t rows,
                             int64_t cols, const pds_landweber* p, void* ws, size_t ws_bytes,
                             void* stream) {
    if (!p) return fail(PDS_ERR_INVALID_ARGUMENT, "null Landweber parameters");
    if (rows < 1 || cols < 1) return fail(PDS_ERR_INVALID_ARGUMENT, "empty height field");
    if (!d || !grad || !mask) return fail(PDS_ERR_INVALID_ARGUMENT, "null height-field array");
    if (p->radius < 0 || p->radius > 64)
        return fail(PDS_ERR_INVALID_ARGUMENT, "volume radius outside [0, 64]");
    if (!(p->d1 != 0.f) || !(p->d2 != 0.f))
        return fail(PDS_ERR_INVALID_ARGUMENT, "volume bounds d1, d2 must be nonzero");
    const int64_t n = rows * cols;
    int rc = check_ws(ws, ws_bytes, pds::landweber_scratch_bytes(n));
    if (rc) return rc;
    float* t = static_cast<float*>(ws);
    float* partial = reinterpret_cast<float*>(static_cast<char*>(ws) +
                                              pds::align_up(size_t(n) * sizeof(float), 256));
    cudaError_t e = pds::launch_landweber(d, grad, mask, rows, cols, *p, t, partial,
                                          static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "landweber kernels");
    return PDS_OK;
}

int pds_landweber_update_noalloc_f32(float* d, const float* grad, const float* mask,
                                     int64_t rows, int64_t cols, const pds_landweber* p,
                                     void* stream) {
    if (!p) return fail(PDS_ERR_INVALID_ARGUMENT, "null Landweber parameters");
    if (rows < 1 || cols < 1) return fail(PDS_ERR_INVALID_ARGUMENT, "empty height field");
    if (!d || !grad || !mask) return fail(PDS_ERR_INVALID_ARGUMENT, "null height-field array");
    if (p->radius < 0 || p->radius > 64)
        return fail(PDS_ERR_INVALID_ARGUMENT, "volume radius outside [0, 64]");
    if (!(p->d1 != 0.f) || !(p->d2 != 0.f))
        return fail(PDS_ERR_INVALID_ARGUMENT, "volume bounds d1, d2 must be nonzero");
    const int64_t maxpx = pds::landweber_noalloc_max_pixels();
    if (rows > maxpx || cols > maxpx || rows * cols > maxpx)
        return fail(PDS_ERR_UNSUPPORTED,
                    "pds_landweber_update_noalloc_f32: field of " + std::to_string(rows) + " x " +
                        std::to_string(cols) + " exceeds its static scratch of " +
                        std::to_string(maxpx) + " pixels; use pds_landweber_update_f32");
    float* t = nullptr;
    float* partial = nullptr;
    cudaError_t e = pds::landweber_noalloc_scratch(&t, &partial);
    if (e != cudaSuccess) return cuda_fail(e, "noalloc scratch address (cudaGetSymbolAddress)");
    e = pds::launch_landweber(d, grad, mask, rows, cols, *p, t, partial,
                              static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "landweber kernels (noalloc)");
    return PDS_OK;
}

int pds_plan_export(const void* ws, size_t ws_bytes, int64_t n, int64_t n_tiles, int32_t mpr,
                    const pds_config* cfg, uint32_t* bucket, uint32_t* slot, void* stream) {
    if (n < 0 || n >= int64_t(0x7FFFFFFFll))
        return fail(PDS_ERR_INVALID_ARGUMENT, "photon count outside [0, 2^31 - 1)");
    if (n > 0 && (!bucket || !slot)) return fail(PDS_ERR_INVALID_ARGUMENT, "null output array");
    Resolved r;
    int rc = resolve(cfg, mpr, n_tiles, n, r);
    if (rc) return rc;
    const Layout L = make_layout(n, r.n_buckets);
    rc = check_ws(const_cast<void*>(ws), ws_bytes, L.total);
    if (rc) return rc;
    const Bufs b = bufs(const_cast<void*>(ws), L);
    cudaError_t e = pds::launch_plan_export(b.inv, b.start, r.n_buckets, r.key_big, r.key_invalid,
                                            n, bucket, slot, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "plan_export_kernel");
    return PDS_OK;
}

}  // extern "C"
