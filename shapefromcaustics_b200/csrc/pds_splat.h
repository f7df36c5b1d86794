// Kernel argument blocks and launchers of the splatting kernels (pds_plan.cu, pds_splat.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pds_device.cuh"

namespace pds {

// Photon arrays in the reference's layouts (photon index fastest, stride n).
struct Photons {
    const float* E;     // [n]
    const float* X;     // [2][n]
    const float* M;     // [2][3][n]
    const int64_t* cp;  // [n]
    const float* R;     // [n]
    int64_t n;
};

struct PlanArgs {
    Photons ph;
    SimTable sims;
    int32_t mpr;
    Cfg cfg;
    uint32_t key_big, key_invalid;  // bucket count (wide photons), and the untouched key
    uint32_t* counts;    // [key_big] photons per bucket; zeroed by the caller (count pass)
    uint32_t* inv;       // [n] out: sorted position (place pass), kWideBit | k for wide and
                         // kInvalidPos for untouched photons (count pass)
    uint32_t* wide;      // [n] out: photon index of the k-th wide photon (count pass)
    uint32_t* counters;  // [0] tile-path, [1] wide, [2] untouched photons; zeroed by caller
    uint32_t* cta_hist;  // [plan_hist_entries] each CTA's window histogram, count -> place
    uint32_t* cursor;    // [key_big] place cursors (the bucket starts, from the scan)
    Rec* srecs;          // [n] out: records in sorted order (place pass)
    uint32_t* tile_r;    // [tiles] out: the largest box radius max(rx, ry) of each tile's
                         // tile-path photons (count pass); zeroed by the caller
    int64_t range;       // photons per CTA (plan_shape)
    int32_t window;      // buckets of each CTA's shared histogram (plan_shape)
};

// Bucket scan and the chunks' tiles.
struct ScanArgs {
    const uint32_t* counts;
    const uint32_t* counters;
    uint32_t* part;        // [bucket_scan_parts(nb)] scan partials
    uint32_t* start;       // [nb + 1] out: first sorted position of each bucket, then the total
    uint32_t* cursor;      // [nb] out: a copy of the starts for the place pass
    uint32_t* chunk_tile;  // [n / chunk + 1] out: tile of each work chunk's first photon
    int64_t n, nb, n_tiles;
    int32_t chunk, cb;
};

struct TileArgs {
    Photons ph;
    SimTable sims;
    int32_t mpr;
    Cfg cfg;
    int64_t n_tiles;
    const Rec* srecs;            // records in sorted order
    const uint32_t* start;       // [(n_tiles << class_bits) + 1] bucket starts
    const uint32_t* chunk_tile;  // tile of each chunk's first photon
    const uint32_t* inv;         // per photon: sorted position, kWideBit | k, or kInvalidPos
    const uint32_t* wide;        // photon index of each wide photon
    const uint32_t* tile_r;      // largest box radius of each tile's photons (plan)
    const uint32_t* counters;
    uint32_t* queue;             // chunk work counter of the tile kernel (zeroed before launch)
    float* out;                  // forward: flat image buffer (zeroed by caller)
    const float* grad;           // backward: flat upstream gradient buffer
    int64_t image_elems;         // elements of out / grad: image planes past it are not touched
    float* gE;                   // backward outputs
    float* gX;
    float* gM;
    GradRec* stage;              // backward: gradient records, sorted positions then the wide
                                 // photons (workspace)
};

int64_t bucket_scan_parts(int64_t nb);
void plan_shape(int64_t n, int64_t nb, int32_t* window, int64_t* range);
int64_t plan_hist_entries(int64_t n, int64_t nb);
cudaError_t launch_plan_count(const PlanArgs& a, cudaStream_t st);
cudaError_t launch_bucket_scan(const ScanArgs& a, cudaStream_t st);
cudaError_t launch_plan_place(const PlanArgs& a, cudaStream_t st);
cudaError_t launch_chunk_tiles(const ScanArgs& a, cudaStream_t st);
cudaError_t launch_plan_export(const uint32_t* inv, const uint32_t* start, int64_t nb,
                               uint32_t key_big, uint32_t key_invalid, int64_t n,
                               uint32_t* bucket, uint32_t* slot, cudaStream_t st);
cudaError_t launch_forward(const TileArgs& a, cudaStream_t st);
cudaError_t launch_backward(const TileArgs& a, cudaStream_t st);

}  // namespace pds
