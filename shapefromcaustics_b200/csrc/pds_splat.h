// Kernel argument blocks and launchers of the splatting kernels (pds_splat.cu).
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
    uint32_t key_big, key_invalid;
    uint32_t* keys;      // [n] out
    Rec* recs;           // [n] out (tile-path photons only)
    uint32_t* counters;  // [0] tile-path, [1] wide, [2] untouched photons; zeroed by caller
};

struct TileArgs {
    Photons ph;
    SimTable sims;
    int32_t mpr;
    Cfg cfg;
    const uint32_t* skeys;     // sorted keys
    const uint32_t* sidx;      // sorted photon indices
    const Rec* srecs;          // records in sorted order
    const uint32_t* counters;
    uint32_t* queue;           // chunk work counter of the tile kernel (zeroed before launch)
    float* out;                // forward: flat image buffer (zeroed by caller)
    const float* grad;         // backward: flat upstream gradient buffer
    float* gE;                 // backward outputs
    float* gX;
    float* gM;
    GradRec* stage;            // backward: per-photon gradient records (workspace)
};

cudaError_t launch_plan(const PlanArgs& a, cudaStream_t st);
cudaError_t launch_sort_records(const Rec* recs, const uint32_t* sidx, const uint32_t* counters,
                                int64_t n, Rec* srecs, cudaStream_t st);
cudaError_t launch_forward(const TileArgs& a, cudaStream_t st);
cudaError_t launch_backward(const TileArgs& a, cudaStream_t st);

}  // namespace pds
