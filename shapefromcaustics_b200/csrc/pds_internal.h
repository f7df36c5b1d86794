// Internal (non-ABI) declarations shared by the library's translation units.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pds_b200.h"

namespace pds {

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// refraction to the receiver (pds_refract.cu)
// A splat plan's per-photon gradient records (the backward's output before the spread into
// grad_Ep / grad_xp / grad_Mp): the inverse map, the 32-byte records, the plan's counters.
struct GradRecords {
    const uint32_t* inv;
    const float* stage;
    const uint32_t* counters;
};

// backward: the splat gradients from gE / gX / gM, or from rec when rec is non-null
cudaError_t launch_refract(bool backward, const float* h, int H, int W, const pds_plate& plate,
                           const pds_plate* plates, const int64_t* begins, int32_t n_sims,
                           const float* px, const float* py, const float* flux,
                           const int64_t* channel, int64_t n, float* Ep, float* xp, float* Mp,
                           int64_t* cp, float* radius, const float* gE, const float* gX,
                           const float* gM, float* gh, cudaStream_t st,
                           const GradRecords* rec = nullptr);

cudaError_t launch_refract_point(bool backward, const float* h, int H, int W,
                                 const pds_plate& plate, const pds_point_light& light,
                                 const float* dir, const float* dth, const float* dph,
                                 const float* flux, const int64_t* channel, int64_t n, float* Ep,
                                 float* xp, float* Mp, int64_t* cp, float* radius,
                                 const float* gE, const float* gX, const float* gM, float* gh,
                                 cudaStream_t st);

// photon source (pds_source.cu)
cudaError_t launch_source(int32_t rows, int32_t cols, int32_t per_texel, float texel,
                          uint64_t seed, uint64_t offset, int64_t n, float* px, float* py,
                          cudaStream_t st);

cudaError_t launch_point_light(const pds_point_light& L, int64_t n_dir, uint64_t seed,
                               uint64_t offset, const float* coeffs, float* dir, float* dth,
                               float* dph, float* flux, cudaStream_t st);

// Landweber update (pds_landweber.cu)
size_t landweber_scratch_bytes(int64_t n);
cudaError_t launch_landweber(float* d, const float* g, const float* mask, int64_t rows,
                             int64_t cols, const pds_landweber& p, float* t, float* partial,
                             cudaStream_t st);
int64_t landweber_noalloc_max_pixels();
cudaError_t landweber_noalloc_scratch(float** t, float** partial);

}  // namespace pds
