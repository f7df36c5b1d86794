/*
 * pds_b200.h -- C ABI of the B200 (sm_100a) photon-differential splatting library
 * (libpds_b200.so).
 *
 * Drop-in boundary for the reference's torch extension module `PhotonDifferentialSplatting`
 * (PyOptix/PhotonDifferentialSplattig.cpp:34-38), whose two ops are
 *   pds_forward(Ep, xp, Mp, cp, radius, output_size, max_pixel_radius) -> [pds_grid]
 *     (PhotonDifferentialSplattig.cpp:12-25 -> PyOptix/kernel/photon_differentials.cu:115-134)
 *   pds_backward(grad_pds, Ep, xp, Mp, cp, radius, max_pixel_radius) -> [gE, gx, gM]
 *     (PhotonDifferentialSplattig.cpp:27-32 -> PyOptix/kernel/photon_differentials.cu:223-247)
 *
 * Layouts are the reference's (all contiguous, photon index fastest):
 *   Ep[N] f32, xp[2][N] f32 (normalised receiver coordinates in [-1,1]), Mp[2][3][N] f32
 *   (change-of-basis rows; column 2 multiplies zero and is never read), cp[1][N] int64
 *   (channel), radius[N] f32, images [C][H][W] f32.
 *
 * Conventions of every entry point:
 *   - Nothing is allocated. Outputs and a device workspace come from the caller; the
 *     workspace size comes from the *_workspace_bytes queries.
 *   - Work is enqueued on `stream` (a cudaStream_t passed as void*; NULL = legacy default
 *     stream) and is asynchronous. No entry point synchronises, so every entry point can be
 *     captured into a CUDA graph.
 *   - Return 0 (PDS_OK) on success, a PDS_ERR_* code otherwise; pds_last_error() gives the
 *     message of the calling thread's last failure.
 *   - Photons whose channel lies outside [0, C) contribute nothing and get zero gradients
 *     (the reference checks only c < C, photon_differentials.cu:75, and leaves its
 *     empty_like gradient outputs unwritten for them).
 *   - A call takes fewer than 2^31 - 1 photons (PDS_ERR_UNSUPPORTED otherwise).
 */
#ifndef PDS_B200_H
#define PDS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PDS_OK 0
#define PDS_ERR_INVALID_ARGUMENT 1 /* shapes, sizes, pointers or alignment */
#define PDS_ERR_WORKSPACE 2        /* workspace missing or smaller than required */
#define PDS_ERR_CUDA 3             /* a CUDA launch or runtime call failed */
#define PDS_ERR_UNSUPPORTED 4      /* configuration outside what the kernels handle */

/* Kernel tuning. A NULL pointer or a zero field selects the default. */
typedef struct pds_config {
    int32_t tile;       /* screen-tile edge in pixels: 16, 32 or 64 (default 64) */
    int32_t chunk;      /* sorted photons per CTA work item, multiple of 256 (default 2048;
                           lowered, to no less than 256, when the call has too few photons to
                           give every resident tile CTA about four work items) */
    int32_t class_bits; /* footprint-size bits appended to the sort key (photons of a tile
                           are then grouped by footprint size; with the band walk, classes
                           of 1/k octave of the band's area, k = 1 up to 3 bits, 2 for 4,
                           3 for 5; 6: the row walk's classes, 3 bits of band rows and 3
                           of row width inside the box): 1..6, or -1 for none (default 5) */
    int32_t apron_max;  /* largest footprint radius (px) the tile path holds (default 32);
                           larger footprints take the direct path */
    int32_t walk;       /* pixels visited per photon: 1 = the reference's whole box,
                           2 = only the rows / row spans that can hold the kernel's support,
                           3 = a sheared band of equal-width rows around the support,
                           4 = the band's rows inside the box, each warp's photons padded to a
                           common row count and width (best with class_bits 6)
                           (2, 3 and 4 give the same result: pixels outside the support add
                           exactly zero); default 3 */
    int32_t min_blocks; /* resident CTAs per SM the tile kernels are compiled for: 2, 3 or 4
                           (fewer: more registers per thread; more: more warps); a value sets
                           both directions; default (0): 3 for the forward, whose CTAs also
                           stage their next records in shared memory, and 4 for the backward */
    int32_t coop_radius; /* footprints with a radius (px) of at least this are splatted by a
                           whole warp instead of one thread; -1 never; default -1 */
} pds_config;

/* One simulation of a batch. The caller fills photon_begin, n_photons, image_offset,
 * channels, height, width; pds_batch_layout fills the tile fields. */
typedef struct pds_sim {
    int64_t photon_begin; /* first photon of this simulation in the concatenated arrays */
    int64_t n_photons;
    int64_t image_offset; /* element offset of this simulation's [C][H][W] image */
    int32_t channels, height, width;
    int32_t tiles_x, tiles_y; /* filled by pds_batch_layout */
    int32_t tile_base;        /* filled by pds_batch_layout */
    int32_t reserved[2];
} pds_sim;

/* Message of the calling thread's last failure ("" if none). */
const char* pds_last_error(void);

/* Library version string. */
const char* pds_version(void);

/* ---- single simulation: the reference's two ops ---------------------------------- */

/* Workspace bytes for one forward or backward call over N photons into [C][H][W]. */
size_t pds_workspace_bytes(int64_t n_photons, int64_t channels, int64_t height, int64_t width,
                           const pds_config* cfg);

/* pds_forward (PhotonDifferentialSplattig.cpp:12-25, photon_differentials.cu:60-134):
 * out[C][H][W] is overwritten (the callee zeroes it). */
int pds_forward_f32(const float* Ep, const float* xp, const float* Mp, const int64_t* cp,
                    const float* radius, int64_t n_photons, int64_t channels, int64_t height,
                    int64_t width, int32_t max_pixel_radius, float* out, void* workspace,
                    size_t workspace_bytes, const pds_config* cfg, void* stream);

/* pds_backward (PhotonDifferentialSplattig.cpp:27-32, photon_differentials.cu:136-247):
 * grad_pds[C][H][W] in; grad_Ep[N], grad_xp[2][N], grad_Mp[2][3][N] overwritten
 * (grad_Mp[.][2] = 0). */
int pds_backward_f32(const float* grad_pds, const float* Ep, const float* xp, const float* Mp,
                     const int64_t* cp, const float* radius, int64_t n_photons,
                     int64_t channels, int64_t height, int64_t width, int32_t max_pixel_radius,
                     float* grad_Ep, float* grad_xp, float* grad_Mp, void* workspace,
                     size_t workspace_bytes, const pds_config* cfg, void* stream);

/* ---- plan reuse: one binning + sort shared by a forward and its backward ------------ */
/* The plan lives in the workspace. pds_plan_f32 builds it; the *_planned calls use it and
 * must get the same photon arrays, sizes, max_pixel_radius and config. Same references as
 * the two ops above (the reference recomputes the footprints in each kernel,
 * photon_differentials.cu:76-89 and :155-167). */
int pds_plan_f32(const float* Ep, const float* xp, const float* Mp, const int64_t* cp,
                 const float* radius, int64_t n_photons, int64_t channels, int64_t height,
                 int64_t width, int32_t max_pixel_radius, void* workspace,
                 size_t workspace_bytes, const pds_config* cfg, void* stream);
int pds_forward_planned_f32(const float* Ep, const float* xp, const float* Mp,
                            const int64_t* cp, const float* radius, int64_t n_photons,
                            int64_t channels, int64_t height, int64_t width,
                            int32_t max_pixel_radius, float* out, void* workspace,
                            size_t workspace_bytes, const pds_config* cfg, void* stream);
/* grad_Ep, grad_xp and grad_Mp all NULL: the gradients stay in the workspace as per-photon
 * records for pds_refract_backward_planned_f32 (the batch variant likewise). */
int pds_backward_planned_f32(const float* grad_pds, const float* Ep, const float* xp,
                             const float* Mp, const int64_t* cp, const float* radius,
                             int64_t n_photons, int64_t channels, int64_t height,
                             int64_t width, int32_t max_pixel_radius, float* grad_Ep,
                             float* grad_xp, float* grad_Mp, void* workspace,
                             size_t workspace_bytes, const pds_config* cfg, void* stream);

/* The binning of a plan built by pds_plan_f32 or pds_batch_plan_f32 (the same n, tile count,
 * max_pixel_radius and config), per photon, for checks of its exactness; it has no
 * counterpart in the reference, whose kernels do not bin. bucket[i] is the photon's sort key:
 * (tile << class_bits) | footprint class for photons of the tile path, with tile = the
 * simulation's tile_base + (channel * tiles_y + ty) * tiles_x + tx of the photon's centre pixel
 * clamped into the image; n_tiles << class_bits for photons whose footprint is wider than the
 * tile path holds; (n_tiles + 1) << class_bits for photons that touch no pixel (channel out of
 * range or an empty clipped box). slot[i] is the photon's position in the sorted order (tile
 * path), its index in the wide list, or 0xFFFFFFFF. n_tiles: C * tiles_y * tiles_x for a single
 * simulation, the total from pds_batch_layout for a batch. */
int pds_plan_export(const void* workspace, size_t workspace_bytes, int64_t n_photons,
                    int64_t n_tiles, int32_t max_pixel_radius, const pds_config* cfg,
                    uint32_t* bucket, uint32_t* slot, void* stream);

/* ---- batches of uneven simulations in one launch sequence -------------------------- */
/* The reference runs its simulations one after another and sums them
 * (shape_from_caustics.py:351-353); these entry points run many simulations, each with
 * its own photon count and image size, through one binning, one sort and one persistent
 * launch per direction. Photon arrays are the simulations' arrays concatenated (stride
 * n_total); images live in one flat buffer at each simulation's image_offset. */

/* Fills tiles_x, tiles_y, tile_base of sims[0..n_sims) (host memory) for cfg and returns
 * the total tile count in *n_tiles_total. Each simulation's image range
 * [image_offset, image_offset + C*H*W) must be identical to or disjoint from every other's
 * (simulations that share an image are summed into it); PDS_ERR_INVALID_ARGUMENT otherwise. */
int pds_batch_layout(pds_sim* sims, int32_t n_sims, const pds_config* cfg,
                     int64_t* n_tiles_total);

/* The element count the batch's image buffers (the forward's out, the backward's grad) must
 * hold: the end of the last image range of sims[0..n_sims) (host memory), after the same range
 * checks as pds_batch_layout. */
int pds_batch_image_elems(const pds_sim* sims, int32_t n_sims, int64_t* image_elems);

size_t pds_batch_workspace_bytes(int64_t n_total, int64_t n_tiles_total, const pds_config* cfg);

/* sims_dev: the laid-out table in device memory. out: flat image buffer, overwritten over
 * [0, image_elems) where image_elems = max(image_offset + C*H*W) (pds_batch_image_elems).
 * Image planes of a table that reach past image_elems are not written (their photons add
 * nothing), so an inconsistent device table cannot write outside the buffer. */
int pds_batch_plan_f32(const float* Ep, const float* xp, const float* Mp, const int64_t* cp,
                       const float* radius, int64_t n_total, const pds_sim* sims_dev,
                       int32_t n_sims, int64_t n_tiles_total, int32_t max_pixel_radius,
                       void* workspace, size_t workspace_bytes, const pds_config* cfg,
                       void* stream);
int pds_batch_forward_planned_f32(const float* Ep, const float* xp, const float* Mp,
                                  const int64_t* cp, const float* radius, int64_t n_total,
                                  const pds_sim* sims_dev, int32_t n_sims,
                                  int64_t n_tiles_total, int64_t image_elems,
                                  int32_t max_pixel_radius, float* out, void* workspace,
                                  size_t workspace_bytes, const pds_config* cfg, void* stream);
/* grad: the flat upstream gradient of the batch's images, image_elems elements (image planes
 * past it are not read: their photons get zero gradients). */
int pds_batch_backward_planned_f32(const float* grad, const float* Ep, const float* xp,
                                   const float* Mp, const int64_t* cp, const float* radius,
                                   int64_t n_total, const pds_sim* sims_dev, int32_t n_sims,
                                   int64_t n_tiles_total, int64_t image_elems,
                                   int32_t max_pixel_radius,
                                   float* grad_Ep, float* grad_xp, float* grad_Mp,
                                   void* workspace, size_t workspace_bytes,
                                   const pds_config* cfg, void* stream);

/* ---- refraction to the receiver for a height-field glass plate --------------------- */
/* Replaces, for a plate whose top face is a height field lit by collimated light, the
 * reference's refraction chain from the traced hit to the splat inputs:
 * Sobel normals (model/caustics.py:215-221), differential transfer
 * (model/photon_differential.py:69-78), Snell + Igehy differentials (model/caustics.py:152-212),
 * normal derivatives (model/renderable_object.py:391-401) and the splat inputs
 * (model/caustics.py:224-239). The OptiX trace that finds the hits (PyOptix/RayTrace.cpp:233-291)
 * is replaced by the analytic plate: entry at (px, py, h(px, py)), exit through the flat face
 * z = 0, receiver plane z = -receiver_distance. */
typedef struct pds_plate {
    float texel;             /* height-field texel edge (world units); the field is centred */
    float ior;               /* refractive index of the plate */
    float receiver_distance; /* from the flat bottom face (z = 0) down to the receiver */
    float receiver_half;     /* receiver half-extent; receiver coordinates are divided by it */
    float light_dir[3];      /* unit propagation direction of the collimated light */
    float du0;               /* length of each photon's initial positional differentials (x, y) */
} pds_plate;

/* Splat inputs of n photons entering at (px[i], py[i]) with flux[i] (channel[i], or 0 when
 * channel is NULL): Ep[N], xp[2][N], Mp[2][3][N], cp[1][N] (-1 for degenerate photons),
 * radius[N]. height: [rows][cols] row-major. */
int pds_refract_forward_f32(const float* height, int32_t rows, int32_t cols, const pds_plate* plate,
                            const float* px, const float* py, const float* flux,
                            const int64_t* channel, int64_t n_photons, float* Ep, float* xp,
                            float* Mp, int64_t* cp, float* radius, void* stream);

/* Adds d L / d height to grad_height[rows][cols] given the splat-input gradients
 * (grad_Ep[N], grad_xp[2][N], grad_Mp[2][3][N], e.g. from pds_backward_f32). The chain is
 * recomputed from the height field; nothing from the forward is needed. */
int pds_refract_backward_f32(const float* height, int32_t rows, int32_t cols,
                             const pds_plate* plate, const float* px, const float* py,
                             const float* flux, int64_t n_photons, const float* grad_Ep,
                             const float* grad_xp, const float* grad_Mp, float* grad_height,
                             void* stream);

/* The two calls above for a batch of simulations that share one height field but each have
 * their own plate parameters (light direction, refractive index for its wavelength, initial
 * differential length, receiver), in one launch: simulation k holds the photons
 * begins_dev[k] .. begins_dev[k + 1] - 1 (the last ends at n_photons; begins_dev[0] = 0,
 * ascending) and uses plates_dev[k]; both tables live in device memory. The reference runs
 * its simulations, each with its own light sample and wavelengths, one after another
 * (shape_from_caustics.py:351-353). Every plate must have the field's texel. */
int pds_batch_refract_forward_f32(const float* height, int32_t rows, int32_t cols,
                                  const pds_plate* plates_dev, const int64_t* begins_dev,
                                  int32_t n_sims, const float* px, const float* py,
                                  const float* flux, const int64_t* channel, int64_t n_photons,
                                  float* Ep, float* xp, float* Mp, int64_t* cp, float* radius,
                                  void* stream);
int pds_batch_refract_backward_f32(const float* height, int32_t rows, int32_t cols,
                                   const pds_plate* plates_dev, const int64_t* begins_dev,
                                   int32_t n_sims, const float* px, const float* py,
                                   const float* flux, int64_t n_photons, const float* grad_Ep,
                                   const float* grad_xp, const float* grad_Mp,
                                   float* grad_height, void* stream);

/* The refraction backward reading the splat gradients from a plan's gradient records instead
 * of grad_Ep / grad_xp / grad_Mp: pds_backward_planned_f32 (or the batch variant) called with
 * grad_Ep = grad_xp = grad_Mp = NULL leaves each photon's gradients in the workspace as a
 * 32-byte record, and these calls read them there, so the spread into the reference's layouts
 * and its re-read are skipped. The plan must be of the refracted photons of these calls, in
 * the same order, on the same workspace: channels, height, width and cfg (one simulation) or
 * n_tiles_total and cfg (a batch) as passed to the splat calls. Photons that touch no pixel
 * add nothing. */
int pds_refract_backward_planned_f32(const float* height, int32_t rows, int32_t cols,
                                     const pds_plate* plate, const float* px, const float* py,
                                     const float* flux, int64_t n_photons, int64_t channels,
                                     int64_t image_height, int64_t image_width,
                                     const void* workspace, size_t workspace_bytes,
                                     const pds_config* cfg, float* grad_height, void* stream);
int pds_batch_refract_backward_planned_f32(const float* height, int32_t rows, int32_t cols,
                                           const pds_plate* plates_dev,
                                           const int64_t* begins_dev, int32_t n_sims,
                                           const float* px, const float* py, const float* flux,
                                           int64_t n_photons, int64_t n_tiles_total,
                                           const void* workspace, size_t workspace_bytes,
                                           const pds_config* cfg, float* grad_height,
                                           void* stream);

/* Entry points of rows * cols * per_texel photons (per_texel per texel of a rows x cols
 * height field of edge `texel`, centred on the origin), each jittered uniformly inside its
 * texel (the reference's per-pixel random surface samples, model/caustics.py:78-83):
 * px[i], py[i] for photon i = k * rows * cols + texel index (per_texel samples of one photon
 * per texel in raster order, as the reference's simulations sample). The offsets come from Philox4x32-10
 * (Salmon et al., SC 2011) keyed by `seed`; photons 2j and 2j + 1 use counter block
 * offset + j, so a call is a pure function of (seed, offset) and calls with offsets advanced
 * by ceil(n / 2) draw disjoint streams. */
int pds_photon_source_f32(int32_t rows, int32_t cols, int32_t per_texel, float texel,
                          uint64_t seed, uint64_t offset, float* px, float* py, void* stream);

/* A point light whose photons spread over a rectangle of the plane z = plane_z
 * (model/caustics.py:26-70, compute_point_light_dirs; the rectangle is the height field's
 * extent, the plane its base height). */
typedef struct pds_point_light {
    float position[3];                /* light position */
    float plane_z;                    /* plane the directions are spread over */
    float xmin, ymin, xmax, ymax;     /* the rectangle on that plane */
    float smoothing;                  /* splat smoothing (scales the direction differentials) */
    float energy;                     /* light energy; each photon carries
                                         energy / (simulations * inner) */
    int32_t simulations;              /* simulations whose photons share the light's energy */
    int32_t inner;                    /* inner simulations per simulation */
    int32_t wavelengths;              /* photons per direction, one per wavelength */
} pds_point_light;

/* Photon directions and direction differentials of a point light (model/caustics.py:26-70):
 * direction k is the bilinear slerp of the rectangle's corner directions by two uniform
 * numbers (u0, u1); its differentials are the Frisvad orthonormal basis of the direction
 * (model/utils.py compute_orthonormal_basis) scaled by 2 smoothing sqrt(omega / (pi N)), with
 * omega the rectangle's solid angle seen from the light (model/utils.py subtended_angle,
 * computed on the device: no host read-back) and N = n_directions * simulations * wavelengths.
 * Each direction is repeated for each wavelength (photon k * wavelengths + w). The uniform
 * numbers are coeffs[0][k], coeffs[1][k] when coeffs is not NULL, else Philox4x32-10 keyed by
 * seed (directions 2j and 2j + 1 use counter block offset + j). Outputs: direction[3][n],
 * dtheta[3][n], dphi[3][n], flux[n] with n = n_directions * wavelengths. */
int pds_point_light_source_f32(const pds_point_light* light, int64_t n_directions, uint64_t seed,
                               uint64_t offset, const float* coeffs, float* direction,
                               float* dtheta, float* dphi, float* flux, void* stream);

/* Splat inputs of n point-light photons (direction[3][n], dtheta[3][n], dphi[3][n], flux[n],
 * e.g. from pds_point_light_source_f32; channel[n] or NULL for 0) on the plate: each photon's
 * first hit with the bilinear height-field surface is traced from the light (Newton steps from
 * the plane z = light->plane_z; the reference traces with OptiX, PyOptix/RayTrace.cpp:233-291,
 * on the plate's mesh), its positional differentials are carried from the light to the hit
 * (model/photon_differential.py:69-78, zero at the light), and the chain continues as in
 * pds_refract_forward_f32 with the photon's direction differentials. plate->light_dir and
 * plate->du0 are not used. Photons whose hit lies outside the field get channel -1. */
int pds_refract_point_forward_f32(const float* height, int32_t rows, int32_t cols,
                                  const pds_plate* plate, const pds_point_light* light,
                                  const float* direction, const float* dtheta, const float* dphi,
                                  const float* flux, const int64_t* channel, int64_t n_photons,
                                  float* Ep, float* xp, float* Mp, int64_t* cp, float* radius,
                                  void* stream);

/* Adds d L / d height for point-light photons given their splat-input gradients; the trace and
 * the chain are recomputed (nothing from the forward is needed), and the hit's dependence on
 * the heights (dt/dh = w / f'(t) for the hit cell's bilinear weights w) is included. */
int pds_refract_point_backward_f32(const float* height, int32_t rows, int32_t cols,
                                   const pds_plate* plate, const pds_point_light* light,
                                   const float* direction, const float* dtheta,
                                   const float* dphi, const float* flux, int64_t n_photons,
                                   const float* grad_Ep, const float* grad_xp,
                                   const float* grad_Mp, float* grad_height, void* stream);

/* ---- projected Landweber update of the height field ------------------------------- */
/* One update of the reference's pixel-basis Landweber loop (shape_from_caustics.py:386-398):
 * d <- VconsHeur(mask * extShrink(d - tau * grad, shrink, lower, upper)), with extShrink
 * (:184-189) and the volume heuristic VconsHeur (:228-241). */
typedef struct pds_landweber {
    float tau;          /* gradient step (the reference's tau_pixel) */
    float shrink;       /* soft-shrinkage threshold (tau_pixel * alpha_pixel) */
    float lower, upper; /* clamp of the extended shrinkage */
    float d1, d2;       /* volume window, in units of the summed offsets */
    float gamma;        /* volume heuristic step */
    int32_t radius;     /* volume heuristic box radius (pixels) */
} pds_landweber;

size_t pds_landweber_workspace_bytes(int64_t rows, int64_t cols);

/* d[rows][cols] updated in place; grad, mask (0/1 floats) same shape. */
int pds_landweber_update_f32(float* d, const float* grad, const float* mask, int64_t rows,
                             int64_t cols, const pds_landweber* params, void* workspace,
                             size_t workspace_bytes, void* stream);

/* Allocation-free variant of pds_landweber_update_f32. It has no counterpart in the
 * reference. It is for callers that cannot allocate device memory: code whose device memory
 * is owned by another allocator (a framework's caching allocator that must not be bypassed),
 * or a fixed-memory loop that may not allocate after start-up. It takes no workspace: its
 * scratch is a static device array of this library, 4 MiB + 4 KiB, present on every GPU that
 * loads the library until the process exits, so fields are limited to rows * cols <=
 * 1048576 (1024 x 1024); larger fields return PDS_ERR_UNSUPPORTED. The first call on a
 * device looks up that device's scratch address (a CUDA runtime query, no allocation); make
 * that first call before any stream capture. All calls share the one scratch array, which
 * keeps the previous call's contents (every byte this update reads there is written first in
 * the same call), so calls that overlap on the GPU, from several streams or threads at once,
 * race and give wrong results: serialise them. */
int pds_landweber_update_noalloc_f32(float* d, const float* grad, const float* mask,
                                     int64_t rows, int64_t cols, const pds_landweber* params,
                                     void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PDS_B200_H */
