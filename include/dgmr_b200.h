/* C ABI of the B200 Gaussian-mixture renderer (libdgmr_b200.so).
 *
 * Plain structs, device pointers, sizes and a cudaStream_t.  No exception,
 * allocation or host synchronisation happens inside these calls: the caller
 * owns every buffer, including one workspace per frame sized by the
 * *_workspace_size queries, and reads results whenever it synchronises.
 *
 * Layouts are the reference's (python_bindings/vol_marcher.cu:42-104):
 *   centroids [N,3], sh [N,sh_stride,3] (sh_stride <= 16 coefficients),
 *   weights [N] (opacity), scales [N,3], rotations [N,4] stored (w,x,y,z),
 *   framebuffer [3,H,W], 4x4 matrices in glm order: element (row r, col c)
 *   at index c*4+r -- i.e. the row-major bytes of the torch tensors the
 *   reference's Python op receives.
 */
#ifndef DGMR_B200_H
#define DGMR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* dgmr_stream;

typedef enum dgmr_status {
    DGMR_OK = 0,
    DGMR_ERR_BAD_ARG = 1, /* null pointer, negative size, sh_stride/degree out of range */
    DGMR_ERR_WORKSPACE = 2, /* workspace smaller than the query returned */
    DGMR_ERR_CUDA = 3, /* a launch failed; cudaGetLastError() holds the cause */
    DGMR_ERR_STATIC_SCRATCH = 4, /* frame too large for dgmr_splat_forward_noalloc's 64 MiB scratch */
    DGMR_ERR_PAIR_OVERFLOW = 5, /* dgmr_splat_forward_noalloc without stats: the frame had more pairs than pair_capacity */
} dgmr_status;

/* Device-side frame statistics (caller-owned, 16 bytes, written by the calls
 * that take it).  flags: bit 0 = more (tile, Gaussian) pairs than the pair
 * capacity (pairs beyond it were dropped; re-run with a larger capacity),
 * bit 1 = some ray march hit the large-step limit. */
typedef struct dgmr_frame_stats {
    uint32_t n_pairs;
    uint32_t flags;
    uint32_t n_visible;
    uint32_t reserved;
} dgmr_frame_stats;

#define DGMR_FLAG_PAIR_OVERFLOW 1u
#define DGMR_FLAG_STEP_LIMIT 2u

typedef enum dgmr_dtype { DGMR_F32 = 0, DGMR_F64 = 1 } dgmr_dtype;

/* The Gaussian mixture (all device pointers, element type = dtype). */
typedef struct dgmr_scene {
    int32_t n_gaussians;
    int32_t sh_stride; /* coefficients stored per Gaussian, 1..16 */
    int32_t sh_degree; /* active SH degree, 0..3 */
    int32_t dtype; /* dgmr_dtype; the splat renderer takes DGMR_F32 only */
    const void* centroids;
    const void* sh;
    const void* weights;
    const void* scales;
    const void* rotations;
    int32_t formulation; /* dgmr_formulation: how weights become masses / opacities */
    int32_t reserved;
} dgmr_scene;

/* types.h:26-32.  The reference fixes one per renderer at compile time: Ots for
 * the splat (splat_forward.h:58) and vol_raster (vol_raster_forward.h:66),
 * Opacity for vol_marcher (vol_marcher.h:66); DGMR_FORMULATION_DEFAULT (0, a
 * zero-initialised scene) selects exactly those. */
typedef enum dgmr_formulation {
    DGMR_FORMULATION_DEFAULT = 0,
    DGMR_FORMULATION_OPACITY = 1,
    DGMR_FORMULATION_MASS = 2,
    DGMR_FORMULATION_DENSITY = 3,
    DGMR_FORMULATION_OTS = 4,
    DGMR_FORMULATION_OLS = 5,
} dgmr_formulation;

/* One camera (host values). */
typedef struct dgmr_camera {
    int32_t width, height;
    double view[16]; /* world -> view, glm order */
    double proj[16]; /* full view-projection (P * V), glm order */
    double campos[3];
    double background[3];
    double tan_fovx, tan_fovy;
    double cov_scale_multiplier; /* 1.0 in the reference's Python path */
} dgmr_camera;

/* ---------------------------------------------------------------- splat */

/* Replaces dgmr::splat_forward(SplatForwardData&) (src/dgmr/splat_forward.h:62,
 * reached through dgmr::sibr_interfaces::splat, src/dgmr/sibr_interfaces.h:25).
 *
 * Two caller-owned workspaces per frame: the frame workspace holds the
 * per-Gaussian, per-tile and per-pixel state (sized by the Gaussian count and
 * the resolution); the pair workspace holds the (tile, Gaussian) pairs and the
 * sort scratch (sized by pair_capacity).  Both must stay alive between a
 * forward and its backward. */
size_t dgmr_splat_frame_workspace_size(int32_t n_gaussians, int32_t width, int32_t height);
size_t dgmr_splat_pair_workspace_size(int32_t n_gaussians, int64_t pair_capacity);

/* Forward splat in one call: framebuffer [3,H,W] f32 (device).  If the frame
 * has more pairs than pair_capacity, stats->flags gets DGMR_FLAG_PAIR_OVERFLOW
 * (pairs beyond the capacity are dropped).  stats may be NULL. */
dgmr_status dgmr_splat_forward(const dgmr_scene* scene, const dgmr_camera* camera, float* framebuffer, void* frame_workspace, size_t frame_workspace_bytes,
    void* pair_workspace, size_t pair_workspace_bytes, int64_t pair_capacity, dgmr_frame_stats* stats, dgmr_stream stream);

/* The same forward in two halves, for callers that size the pair workspace
 * from the frame itself (the reference reads the pair count back with .item(),
 * splat_forward.cu:141): preprocess (splat_forward.cu:70-139) leaves the pair
 * count in stats->n_pairs and in point_offsets[N-1]; render (:145-335) does
 * the binning and the blend. */
dgmr_status dgmr_splat_preprocess(const dgmr_scene* scene, const dgmr_camera* camera, void* frame_workspace, size_t frame_workspace_bytes,
    dgmr_frame_stats* stats, dgmr_stream stream);
dgmr_status dgmr_splat_render(const dgmr_scene* scene, const dgmr_camera* camera, float* framebuffer, void* frame_workspace, size_t frame_workspace_bytes,
    void* pair_workspace, size_t pair_workspace_bytes, int64_t pair_capacity, dgmr_frame_stats* stats, dgmr_stream stream);

/* Views into the workspaces after a forward (device pointers): the
 * per-Gaussian cache and the binning result, in the reference's layouts
 * (splat_forward.cu:96-107, :159-191, :218-239). */
typedef struct dgmr_splat_views {
    int32_t* rects; /* [N,2] */
    float* rgb; /* [N,3] */
    uint8_t* rgb_sh_clamped; /* [N,3] */
    float* depths; /* [N] */
    float* points_xy_image; /* [N,2] */
    float* conic_opacity; /* [N,4] */
    int32_t* tiles_touched; /* [N] */
    int32_t* point_offsets; /* [N] inclusive scan */
    int32_t* i_ranges; /* [tiles,2] */
    int32_t* point_list; /* [pair_capacity] Gaussian ids sorted by (tile, depth) */
    uint32_t* point_list_tiles; /* [pair_capacity] tile id of each point_list entry */
    float* final_transmittance; /* [H,W] */
    int32_t* n_contrib; /* [H,W] */
} dgmr_splat_views;

dgmr_status dgmr_splat_workspace_views(int32_t n_gaussians, int32_t width, int32_t height, int64_t pair_capacity, void* frame_workspace,
    size_t frame_workspace_bytes, void* pair_workspace, size_t pair_workspace_bytes, dgmr_splat_views* views);

/* Re-runs only the blend stage of the last forward made in these workspaces
 * (same camera, Gaussian count and capacity), e.g. to time the blend kernel
 * by itself.  Splits splat_forward.cu:242-335 out of the frame. */
dgmr_status dgmr_splat_blend(const dgmr_camera* camera, int32_t n_gaussians, float* framebuffer, void* frame_workspace, size_t frame_workspace_bytes,
    void* pair_workspace, size_t pair_workspace_bytes, int64_t pair_capacity, dgmr_stream stream);

/* Splat forward that allocates nothing -- no counterpart in the reference.
 * For callers that cannot provide or allocate device memory on the render
 * path (a plugin whose host application owns all GPU memory; a per-frame
 * callback where cudaMalloc would synchronise the device).  Both workspaces
 * live in one static 64 MiB device array that every GPU loading the library
 * holds until exit; frames whose frame + pair workspaces
 * (dgmr_splat_frame_workspace_size + dgmr_splat_pair_workspace_size) exceed
 * it return DGMR_ERR_STATIC_SCRATCH.  The first call on each device looks up
 * the array's device address (make that first call before any stream
 * capture).  All calls on a device share the array: calls that overlap on the
 * GPU race and corrupt each other; calls ordered on one stream are fine.
 * Results equal dgmr_splat_forward's; the workspace views are not available.
 * With a device `stats` the call is asynchronous and the caller reads
 * DGMR_FLAG_PAIR_OVERFLOW there.  With stats == NULL the frame's statistics
 * stay in the static array, which the caller cannot read, so the call waits
 * for the stream and returns DGMR_ERR_PAIR_OVERFLOW when pair_capacity was too
 * small (the image is then incomplete) instead of dropping pairs silently. */
dgmr_status dgmr_splat_forward_noalloc(const dgmr_scene* scene, const dgmr_camera* camera, float* framebuffer, int64_t pair_capacity,
    dgmr_frame_stats* stats, dgmr_stream stream);

/* Backward splat (no reference kernel; the reference only has the pieces:
 * grad/math.h:333-527, :203-282).  grad_framebuffer [3,H,W]; grads written
 * (not accumulated) for sh [N,sh_stride,3], weights [N], centroids [N,3],
 * scales [N,3], rotations [N,4]. */
dgmr_status dgmr_splat_backward(const dgmr_scene* scene, const dgmr_camera* camera, const float* grad_framebuffer, float* grad_sh, float* grad_weights,
    float* grad_centroids, float* grad_scales, float* grad_rotations, void* frame_workspace, size_t frame_workspace_bytes, void* pair_workspace,
    size_t pair_workspace_bytes, int64_t pair_capacity, dgmr_stream stream);

/* ------------------------------------------------------- batched splat */

/* Many views of one or several scenes rendered by ONE launch sequence (no
 * reference counterpart: the reference renders one view per call,
 * splat_forward.cu:30-338).  Each view's image, point list and tile ranges are
 * bit-identical to a dgmr_splat_forward of that view alone.  All views share one
 * frame workspace and one pair workspace (pair_capacity = pairs of all views
 * together), sized by dgmr_splat_batch_workspace_size.  No allocation, no host
 * synchronisation: the calls can be captured in a CUDA graph. */
#define DGMR_BATCH_MAX_VIEWS 64
#define DGMR_BATCH_MAX_SCENES 16

typedef struct dgmr_batch_view {
    int32_t scene; /* index into the scenes array */
    int32_t blend_block; /* splat batches: side of the blend's pixel blocks, 8 or 16 (0 = the library default, 8); the
                            first view's value holds for the batch, and later views carry 0 or the same value.  Every
                            block shape gives the same bits (each pixel sees the same splats in the same order); only
                            the speed differs.  The volume marcher ignores it. */
    dgmr_camera camera;
    float* framebuffer; /* [3,H,W] device, written by the forward */
    const float* grad_framebuffer; /* [3,H,W] device, read by the backward; NULL = no gradient for this view */
} dgmr_batch_view;

typedef struct dgmr_scene_grads { /* device outputs of the batched backward, per scene */
    float* sh; /* [N,sh_stride,3] */
    float* weights; /* [N] */
    float* centroids; /* [N,3] */
    float* scales; /* [N,3] */
    float* rotations; /* [N,4] */
} dgmr_scene_grads;

dgmr_status dgmr_splat_batch_workspace_size(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views, int64_t pair_capacity,
    size_t* frame_workspace_bytes, size_t* pair_workspace_bytes);

/* First half only: preprocess of every view and the pair count of the whole
 * batch into stats->n_pairs (to size pair_capacity, like the reference's
 * .item() read of the pair count, splat_forward.cu:141). */
dgmr_status dgmr_splat_batch_preprocess(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views, void* frame_workspace,
    size_t frame_workspace_bytes, dgmr_frame_stats* stats, dgmr_stream stream);

dgmr_status dgmr_splat_batch_forward(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views, void* frame_workspace,
    size_t frame_workspace_bytes, void* pair_workspace, size_t pair_workspace_bytes, int64_t pair_capacity, dgmr_frame_stats* stats, dgmr_stream stream);

/* Backward of the last batched forward run in these workspaces.  Gradients of
 * every scene entry are written (not accumulated): the sum over that entry's
 * views, added in view order.  A view with grad_framebuffer == NULL takes no
 * part (its tiles are skipped), and a scene entry whose grads[s].sh is NULL
 * gets no gradient -- so one batch can mix plain renders with gradient
 * requests.  The same scene tensors may appear in several entries (one per
 * gradient request) to keep their gradients apart. */
dgmr_status dgmr_splat_batch_backward(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views,
    const dgmr_scene_grads* grads, void* frame_workspace, size_t frame_workspace_bytes, void* pair_workspace, size_t pair_workspace_bytes,
    int64_t pair_capacity, dgmr_stream stream);

/* --------------------------------------------------- batched vol_marcher */

/* Many views of one or several scenes marched by ONE launch sequence (no
 * reference counterpart: the reference's vol_marcher.apply marches one view
 * per call, python_bindings/vol_marcher.py:19-65, vol_marcher_forward.cu:42-503).
 * Float32, RenderMode::Full, a scene with DGMR_FORMULATION_DEFAULT gets the
 * marcher's default (Opacity).  Same view table, workspaces and rules as the
 * batched splat above: each view's image is bit-identical to a
 * dgmr_vm_forward_render of that view alone; no allocation, no host
 * synchronisation, capturable in a CUDA graph. */
dgmr_status dgmr_vm_batch_workspace_size(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views, int64_t pair_capacity,
    size_t* frame_workspace_bytes, size_t* pair_workspace_bytes);

/* Preprocess of every view and the batch's pair count into stats->n_pairs. */
dgmr_status dgmr_vm_batch_preprocess(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views, void* frame_workspace,
    size_t frame_workspace_bytes, dgmr_frame_stats* stats, dgmr_stream stream);

dgmr_status dgmr_vm_batch_forward(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views, void* frame_workspace,
    size_t frame_workspace_bytes, void* pair_workspace, size_t pair_workspace_bytes, int64_t pair_capacity, dgmr_frame_stats* stats, dgmr_stream stream);

/* Backward of the last batched march run in these workspaces (replaces
 * dgmr::vol_marcher_backward per view, vol_marcher_backward.cu:53-386, the
 * march recomputed).  Gradients of every scene entry are written, not
 * accumulated: the sum over that entry's views with a grad_framebuffer, added
 * in view order, each term the value the single-view dgmr_vm_backward gives.
 * Views without a grad_framebuffer and scene entries whose grads[s].sh is NULL
 * take no part.  stats (may be NULL) receives the step-limit flag. */
dgmr_status dgmr_vm_batch_backward(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views,
    const dgmr_scene_grads* grads, void* frame_workspace, size_t frame_workspace_bytes, void* pair_workspace, size_t pair_workspace_bytes,
    int64_t pair_capacity, dgmr_frame_stats* stats, dgmr_stream stream);

/* ------------------------------------------------------ batch autotuner */

/* Picks the launch structure of a view set (no reference counterpart: the
 * reference renders one view per call).  For every candidate (depths[d],
 * blend_blocks[b]) the views are cut into consecutive batches of at most
 * depths[d] views (each batch passing only the scenes its views use) with
 * that blend block, and the whole set is rendered -- forward, and backward
 * when grads != NULL -- once untimed and reps times timed with CUDA events on
 * stream.  ms[d * n_blocks + b] receives the candidate's best time,
 * *best_depth and *best_block the fastest candidate.  kind is
 * DGMR_SERVE_SPLAT (blend blocks 0, 8 or 16) or DGMR_SERVE_MARCH (the marcher
 * has no blend block: pass 0).  Every candidate gives the same images and
 * gradients; the runs overwrite the views' framebuffers and the gradient
 * outputs.  The workspaces are those of one batch of all the views (at most
 * DGMR_BATCH_MAX_VIEWS, sized by the kind's *_batch_workspace_size with the
 * pair capacity of the whole set).  The call waits for the stream (it reads
 * the events), so it cannot be captured in a CUDA graph. */
dgmr_status dgmr_batch_autotune(int32_t kind, const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views,
    const dgmr_scene_grads* grads, const int32_t* depths, int32_t n_depths, const int32_t* blend_blocks, int32_t n_blocks, int32_t reps,
    void* frame_workspace, size_t frame_workspace_bytes, void* pair_workspace, size_t pair_workspace_bytes, int64_t pair_capacity, float* ms,
    int32_t* best_depth, int32_t* best_block, dgmr_stream stream);

/* ---------------------------------------------------------- vol_raster */

/* Replaces dgmr::vol_raster_forward(VolRasterForwardData&)
 * (src/dgmr/vol_raster_forward.h:70, .cu:39-520): forward-only volume
 * rasteriser, float.  Per pixel 32 depth bins placed by a RasterBinSizer,
 * piecewise-linear blend with 256 steps per bin.  Same two-workspace scheme as
 * the splat renderer (the binning is the same); dgmr_vr_preprocess leaves the
 * pair count in stats->n_pairs for callers that size the pair workspace from
 * the frame.  An empty frame renders the background (the reference leaves the
 * framebuffer unwritten). */
typedef enum dgmr_render_mode {
    DGMR_RENDER_FULL = 0, /* RenderMode::Full */
    DGMR_RENDER_BINS = 1, /* RenderMode::Bins (vol_raster: nothing drawn, background; marcher: one bin's sum) */
    DGMR_RENDER_DEPTH = 2, /* RenderMode::Depth (vol_raster: end of debug_bin; marcher: distance marched), over max_depth */
} dgmr_render_mode;

/* The debug fields of VolRasterForwardData (vol_raster_forward.h:46-54) and of
 * vol_marcher::ForwardData (vol_marcher.h:48-56).  NULL options = Full. */
typedef struct dgmr_render_options {
    int32_t render_mode; /* dgmr_render_mode */
    int32_t debug_bin; /* -1 = last bin */
    double max_depth; /* 20 in the reference */
    /* Optional device counter (NULL = none), marcher forward only: the march
     * adds the number of (ray, Gaussian, large step) bin fills it makes, each
     * 128 CDF evaluations and 127 bin updates -- the work unit its roofline
     * is stated in.  No reference counterpart. */
    unsigned long long* work_counter;
} dgmr_render_options;

size_t dgmr_vr_frame_workspace_size(int32_t n_gaussians, int32_t width, int32_t height);
size_t dgmr_vr_pair_workspace_size(int32_t n_gaussians, int64_t pair_capacity);
dgmr_status dgmr_vr_preprocess(const dgmr_scene* scene, const dgmr_camera* camera, void* frame_workspace, size_t frame_workspace_bytes,
    dgmr_frame_stats* stats, dgmr_stream stream);
dgmr_status dgmr_vr_forward(const dgmr_scene* scene, const dgmr_camera* camera, const dgmr_render_options* options, float* framebuffer, void* frame_workspace,
    size_t frame_workspace_bytes, void* pair_workspace, size_t pair_workspace_bytes, int64_t pair_capacity, dgmr_frame_stats* stats, dgmr_stream stream);

/* ---------------------------------------------------------- vol_marcher */

/* The reference's ForwardCache plus framebuffer (vol_marcher_forward.h:28-41,
 * returned in this order by python_bindings/vol_marcher.cu:109-122).  All
 * caller-owned device buffers; element type T = scene dtype. */
typedef struct dgmr_vm_cache {
    void* framebuffer; /* [3,H,W] T */
    int32_t* rects; /* [N,2] */
    void* rgb; /* [N,3] T */
    uint8_t* rgb_sh_clamped; /* [N,3] bool */
    void* depths; /* [N] T */
    void* points_xy_image; /* [N,2] T */
    void* inverse_filtered_cov3d; /* [N,6] T, packed 00 01 02 11 12 22 */
    void* filtered_masses; /* [N] T */
    int32_t* tiles_touched; /* [N] */
    int32_t* point_offsets; /* [N] inclusive scan */
    int32_t* i_ranges; /* [tiles,2] */
    int32_t* b_point_list; /* [pair_capacity] */
    void* remaining_transparency; /* [H,W] T */
} dgmr_vm_cache;

/* Workspace for forward (binning) and backward (per-Gaussian accumulators). */
size_t dgmr_vm_workspace_size(int32_t n_gaussians, int32_t width, int32_t height, int64_t pair_capacity, int32_t dtype);

/* Replaces the first half of dgmr::vol_marcher::forward<T>
 * (vol_marcher_forward.cu:98-191): per-Gaussian preprocess and the scan.
 * Afterwards point_offsets[N-1] (also stats->n_pairs) is the pair count. */
dgmr_status dgmr_vm_forward_preprocess(const dgmr_scene* scene, const dgmr_camera* camera, dgmr_vm_cache* cache, void* workspace, size_t workspace_bytes,
    dgmr_frame_stats* stats, dgmr_stream stream);

/* Second half (vol_marcher_forward.cu:197-501): binning into b_point_list and
 * i_ranges, then the ray march into framebuffer and remaining_transparency. */
dgmr_status dgmr_vm_forward_render(const dgmr_scene* scene, const dgmr_camera* camera, dgmr_vm_cache* cache, int64_t pair_capacity, void* workspace,
    size_t workspace_bytes, dgmr_frame_stats* stats, dgmr_stream stream);

/* dgmr_vm_forward_render with the reference's debug render modes
 * (vol_marcher_forward.cu:448-482): Full, Bins (the sum of one bin's channels
 * of the first large step, times max_depth) or Depth (distance marched over
 * max_depth).  options = NULL is Full. */
dgmr_status dgmr_vm_forward_render_options(const dgmr_scene* scene, const dgmr_camera* camera, const dgmr_render_options* options,
    dgmr_vm_cache* cache, int64_t pair_capacity, void* workspace, size_t workspace_bytes, dgmr_frame_stats* stats, dgmr_stream stream);

/* Replaces dgmr::vol_marcher::backward<T> (vol_marcher_backward.cu:53-386).
 * grad_framebuffer [3,H,W] T.  Grads are written (not accumulated): sh
 * [N,sh_stride,3] (SH coefficients beyond sh_stride read as 1.0, as the
 * reference pads with ones, vol_marcher.cu:177), weights [N], centroids [N,3],
 * scales [N,3], rotations [N,4]. */
dgmr_status dgmr_vm_backward(const dgmr_scene* scene, const dgmr_camera* camera, const dgmr_vm_cache* cache, const void* grad_framebuffer, void* grad_sh,
    void* grad_weights, void* grad_centroids, void* grad_scales, void* grad_rotations, void* workspace, size_t workspace_bytes, dgmr_frame_stats* stats,
    dgmr_stream stream);

/* Sample-step store -- no reference counterpart.  The reference's backward
 * recomputes every ray's section set and its 128 sample positions per large
 * step (vol_marcher_backward.cu:172-230) before the bin adjoints.  When the
 * memory is there, the forward can keep them instead: for the first
 * store_steps large steps of each ray, its sample borders and its section
 * count; the backward given the same store reads them and recomputes only
 * steps beyond store_steps.  Results are the same bits as without a store.
 * Bytes of a store: dgmr_vm_step_store_size (W*H rays x store_steps x
 * (128 borders + a count)). */
size_t dgmr_vm_step_store_size(int32_t width, int32_t height, int32_t store_steps, int32_t dtype);
dgmr_status dgmr_vm_forward_render_stored(const dgmr_scene* scene, const dgmr_camera* camera, const dgmr_render_options* options,
    dgmr_vm_cache* cache, int64_t pair_capacity, void* workspace, size_t workspace_bytes, void* step_store, size_t step_store_bytes,
    int32_t store_steps, dgmr_frame_stats* stats, dgmr_stream stream);
dgmr_status dgmr_vm_backward_stored(const dgmr_scene* scene, const dgmr_camera* camera, const dgmr_vm_cache* cache, const void* grad_framebuffer,
    void* grad_sh, void* grad_weights, void* grad_centroids, void* grad_scales, void* grad_rotations, void* workspace, size_t workspace_bytes,
    const void* step_store, size_t step_store_bytes, int32_t store_steps, dgmr_frame_stats* stats, dgmr_stream stream);

/* Gradient-check mode of the marcher (the reference's compile-time
 * DGMR_TORCH_GRAD_CHECK_CONST_SAMPLES, vol_marcher_forward.cu:343-350): with
 * n_sections > 0 every large step uses these fixed (start, end, delta_t)
 * sections instead of collecting them from the Gaussians.  n_sections = 0
 * restores adaptive sampling.  Process-wide; at most 4 sections. */
dgmr_status dgmr_vm_set_const_samples(int32_t n_sections, const double* sections);

/* ------------------------------------------------------------- serving */

/* A continuous-batching request server over resident scenes -- no reference
 * counterpart (the reference renders one view per call from its training loop
 * or viewer).  Requests wait in a queue; whenever one of n_slots slots (a CUDA
 * stream with grow-only workspaces) is free, the queue head is cut into one
 * batch of requests of one kind (splat or vol_marcher) for the batched entry
 * points above, as many as fit max_views, DGMR_BATCH_MAX_SCENES scene
 * entries, max_batch_pixels and the HBM budget (arrival order kept; a
 * gradient request gets a scene entry of its own); a batch of one request
 * takes the single-frame entry points.  Pair capacities are learnt per (scene,
 * resolution, renderer): the first request of such a key reads its pair count
 * back once (a host synchronisation); later ones launch without one, and a
 * batch that overflowed renders again, exactly sized, before it completes.
 * Each result equals the plain call's: images bit-identical, gradients up to
 * the order of atomic additions.  The caller owns every output buffer and must
 * not touch it before the request's completion is returned.  One thread
 * drives a server; the server allocates its own workspaces (cudaMalloc). */
typedef struct dgmr_server dgmr_server;

typedef struct dgmr_server_config {
    int32_t device; /* CUDA device of the server and its scenes */
    int32_t n_slots; /* batches in flight, one stream each (0 = 4) */
    int32_t max_views; /* views per batch, <= DGMR_BATCH_MAX_VIEWS (0 = 8) */
    int32_t reserved;
    size_t hbm_budget_bytes; /* device memory held for work in flight (0 = 80 % of free memory at creation) */
    double capacity_margin; /* pair capacity = pairs seen x margin + 1024 (<= 0 = 2.0; below 1 forces re-renders) */
    int64_t max_batch_pixels; /* a batch takes no further view once its pixels would pass this (0 = no limit; a
                                 batch always takes one); large frames gain nothing from sharing a launch sequence */
} dgmr_server_config;

typedef enum dgmr_serve_kind {
    DGMR_SERVE_SPLAT = 0, /* splat forward (+ backward); dgmr_splat_forward / dgmr_splat_backward */
    DGMR_SERVE_MARCH = 1, /* vol_marcher forward (+ backward), Full mode; dgmr_vm_forward_* / dgmr_vm_backward, or dgmr_vm_batch_* */
} dgmr_serve_kind;

typedef struct dgmr_server_request {
    int32_t kind; /* dgmr_serve_kind */
    int32_t scene; /* index from dgmr_server_add_scene */
    dgmr_camera camera; /* camera and background */
    float* framebuffer; /* [3,H,W] device, written */
    const float* grad_image; /* [3,H,W] device image gradient, or NULL for a render only */
    dgmr_scene_grads grads; /* gradient outputs (written) when grad_image != NULL; weights [N] */
    void* host_image; /* optional pinned host [3,H,W] float: the image is copied there as well */
    uint64_t tag; /* the caller's identifier, returned in the completion */
} dgmr_server_request;

typedef struct dgmr_server_completion {
    uint64_t tag;
    dgmr_status status;
    uint32_t n_pairs; /* pairs of the request's batch */
    int32_t batch_size; /* requests in that batch */
    int32_t rerendered; /* 1 if the batch rendered again after a pair overflow */
    double submit_s, launch_s, done_s; /* host clock, seconds since the server's creation */
} dgmr_server_completion;

typedef struct dgmr_server_stats {
    int64_t submitted, batches, rerenders, deferred;
    int32_t reallocs; /* workspace growths */
    int32_t reserved;
    size_t hbm_budget_bytes, hbm_in_use_bytes, hbm_peak_bytes;
} dgmr_server_stats;

dgmr_status dgmr_server_create(const dgmr_server_config* config, dgmr_server** out);
/* float32 scenes only; the tensors stay the caller's and must outlive the server's use */
dgmr_status dgmr_server_add_scene(dgmr_server* server, const dgmr_scene* scene, int32_t* index);
dgmr_status dgmr_server_submit(dgmr_server* server, const dgmr_server_request* request);
/* Completes finished batches, launches new ones, returns up to max_out
 * completions (never blocks). */
int32_t dgmr_server_poll(dgmr_server* server, dgmr_server_completion* out, int32_t max_out);
/* As poll, but waits until at least one request completes; 0 when nothing is queued or in flight. */
int32_t dgmr_server_wait(dgmr_server* server, dgmr_server_completion* out, int32_t max_out);
/* Requests queued, in flight or completed and not yet returned. */
int64_t dgmr_server_pending(const dgmr_server* server);
/* The server's clock now (seconds since its creation), the clock of the completions' times. */
double dgmr_server_now(const dgmr_server* server);
dgmr_status dgmr_server_get_stats(const dgmr_server* server, dgmr_server_stats* out);
/* Waits for work in flight, frees the server's memory. */
dgmr_status dgmr_server_destroy(dgmr_server* server);

/* ---------------------------------------------------------------- misc */
const char* dgmr_status_string(dgmr_status status);
/* Library version, e.g. "dgmr_b200 0.1 sm_100a". */
const char* dgmr_version(void);
/* Number of kernels this library has launched in this process so far. */
uint64_t dgmr_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* DGMR_B200_H */
