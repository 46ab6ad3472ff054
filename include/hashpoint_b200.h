/*
 * hashpoint_b200 -- C ABI of the B200 (sm_100a) HashPoint point searching and
 * sampling library.
 *
 * Every entry point takes plain device pointers and sizes, runs asynchronously
 * on the caller's stream and allocates nothing: outputs and scratch
 * ("workspace") are provided by the caller.  Each returns HP_OK (0) or a
 * negative HP_ERR_* code; hp_last_error() then describes the failure (the
 * message is per calling thread).  Launch failures are reported; faults that
 * happen later on the device surface at the caller's next synchronisation.
 *
 * Layouts follow the reference's tensors exactly:
 *   xyz               float32 [n_points, 3]
 *   sorted_point_idx  int32   [n_points]     point ids grouped by pixel, -1 tail
 *   sorted_depth      float32 [n_points]     camera depth of those ids, -1 tail
 *   hash_table        int32   [H*W, 2]       (start, count) per pixel, (-1,-1) empty
 *   sp_xyz            float32 [H, W, S, 3]   sample positions (0 when unused)
 *   pc_idx            int32   [H, W, S, P]   point ids near each sample (-1 when unused)
 *   sp_t              float32 [H, W, S]      sample depths along the ray (0 when unused)
 *   mask              uint8   [H, W, S]      1 where a sample was emitted (torch.bool layout)
 * where S = num_sample_points_per_ray and P = num_point_cloud_per_sp.
 */
#ifndef HASHPOINT_B200_H
#define HASHPOINT_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define HP_API __attribute__((visibility("default")))
#else
#define HP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* hp_stream_t; /* a cudaStream_t; NULL = legacy default stream */

enum {
  HP_OK = 0,
  HP_ERR_INVALID_ARGUMENT = -1, /* null pointer, bad size, unsupported option value */
  HP_ERR_WORKSPACE = -2,        /* workspace missing or smaller than the *_workspace_size query */
  HP_ERR_CUDA = -3,             /* a CUDA launch or runtime call failed */
  HP_ERR_UNSUPPORTED = -4       /* valid input outside what this build supports */
};

/* Camera of the reference's CameraSpec (epcq/csrc/include/data_spec.hpp:15-31,
 * epcq/epcq.py:16-37).  c2w / w2c: device pointers to row-major matrices with a
 * row stride of 4 floats (a [3,4] or [4,4] float32 tensor); rows 0..2 are read.
 * K: device pointer to the row-major 3x3 intrinsics, read only by the
 * projection (epcq.py:261); may be NULL for the other entry points. */
typedef struct hp_camera {
  const float* c2w;
  const float* w2c;
  const float* K;
  float fx, fy, cx, cy;
  int32_t width, height;
} hp_camera;

/* The RenderOptions fields the path reads (data_spec.hpp:49-69, epcq.py:82-96). */
typedef struct hp_options {
  int32_t kernel_size;              /* search window side k, 1..5 */
  float t_intvl;                    /* t-histogram bin width, > 0 */
  float radius_threshold;           /* ray / ball radius */
  int32_t num_sample_points_per_ray;/* S >= 1 */
  int32_t num_point_cloud_per_sp;   /* P >= 1 */
  int32_t num_point_per_ray;        /* ray-query capacity per ray, >= 0 */
  float sdf2weight_gaussian_alpha;
  float sdf2weight_gaussian_gamma;
} hp_options;

/* Library version (major*10000 + minor*100 + patch). */
HP_API int32_t hp_version(void);

/* Message for the calling thread's last failing call ("" if none). */
HP_API const char* hp_last_error(void);

/* Which arithmetic the projection uses for its two 3x3 @ 3xN products at this
 * point count: 1 = fused multiply-add chain, 0 = separately rounded products.
 * This reproduces what torch's cuBLAS GEMM did for the reference's projection
 * (epcq/epcq.py:253,261) on B200, so pixel ids and depths match bit for bit. */
HP_API void hp_projection_rounding(int64_t n_points, int32_t* fused_world, int32_t* fused_image);

/* Scratch bytes hp_pts2plane needs for this problem size. */
HP_API size_t hp_pts2plane_workspace_size(int64_t n_points, int32_t height, int32_t width);

/* Projection + per-pixel hash table.  Replaces NeuralPoints.pts2plane
 * (epcq/epcq.py:279-295: _world2cam :251, _cam2image :259, _convetpixel :267,
 * torch.sort :284, gathers :285-286) followed by _C.scatter_hashtable
 * (epcq/csrc/rasterization.cu:130-171).  Buckets list point ids in ascending
 * id order (sort == 0, the stable sort's order) or by (depth, id) (sort != 0,
 * the reference's stable bubble sort).  Writes every element of the three
 * outputs.  n_points <= 2^30. */
HP_API int32_t hp_pts2plane(const float* xyz, int64_t n_points, const hp_camera* cam, int32_t sort,
                     int32_t* sorted_point_idx, float* sorted_depth, int32_t* hash_table,
                     void* workspace, size_t workspace_bytes, hp_stream_t stream);

/* Reports whether the hash-table scan of the last hp_pts2plane on this
 * workspace (same n_points, height and width) had to give up waiting for one
 * of its blocks (its waits are bounded; the table is then wrong): HP_OK, or
 * HP_ERR_CUDA with the reason in hp_last_error().  Synchronises on stream.
 * This does not happen while the GPU runs the call's blocks; the check exists
 * so that a failure would be seen.  No counterpart in the reference. */
HP_API int32_t hp_pts2plane_status(const void* workspace, int64_t n_points, int32_t height, int32_t width,
                                   hp_stream_t stream);

/* hp_pts2plane for callers that cannot allocate device memory: a host plugin
 * that only receives device pointers for its inputs and outputs from the
 * application embedding it, or a service that must not grow its device
 * footprint after start-up, has no way to provide hp_pts2plane's workspace.
 * This entry point takes the same inputs and outputs and allocates nothing;
 * its scratch is an array built into the library (about 11 MB of device
 * memory on every GPU that loads the library, held until the process exits),
 * so it accepts at most HP_NOALLOC_MAX_POINTS points and HP_NOALLOC_MAX_PIXELS
 * pixels and returns HP_ERR_INVALID_ARGUMENT beyond that.  A call looks up its
 * device's address of the array unless its stream is being captured; a
 * captured call uses the address the device's last uncaptured call found, so
 * make one call outside capture first (a captured call with none before it
 * fails with HP_ERR_CUDA).  All calls share the one array, so calls that
 * overlap on the GPU (on different streams, or from different threads) race:
 * serialise them.  Each call clears the parts of the array that must start at
 * zero.
 * No counterpart in the reference. */
#define HP_NOALLOC_MAX_POINTS 262144
#define HP_NOALLOC_MAX_PIXELS 1048576
HP_API int32_t hp_pts2plane_noalloc(const float* xyz, int64_t n_points, const hp_camera* cam, int32_t sort,
                                    int32_t* sorted_point_idx, float* sorted_depth, int32_t* hash_table,
                                    hp_stream_t stream);

/* hp_pts2plane_status for the last hp_pts2plane_noalloc on the current
 * device (same n_points, height and width).  Synchronises on stream. */
HP_API int32_t hp_pts2plane_noalloc_status(int64_t n_points, int32_t height, int32_t width, hp_stream_t stream);

/* Per-pixel hash table from inputs already sorted by pixel id.  Replaces
 * _C.scatter_hashtable (epcq/csrc/rasterization.cu:130-171, kernel :7-34):
 * point_idx / point2img / depth [n] sorted by point2img ascending; entries with
 * point2img outside [0, H*W) are left -1.  Writes every element of the outputs.
 * n <= 2^30. */
HP_API int32_t hp_scatter_hashtable(const int32_t* point_idx, const int32_t* point2img, const float* depth, int64_t n,
                             int32_t height, int32_t width, int32_t sort,
                             int32_t* sorted_point_idx, float* sorted_depth, int32_t* hash_table,
                             hp_stream_t stream);

/* Window search, primary-surface selection, K-sample emission and per-sample
 * point selection for every pixel ray.  Replaces _C.quick_sampling
 * (epcq/csrc/epcq_render_topk.cu:341-417: quick_sampling_kernel :82-220 then
 * quick_search_nearby_pc :10-81).  hash_table may come from hp_pts2plane,
 * hp_scatter_hashtable or the reference.  Writes every element of the four
 * outputs (no separate fill is needed).  For P < 8 the first P of the up to 8
 * selected ids are kept (the reference writes 8 ids into a P-wide row there).
 * n_sorted is the length of sorted_point_idx: bucket ranges are clipped to it
 * and ids outside [0, n_points) are skipped, so a malformed hash table cannot
 * make the kernel read out of bounds. */
HP_API int32_t hp_quick_sampling(const float* xyz, int64_t n_points, const hp_camera* cam, const hp_options* opt,
                                 const int32_t* sorted_point_idx, int64_t n_sorted, const int32_t* hash_table,
                                 float* sp_xyz, int32_t* pc_idx, float* sp_t, uint8_t* mask, void* workspace,
                                 size_t workspace_bytes, hp_stream_t stream);

/* Point attributes read by hp_feature_query: xyz, rgb, dir f32 [n_points, 3]
 * and feat [n_points, feat_dim] in f32 or (feat_half != 0) f16. */
typedef struct hp_point_attrs {
  const float* xyz;
  const float* rgb;
  const float* dir;
  const void* feat;
  int32_t feat_dim;
  int32_t feat_half;
  int64_t n_points;
} hp_point_attrs;

/* offsets[i] = number of nonzero bytes of mask[0..i) (an exclusive scan), and
 * *count (device) = all of them.  Numbers the valid samples for
 * hp_feature_query, in place of the reference's boolean indexing
 * (epcq/epcq.py:347-351).  workspace: hp_mask_scan_workspace_size(n) bytes. */
HP_API int32_t hp_mask_scan(const uint8_t* mask, int64_t n, int32_t* offsets, int32_t* count, void* workspace,
                            size_t workspace_bytes, hp_stream_t stream);
HP_API size_t hp_mask_scan_workspace_size(int64_t n);

/* FeatureQuery.forward (epcq/epcq.py:345-387): for every sample with mask set
 * (n_rays x S samples; offsets from hp_mask_scan give its output row m), write
 * out_sp_xyz[m] = sp_xyz of the sample, rays_d[m] = the direction of its
 * pixel ray as generate_rays builds it (epcq.py:333-341: ((u - cx) / fx,
 * (v - cy) / fy, 1) times the rotation of cam->c2w, pixel corners, not
 * centres), and for each of its P ids: valid[m, p] and the id's xyz / rgb /
 * dir / feat rows in pc_xyz / pc_rgb / pc_dir [M, P, 3] and pc_feat
 * [M, P, feat_dim] (f32), or zeros for an id of -1 (any id outside
 * [0, n_points) is treated as -1).  ray_uv: [n_rays, 2] (u, v) of each ray
 * (the reference's ray_index_uv), or NULL for the image's pixels in row-major
 * order (then cam->width is used). */
HP_API int32_t hp_feature_query(const hp_point_attrs* pts, const float* sp_xyz, const int32_t* pc_idx,
                                const uint8_t* mask, int64_t n_rays, int32_t S, int32_t P, const int32_t* offsets,
                                const hp_camera* cam, const int32_t* ray_uv, float* pc_xyz, float* pc_rgb,
                                float* pc_dir, float* pc_feat, float* out_sp_xyz, uint8_t* valid, float* rays_d,
                                hp_stream_t stream);

/* clamp_t (epcq/epcq.py:508-515): t_dist[r, s] = t[r, s+1] - t[r, s], the
 * last one vsize, and any gap below 1e-8 or above 2 * vsize replaced by vsize. */
HP_API int32_t hp_clamp_t(const float* t_val, int64_t n_rays, int32_t S, float vsize, float* t_dist,
                          hp_stream_t stream);

/* render (epcq/epcq.py:517-529): colour [n_rays, 3] of sigmas [n_rays, S] and
 * rgbs [n_rays, S, 3] composited front to back with the spacings `deltas`
 * [n_rays, S] -- or, when deltas is NULL, with clamp_t(t_val, vsize) computed
 * on the fly -- over a black (white_bg = 0) or white background. */
HP_API int32_t hp_render(const float* deltas, const float* t_val, float vsize, const float* sigmas,
                         const float* rgbs, int64_t n_rays, int32_t S, int32_t white_bg, float* color,
                         hp_stream_t stream);

/* Aggregator (epcq/epcq.py:406-507): the per-point MLP, alpha branch,
 * inverse-distance aggregation and colour branch over FeatureQuery's outputs,
 * on the tensor cores (bf16 operands, fp32 accumulation).
 *
 * The nine nn.Linear layers as row-major fp32 [out, in] device arrays and
 * their biases, in module order: block1.0 (256x284), block1.2 (256x256),
 * block3.0 (256x263), block3.2 (256x256), alpha_branch.0 (1x256),
 * color_branch.0 (128x280), .2 (128x128), .4 (128x128), .6 (3x128). */
typedef struct hp_aggregator_weights {
  const float* weight[9];
  const float* bias[9];
} hp_aggregator_weights;

/* Bytes of the packed weights (bf16 operand tiles + fp32 biases). */
HP_API size_t hp_aggregator_packed_size(void);
/* Pack the weights once (after every change); packed: 256-byte aligned. */
HP_API int32_t hp_aggregator_pack(const hp_aggregator_weights* w, void* packed, size_t packed_bytes,
                                  hp_stream_t stream);
HP_API size_t hp_aggregator_workspace_size(int64_t n_samples);
/* Aggregator.forward: n_samples valid samples (FeatureQuery's M) with P points
 * each -- pc_xyz / pc_rgb / pc_dir f32 [M, P, 3], pc_feat f32 [M, P, 32]
 * (16-byte aligned), sp_xyz and rays_d f32 [M, 3], valid u8 [M, P] -- then
 * alpha_out f32 [n_positions] and color_out f32 [n_positions, 3]: sample
 * mask_offsets[i] at every set position i of mask_out (the sampling mask,
 * mask_offsets from hp_mask_scan of it), zeros elsewhere.  P: 1, 2, 4, ..., 32.
 * Waits inside the kernels are bounded; hp_aggregator_status (synchronising)
 * reports one that gave up. */
HP_API int32_t hp_aggregator_forward(const void* packed, const float* pc_xyz, const float* pc_rgb,
                                     const float* pc_dir, const float* pc_feat, int32_t feat_dim,
                                     const float* sp_xyz, const uint8_t* valid, const float* rays_d,
                                     int64_t n_samples, int32_t P, const uint8_t* mask_out,
                                     const int32_t* mask_offsets, int64_t n_positions, float* alpha_out,
                                     float* color_out, void* workspace, size_t workspace_bytes, hp_stream_t stream);
HP_API int32_t hp_aggregator_status(const void* workspace, int64_t n_samples, hp_stream_t stream);

/* Scratch bytes hp_quick_sampling needs for n_sorted ids and an image of this
 * size (its tile schedule and the ids' points packed as 16-byte records);
 * workspace must be 256-byte aligned. */
HP_API size_t hp_quick_sampling_workspace_size(int64_t n_sorted, int32_t height, int32_t width);

/* Launch tuning of hp_quick_sampling_tuned and hp_quick_sampling_batch (NULL
 * or 0 fields = defaults).  Outputs never depend on it.
 *   heavy_window   rays whose window holds more candidates are served by a
 *                  whole warp instead of one thread (0..4096; default 320).
 *   blocks_per_sm  resident blocks of the persistent sampling kernel per SM
 *                  (default: as many as fit).
 *   stage_config   stage and tile of the sampling kernel (0 = 4):
 *                  1: 2560 staged points per tile, 4 blocks per SM, 8 x 32 tiles;
 *                  2: 3712 points, 3 blocks per SM, 8 x 32;
 *                  3: 5888 points, 2 blocks per SM, 8 x 32;
 *                  4: 2560 points, 4 blocks per SM, 16 x 16 tiles;
 *                  5: 3712 points, 3 blocks per SM, 16 x 16.
 *                  Tiles whose window halo holds more points are split into
 *                  row bands and column ranges, or read from global memory. */
typedef struct hp_tuning {
  int32_t heavy_window;
  int32_t blocks_per_sm;
  int32_t stage_config;
} hp_tuning;

/* The tile (tile_h x tile_w pixels), staged points per tile and resident
 * blocks per SM of a stage configuration (0 reads as 4); any output pointer
 * may be NULL.  HP_ERR_INVALID_ARGUMENT outside 0..5.  No counterpart in the
 * reference. */
HP_API int32_t hp_stage_config_info(int32_t config, int32_t* tile_h, int32_t* tile_w, int32_t* stage_points,
                                    int32_t* blocks_per_sm);

/* hp_quick_sampling with launch tuning (see hp_tuning; NULL = defaults).
 * No counterpart in the reference. */
HP_API int32_t hp_quick_sampling_tuned(const float* xyz, int64_t n_points, const hp_camera* cam,
                                       const hp_options* opt, const int32_t* sorted_point_idx, int64_t n_sorted,
                                       const int32_t* hash_table, float* sp_xyz, int32_t* pc_idx, float* sp_t,
                                       uint8_t* mask, const hp_tuning* tuning, void* workspace,
                                       size_t workspace_bytes, hp_stream_t stream);

/* One view of a batched hp_quick_sampling: the arguments of hp_quick_sampling
 * for that view (cloud, camera, options, its hash table and its outputs). */
typedef struct hp_view {
  const float* xyz;
  int64_t n_points;
  const int32_t* sorted_point_idx;
  int64_t n_sorted;
  const int32_t* hash_table;
  float* sp_xyz;
  int32_t* pc_idx;
  float* sp_t;
  uint8_t* mask;
  hp_camera cam;
  hp_options opt;
} hp_view;

/* hp_quick_sampling for many views -- different clouds, cameras, image sizes
 * and options -- in one persistent launch over the tiles of all views, so one
 * view's tail overlaps the next views' work.  Tiles are taken view by view in
 * table order (heaviest first within a view), so put heavy views first.  Each
 * view's outputs are bit-identical to hp_quick_sampling's for that view.  No
 * counterpart call in the reference, which launches quick_sampling once per
 * view (epcq/csrc/epcq_render_topk.cu:341-417).  `views` (host) is checked and
 * sizes the launch; the kernels read `views_device`, the same table in device
 * memory (for example copied there from pinned memory, so the call can be
 * captured in a CUDA graph), or, when it is NULL, a copy of `views` made into
 * the workspace on `stream`.  `tuning` may be NULL. */
HP_API int32_t hp_quick_sampling_batch(const hp_view* views, const hp_view* views_device, int32_t n_views,
                                       const hp_tuning* tuning, void* workspace, size_t workspace_bytes,
                                       hp_stream_t stream);

/* Scratch bytes hp_quick_sampling_batch needs for these views (0 if invalid);
 * 256-byte aligned. */
HP_API size_t hp_quick_sampling_batch_workspace_size(const hp_view* views, int32_t n_views);

/* Ray query for a list of pixel rays (linear ids v*W+u).  Replaces
 * _C.quick_query_for_nearby_point (epcq/csrc/epcq_render_topk.cu:287-339,
 * kernel :222-283).  out [n_rays, num_point_per_ray]: ids with ray distance
 * below the radius, at most 32 per window cell, in window-cell then bucket
 * order (the reference's order is that of its atomics), -1 padded.
 * kernel_size may be 1..31 here.  Ray ids outside the image give a row of -1. */
HP_API int32_t hp_quick_query_for_nearby_point(const float* xyz, int64_t n_points, const hp_camera* cam,
                                               const hp_options* opt, const int32_t* sorted_point_idx,
                                               int64_t n_sorted, const int32_t* hash_table, const int32_t* ray_ids,
                                               int64_t n_rays, int32_t* out, hp_stream_t stream);

/* Multi-bin z-buffer: per pixel the `bins` nearest-depth points, ascending.
 * Replaces _C.scatter (epcq/csrc/rasterization.cu:88-128, kernel :36-86).
 * Inputs sorted by point2img as for hp_scatter_hashtable.  Points with negative
 * depth are skipped (the reference never advances past one).  Outputs
 * [H*W, bins], -1 padded.  1 <= bins <= 64. */
HP_API int32_t hp_scatter(const int32_t* point_idx, const int32_t* point2img, const float* depth, int64_t n,
                   int32_t height, int32_t width, int32_t bins, float* buffer_depth, int32_t* buffer_point_index,
                   hp_stream_t stream);

/* Normalised world-space direction of every pixel's ray, [H*W, 3], exactly as
 * the sampling kernels compute it (cam2world_ray, cuda_util.cuh:338-354). */
HP_API int32_t hp_ray_directions(const hp_camera* cam, float* dirs, hp_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* HASHPOINT_B200_H */
