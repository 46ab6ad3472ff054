/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle for the HashPoint search+sample path.
 *
 * A CPU restatement of the reference's algorithm, used by tests/, the smoke
 * check and bench.py's CPU-baseline leg as the checker.  It is never linked
 * into, called by or shipped with the CUDA product path.
 *
 * Parity: pinned against golden fixtures produced by the reference's own CUDA
 * extension (compiled from its sources by oracle/build_ref.py and run on a
 * B200; see tests/golden/make_golden.py).  The FP32 functions mirror the GPU
 * arithmetic operation by operation (explicit fmaf where nvcc/cuBLAS fuse).
 * CUDA's norm3df / rnorm3df / __expf are replaced by correctly rounded
 * double-precision evaluations, so a ray whose decision lies within a few ulp
 * of a threshold can legitimately differ; every sampling routine reports a
 * per-ray decision margin so tests can tell such rays apart.
 */
#ifndef HP_ORACLE_H
#define HP_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  float c2w[12];   /* rows 0..2 of the 4x4 camera-to-world matrix, row-major */
  float w2c[12];   /* rows 0..2 of the world-to-camera matrix */
  float K[9];      /* 3x3 intrinsics, row-major (used by the projection only) */
  float fx, fy, cx, cy;
  int32_t width, height;
} ora_camera;

typedef struct {
  int32_t kernel_size;
  float t_intvl;
  float radius_threshold;
  int32_t num_sample_points_per_ray;   /* S */
  int32_t num_point_cloud_per_sp;      /* P */
  int32_t num_point_per_ray;
  float sdf2weight_gaussian_alpha;
  float sdf2weight_gaussian_gamma;
} ora_options;

/* epcq/epcq.py:251-274: world->camera (cuBLAS 3x3 GEMM + bias), K projection,
 * divide, truncating int32 cast, out-of-image -> H*W.  depth = camera z. */
void ora_project(const float* xyz, int64_t n, const ora_camera* cam, int32_t* point2img, float* depth);
/* Same in float64 (error yardstick); depth only. */
void ora_project_f64(const float* xyz, int64_t n, const ora_camera* cam, double* depth);

/* Stable sort of point ids by pixel id (epcq.py:283-286; torch.sort, radix). */
void ora_sort_by_pixel(const int32_t* point2img, const float* depth, int64_t n, int32_t hw,
                       int32_t* pid_sorted, float* depth_sorted, int32_t* idx_sorted);

/* rasterization.cu:7-34 + :130-171.  Inputs sorted by pixel id.
 * Outputs: out_idx/out_depth [n] (-1 where no pixel claims the slot), hash [hw*2]. */
void ora_scatter_hashtable(const int32_t* point_idx, const int32_t* point2img, const float* depth, int64_t n,
                           int32_t height, int32_t width, int32_t sort,
                           int32_t* out_idx, float* out_depth, int32_t* hash);

/* epcq.py:279-295: projection + sort + scatter_hashtable. */
void ora_pts2plane(const float* xyz, int64_t n, const ora_camera* cam, int32_t sort,
                   int32_t* out_idx, float* out_depth, int32_t* hash);

/* epcq_render_topk.cu:341-417 (quick_sampling_kernel :82-220 followed by
 * quick_search_nearby_pc :10-81).  Outputs are fully written (defaults 0/-1/0).
 * margin [hw] (optional): smallest relative slack of any decision on the ray.
 * rays [n_rays] (optional): only these linear pixel ids; outputs (and margin)
 * are then compact, indexed by position in `rays`.
 * Returns 0, or a negative error code for invalid options. */
int ora_quick_sampling(const float* xyz, int64_t n_points, const ora_camera* cam, const ora_options* opt,
                       const int32_t* sorted_idx, const int32_t* hash,
                       float* sp_xyz, int32_t* pc_idx, float* sp_t, uint8_t* mask, float* margin,
                       const int32_t* rays, int64_t n_rays, int32_t nthreads);

/* Float64 twin: emitted t and sample xyz in double for the error statement. */
int ora_quick_sampling_f64(const float* xyz, int64_t n_points, const ora_camera* cam, const ora_options* opt,
                           const int32_t* sorted_idx, const int32_t* hash,
                           double* sp_xyz, double* sp_t, uint8_t* mask, int32_t nthreads);

/* epcq_render_topk.cu:222-283 + :287-339.  Deterministic order: window-cell
 * order, then bucket order; per cell at most 32 ids; per ray at most
 * num_point_per_ray.  out [n_rays * num_point_per_ray] (-1 padded),
 * count [n_rays] = ids written. */
int ora_quick_query(const float* xyz, int64_t n_points, const ora_camera* cam, const ora_options* opt,
                    const int32_t* sorted_idx, const int32_t* hash, const int32_t* ray_ids, int64_t n_rays,
                    int32_t* out, int32_t* count, float* margin);

/* rasterization.cu:36-128: per pixel the `bins` nearest-depth points, ascending.
 * Negative-depth points are skipped.  out_depth/out_idx [hw*bins] (-1 padded). */
void ora_scatter_multibin(const int32_t* point_idx, const int32_t* point2img, const float* depth, int64_t n,
                          int32_t height, int32_t width, int32_t bins, float* out_depth, int32_t* out_idx);

#ifdef __cplusplus
}
#endif
#endif
