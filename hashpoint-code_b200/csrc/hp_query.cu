// Ray query for listed pixel rays, and the multi-bin z-buffer.
//
// hp_quick_query_for_nearby_point replaces _C.quick_query_for_nearby_point
// (epcq/csrc/epcq_render_topk.cu:287-339, kernel :222-283).  The reference
// gives each window cell a lane that gathers up to 32 ids within the ray
// radius and then reserves output slots with atomicAdd, so the order of a
// row -- and which ids survive when the row overflows -- depends on atomic
// timing.  Here one warp serves one ray: lanes count their cell's ids, a warp
// prefix sum assigns each cell its offset in window-cell order, and a second
// pass writes the ids, so rows are deterministic (window-cell order, bucket
// order) and an overflowing row keeps its first num_point_per_ray ids.
//
// hp_scatter replaces _C.scatter (epcq/csrc/rasterization.cu:88-128, kernel
// :36-86): per pixel the `bins` nearest points by depth, sorted ascending.
#include "hp_common.cuh"

namespace hp {

int32_t check_camera(const hp_camera* cam, const char* who);
DevCamera dev_camera(const hp_camera* cam);
DevOptions dev_options(const hp_options* o);

constexpr int kQueryWarps = 4;

__global__ void __launch_bounds__(kQueryWarps * 32) k_quick_query(const float* __restrict__ xyz, int n_points,
                                                                  const int* __restrict__ sidx, int n_sorted,
                                                                  const int2* __restrict__ hash, DevCamera cam,
                                                                  DevOptions opt, const int* __restrict__ ray_ids,
                                                                  int n_rays, int* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * kQueryWarps + (threadIdx.x >> 5);
  if (i >= n_rays) return;
  const int cap = opt.num_point_per_ray;
  int* row = out + (size_t)i * cap;
  const int W = cam.width, H = cam.height;
  const int ray = ray_ids[i];
  int written = 0;
  if (0 <= ray && ray < W * H) {
    const int u = ray % W, v = ray / W;
    Ray r;
    make_ray(cam.c2w, cam.fx, cam.fy, cam.cx, cam.cy, u, v, r);
    const int k2 = opt.k * opt.k;
    int base = 0;
    for (int c0 = 0; c0 < k2 && base < cap; c0 += 32) {
      const int l = c0 + lane;
      int2 h = make_int2(0, -1);
      if (l < k2) {
        int vv, uu;
        window_cell(v, u, opt.k, H, W, l, vv, uu);
        h = __ldg(hash + (size_t)vv * W + uu);
        if (h.x < 0) h.y = -1;
        h.y = min(h.y, n_sorted - h.x);  // clip the range to the id list
      }
      // count this cell's ids (<= 32)
      int cnt = 0;
      for (int j = h.x; j < h.x + h.y && cnt < kQueryPerCell; j++) {
        const int id = __ldg(sidx + j);
        if ((unsigned)id >= (unsigned)n_points) continue;
        const float4 p = load_point(xyz, id);
        float t, dist;
        intersect(r, p.x, p.y, p.z, t, dist);
        if (dist < opt.radius) cnt++;
      }
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      int pos = base + incl - cnt;
      for (int j = h.x, c = 0; j < h.x + h.y && c < cnt && pos < cap; j++) {
        const int id = __ldg(sidx + j);
        if ((unsigned)id >= (unsigned)n_points) continue;
        const float4 p = load_point(xyz, id);
        float t, dist;
        intersect(r, p.x, p.y, p.z, t, dist);
        if (dist < opt.radius) {
          row[pos++] = id;
          c++;
        }
      }
      base += __shfl_sync(0xffffffffu, incl, 31);
    }
    written = base < cap ? base : cap;
  }
  for (int q = written + lane; q < cap; q += 32) row[q] = -1;
}

// Per pixel: first index of its run by binary search over the sorted pixel
// ids (cuda_util.cuh:558-579), then the reference's buffer of the `bins`
// nearest depths, then a stable ascending sort (its bubble sort's result).
constexpr int kMaxBins = 64;

__global__ void __launch_bounds__(128) k_scatter_multibin(const int* __restrict__ point_idx,
                                                          const int* __restrict__ point2img,
                                                          const float* __restrict__ depth, int n, int hw, int bins,
                                                          float* __restrict__ out_depth, int* __restrict__ out_idx) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= hw) return;
  int lo = 0, hi = n;  // lower_bound of p
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (point2img[mid] < p)
      lo = mid + 1;
    else
      hi = mid;
  }
  float bd[kMaxBins];
  int bi[kMaxBins];
  int size = 0, maxi = -1;
  float maxz = -1000.0f;
  for (int j = lo; j < n && point2img[j] == p; j++) {
    const float d = depth[j];
    if (d < 0) continue;  // the reference spins forever here; the point is skipped instead
    if (size < bins) {
      bd[size] = d;
      bi[size] = point_idx[j];
      if (d > maxz) maxz = d, maxi = size;
      size++;
    } else if (d < maxz) {
      bd[maxi] = d;
      bi[maxi] = point_idx[j];
      maxz = d;
      for (int q = 0; q < bins; q++)
        if (bd[q] > maxz) maxz = bd[q], maxi = q;
    }
  }
  // stable insertion sort ascending by depth (same result as a stable bubble sort)
  for (int a = 1; a < size; a++) {
    const float kd = bd[a];
    const int ki = bi[a];
    int b = a - 1;
    while (b >= 0 && bd[b] > kd) {
      bd[b + 1] = bd[b];
      bi[b + 1] = bi[b];
      b--;
    }
    bd[b + 1] = kd;
    bi[b + 1] = ki;
  }
  float* od = out_depth + (size_t)p * bins;
  int* oi = out_idx + (size_t)p * bins;
  for (int q = 0; q < bins; q++) {
    od[q] = q < size ? bd[q] : -1.0f;
    oi[q] = q < size ? bi[q] : -1;
  }
}

}  // namespace hp

using namespace hp;

extern "C" int32_t hp_quick_query_for_nearby_point(const float* xyz, int64_t n_points, const hp_camera* cam,
                                                   const hp_options* opt, const int32_t* sorted_point_idx,
                                                   int64_t n_sorted, const int32_t* hash_table, const int32_t* ray_ids,
                                                   int64_t n_rays, int32_t* out, hp_stream_t stream) {
  if (int32_t rc = check_camera(cam, "hp_quick_query_for_nearby_point")) return rc;
  if (!opt) return set_error(HP_ERR_INVALID_ARGUMENT, "hp_quick_query_for_nearby_point: opt is NULL");
  // the reference rejects windows that need 1024 threads per block (epcq_render_topk.cu:321-323)
  if (opt->kernel_size < 1 || opt->kernel_size > 31)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_quick_query_for_nearby_point: kernel_size %d outside 1..31",
                     opt->kernel_size);
  if (opt->num_point_per_ray < 0)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_quick_query_for_nearby_point: num_point_per_ray < 0");
  if (n_rays < 0 || n_rays >= (1ll << 31) || n_points < 0 || n_points >= (1ll << 31) || n_sorted < 0 ||
      n_sorted >= (1ll << 31))
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_quick_query_for_nearby_point: bad sizes");
  if (n_rays == 0 || opt->num_point_per_ray == 0) return HP_OK;
  if (!hash_table || !ray_ids || !out || (n_points > 0 && !xyz) || (n_sorted > 0 && !sorted_point_idx))
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_quick_query_for_nearby_point: null pointer");
  if (((uintptr_t)hash_table & 7) != 0)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_quick_query_for_nearby_point: hash_table must be 8-byte aligned");
  const int blocks = (int)((n_rays + kQueryWarps - 1) / kQueryWarps);
  k_quick_query<<<blocks, kQueryWarps * 32, 0, (cudaStream_t)stream>>>(
      xyz, (int)n_points, sorted_point_idx, (int)n_sorted, (const int2*)hash_table, dev_camera(cam), dev_options(opt),
      ray_ids, (int)n_rays, out);
  return check_launch("k_quick_query");
}

extern "C" int32_t hp_scatter(const int32_t* point_idx, const int32_t* point2img, const float* depth, int64_t n,
                              int32_t height, int32_t width, int32_t bins, float* buffer_depth,
                              int32_t* buffer_point_index, hp_stream_t stream) {
  if (height <= 0 || width <= 0 || (int64_t)height * width >= (1ll << 31))
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_scatter: bad image size %dx%d", height, width);
  if (bins < 1 || bins > kMaxBins)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_scatter: bins %d outside 1..%d", bins, kMaxBins);
  if (n < 0 || n >= (1ll << 31)) return set_error(HP_ERR_INVALID_ARGUMENT, "hp_scatter: n out of range");
  if (!buffer_depth || !buffer_point_index || (n > 0 && (!point_idx || !point2img || !depth)))
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_scatter: null pointer");
  const int hw = height * width;
  k_scatter_multibin<<<(hw + 127) / 128, 128, 0, (cudaStream_t)stream>>>(point_idx, point2img, depth, (int)n, hw,
                                                                          bins, buffer_depth, buffer_point_index);
  return check_launch("k_scatter_multibin");
}
