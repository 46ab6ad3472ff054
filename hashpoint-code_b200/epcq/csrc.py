"""Drop-in for the reference's compiled `epcq.csrc` extension module.

Same surface as the reference's pybind registration (epcq/csrc/epcq.cpp:10-56):
four functions -- scatter, scatter_hashtable, quick_sampling,
quick_query_for_nearby_point -- and four spec classes with the same
read/write fields.  Every function runs on the B200 CUDA library through its
C ABI (hashpoint.native); nothing falls back to the CPU.

Like pybind11's float/int casters, the spec setters accept Python numbers
and 0-d tensors (the reference's callers pass 0-d tensors for fx..height).
"""
import torch

from hashpoint import ops


def _as_float(v):
    return float(v.item() if isinstance(v, torch.Tensor) else v)


def _as_int(v):
    return int(v.item() if isinstance(v, torch.Tensor) else v)


class _Spec:
    _floats = ()
    _ints = ()
    _tensors = ()

    def __init__(self):
        for f in self._floats:
            object.__setattr__(self, f, 0.0)
        for f in self._ints:
            object.__setattr__(self, f, 0)
        for f in self._tensors:
            object.__setattr__(self, f, None)

    def __setattr__(self, name, value):
        if name in self._floats:
            value = _as_float(value)
        elif name in self._ints:
            value = _as_int(value)
        elif name in self._tensors:
            if not isinstance(value, torch.Tensor):
                raise TypeError("%s.%s must be a torch.Tensor" % (type(self).__name__, name))
        else:
            raise AttributeError("%s has no field %r" % (type(self).__name__, name))
        object.__setattr__(self, name, value)


class NeuralPointsSpec(_Spec):
    """data_spec.hpp:8-13: xyz_data [N, 3]."""
    _tensors = ("xyz_data",)

    def check(self):
        ops.check_input(self.xyz_data, "xyz_data", torch.float32)


class CameraSpec(_Spec):
    """data_spec.hpp:15-31."""
    _tensors = ("c2w", "w2c")
    _floats = ("fx", "fy", "cx", "cy")
    _ints = ("width", "height")

    def check(self):
        # CHECK_INPUT(c2w), CHECK_INPUT(w2c), c2w floating, 2-D, size(1) == 4
        ops.check_input(self.c2w, "c2w")
        ops.check_input(self.w2c, "w2c")
        if not self.c2w.is_floating_point():
            raise RuntimeError("c2w must be floating point")
        if self.c2w.dim() != 2 or self.c2w.shape[1] != 4:
            raise RuntimeError("c2w must be [*, 4]")


class RenderOptions(_Spec):
    """data_spec.hpp:49-69."""
    _ints = ("kernel_size", "num_sample_points_per_ray", "num_point_cloud_per_sp", "num_point_per_ray", "topK")
    _floats = ("t_intvl", "radius_threshold", "sigma_threshold", "background_brightness", "stop_threshold",
               "sdf2weight_gaussian_alpha", "sdf2weight_gaussian_gamma")


class NeuralPointsGrads(_Spec):
    """data_spec.hpp:72-81 (carried for API compatibility; no entry point reads it)."""
    _tensors = ("grad_sigma_out", "grad_sh_out", "mask_out")


def _img_size(img_size):
    if len(img_size) != 2:
        raise RuntimeError("img_size must be (height, width)")
    return _as_int(img_size[0]), _as_int(img_size[1])


def scatter(point_idx_list, point2img_idx_list, depth_list, img_size, bins):
    """rasterization.cu:88-128 -> (buffer_depth f32[H*W, bins], buffer_point_index i32[H*W, bins])."""
    H, W = _img_size(img_size)
    return ops.scatter_multibin(point_idx_list, point2img_idx_list, depth_list, H, W, _as_int(bins))


def scatter_hashtable(point_idx_list, point2img_idx_list, depth_list, img_size, sort):
    """rasterization.cu:130-171 -> (sorted_point_idx_list, sorted_depth_list, hash_table [H*W, 2])."""
    H, W = _img_size(img_size)
    return ops.scatter_hashtable(point_idx_list, point2img_idx_list, depth_list, H, W, bool(sort))


def quick_sampling(neural_points, cam, options, sorted_point_idx_list, hashtable):
    """epcq_render_topk.cu:341-417 -> (output_sp_xyz, output_pc_idx, output_sp_t, mask_out)."""
    neural_points.check()
    cam.check()
    return ops.quick_sampling(neural_points.xyz_data, cam.c2w, cam.fx, cam.fy, cam.cx, cam.cy, cam.width, cam.height,
                              options, sorted_point_idx_list, hashtable)


def quick_query_for_nearby_point(neural_points, cam, options, sorted_point_idx_list, hashtable, indices_of_ray):
    """epcq_render_topk.cu:287-339 -> output_pc_idx i32[R, num_point_per_ray]."""
    neural_points.check()
    cam.check()
    return ops.quick_query(neural_points.xyz_data, cam.c2w, cam.fx, cam.fy, cam.cx, cam.cy, cam.width, cam.height,
                           options, sorted_point_idx_list, hashtable, indices_of_ray)
