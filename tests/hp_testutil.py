"""Shared helpers of the test suite: golden fixtures and the oracle's view of them."""
import glob
import json
import os

import numpy as np

from hashpoint import synth

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_files():
    """Search+sample fixtures (make_golden.py)."""
    return sorted(f for f in glob.glob(os.path.join(GOLDEN_DIR, "*.npz")) if not os.path.basename(f).startswith("fd_"))


def downstream_files(kind):
    """FeatureQuery / render / Aggregator fixtures (make_golden_downstream.py) of a kind ('feature',
    'render' or 'aggregator')."""
    out = []
    for f in sorted(glob.glob(os.path.join(GOLDEN_DIR, "fd_*.npz"))):
        if str(np.load(f)["kind"]) == kind:
            out.append(f)
    return out


def golden_names():
    return [os.path.basename(f)[:-4] for f in golden_files()]


class Golden:
    """One fixture written by tests/golden/make_golden.py (reference CUDA outputs)."""

    def __init__(self, name):
        self.name = name
        self.g = np.load(os.path.join(GOLDEN_DIR, name + ".npz"))
        g = self.g
        self.H, self.W = int(g["hw"][0]), int(g["hw"][1])
        self.fx, self.fy, self.cx, self.cy = [float(x) for x in g["cam_f"]]
        self.opt = synth.Options(**json.loads(str(g["options"])))
        self.sort = bool(g["sort"])

    def __getitem__(self, k):
        return self.g[k]

    def __contains__(self, k):
        return k in self.g.files

    def ora_camera(self):
        import oracle
        return oracle.camera(self["c2w"], self["w2c"], self["K"], self.W, self.H, self.fx, self.fy, self.cx, self.cy)


def ray_mismatch(mask_a, idx_a, mask_b, idx_b, H, W):
    """Per-ray bool: any mask or pc_idx difference."""
    ma = mask_a.reshape(H * W, -1)
    mb = mask_b.reshape(H * W, -1)
    ia = idx_a.reshape(H * W, -1)
    ib = idx_b.reshape(H * W, -1)
    return ~(np.all(ma == mb, 1) & np.all(ia == ib, 1))


def bits(a):
    a = np.ascontiguousarray(a, np.float32)
    return a.view(np.int32)


def aggregator_params(g):
    """{layer: (weight, bias)} float32 of an Aggregator fixture (stored as fp16-representable fp16)."""
    import oracle_downstream as OD
    return {k: (g["w_" + k].astype(np.float32), g["b_" + k].astype(np.float32)) for k, _, _ in OD.AGG_LAYERS}


def aggregator_inputs(g):
    """(pc_xyz, pc_rgb, pc_dir, pc_feat, sp_xyz, valid) float32 / bool of an Aggregator fixture."""
    return (g["pc_xyz"], g["pc_rgb"], g["pc_dir"], g["pc_feat"].astype(np.float32), g["sp_xyz"], g["valid"])
