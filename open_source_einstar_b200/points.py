"""Organised points, normals and weights from a disparity map, and the recording layout of depth frames.

disparity_to_points mirrors depth::disparity_to_points (libs/depth/src/point_image.cpp:10-54), which
produces the point image that tracking and fusion consume. pack_depth mirrors depth_metal::DepthPacker
(libs/depth_metal/src/depth_packer.cpp:10-21), the uncompressed depth layout of session recordings.
Both run on device tensors through libdepth_cuda (ds_disparity_to_points, ds_pack_depth) and allocate
nothing in the library; the caller owns every buffer.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import _native as N
from .stereo import CUDA_STREAM_LEGACY, RectifiedGeometry, StereoError


@dataclass
class PointImageParams:
    """depth::PointImageParams (libs/depth/include/einstar/depth/point_image.hpp:41-47)."""
    min_depth: float = 150.0
    max_depth: float = 700.0
    max_depth_jump: float = 4.0
    edge_weight: float = 0.25
    weight_reference_depth: float = 0.0

    def c(self) -> N.PointParamsC:
        return N.PointParamsC(self.min_depth, self.max_depth, self.max_depth_jump, self.edge_weight,
                              self.weight_reference_depth)


def _stream(stream):
    if stream is None:
        return None
    h = int(stream.cuda_stream)
    return CUDA_STREAM_LEGACY if h == 0 else h


def disparity_to_points(disparity, confidence, geometry: RectifiedGeometry, params: PointImageParams | None = None,
                        out: dict | None = None, stream=None) -> dict:
    """Device float32 disparity (H x W) and confidence (or None) -> {"points": H x W x 4, "normals": H x W x 4,
    "weights": H x W} device float32 tensors (points w = 1 where valid)."""
    import torch
    h, w = disparity.shape
    params = params or PointImageParams()
    if out is None:
        out = {"points": torch.empty((h, w, 4), dtype=torch.float32, device=disparity.device),
               "normals": torch.empty((h, w, 4), dtype=torch.float32, device=disparity.device),
               "weights": torch.empty((h, w), dtype=torch.float32, device=disparity.device)}
    g = N.GeometryC(geometry.f, geometry.cx, geometry.cy, geometry.baseline, geometry.cx_offset)
    rc = N.lib().ds_disparity_to_points(disparity.data_ptr(), None if confidence is None else confidence.data_ptr(),
                                        w, h, C.byref(g), C.byref(params.c()), out["points"].data_ptr(),
                                        out["normals"].data_ptr(), out["weights"].data_ptr(), _stream(stream))
    if rc != 0:
        raise StereoError(rc, N.lib().ds_last_global_error().decode())
    return out


def pack_depth(points, weights, out=None, stream=None):
    """Device points (H x W x 4) and weights (H x W) -> H*W*3 bytes: u16 depth in 1/50 mm delta-coded along
    rows, then u8 confidence (the session file's uncompressed layout)."""
    import torch
    h, w = weights.shape
    if out is None:
        out = torch.empty(h * w * 3, dtype=torch.uint8, device=weights.device)
    rc = N.lib().ds_pack_depth(points.data_ptr(), weights.data_ptr(), w, h, out.data_ptr(), _stream(stream))
    if rc != 0:
        raise StereoError(rc, N.lib().ds_last_global_error().decode())
    return out


def unpack_depth(packed, width: int, height: int):
    """Host inverse of the packed layout: (depth in mm as float32, confidence u8); 0 = no depth."""
    import numpy as np
    b = np.asarray(packed, np.uint8)
    dq = b[: 2 * width * height].view(np.uint16).reshape(height, width)
    q = (np.cumsum(dq.astype(np.int64), axis=1) % 65536).astype(np.float32)
    return q / 50.0, b[2 * width * height:].reshape(height, width)
