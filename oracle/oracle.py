"""numpy front end of the test oracle (ctypes over oracle/_bin/liboracle.so and oracle/_ref/libref_stereo.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the bench's CPU-baseline leg, as
the checker or the timed CPU arm. The product package never imports it.

Two implementations of the same functions:
  Port(): this repository's C restatement (oracle/sgm_oracle.c), always buildable with gcc.
  Ref():  the reference's own libs/depth/src/stereo.cpp compiled unmodified (oracle/_ref), for
          census, sgm_disparity and median3; remap and depth (whose reference files need Eigen) come
          from the port in both.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_bin", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_stereo.so")

INVALID = np.float32(-1.0e9)
NO_MATCH = np.int32(-(2**31))


class _Sgm(C.Structure):
    _fields_ = [
        ("min_disparity", C.c_int), ("num_disparities", C.c_int),
        ("census_radius_x", C.c_int), ("census_radius_y", C.c_int),
        ("p1", C.c_int), ("p2", C.c_int), ("adaptive_p2", C.c_int),
        ("eight_paths", C.c_int), ("slant_steps", C.c_int),
        ("uniqueness", C.c_float), ("lr_max_diff", C.c_int),
    ]


@dataclass
class OracleSgm:
    """Fields of depth::SgmParams (libs/depth/include/einstar/depth/stereo.hpp:26-40), same defaults."""
    min_disparity: int = 0
    num_disparities: int = 64
    census_radius_x: int = 2
    census_radius_y: int = 2
    p1: int = 8
    p2: int = 96
    adaptive_p2: bool = True
    eight_paths: bool = False
    slant_steps: bool = True
    uniqueness: float = 0.9
    lr_max_diff: int = 1

    def c(self) -> _Sgm:
        return _Sgm(self.min_disparity, self.num_disparities, self.census_radius_x, self.census_radius_y,
                    self.p1, self.p2, int(bool(self.adaptive_p2)), int(bool(self.eight_paths)),
                    int(bool(self.slant_steps)), float(self.uniqueness), self.lr_max_diff)


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _u8(a) -> np.ndarray:
    a = np.ascontiguousarray(a)
    assert a.dtype == np.uint8 and a.ndim == 2
    return a


def build(ref: str | None = None) -> None:
    """Builds the port (and, when the reference tree is present, oracle/_ref) with make."""
    import subprocess
    cmd = ["make", "-s", "-C", HERE, "all"]
    if ref:
        cmd.append(f"REF={ref}")
    subprocess.run(cmd, check=True)


class _BlobParams(C.Structure):
    _fields_ = [("threshold", C.c_uint32), ("min_diameter", C.c_uint32), ("max_diameter", C.c_uint32),
                ("max_aspect", C.c_float), ("min_fill", C.c_float), ("border", C.c_uint32), ("max_axis_ratio", C.c_float),
                ("ring_scale", C.c_float), ("ring_contrast", C.c_float), ("ring_max_bright", C.c_float),
                ("max_blobs", C.c_uint32)]


def blob_params_c(bp=None) -> _BlobParams:
    """orc_blob_params from an object with depth_metal::BlobParams' fields (defaults when None)."""
    d = dict(threshold=150, min_diameter=3, max_diameter=60, max_aspect=4.0, min_fill=0.5, border=4, max_axis_ratio=3.0,
             ring_scale=1.4, ring_contrast=0.5, ring_max_bright=0.3, max_blobs=1024)
    if bp is not None:
        d.update({k: getattr(bp, k) for k in d})
    return _BlobParams(int(d["threshold"]), int(d["min_diameter"]), int(d["max_diameter"]), float(d["max_aspect"]),
                       float(d["min_fill"]), int(d["border"]), float(d["max_axis_ratio"]), float(d["ring_scale"]),
                       float(d["ring_contrast"]), float(d["ring_max_bright"]), int(d["max_blobs"]))


class Port:
    """The C restatement (oracle/sgm_oracle.c)."""

    def __init__(self, path: str = PORT_SO):
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        self.lib = L
        vp, i, f, d = C.c_void_p, C.c_int, C.c_float, C.c_double
        L.orc_census.argtypes = [vp, i, i, i, i, vp]
        L.orc_cost_volume.argtypes = [vp, vp, i, i, C.POINTER(_Sgm), vp]
        L.orc_aggregate.argtypes = [vp, vp, i, i, C.POINTER(_Sgm), vp]
        L.orc_wta.argtypes = [vp, i, i, C.POINTER(_Sgm), i, vp, vp]
        L.orc_lr_check.argtypes = [vp, vp, i, i, i]
        L.orc_sgm_disparity.argtypes = [vp, vp, i, i, C.POINTER(_Sgm), i, vp]
        L.orc_sgm_disparity.restype = i
        L.orc_median3.argtypes = [vp, i, i, vp]
        L.orc_remap.argtypes = [vp, i, i, vp, vp, i, i, vp]
        L.orc_depth.argtypes = [vp, i, i, d, d, d, f, f, vp]
        L.orc_encode_u16.argtypes = [vp, C.c_long, i, vp]
        L.orc_points.argtypes = [vp, vp, i, i, d, d, d, d, d, f, f, f, f, f, vp, vp, vp]
        L.orc_pack_depth.argtypes = [vp, vp, i, i, vp]
        L.orc_find_blobs.argtypes = [vp, i, i, i, vp, i]
        L.orc_find_blobs.restype = i
        L.orc_blob_candidates.argtypes = [vp, i, i, C.POINTER(_BlobParams), vp, i]
        L.orc_blob_candidates.restype = i

    def census(self, img, rx=2, ry=2) -> np.ndarray:
        img = _u8(img)
        h, w = img.shape
        out = np.empty((h, w), np.uint64)
        self.lib.orc_census(_p(img), w, h, rx, ry, _p(out))
        return out

    def cost_volume(self, cl, cr, p: OracleSgm) -> np.ndarray:
        h, w = cl.shape
        out = np.empty((h, w, p.num_disparities), np.uint16)
        self.lib.orc_cost_volume(_p(np.ascontiguousarray(cl)), _p(np.ascontiguousarray(cr)), w, h, C.byref(p.c()), _p(out))
        return out

    def aggregate(self, cost, guide, p: OracleSgm) -> np.ndarray:
        h, w, nd = cost.shape
        out = np.empty_like(cost)
        self.lib.orc_aggregate(_p(np.ascontiguousarray(cost)), _p(_u8(guide)), w, h, C.byref(p.c()), _p(out))
        return out

    def wta(self, sums, p: OracleSgm, subpixel=True):
        h, w, nd = sums.shape
        disp = np.empty((h, w), np.float32)
        rd = np.empty((h, w), np.int32)
        self.lib.orc_wta(_p(np.ascontiguousarray(sums)), w, h, C.byref(p.c()), int(subpixel), _p(disp), _p(rd))
        return disp, rd

    def lr_check(self, disp, rd, lr_max_diff=1) -> np.ndarray:
        d = np.array(disp, np.float32, copy=True)
        h, w = d.shape
        self.lib.orc_lr_check(_p(d), _p(np.ascontiguousarray(rd, np.int32)), w, h, lr_max_diff)
        return d

    def sgm_disparity(self, left, right, p: OracleSgm, subpixel=True) -> np.ndarray:
        left, right = _u8(left), _u8(right)
        h, w = left.shape
        out = np.empty((h, w), np.float32)
        if self.lib.orc_sgm_disparity(_p(left), _p(right), w, h, C.byref(p.c()), int(subpixel), _p(out)) != 0:
            raise MemoryError("oracle allocation failed")
        return out

    def median3(self, disp) -> np.ndarray:
        d = np.ascontiguousarray(disp, np.float32)
        h, w = d.shape
        out = np.empty_like(d)
        self.lib.orc_median3(_p(d), w, h, _p(out))
        return out

    def remap(self, src, map_x, map_y) -> np.ndarray:
        src = _u8(src)
        mx = np.ascontiguousarray(map_x, np.float32)
        my = np.ascontiguousarray(map_y, np.float32)
        h, w = mx.shape
        out = np.empty((h, w), np.uint8)
        self.lib.orc_remap(_p(src), src.shape[1], src.shape[0], _p(mx), _p(my), w, h, _p(out))
        return out

    def depth(self, disp, f, baseline, cx_offset=0.0, min_depth=150.0, max_depth=700.0) -> np.ndarray:
        d = np.ascontiguousarray(disp, np.float32)
        h, w = d.shape
        out = np.empty_like(d)
        self.lib.orc_depth(_p(d), w, h, float(f), float(baseline), float(cx_offset), float(min_depth), float(max_depth), _p(out))
        return out

    def points(self, disp, conf, f, cx, cy, baseline, cx_offset=0.0, min_depth=150.0, max_depth=700.0,
               max_jump=4.0, edge_weight=0.25, weight_reference_depth=0.0):
        """depth::disparity_to_points restated (point_image.cpp:10-54): (points xyzw, normals xyzw, weights)."""
        dd = np.ascontiguousarray(disp, np.float32)
        h, w = dd.shape
        cf = None if conf is None else np.ascontiguousarray(conf, np.float32)
        pts = np.empty((h, w, 4), np.float32)
        nrm = np.empty((h, w, 4), np.float32)
        wts = np.empty((h, w), np.float32)
        self.lib.orc_points(_p(dd), None if cf is None else _p(cf), w, h, float(f), float(cx), float(cy), float(baseline),
                            float(cx_offset), float(min_depth), float(max_depth), float(max_jump), float(edge_weight),
                            float(weight_reference_depth), _p(pts), _p(nrm), _p(wts))
        return pts, nrm, wts

    def find_blobs(self, img, threshold=150) -> np.ndarray:
        """markers::find_blobs restated (detect.cpp:14-45): (n, 12) int32 rows of x0, y0, x1, y1, pixels,
        peak, first pixel, five moment sums, in the CPU detector's order."""
        img = _u8(img)
        h, w = img.shape
        n = self.lib.orc_find_blobs(_p(img), w, h, int(threshold), None, 0)
        out = np.zeros((max(n, 1), 12), np.int32)
        self.lib.orc_find_blobs(_p(img), w, h, int(threshold), _p(out), n)
        return out[:n]

    def blob_candidates(self, img, params=None, cap=None):
        """The GPU blob search's candidates restated: ((k, 6) uint32 boxes, number that passed)."""
        img = _u8(img)
        h, w = img.shape
        bp = blob_params_c(params)
        cap = int(bp.max_blobs if cap is None else cap)
        out = np.zeros((max(cap, 1), 6), np.uint32)
        n = self.lib.orc_blob_candidates(_p(img), w, h, C.byref(bp), _p(out), cap)
        return out[:min(n, cap)], n

    def pack_depth(self, points_xyzw, weights) -> np.ndarray:
        """depth_metal::DepthPacker restated (depth_packer.cpp:10-21): w*h*3 bytes."""
        p = np.ascontiguousarray(points_xyzw, np.float32)
        wt = np.ascontiguousarray(weights, np.float32)
        h, w = wt.shape
        out = np.empty(h * w * 3, np.uint8)
        self.lib.orc_pack_depth(_p(p), _p(wt), w, h, _p(out))
        return out

    def encode_u16(self, disp, min_disparity) -> np.ndarray:
        d = np.ascontiguousarray(disp, np.float32)
        out = np.empty(d.shape, np.uint16)
        self.lib.orc_encode_u16(_p(d), d.size, int(min_disparity), _p(out))
        return out

    def pipeline(self, left, right, p: OracleSgm, *, subpixel=True, median=True, geometry=None,
                 min_depth=150.0, max_depth=700.0, maps=None):
        """The whole hot path: [remap] -> sgm_disparity -> [median3] -> u16 encoding -> depth."""
        return _pipeline(self, left, right, p, subpixel, median, geometry, min_depth, max_depth, maps)


class _RefStereo(C.Structure):
    """ref_stereo_params of oracle/ref_shim.cpp (depth::StereoParams, stereo.hpp:41-88)."""
    _fields_ = [("pyramid_levels", C.c_int), ("sgm", _Sgm), ("refine_search_radius", C.c_int),
                ("refine_zncc_radius", C.c_int), ("refine_min_zncc", C.c_float), ("refine_reject_edge_winners", C.c_int),
                ("detail_enabled", C.c_int), ("detail_radius", C.c_int), ("detail_search", C.c_float),
                ("detail_step", C.c_float), ("detail_min_zncc", C.c_float), ("filter_occlusion", C.c_int),
                ("filter_occlusion_tolerance", C.c_float), ("filter_spikes", C.c_int), ("filter_spike_threshold", C.c_float),
                ("speckle_max_region_size", C.c_int), ("speckle_max_diff", C.c_float), ("subpixel", C.c_int)]


def ref_stereo_params(sp) -> _RefStereo:
    """From the package's StereoParams (field names of depth::StereoParams)."""
    g = sp.sgm
    sgm = OracleSgm(min_disparity=g.min_disparity, num_disparities=g.num_disparities, census_radius_x=g.census_radius_x,
                    census_radius_y=g.census_radius_y, p1=g.p1, p2=g.p2, adaptive_p2=g.adaptive_p2,
                    eight_paths=g.eight_paths, slant_steps=g.slant_steps, uniqueness=g.uniqueness,
                    lr_max_diff=g.lr_max_diff).c()
    return _RefStereo(int(sp.pyramid_levels), sgm, int(sp.refine.search_radius), int(sp.refine.zncc_radius),
                      float(sp.refine.min_zncc), int(bool(sp.refine.reject_edge_winners)), int(bool(sp.detail_enabled)),
                      int(sp.detail.radius), float(sp.detail.search), float(sp.detail.step), float(sp.detail.min_zncc),
                      int(bool(sp.filter_occlusion)), float(sp.occlusion_tolerance), int(bool(sp.filter_spikes)),
                      float(sp.spike_threshold), int(sp.speckle_max_region_size), float(sp.speckle_max_diff),
                      int(bool(sp.subpixel)))


class Ref(Port):
    """The reference's own stereo.cpp (oracle/_ref): census, sgm_disparity, median3, downsample2, the refinement
    stages and compute_disparity."""

    def __init__(self, path: str = REF_SO, port_path: str = PORT_SO):
        super().__init__(port_path)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (needs the reference tree at build time)")
        R = C.CDLL(path)
        self.ref = R
        vp, i = C.c_void_p, C.c_int
        R.ref_census.argtypes = [vp, i, i, i, i, vp]
        R.ref_sgm_disparity.argtypes = [vp, vp, i, i, C.POINTER(_Sgm), i, vp]
        R.ref_median3.argtypes = [vp, i, i, vp]
        R.ref_threads.restype = i
        P = C.POINTER(_RefStereo)
        R.ref_downsample2.argtypes = [vp, i, i, vp]
        R.ref_refine_level.argtypes = [vp, vp, i, i, vp, i, i, P, vp, vp]
        R.ref_refine_detail.argtypes = [vp, vp, i, i, vp, i, i, P]
        R.ref_filter_disparity.argtypes = [vp, i, i, P]
        R.ref_remove_speckles.argtypes = [vp, i, i, P]
        R.ref_compute_disparity.argtypes = [vp, vp, i, i, vp, vp, P, vp, vp]

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_SO)

    def threads(self) -> int:
        return int(self.ref.ref_threads())

    def census(self, img, rx=2, ry=2) -> np.ndarray:
        img = _u8(img)
        h, w = img.shape
        out = np.empty((h, w), np.uint64)
        self.ref.ref_census(_p(img), w, h, rx, ry, _p(out))
        return out

    def sgm_disparity(self, left, right, p: OracleSgm, subpixel=True) -> np.ndarray:
        left, right = _u8(left), _u8(right)
        h, w = left.shape
        out = np.empty((h, w), np.float32)
        self.ref.ref_sgm_disparity(_p(left), _p(right), w, h, C.byref(p.c()), int(subpixel), _p(out))
        return out

    def median3(self, disp) -> np.ndarray:
        d = np.ascontiguousarray(disp, np.float32)
        h, w = d.shape
        out = np.empty_like(d)
        self.ref.ref_median3(_p(d), w, h, _p(out))
        return out

    def downsample2(self, img) -> np.ndarray:
        img = _u8(img)
        h, w = img.shape
        out = np.empty((h // 2, w // 2), np.uint8)
        self.ref.ref_downsample2(_p(img), w, h, _p(out))
        return out

    def filter_disparity(self, disp, sp) -> np.ndarray:
        d = np.array(disp, np.float32, order="C")
        h, w = d.shape
        self.ref.ref_filter_disparity(_p(d), w, h, C.byref(ref_stereo_params(sp)))
        return d

    def remove_speckles(self, disp, sp) -> np.ndarray:
        d = np.array(disp, np.float32, order="C")
        h, w = d.shape
        self.ref.ref_remove_speckles(_p(d), w, h, C.byref(ref_stereo_params(sp)))
        return d

    def compute_disparity(self, left, right, sp, full_left=None, full_right=None):
        """depth::compute_disparity (stereo.cpp:501-536): (disparity, confidence)."""
        left, right = _u8(left), _u8(right)
        h, w = left.shape
        fl = None if full_left is None else _u8(full_left)
        fr = None if full_right is None else _u8(full_right)
        disp = np.empty((h, w), np.float32)
        conf = np.empty((h, w), np.float32)
        self.ref.ref_compute_disparity(_p(left), _p(right), w, h, None if fl is None else _p(fl),
                                       None if fr is None else _p(fr), C.byref(ref_stereo_params(sp)), _p(disp), _p(conf))
        return disp, conf


def _pipeline(o, left, right, p, subpixel, median, geometry, min_depth, max_depth, maps):
    if maps is not None:
        (lx, ly), (rx, ry) = maps
        left, right = o.remap(left, lx, ly), o.remap(right, rx, ry)
    disp = o.sgm_disparity(left, right, p, subpixel)
    if median:
        disp = o.median3(disp)
    out = {"left": left, "right": right, "disparity": disp, "disparity_u16": o.encode_u16(disp, p.min_disparity)}
    if geometry is not None:
        f, baseline, cx_offset = geometry
        out["depth"] = o.depth(disp, f, baseline, cx_offset, min_depth, max_depth)
    return out


def metal_blob_candidates(port: Port, img, params=None) -> np.ndarray:
    """The reference GPU search's candidate rule as its own kernel states it: blob_select in
    libs/depth_metal/src/stereo_kernels.metal.inc:847-901, with the ellipse orientation from
    th = atan2(2 cxy, cxx - cyy) / 2 and cos/sin of th and of the 16 ring angles 2 pi k / 16 (numpy float32,
    one rounding per operation), ring samples at the nearest pixel (round half away from zero, clamped).
    Blobs and their statistics come from the restated markers::find_blobs. Returns the (k, 6) uint32 rows
    (x0, y0, x1, y1, pixels, peak) of the blobs that pass, sorted. Pure Python per blob: small images only."""
    import math
    f32 = np.float32
    img = _u8(img)
    h, w = img.shape
    d = dict(threshold=150, min_diameter=3, max_diameter=60, max_aspect=4.0, min_fill=0.5, border=4, max_axis_ratio=3.0,
             ring_scale=1.4, ring_contrast=0.5, ring_max_bright=0.3)
    if params is not None:
        d.update({k: v for k, v in (params.items() if isinstance(params, dict) else vars(params).items()) if k in d})
    blobs = port.find_blobs(img, int(d["threshold"]))
    pi = f32(math.pi)

    def sample(x, y):  # stereo_kernels.metal.inc:840-843
        def rnd(v):
            v = float(v)
            return math.floor(v + 0.5) if v >= 0 else math.ceil(v - 0.5)
        sx = min(max(rnd(x), 0), w - 1) if math.isfinite(float(x)) else (w - 1 if x > 0 else 0)
        sy = min(max(rnd(y), 0), h - 1) if math.isfinite(float(y)) else (h - 1 if y > 0 else 0)
        return f32(img[sy, sx])

    out = []
    for b in blobs:
        x0, y0, x1, y1, px, pk, first = (int(v) for v in b[:7])
        mo = [f32(np.int32(v)) for v in b[7:12]]
        bw, bh = f32(x1 - x0 + 1), f32(y1 - y0 + 1)
        if bw < f32(d["min_diameter"]) or bh < f32(d["min_diameter"]) or bw > f32(d["max_diameter"]) or bh > f32(d["max_diameter"]):
            continue
        if max(bw, bh) > f32(d["max_aspect"]) * min(bw, bh):
            continue
        if f32(px) < f32(d["min_fill"]) * bw * bh * pi / f32(4.0):
            continue
        m = max(3, int(max(bw, bh)) // 2)
        bd = int(d["border"])
        if x0 - m < bd or y0 - m < bd or x1 + m >= w - bd or y1 + m >= h - bd:
            continue
        n = f32(px)
        mx, my = mo[0] / n, mo[1] / n
        cxx, cxy, cyy = mo[2] / n - mx * mx, mo[3] / n - mx * my, mo[4] / n - my * my
        tr = f32(0.5) * (cxx + cyy)
        det = np.sqrt(max(f32(0.0), f32(0.25) * (cxx - cyy) * (cxx - cyy) + cxy * cxy))
        l1, l2 = tr + det, max(tr - det, f32(0.0625))
        ea = f32(2.0) * np.sqrt(l1) + f32(0.5)
        eb = f32(2.0) * np.sqrt(l2) + f32(0.5)
        if ea / eb > f32(d["max_axis_ratio"]) * f32(1.2):
            continue
        th = f32(0.5) * np.arctan2(f32(2.0) * cxy, cxx - cyy)
        ct, st = np.cos(th), np.sin(th)
        cx, cy = f32(first % w) + mx, f32(first // w) + my

        def ring(scale_u, scale_v, k):
            t = f32(2.0) * pi * f32(k) / f32(16.0)
            u, v = scale_u * np.cos(t), scale_v * np.sin(t)
            return sample(cx + ct * u - st * v, cy + st * u + ct * v)

        bg = sorted(ring(f32(2.2) * ea, f32(2.2) * eb, k) for k in range(16))
        level = bg[3] + f32(d["ring_contrast"]) * (f32(pk) - bg[3])
        ru, rv = f32(d["ring_scale"]) * ea, f32(d["ring_scale"]) * eb
        bright = sum(1 for k in range(16) if ring(ru, rv, k) > level)
        if f32(bright) > f32(d["ring_max_bright"]) * f32(16.0):
            continue
        out.append((x0, y0, x1, y1, px, pk))
    return np.array(sorted(out), np.uint32).reshape(-1, 6)
