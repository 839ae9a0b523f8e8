"""Host-side mirror of the reference's stereo-matcher interface, over the C ABI (include/depth_cuda.h).

Names, argument meaning and error behaviour follow:
  depth::SgmParams / StereoParams / StereoResult   libs/depth/include/einstar/depth/stereo.hpp:26-93
  depth::RectifiedGeometry                         libs/depth/include/einstar/depth/point_image.hpp:12-26
  calib::RemapTable                                libs/calib/include/einstar/calib/rectify.hpp:40-44
  depth_metal::MetalStereo, StereoTimings          libs/depth_metal/include/einstar/depth_metal/metal_stereo.hpp:61-107
  einstar::Errc / Result                           libs/core/include/einstar/core/error.hpp:8-33
A Result error becomes a StereoError carrying the Errc and the message.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field

import numpy as np

from . import _native as N

INVALID_DISPARITY = np.float32(-1.0e9)  # depth::kInvalidDisparity


def valid_disparity(d):
    """depth::valid_disparity (stereo.hpp:24)."""
    return d > -1.0e8


class Errc(enum.IntEnum):
    ok = 0
    not_found = 1
    io = 2
    timeout = 3
    protocol = 4
    invalid_argument = 5
    blocked = 6
    unsupported = 7
    busy = 8
    disconnected = 9


class StereoError(RuntimeError):
    def __init__(self, code: int, message: str):
        self.code = Errc(code)
        self.message = message
        super().__init__(f"{self.code.name}: {message}")


@dataclass
class SgmParams:
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


@dataclass
class RefineParams:
    """depth::RefineParams (libs/depth/include/einstar/depth/stereo.hpp:41-47)."""
    search_radius: int = 2
    zncc_radius: int = 3
    min_zncc: float = 0.5
    reject_edge_winners: bool = True


@dataclass
class DetailParams:
    """depth::DetailParams (stereo.hpp:53-61) without `enabled` (StereoParams.detail_enabled)."""
    radius: int = 5
    search: float = 1.0
    step: float = 0.5
    min_zncc: float = 0.5


@dataclass
class StereoParams:
    """depth::StereoParams. The defaults are the hot path (pyramid 0, later stages off, subpixel, median).
    pyramid_levels > 0, detail_enabled, the filters or speckle_max_region_size > 1 select the full
    depth::compute_disparity (ZNCC refinement, detail, filters, speckles) instead; see ds_stereo_params."""
    pyramid_levels: int = 0
    sgm: SgmParams = field(default_factory=SgmParams)
    subpixel: bool = True
    median: bool = True
    detail_enabled: bool = False
    filter_occlusion: bool = False
    filter_spikes: bool = False
    speckle_max_region_size: int = 0
    wide_costs: bool = False
    refine: RefineParams = field(default_factory=RefineParams)
    detail: DetailParams = field(default_factory=DetailParams)
    occlusion_tolerance: float = 1.0
    spike_threshold: float = 1.0
    speckle_max_diff: float = 1.0

    @property
    def refines(self) -> bool:
        return bool(self.pyramid_levels > 0 or self.detail_enabled or self.filter_occlusion or self.filter_spikes
                    or self.speckle_max_region_size > 1)

    def c(self) -> N.StereoParamsC:
        s = self.sgm
        return N.StereoParamsC(
            self.pyramid_levels,
            N.SgmParamsC(s.min_disparity, s.num_disparities, s.census_radius_x, s.census_radius_y, s.p1, s.p2,
                         int(bool(s.adaptive_p2)), int(bool(s.eight_paths)), int(bool(s.slant_steps)),
                         float(s.uniqueness), s.lr_max_diff),
            int(bool(self.subpixel)), int(bool(self.median)), int(bool(self.detail_enabled)),
            int(bool(self.filter_occlusion)), int(bool(self.filter_spikes)), int(self.speckle_max_region_size),
            int(bool(self.wide_costs)), int(self.refine.search_radius), int(self.refine.zncc_radius),
            float(self.refine.min_zncc), int(bool(self.refine.reject_edge_winners)), int(self.detail.radius),
            float(self.detail.search), float(self.detail.step), float(self.detail.min_zncc),
            float(self.occlusion_tolerance), float(self.spike_threshold), float(self.speckle_max_diff))


@dataclass
class RectifiedGeometry:
    f: float = 0.0
    cx: float = 0.0
    cy: float = 0.0
    baseline: float = 0.0
    cx_offset: float = 0.0

    def depth_from_disparity(self, d):
        return self.f * self.baseline / (d + self.cx_offset)

    def disparity_from_depth(self, z):
        return self.f * self.baseline / z - self.cx_offset


@dataclass
class RemapTable:
    """calib::RemapTable: for each rectified pixel the source pixel in the raw image (float32)."""
    map_x: np.ndarray
    map_y: np.ndarray

    @property
    def width(self) -> int:
        return int(self.map_x.shape[1])

    @property
    def height(self) -> int:
        return int(self.map_x.shape[0])


@dataclass
class StereoTimings:
    gpu_ms: float = 0.0
    speckle_ms: float = 0.0
    total_ms: float = 0.0


@dataclass
class StereoResult:
    """depth::StereoResult (disparity, confidence) plus this library's u16 disparity and depth."""
    disparity: np.ndarray
    confidence: np.ndarray
    disparity_u16: np.ndarray | None = None
    depth: np.ndarray | None = None
    rect_left: np.ndarray | None = None
    rect_right: np.ndarray | None = None
    # compute_raw(blobs=True): candidate boxes (x0, y0, x1, y1, pixels, peak) of the left and right raw
    # images, and how many passed before the max_blobs cap (depth_metal::FrameOutputs::blobs / blobs_found)
    blobs: tuple | None = None
    blobs_found: tuple | None = None


@dataclass
class BlobParams:
    """depth_metal::BlobParams (libs/depth_metal/include/einstar/depth_metal/metal_stereo.hpp:21-35)."""
    threshold: int = 150
    min_diameter: int = 3
    max_diameter: int = 60
    max_aspect: float = 4.0
    min_fill: float = 0.5
    border: int = 4
    max_axis_ratio: float = 3.0
    ring_scale: float = 1.4
    ring_contrast: float = 0.5
    ring_max_bright: float = 0.3
    max_blobs: int = 1024

    def c(self) -> N.BlobParamsC:
        return N.BlobParamsC(int(self.threshold), int(self.min_diameter), int(self.max_diameter), float(self.max_aspect),
                             float(self.min_fill), int(self.border), float(self.max_axis_ratio), float(self.ring_scale),
                             float(self.ring_contrast), float(self.ring_max_bright), int(self.max_blobs))


BLOB_FIELDS = ("x0", "y0", "x1", "y1", "pixels", "peak")


def _ptr(a) -> int | None:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a.data_ptr())  # a device tensor (plumbing only: just its address crosses the ABI)


def _check_u8(img: np.ndarray, w: int, h: int, what: str) -> np.ndarray:
    img = np.asarray(img)
    if img.dtype != np.uint8 or img.ndim != 2:
        raise StereoError(Errc.invalid_argument, f"{what}: expected a 2-D uint8 image")
    if img.shape != (h, w):
        raise StereoError(Errc.invalid_argument, f"{what}: image size does not match the configured size")
    if img.strides[1] != 1:
        img = np.ascontiguousarray(img)
    return img


class CudaStereo:
    """Drop-in for depth_metal::MetalStereo on the hot path (create / set_rectification / compute /
    compute_raw / set_point_params / last_timings)."""

    def __init__(self, handle: int, params: StereoParams, width: int, height: int):
        self._h = C.c_void_p(handle)
        self.params = params
        self.width = width
        self.height = height
        self.raw_size: tuple[int, int] | None = None
        self.geometry: RectifiedGeometry | None = None
        self.blob_params: BlobParams | None = None

    # --- life cycle ---------------------------------------------------------------------------------
    @classmethod
    def create(cls, params: StereoParams, width: int, height: int, tuned: bool = True) -> "CudaStereo":
        """MetalStereo::create (metal_stereo.cpp:108-201): validates and allocates device buffers. With
        `tuned`, the autotuner's table entry for this kind of frame on this GPU (if any) sets the kernel
        configuration; results do not depend on it."""
        L = N.lib()
        h = C.c_void_p()
        rc = L.ds_create(C.byref(params.c()), int(width), int(height), C.byref(h))
        if rc != 0:
            raise StereoError(rc, L.ds_last_global_error().decode())
        s = cls(h.value, params, int(width), int(height))
        if tuned:
            from .autotune import apply, tuned_config
            lv = params.pyramid_levels if params.refines else 0  # SGM runs at the pyramid's coarsest level
            cfg = tuned_config(int(width) >> lv, int(height) >> lv, params)
            if cfg:
                apply(s, cfg)
        return s

    def close(self) -> None:
        if self._h:
            N.lib().ds_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise StereoError(rc, N.lib().ds_last_error(self._h).decode())

    # --- configuration ------------------------------------------------------------------------------
    def set_rectification(self, left: RemapTable, right: RemapTable, raw_width: int, raw_height: int) -> None:
        """MetalStereo::set_rectification (metal_stereo.cpp:203-231): tables resident on the device."""
        if (left.width, left.height) != (right.width, right.height):
            raise StereoError(Errc.invalid_argument, "left and right remap tables differ in size")
        arrs = [np.ascontiguousarray(a, np.float32) for a in (left.map_x, left.map_y, right.map_x, right.map_y)]
        self._check(N.lib().ds_set_rectification(self._h, *[a.ctypes.data for a in arrs], left.width, left.height,
                                                 int(raw_width), int(raw_height)))
        self.raw_size = (int(raw_width), int(raw_height))

    def set_point_params(self, geometry: RectifiedGeometry, min_depth_mm: float = 150.0, max_depth_mm: float = 700.0,
                         max_depth_jump_mm: float = 4.0) -> None:
        """MetalStereo::set_point_params (metal_stereo.cpp:243-249)."""
        g = N.GeometryC(geometry.f, geometry.cx, geometry.cy, geometry.baseline, geometry.cx_offset)
        self._check(N.lib().ds_set_point_params(self._h, C.byref(g), float(min_depth_mm), float(max_depth_mm),
                                                float(max_depth_jump_mm)))
        self.geometry = geometry

    # --- per frame ----------------------------------------------------------------------------------
    def _outputs(self, rect: bool):
        n = (self.height, self.width)
        res = StereoResult(np.empty(n, np.float32), np.empty(n, np.float32), np.empty(n, np.uint16),
                           np.empty(n, np.float32) if self.geometry is not None else None,
                           np.empty(n, np.uint8) if rect else None, np.empty(n, np.uint8) if rect else None)
        o = N.OutputsC(_ptr(res.disparity), _ptr(res.confidence), _ptr(res.disparity_u16), _ptr(res.depth),
                       _ptr(res.rect_left), _ptr(res.rect_right))
        return res, o

    @staticmethod
    def _outputs_of(res: StereoResult):
        return N.OutputsC(_ptr(res.disparity), _ptr(res.confidence), _ptr(res.disparity_u16), _ptr(res.depth),
                          _ptr(res.rect_left), _ptr(res.rect_right))

    def compute(self, left: np.ndarray, right: np.ndarray, out: StereoResult | None = None) -> StereoResult:
        """MetalStereo::compute (metal_stereo.cpp:233-241) on an already rectified pair. `out` may hold
        preallocated host arrays (None entries are not produced)."""
        left = _check_u8(left, self.width, self.height, "left")
        right = _check_u8(right, self.width, self.height, "right")
        if left.strides[0] != right.strides[0]:
            left, right = np.ascontiguousarray(left), np.ascontiguousarray(right)
        res, o = (out, self._outputs_of(out)) if out is not None else self._outputs(False)
        self._check(N.lib().ds_compute(self._h, left.ctypes.data, right.ctypes.data, left.strides[0], C.byref(o)))
        return res

    def compute_raw(self, raw_left: np.ndarray, raw_right: np.ndarray, rectified: bool = False,
                    out: StereoResult | None = None, blobs: bool = False) -> StereoResult:
        """MetalStereo::compute_raw (metal_stereo.cpp:340-349): rectify on the device, then stereo. With
        `rectified`, the rectified pair is returned too (the rect_left / rect_right out-parameters).
        `out` may hold preallocated host arrays (None entries are not produced). With `blobs`, the marker
        blob search runs on both raw images concurrently (FrameRequest::marker_blobs; set_blob_params first)
        and res.blobs holds the candidates, (k, 6) uint32 arrays of BLOB_FIELDS."""
        if self.raw_size is None:
            raise StereoError(Errc.invalid_argument, "set_rectification() not called")
        rw, rh = self.raw_size
        raw_left = _check_u8(raw_left, rw, rh, "raw left")
        raw_right = _check_u8(raw_right, rw, rh, "raw right")
        if raw_left.strides[0] != raw_right.strides[0]:
            raw_left, raw_right = np.ascontiguousarray(raw_left), np.ascontiguousarray(raw_right)
        res, o = (out, self._outputs_of(out)) if out is not None else self._outputs(rectified)
        if not blobs:
            self._check(N.lib().ds_compute_raw(self._h, raw_left.ctypes.data, raw_right.ctypes.data, raw_left.strides[0],
                                               C.byref(o)))
            return res
        if self.blob_params is None:
            raise StereoError(Errc.invalid_argument, "set_blob_params() not called")
        cap = self.blob_params.max_blobs
        bl, br = np.zeros((cap, 6), np.uint32), np.zeros((cap, 6), np.uint32)
        bb = N.BlobBoxesC(bl.ctypes.data, br.ctypes.data, cap)
        self._check(N.lib().ds_compute_raw_blobs(self._h, raw_left.ctypes.data, raw_right.ctypes.data, raw_left.strides[0],
                                                 C.byref(o), C.byref(bb)))
        res.blobs = (bl[:bb.kept[0]].copy(), br[:bb.kept[1]].copy())
        res.blobs_found = (int(bb.found[0]), int(bb.found[1]))
        return res

    def compute_frame(self, raw_left: np.ndarray, raw_right: np.ndarray, points=None, normals=None, weights=None,
                      blobs: bool = False, on_blobs=None, rectified: bool = False) -> StereoResult:
        """MetalStereo::compute_frame (metal_stereo.hpp:92-95), the scanner frontend's per-frame call: raw pair
        in; points / normals (H x W x 4 float32) and weights (H x W float32), device tensors of the caller,
        receive the frame and stay on the device; the host result holds disparity, confidence, u16 (and
        depth, the rectified pair) as compute_raw. With `blobs`, res.blobs has the marker candidates, and
        `on_blobs(left, right)` (if given) is called with them while the stereo may still run."""
        if self.raw_size is None:
            raise StereoError(Errc.invalid_argument, "set_rectification() not called")
        rw, rh = self.raw_size
        raw_left = _check_u8(raw_left, rw, rh, "raw left")
        raw_right = _check_u8(raw_right, rw, rh, "raw right")
        if raw_left.strides[0] != raw_right.strides[0]:
            raw_left, raw_right = np.ascontiguousarray(raw_left), np.ascontiguousarray(raw_right)
        res, o = self._outputs(rectified)
        fo = N.FrameOutputsC(_ptr(points), _ptr(normals), _ptr(weights), o, None)
        req = N.FrameRequestC(0, N.BLOB_CALLBACK(), None)
        keep = []
        if blobs:
            if self.blob_params is None:
                raise StereoError(Errc.invalid_argument, "set_blob_params() not called")
            cap = self.blob_params.max_blobs
            bl, br = np.zeros((cap, 6), np.uint32), np.zeros((cap, 6), np.uint32)
            bb = N.BlobBoxesC(bl.ctypes.data, br.ctypes.data, cap)
            fo.blobs = C.pointer(bb)
            req.marker_blobs = 1
            if on_blobs is not None:
                def cb(p, _user):
                    b = p.contents
                    on_blobs(bl[:b.kept[0]].copy(), br[:b.kept[1]].copy())
                req.on_blobs = N.BLOB_CALLBACK(cb)
                keep.append(req.on_blobs)
        self._check(N.lib().ds_compute_frame(self._h, raw_left.ctypes.data, raw_right.ctypes.data, raw_left.strides[0],
                                             C.byref(req), C.byref(fo)))
        if blobs:
            res.blobs = (bl[:bb.kept[0]].copy(), br[:bb.kept[1]].copy())
            res.blobs_found = (int(bb.found[0]), int(bb.found[1]))
        return res

    def compute_frame_raw(self, raw_left: np.ndarray, raw_right: np.ndarray, points, normals, weights,
                          rectified: bool = False):
        """MetalStereo::compute_frame_raw (metal_stereo.hpp:86-90): raw pair in; points / normals (H x W x 4
        float32) and weights (H x W float32), device tensors of the caller, receive the frame and stay on the
        device. With `rectified`, returns the rectified pair (host arrays), else None."""
        if self.raw_size is None:
            raise StereoError(Errc.invalid_argument, "set_rectification() not called")
        rw, rh = self.raw_size
        raw_left = _check_u8(raw_left, rw, rh, "raw left")
        raw_right = _check_u8(raw_right, rw, rh, "raw right")
        if raw_left.strides[0] != raw_right.strides[0]:
            raw_left, raw_right = np.ascontiguousarray(raw_left), np.ascontiguousarray(raw_right)
        rl = np.empty((self.height, self.width), np.uint8) if rectified else None
        rr = np.empty((self.height, self.width), np.uint8) if rectified else None
        self._check(N.lib().ds_compute_frame_raw(self._h, raw_left.ctypes.data, raw_right.ctypes.data, raw_left.strides[0],
                                                 _ptr(points), _ptr(normals), _ptr(weights), _ptr(rl), _ptr(rr)))
        return (rl, rr) if rectified else None

    def set_blob_params(self, params: "BlobParams | None" = None) -> None:
        """MetalStereo::set_blob_params (metal_stereo.cpp:279-291)."""
        params = params or BlobParams()
        self._check(N.lib().ds_set_blob_params(self._h, C.byref(params.c())))
        self.blob_params = params

    def find_blobs(self, image: np.ndarray) -> tuple[np.ndarray, int]:
        """The marker blob search alone on one host image: ((k, 6) uint32 candidates of BLOB_FIELDS ordered
        by first pixel, number that passed before the max_blobs cap)."""
        if self.blob_params is None:
            raise StereoError(Errc.invalid_argument, "set_blob_params() not called")
        img = np.asarray(image)
        if img.dtype != np.uint8 or img.ndim != 2:
            raise StereoError(Errc.invalid_argument, "blob image must be a 2-D uint8 array")
        if img.strides[1] != 1:
            img = np.ascontiguousarray(img)
        cap = self.blob_params.max_blobs
        out = np.zeros((cap, 6), np.uint32)
        found, kept = C.c_uint32(), C.c_uint32()
        self._check(N.lib().ds_find_blobs(self._h, img.ctypes.data, img.shape[1], img.shape[0], img.strides[0], out.ctypes.data,
                                          cap, C.byref(found), C.byref(kept)))
        return out[:kept.value].copy(), int(found.value)

    def compute_device(self, left, right, outputs: dict, stream=None, raw: bool = False) -> None:
        """Device-resident frame: `left`/`right` and every tensor in `outputs` (keys of ds_outputs:
        disparity, confidence, disparity_u16, depth, rect_left, rect_right) are device buffers; enqueued on
        `stream` (a torch.cuda.Stream or raw cudaStream_t; None = the handle's stream), not waited for."""
        o = N.OutputsC(*[_ptr(outputs.get(k)) for k in ("disparity", "confidence", "disparity_u16", "depth",
                                                        "rect_left", "rect_right")])
        s = None if stream is None else (stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
        if stream is not None and not s:
            s = CUDA_STREAM_LEGACY  # torch's default stream is the legacy stream; NULL would mean the handle's
        fn = N.lib().ds_compute_raw_device if raw else N.lib().ds_compute_device
        self._check(fn(self._h, _ptr(left), _ptr(right), C.byref(o), s))

    def last_timings(self) -> StereoTimings:
        t = N.TimingsC()
        self._check(N.lib().ds_last_timings(self._h, C.byref(t)))
        return StereoTimings(t.gpu_ms, t.speckle_ms, t.total_ms)

    # --- introspection ------------------------------------------------------------------------------
    def debug_read(self, census=True, sums=True):
        """Census words (u64) and summed path values (u16 [y][x][d]) of the last frame."""
        h, w, nd = self.height, self.width, self.params.sgm.num_disparities
        cl = np.empty((h, w), np.uint64) if census else None
        cr = np.empty((h, w), np.uint64) if census else None
        s = np.empty((h, w, nd), np.uint16) if sums else None
        self._check(N.lib().ds_debug_read(self._h, _ptr(cl), _ptr(cr), _ptr(s)))
        return cl, cr, s

    @property
    def device_bytes(self) -> int:
        return int(N.lib().ds_device_bytes(self._h))

    def set_kernel_config(self, regs_per_lane: int, lanes_per_line: int, materialize_costs: bool = False,
                          path_warps_per_block: int = 4, wta_threads: int = 256, prefetch_steps: int = 4,
                          fused_pairs: bool = False, horz_warps_per_block: int = 4) -> None:
        """ds_set_kernel_config: lanes per scanline (16/32) x 2*regs disparities per lane; results do not change."""
        c = N.KernelConfigC(regs_per_lane, lanes_per_line, int(bool(materialize_costs)), path_warps_per_block, wta_threads,
                            prefetch_steps, int(bool(fused_pairs)), horz_warps_per_block)
        self._check(N.lib().ds_set_kernel_config(self._h, C.byref(c)))

    def kernel_config(self) -> dict:
        c = N.KernelConfigC()
        self._check(N.lib().ds_get_kernel_config(self._h, C.byref(c)))
        return {k: getattr(c, k) for k, _ in c._fields_}

    def profile(self, on: bool = True) -> None:
        """Per-stage CUDA events for every frame (stages: STAGE_NAMES)."""
        self._check(N.lib().ds_profile_enable(self._h, int(bool(on))))

    def profile_collect(self, max_frames: int = 4096) -> np.ndarray:
        """Waits for the profiled frames since the last call; rows of per-stage milliseconds."""
        buf = np.zeros((max_frames, STAGES), np.float64)
        n = C.c_int()
        self._check(N.lib().ds_profile_collect(self._h, buf.ctypes.data, max_frames, C.byref(n)))
        return buf[:n.value].copy()


CUDA_STREAM_LEGACY = 1  # (cudaStream_t)0x1
STAGES = 6
STAGE_NAMES = ("rectify", "census", "costs", "paths", "wta_lr", "median_out")


def kernel_launches() -> int:
    """Kernels the library has launched since it was loaded."""
    return int(N.lib().ds_kernel_launches())
