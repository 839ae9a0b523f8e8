"""Batched stereo: many pairs of uneven size and disparity range per launch (include/depth_cuda.h,
ds_batch_*). Each stage is one persistent launch per kernel variant over the blocks of all pairs; the
batch is captured once as a CUDA graph and replayed. Results equal per-pair CudaStereo runs bit for bit.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .stereo import (CUDA_STREAM_LEGACY, Errc, RectifiedGeometry, RemapTable, StereoError, StereoParams, _ptr)


@dataclass
class PairDesc:
    """One pair of a batch: stereo size, SGM parameters, raw input (rectified with calibration `calib`) or
    rectified input, optional depth geometry, optional kernel configuration (from the autotuner)."""
    width: int
    height: int
    params: StereoParams = field(default_factory=StereoParams)
    raw: bool = False
    calib: int = 0
    geometry: RectifiedGeometry | None = None
    min_depth: float = 150.0
    max_depth: float = 700.0
    kernel: dict | None = None  # keys of ds_kernel_config

    def c(self) -> N.PairDescC:
        g = self.geometry or RectifiedGeometry()
        k = N.KernelConfigC()
        if self.kernel:
            d = {"path_warps_per_block": 4, "wta_threads": 256, "prefetch_steps": 4, "materialize_costs": 0,
                 "fused_pairs": 0, "horz_warps_per_block": 1, **self.kernel}
            for name, _ in k._fields_:
                setattr(k, name, int(d.get(name, 0)))
        return N.PairDescC(self.width, self.height, self.params.c(), int(self.raw), int(self.calib),
                           int(self.geometry is not None), N.GeometryC(g.f, g.cx, g.cy, g.baseline, g.cx_offset),
                           float(self.min_depth), float(self.max_depth), k)


BATCH_STAGES = 6
BATCH_STAGE_NAMES = ("rectify", "census", "costs", "paths", "wta_lr", "median_out")


def _stream_handle(stream):
    if stream is None:
        return None
    s = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
    return s if s else CUDA_STREAM_LEGACY


class StereoBatch:
    def __init__(self, pairs: list[PairDesc], n_calib: int = 0, micro_batch: int = 0, branches: int = 0,
                 tuned: bool = True):
        """micro_batch / branches: see ds_batch_options (0 = the library's defaults). With `tuned`, pairs
        without a kernel configuration take the autotuner's batched-path entry for their kind of frame."""
        L = N.lib()
        if tuned:
            from dataclasses import replace

            from .autotune import tuned_config
            pairs = [p if p.kernel else replace(p, kernel=tuned_config(p.width, p.height, p.params, batch=True))
                     for p in pairs]
        arr = (N.PairDescC * len(pairs))(*[p.c() for p in pairs])
        h = C.c_void_p()
        opt = N.BatchOptionsC(int(micro_batch), int(branches))
        rc = L.ds_batch_create(arr, len(pairs), int(n_calib), C.byref(opt), C.byref(h))
        if rc != 0:
            raise StereoError(rc, L.ds_last_global_error().decode())
        self._b = h
        self.pairs = list(pairs)
        self._bound: dict = {}

    def _check(self, rc):
        if rc != 0:
            raise StereoError(rc, N.lib().ds_batch_last_error(self._b).decode())

    def close(self):
        if self._b:
            N.lib().ds_batch_destroy(self._b)
            self._b = C.c_void_p()
        self._bound = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_rectification(self, calib: int, left: RemapTable, right: RemapTable, raw_width: int, raw_height: int):
        arrs = [np.ascontiguousarray(a, np.float32) for a in (left.map_x, left.map_y, right.map_x, right.map_y)]
        self._check(N.lib().ds_batch_set_rectification(self._b, int(calib), *[a.ctypes.data for a in arrs], left.width,
                                                       left.height, int(raw_width), int(raw_height)))

    def bind(self, i: int, left, right, outputs: dict | None = None):
        """Device buffers of pair i (inputs tightly packed; outputs keyed like ds_outputs). The batch keeps a
        reference to every bound tensor until it is re-bound or the batch closes: the graph holds their device
        addresses, and a tensor freed by its caller would hand its memory to the next allocation."""
        outputs = outputs or {}
        o = N.OutputsC(*[_ptr(outputs.get(k)) for k in ("disparity", "confidence", "disparity_u16", "depth",
                                                        "rect_left", "rect_right")])
        self._check(N.lib().ds_batch_bind(self._b, int(i), _ptr(left), _ptr(right), C.byref(o)))
        self._bound[int(i)] = (left, right, dict(outputs))

    def run(self, stream=None, graph: bool = True):
        fn = N.lib().ds_batch_run if graph else N.lib().ds_batch_run_eager
        self._check(fn(self._b, _stream_handle(stream)))

    def profile(self, on: bool = True):
        """Stage events inside the captured graph (re-captures on the next run)."""
        self._check(N.lib().ds_batch_profile(self._b, int(bool(on))))

    def stage_ms(self) -> np.ndarray:
        """Per-stage milliseconds of the last run: rectify, census, costs, paths, wta_lr, median_out."""
        out = np.zeros(BATCH_STAGES, np.float64)
        self._check(N.lib().ds_batch_stage_ms(self._b, out.ctypes.data))
        return out

    @property
    def device_bytes(self) -> int:
        return int(N.lib().ds_batch_device_bytes(self._b))

    @property
    def launches_per_run(self) -> int:
        return int(N.lib().ds_batch_launches_per_run(self._b))

    def _options(self) -> N.BatchOptionsC:
        o = N.BatchOptionsC()
        self._check(N.lib().ds_batch_get_options(self._b, C.byref(o)))
        return o

    @property
    def micro_batch(self) -> int:
        """Pairs per micro-batch (all stages of a micro-batch run back to back)."""
        return int(self._options().micro_batch)

    @property
    def branches(self) -> int:
        """Parallel graph branches the micro-batches are spread over."""
        return int(self._options().branches)
