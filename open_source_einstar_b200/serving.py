"""Request server: continuous batching of stereo frames as they arrive (ds_server_* in include/depth_cuda.h).

The reference runs one camera pair at a time, synchronously, from its frontend
(libs/pipeline/src/stereo_frontend.cpp:302-330). StereoServer instead serves many frame streams at once.
Frames of mixed sizes and disparity ranges are queued, and a native worker thread admits each one as
soon as a GPU slot is free and its cost volume fits the memory budget. Admitted frames run
concurrently, and the remap tables and geometry of every calibration stay on the device. This module
is a thin host mirror: scheduling, admission and timing all happen in the library.

`poisson_arrivals` and `latency_summary` are the host-side pieces of the serving benchmark
(Poisson arrivals at a given frame rate; p50/p99/p99.9 latency beside frames/s).
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .stereo import Errc, RectifiedGeometry, RemapTable, StereoError, StereoParams

OUTPUT_DTYPES = {"disparity": np.float32, "confidence": np.float32, "disparity_u16": np.uint16, "depth": np.float32}


@dataclass
class Completion:
    ticket: int
    tag: int
    status: int
    queue_ms: float
    gpu_ms: float
    latency_ms: float

    @property
    def ok(self) -> bool:
        return self.status == 0


def pinned_empty(shape, dtype) -> np.ndarray:
    """A numpy array in page-locked host memory (allocated through torch, which keeps it alive), so that
    the server's copies run asynchronously and overlap other frames' work. Pageable arrays work too,
    but their device-to-host copies hold the worker until the frame has finished."""
    import torch
    t = torch.empty(tuple(shape), dtype=getattr(torch, np.dtype(dtype).name), pin_memory=True)
    return t.numpy()


def pinned_copy(a: np.ndarray) -> np.ndarray:
    out = pinned_empty(a.shape, a.dtype)
    out[...] = a
    return out


def _host_ptr(a) -> int:
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if getattr(a, "is_cuda", False):
        raise StereoError(Errc.invalid_argument, "the server takes host buffers (pinned for overlap)")
    return int(a.data_ptr())


def _rows(a) -> tuple[int, int, int]:
    """(height, width, row stride in bytes) of a 2-D u8 host image with unit column stride."""
    if isinstance(a, np.ndarray):
        if a.ndim != 2 or a.dtype != np.uint8 or a.strides[1] != 1:
            raise StereoError(Errc.invalid_argument, "expected a 2-D uint8 image with contiguous rows")
        return a.shape[0], a.shape[1], a.strides[0]
    if a.dim() != 2 or a.element_size() != 1 or a.stride(1) != 1:
        raise StereoError(Errc.invalid_argument, "expected a 2-D uint8 image with contiguous rows")
    return a.shape[0], a.shape[1], a.stride(0)


class StereoServer:
    """Continuous-batching stereo server over libdepth_cuda's ds_server_* entry points."""

    def __init__(self, volume_budget_bytes: int = 40 << 30, max_slots: int = 8, max_pending: int = 4096):
        opt = N.ServerOptionsC(int(volume_budget_bytes), int(max_slots), int(max_pending))
        h = C.c_void_p()
        rc = N.lib().ds_server_create(C.byref(opt), C.byref(h))
        if rc != 0:
            raise StereoError(rc, N.lib().ds_last_global_error().decode())
        self._s = h
        self._live: dict[int, tuple] = {}  # ticket -> buffers kept alive until the completion is polled

    def close(self) -> None:
        if getattr(self, "_s", None):
            N.lib().ds_server_destroy(self._s)
            self._s = None
            self._live.clear()

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
            raise StereoError(rc, N.lib().ds_server_last_error(self._s).decode())

    def add_calibration(self, calib: int, left: RemapTable, right: RemapTable, raw_width: int, raw_height: int,
                        geometry: RectifiedGeometry | None = None, min_depth_mm: float = 150.0,
                        max_depth_mm: float = 700.0) -> None:
        """A resident calibration: remap tables (stereo size or twice it) and the geometry for depth."""
        arrs = [np.ascontiguousarray(a, np.float32) for a in (left.map_x, left.map_y, right.map_x, right.map_y)]
        g = None
        if geometry is not None:
            g = C.byref(N.GeometryC(geometry.f, geometry.cx, geometry.cy, geometry.baseline, geometry.cx_offset))
        self._check(N.lib().ds_server_add_calibration(self._s, int(calib), *[a.ctypes.data for a in arrs], left.width,
                                                      left.height, int(raw_width), int(raw_height), g,
                                                      float(min_depth_mm), float(max_depth_mm)))

    def reserve(self, width: int, height: int, params: StereoParams, calib: int = -1, count: int = 8) -> None:
        """Allocates the slots' buffers for this kind of frame ahead of serving."""
        p = params.c()
        self._check(N.lib().ds_server_reserve(self._s, int(width), int(height), C.byref(p), int(calib), int(count)))

    def submit(self, left, right, width: int, height: int, params: StereoParams, outputs: dict, calib: int = -1,
               tag: int = 0) -> int:
        """Queues one frame; returns its ticket. `left`/`right` are host images (raw when `calib` >= 0);
        `outputs` maps disparity / confidence / disparity_u16 / depth to host arrays of height x width."""
        hl, wl, stride = _rows(left)
        hr, wr, stride_r = _rows(right)
        if (hl, wl, stride) != (hr, wr, stride_r):
            raise StereoError(Errc.invalid_argument, "left and right images differ in size or row stride")
        o = N.OutputsC()
        for name, arr in outputs.items():
            if name not in OUTPUT_DTYPES:
                raise StereoError(Errc.invalid_argument, f"unknown output {name!r}")
            if tuple(arr.shape) != (height, width):
                raise StereoError(Errc.invalid_argument, f"output {name!r} must be {height}x{width}")
            setattr(o, name, _host_ptr(arr))
        r = N.RequestC(int(calib), int(width), int(height), params.c(), _host_ptr(left), _host_ptr(right), int(stride),
                       o, int(tag))
        t = C.c_uint64()
        self._check(N.lib().ds_server_submit(self._s, C.byref(r), C.byref(t)))
        self._live[t.value] = (left, right, outputs)
        return int(t.value)

    def poll(self, timeout_ms: int = 0, max_completions: int = 256) -> list[Completion]:
        buf = (N.CompletionC * max_completions)()
        n = C.c_int()
        self._check(N.lib().ds_server_poll(self._s, buf, max_completions, C.byref(n), int(timeout_ms)))
        out = []
        for c in buf[:n.value]:
            self._live.pop(c.ticket, None)
            out.append(Completion(c.ticket, c.tag, c.status, c.queue_ms, c.gpu_ms, c.latency_ms))
        return out

    def wait_all(self, tickets, timeout_s: float = 60.0) -> dict[int, Completion]:
        """Polls until every ticket in `tickets` has completed."""
        want = set(tickets)
        got: dict[int, Completion] = {}
        deadline = time.monotonic() + timeout_s
        while want - got.keys():
            if time.monotonic() > deadline:
                raise StereoError(Errc.timeout, f"{len(want - got.keys())} frames did not complete")
            for c in self.poll(timeout_ms=50):
                got[c.ticket] = c
        return got

    def stats(self) -> dict:
        s = N.ServerStatsC()
        self._check(N.lib().ds_server_get_stats(self._s, C.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_}


def poisson_arrivals(rate_hz: float, duration_s: float, seed: int) -> np.ndarray:
    """Arrival times (s, from 0) of a Poisson process of `rate_hz` over `duration_s`."""
    rng = np.random.default_rng(seed)
    n = int(rate_hz * duration_s * 1.5) + 16
    t = np.cumsum(rng.exponential(1.0 / rate_hz, n))
    while t[-1] < duration_s:  # extend in the unlikely case the draw fell short
        t = np.concatenate([t, t[-1] + np.cumsum(rng.exponential(1.0 / rate_hz, n))])
    return t[t < duration_s]


def latency_summary(latencies_ms, wall_s: float) -> dict:
    """p50 / p99 / p99.9 / max latency (ms) and completed frames per second."""
    lat = np.asarray(latencies_ms, np.float64)
    if lat.size == 0:
        return {"frames": 0, "fps": 0.0, "p50_ms": None, "p99_ms": None, "p999_ms": None, "max_ms": None}
    return {"frames": int(lat.size), "fps": float(lat.size / wall_s),
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "p999_ms": float(np.percentile(lat, 99.9)), "max_ms": float(lat.max())}


def replay(server: StereoServer, frames: list[dict], arrivals_s: np.ndarray, poll_ms: int = 0) -> tuple[list, float]:
    """Submits frames[i % len(frames)] at arrivals_s[i] (host clock) and collects every completion.

    Each frame dict holds the submit arguments (left, right, width, height, params, outputs, calib).
    Returns (completions, wall seconds from the first arrival to the last completion)."""
    completions: list[Completion] = []
    t0 = time.perf_counter()
    for i, ta in enumerate(arrivals_s):
        while True:
            now = time.perf_counter() - t0
            if now >= ta:
                break
            completions.extend(server.poll(timeout_ms=0))
            if ta - now > 0.0005:
                time.sleep(min(ta - now - 0.0003, 0.002))
        f = frames[i % len(frames)]
        server.submit(f["left"], f["right"], f["width"], f["height"], f["params"], f["outputs"], f.get("calib", -1),
                      tag=i)
    while len(completions) < len(arrivals_s):
        got = server.poll(timeout_ms=100)
        if not got and time.perf_counter() - t0 > arrivals_s[-1] + 60:
            raise StereoError(Errc.timeout, "frames did not complete")
        completions.extend(got)
    return completions, time.perf_counter() - t0
