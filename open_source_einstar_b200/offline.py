"""Offline re-depth of a raw IR recording in large batches (the recording-replay use of the stereo path).

The reference re-runs depth on recorded raw IR pairs one frame at a time through its frontend. OfflineRedepth
runs them in batches of `batch_size` pairs instead, each batch one StereoBatch graph replay. Two batches
alternate over three streams: while one runs, the raw pairs of the next are copied to the device and
the results of the previous one are copied back, on the GPU's separate copy engines. All frames share
one calibration (resident remap tables) and one parameter set. That is typically 8-path SGM with
16-bit path values at D=256 for offline quality.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .batch import PairDesc, StereoBatch
from .stereo import RectifiedGeometry, RemapTable, StereoParams


@dataclass
class OfflineStats:
    frames: int
    batches: int
    device_ms: float          # first H2D issue to last D2H completion, CUDA events on the compute stream
    device_bytes: int


class OfflineRedepth:
    """Double-buffered batched re-depth: feed host raw pairs, get u16 disparity and depth per frame."""

    def __init__(self, width: int, height: int, params: StereoParams, maps, raw_size: tuple[int, int],
                 geometry: RectifiedGeometry | None = None, batch_size: int = 128, kernel: dict | None = None,
                 depth_range=(150.0, 700.0), micro_batch: int = 0, branches: int = 0):
        import torch
        self.torch = torch
        self.w, self.h, self.n = int(width), int(height), int(batch_size)
        self.raw_w, self.raw_h = (int(v) for v in raw_size)
        (lx, ly), (rx, ry) = maps
        dev = torch.device("cuda")
        self.dev = dev
        self.compute = torch.cuda.Stream(dev)
        self.copy = torch.cuda.Stream(dev)       # host -> device
        self.copy_out = torch.cuda.Stream(dev)   # device -> host
        desc = PairDesc(self.w, self.h, params, raw=True, calib=0, geometry=geometry, kernel=kernel,
                        min_depth=depth_range[0], max_depth=depth_range[1])
        self.batches, self.inputs, self.outputs = [], [], []
        for _ in range(2):
            b = StereoBatch([desc] * self.n, n_calib=1, micro_batch=micro_batch, branches=branches)
            b.set_rectification(0, RemapTable(lx, ly), RemapTable(rx, ry), self.raw_w, self.raw_h)
            ins = [(torch.empty((self.raw_h, self.raw_w), dtype=torch.uint8, device=dev),
                    torch.empty((self.raw_h, self.raw_w), dtype=torch.uint8, device=dev)) for _ in range(self.n)]
            outs = [{"disparity_u16": torch.empty((self.h, self.w), dtype=torch.int16, device=dev),
                     **({"depth": torch.empty((self.h, self.w), dtype=torch.float32, device=dev)} if geometry else {})}
                    for _ in range(self.n)]
            for i, ((l, r), o) in enumerate(zip(ins, outs)):
                b.bind(i, l, r, o)
            self.batches.append(b)
            self.inputs.append(ins)
            self.outputs.append(outs)
        self.h2d_done = [torch.cuda.Event(), torch.cuda.Event()]
        self.run_done = [torch.cuda.Event(), torch.cuda.Event()]
        self.d2h_done = [torch.cuda.Event(), torch.cuda.Event()]

    def close(self):
        for b in self.batches:
            b.close()
        self.batches = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def device_bytes(self) -> int:
        return sum(b.device_bytes for b in self.batches)

    def run(self, left_frames, right_frames, out_u16: np.ndarray, out_depth: np.ndarray | None = None,
            delta_coded: bool = False) -> OfflineStats:
        """Re-depths frames[i] for all i. left_frames/right_frames: sequences of host u8 raw images (pinned
        for overlap). out_u16 (N x H x W, uint16) and out_depth (N x H x W, float32) receive the results;
        pinned host arrays let the copies overlap the next batch. A last partial batch is padded with its
        final frame. With `delta_coded`, the images are a session recording's row-delta-coded bytes
        (recording.py) and are decoded on the GPU after their upload, on the copy stream."""
        torch = self.torch
        N = len(left_frames)
        nb = (N + self.n - 1) // self.n
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        self.compute.wait_stream(torch.cuda.current_stream(self.dev))
        start.record(self.compute)
        self.copy.wait_event(start)

        def upload(k):
            s = k % 2
            with torch.cuda.stream(self.copy):
                self.copy.wait_event(self.run_done[s])  # the batch two back has finished reading these inputs
                for j in range(self.n):
                    i = min(k * self.n + j, N - 1)
                    self.inputs[s][j][0].copy_(torch.from_numpy(np.asarray(left_frames[i])), non_blocking=True)
                    self.inputs[s][j][1].copy_(torch.from_numpy(np.asarray(right_frames[i])), non_blocking=True)
                    if delta_coded:
                        from .recording import undelta_rows
                        for img in self.inputs[s][j]:
                            undelta_rows(img, img, self.copy)
                self.h2d_done[s].record(self.copy)

        def download(k):
            s = k % 2
            with torch.cuda.stream(self.copy_out):
                self.copy_out.wait_event(self.run_done[s])
                for j in range(self.n):
                    i = k * self.n + j
                    if i >= N:
                        break
                    o = self.outputs[s][j]
                    torch.from_numpy(out_u16[i].view(np.int16)).copy_(o["disparity_u16"], non_blocking=True)
                    if out_depth is not None and "depth" in o:
                        torch.from_numpy(out_depth[i]).copy_(o["depth"], non_blocking=True)
                self.d2h_done[s].record(self.copy_out)

        # Three streams: inputs in, graph replays, results out. A buffer set is reused two batches later,
        # after its results have left (d2h_done) and its inputs were consumed (run_done).
        upload(0)
        for k in range(nb):
            s = k % 2
            if k + 1 < nb:
                upload(k + 1)
            self.compute.wait_event(self.h2d_done[s])
            self.compute.wait_event(self.d2h_done[s])
            self.batches[s].run(stream=self.compute)
            self.run_done[s].record(self.compute)
            download(k)
        for s in range(min(nb, 2)):
            self.compute.wait_event(self.d2h_done[s])
        end.record(self.compute)
        end.synchronize()
        return OfflineStats(N, nb, start.elapsed_time(end), self.device_bytes)
