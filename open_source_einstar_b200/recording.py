"""Raw IR images of a session recording (`.estr`): reading, writing and replay through the batched stereo.

The session file (libs/session/src/session.cpp) is a little-endian stream: u32 magic "ESTR", u32 version 1,
then records of u32 tag, u32 reserved (0), u64 payload size and the payload (session.cpp:499-506,
603-620). Readers skip tags they do not know and stop at a truncated last record. A RAWI record
(session.cpp:248-272) holds the raw images of one trigger: u64 frame index, f64 timestamp (s), u32 image
count, then per image i32 sensor, i32 width, i32 height, u64 byte count and that many bytes of zstd data,
which decompress to the image with each row delta-coded from its left neighbour (mod 256).

`SessionRawReader` indexes the RAWI records. `read_raw` decodes one on the host as
SessionReader::read_raw does (session.cpp:815-836); `read_coded` stops after zstd, and `replay` uploads
the still delta-coded rows and undoes the coding on the GPU (ds_undelta_rows) on the copy stream of an
OfflineRedepth, so the host only runs zstd. zstd is the system libzstd (the reference's own dependency),
called through its public C API.
"""
from __future__ import annotations

import ctypes as C
import ctypes.util
import os
import struct
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import _native as N

MAGIC = 0x52545345  # "ESTR"
VERSION = 1


def tag(s: str) -> int:
    """Record tag of a four-letter name (session.cpp:19-22)."""
    b = s.encode("ascii")
    return b[0] | b[1] << 8 | b[2] << 16 | b[3] << 24


HEAD, RAWI = tag("HEAD"), tag("RAWI")


class _Zstd:
    """libzstd through its public C API (ZSTD_compress / ZSTD_decompress)."""

    def __init__(self):
        path = ctypes.util.find_library("zstd") or "libzstd.so.1"
        L = C.CDLL(path)
        L.ZSTD_compressBound.restype = C.c_size_t
        L.ZSTD_compressBound.argtypes = [C.c_size_t]
        L.ZSTD_compress.restype = C.c_size_t
        L.ZSTD_compress.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_int]
        L.ZSTD_decompress.restype = C.c_size_t
        L.ZSTD_decompress.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t]
        L.ZSTD_isError.restype = C.c_uint
        L.ZSTD_isError.argtypes = [C.c_size_t]
        self.lib = L

    def compress(self, data: np.ndarray, level: int = 1) -> bytes:
        src = np.ascontiguousarray(data).view(np.uint8).reshape(-1)
        cap = self.lib.ZSTD_compressBound(src.size)
        out = np.empty(cap, np.uint8)
        n = self.lib.ZSTD_compress(out.ctypes.data, cap, src.ctypes.data, src.size, level)
        if self.lib.ZSTD_isError(n):
            raise OSError("zstd compression failed")
        return out[:n].tobytes()

    def decompress_into(self, data: bytes, out: np.ndarray) -> None:
        """Decompresses `data` into the contiguous array `out`, which must be exactly filled."""
        src = np.frombuffer(data, np.uint8)
        n = self.lib.ZSTD_decompress(out.ctypes.data, out.nbytes, src.ctypes.data, src.size)
        if self.lib.ZSTD_isError(n) or n != out.nbytes:
            raise OSError("corrupt zstd image")


_zstd: _Zstd | None = None


def zstd() -> _Zstd:
    global _zstd
    if _zstd is None:
        _zstd = _Zstd()
    return _zstd


def delta_code_rows(img: np.ndarray) -> np.ndarray:
    """Each row minus its left neighbour, mod 256; the first byte of a row as is (session.cpp:255-266)."""
    img = np.asarray(img, np.uint8)
    out = img.copy()
    out[:, 1:] = img[:, 1:] - img[:, :-1]  # uint8 arithmetic wraps mod 256
    return out


def undelta_rows_host(coded: np.ndarray) -> np.ndarray:
    """The running sum of each row, mod 256 (session.cpp:829-833)."""
    return (np.cumsum(np.asarray(coded, np.uint8), axis=1, dtype=np.uint32) & 0xFF).astype(np.uint8)


def undelta_rows(coded, image, stream=None) -> None:
    """ds_undelta_rows on device tensors (torch, uint8, 2-D, rows contiguous); in place when coded is image."""
    h, w = coded.shape
    s = None if stream is None else (stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
    rc = N.lib().ds_undelta_rows(coded.data_ptr(), coded.stride(0), image.data_ptr(), image.stride(0), w, h, s)
    if rc != 0:
        raise RuntimeError(N.lib().ds_last_global_error().decode())


@dataclass
class RawFrame:
    """session::RawFrame (libs/session/include/einstar/session/session.hpp:102-106)."""
    index: int
    timestamp_s: float
    images: list = field(default_factory=list)  # (sensor, uint8 H x W)


@dataclass
class _RawBlock:
    index: int
    timestamp_s: float
    offset: int  # of the RAWI payload in the file
    size: int


class SessionRawReader:
    """The RAWI records of a session file, indexed on open and decoded on demand."""

    def __init__(self, path: str):
        self.path = path
        self.raws: list[_RawBlock] = []
        self.head: bytes | None = None
        size = os.path.getsize(path)
        with open(path, "rb") as f:
            magic, version = struct.unpack("<II", f.read(8) or b"\0" * 8)
            if magic != MAGIC:
                raise ValueError(f"{path} is not an einstar session")
            if version != VERSION:
                raise ValueError(f"session version {version} is not supported")
            pos = 8
            while True:
                hdr = f.read(16)
                if len(hdr) < 16:
                    break
                t, _reserved, n = struct.unpack("<IIQ", hdr)
                payload = pos + 16
                if payload + n > size:
                    break  # truncated last record
                if t == RAWI:
                    index, ts = struct.unpack("<Qd", f.read(16))
                    self.raws.append(_RawBlock(index, ts, payload, n))
                elif t == HEAD and self.head is None:
                    self.head = f.read(n)
                f.seek(payload + n)
                pos = payload + n

    def __len__(self) -> int:
        return len(self.raws)

    def _payload(self, i: int) -> bytes:
        b = self.raws[i]
        with open(self.path, "rb") as f:
            f.seek(b.offset)
            data = f.read(b.size)
        if len(data) != b.size:
            raise OSError(f"raw frame {i}: truncated")
        return data

    def read_coded(self, i: int) -> RawFrame:
        """Frame i with each image zstd-decompressed but still delta-coded along its rows."""
        data = self._payload(i)
        index, ts, n = struct.unpack_from("<QdI", data, 0)
        p = 20
        f = RawFrame(index, ts)
        for _ in range(n):
            sensor, w, h, nb = struct.unpack_from("<iiiQ", data, p)
            p += 20
            if w <= 0 or h <= 0 or p + nb > len(data):
                raise OSError(f"raw frame {i}: corrupt record")
            img = np.empty((h, w), np.uint8)
            zstd().decompress_into(data[p:p + nb], img)
            p += nb
            f.images.append((sensor, img))
        return f

    def read_raw(self, i: int) -> RawFrame:
        """SessionReader::read_raw: frame i decoded on the host."""
        f = self.read_coded(i)
        f.images = [(s, undelta_rows_host(img)) for s, img in f.images]
        return f


class SessionRawWriter:
    """Writes a session file with a HEAD record and RAWI records (SessionWriter's layout for these two)."""

    def __init__(self, path: str, depth_size=(640, 512), intrinsics=(0.0, 0.0, 0.0, 0.0), rect=(0.0, 0.0, 0.0, 0.0),
                 description: str = "", rect_cx_offset: float = 0.0):
        self.f = open(path, "wb")
        self.f.write(struct.pack("<II", MAGIC, VERSION))
        d = description.encode()
        head = struct.pack("<ii4d4dI", depth_size[0], depth_size[1], *intrinsics, *rect, len(d)) + d + struct.pack("<d", rect_cx_offset)
        self.record(HEAD, head)

    def record(self, t: int, payload: bytes) -> None:
        self.f.write(struct.pack("<IIQ", t, 0, len(payload)))
        self.f.write(payload)

    def write_raw(self, index: int, timestamp_s: float, images) -> None:
        """images: (sensor, uint8 H x W) pairs, stored row delta-coded and zstd-compressed (level 1)."""
        parts = [struct.pack("<QdI", index, timestamp_s, len(images))]
        for sensor, img in images:
            img = np.ascontiguousarray(img, np.uint8)
            z = zstd().compress(delta_code_rows(img), 1)
            parts.append(struct.pack("<iiiQ", sensor, img.shape[1], img.shape[0], len(z)))
            parts.append(z)
        self.record(RAWI, b"".join(parts))

    def close(self) -> None:
        self.f.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def replay(reader: SessionRawReader, redepth, out_u16: np.ndarray, out_depth: np.ndarray | None = None, left_sensor: int = 0,
           threads: int = 8, chunk_batches: int = 4):
    """Re-depths every RAWI frame of `reader` through `redepth` (an OfflineRedepth) into out_u16[i] /
    out_depth[i]: zstd on `threads` host threads, the row-delta decode on the GPU as part of each batch's
    upload. Frame i's images are the sensor `left_sensor` and the other one. Frames go through in chunks of
    `chunk_batches` batches, so host memory stays bounded for long recordings. Returns the OfflineStats
    summed over the chunks."""
    from .offline import OfflineStats
    from .serving import pinned_empty
    n = len(reader)
    h, w = redepth.raw_h, redepth.raw_w
    chunk = max(1, chunk_batches) * redepth.n
    lefts, rights = pinned_empty((min(chunk, n), h, w), np.uint8), pinned_empty((min(chunk, n), h, w), np.uint8)

    def load(i, slot):
        f = reader.read_coded(i)
        imgs = dict(f.images)
        if left_sensor not in imgs or len(imgs) != 2:
            raise ValueError(f"raw frame {i}: expected two images including sensor {left_sensor}")
        right_sensor = next(s for s in imgs if s != left_sensor)
        if imgs[left_sensor].shape != (h, w) or imgs[right_sensor].shape != (h, w):
            raise ValueError(f"raw frame {i}: images are not {w}x{h}")
        lefts[slot], rights[slot] = imgs[left_sensor], imgs[right_sensor]

    total = OfflineStats(0, 0, 0.0, 0)
    with ThreadPoolExecutor(max_workers=threads) as pool:
        for start in range(0, n, chunk):
            m = min(chunk, n - start)
            list(pool.map(lambda k: load(start + k, k), range(m)))
            st = redepth.run(lefts[:m], rights[:m], out_u16[start:start + m],
                             None if out_depth is None else out_depth[start:start + m], delta_coded=True)
            total = OfflineStats(total.frames + st.frames, total.batches + st.batches, total.device_ms + st.device_ms, st.device_bytes)
    return total
