"""Raw IR images of a session recording (`.estr` RAWI records, libs/session/src/session.cpp:248-272,
815-836): the row delta coding, the file layout read and written, the row decode on the GPU
(ds_undelta_rows) and a replay of a recording through the batched re-depth."""
import struct

import numpy as np
import pytest

from open_source_einstar_b200 import recording as R


def test_delta_coding_known_answer():
    # session.cpp:255-266: each byte minus its left neighbour, mod 256; the first byte of a row as is
    img = np.array([[10, 12, 5, 5], [0, 255, 1, 0]], np.uint8)
    want = np.array([[10, 2, 249, 0], [0, 255, 2, 255]], np.uint8)
    assert np.array_equal(R.delta_code_rows(img), want)
    assert np.array_equal(R.undelta_rows_host(want), img)
    rng = np.random.default_rng(0)
    x = rng.integers(0, 256, (37, 1281), dtype=np.uint8)
    assert np.array_equal(R.undelta_rows_host(R.delta_code_rows(x)), x)


def test_session_file_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    frames = [[(s, rng.integers(0, 256, (48, 64), dtype=np.uint8)) for s in (1, 0)] for _ in range(3)]
    path = str(tmp_path / "scan.estr")
    with R.SessionRawWriter(path, description="test") as w:
        for i, imgs in enumerate(frames):
            w.write_raw(100 + i, 0.25 * i, imgs)
            w.record(R.tag("FXTR"), b"\x01\x02\x03")  # a record kind this reader skips
        w.f.write(struct.pack("<IIQ", R.RAWI, 0, 1 << 20) + b"\0" * 100)  # truncated last record
    r = R.SessionRawReader(path)
    assert len(r) == 3 and r.head is not None
    for i, imgs in enumerate(frames):
        f = r.read_raw(i)
        assert (f.index, f.timestamp_s) == (100 + i, 0.25 * i)
        assert [s for s, _ in f.images] == [1, 0]
        for (_, got), (_, want) in zip(f.images, imgs):
            assert np.array_equal(got, want)
        coded = r.read_coded(i)
        for (_, got), (_, want) in zip(coded.images, imgs):
            assert np.array_equal(got, R.delta_code_rows(want))


def test_not_a_session(tmp_path):
    p = tmp_path / "x.estr"
    p.write_bytes(b"NOPE" + b"\0" * 12)
    with pytest.raises(ValueError):
        R.SessionRawReader(str(p))


@pytest.mark.gpu
def test_undelta_rows_on_the_gpu(cuda):
    import torch
    rng = np.random.default_rng(2)
    for w in (1, 17, 512, 513, 1280, 2000):
        img = rng.integers(0, 256, (33, w), dtype=np.uint8)
        coded = torch.from_numpy(R.delta_code_rows(img)).to(cuda)
        out = torch.empty((33, w + 7), dtype=torch.uint8, device=cuda)[:, :w]  # a row stride above the width
        R.undelta_rows(coded, out)
        R.undelta_rows(coded, coded)  # in place
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), img), w
        assert np.array_equal(coded.cpu().numpy(), img), w


@pytest.mark.gpu
def test_replay_recording_matches_per_frame_path(cuda, tmp_path):
    from open_source_einstar_b200 import CudaStereo, RectifiedGeometry, RemapTable, SgmParams, StereoParams, synth
    from open_source_einstar_b200.offline import OfflineRedepth
    pairs = [synth.raw_objects_pair(seed=70 + i, width=640, height=512, f=560.0, num_disparities=64, n_objects=6, device="cuda")
             for i in range(5)]
    path = str(tmp_path / "scan.estr")
    with R.SessionRawWriter(path) as w:
        for i, p in enumerate(pairs):
            w.write_raw(i, i / 30.0, [(0, p.left), (1, p.right)])
    reader = R.SessionRawReader(path)
    (lx, ly), (rx, ry) = pairs[0].maps
    sp = StereoParams(sgm=SgmParams(min_disparity=pairs[0].min_disparity, num_disparities=64))
    geom = RectifiedGeometry(pairs[0].f, 0, 0, pairs[0].baseline, 0.0)
    u16 = np.zeros((5, 512, 640), np.uint16)
    depth = np.zeros((5, 512, 640), np.float32)
    with OfflineRedepth(640, 512, sp, pairs[0].maps, (640, 512), geom, batch_size=2) as off:
        st = R.replay(reader, off, u16, depth, left_sensor=0, threads=2, chunk_batches=1)  # chunks of 2 frames
    assert st.frames == 5
    with CudaStereo.create(sp, 640, 512) as s:
        s.set_rectification(RemapTable(lx, ly), RemapTable(rx, ry), 640, 512)
        s.set_point_params(geom, 150.0, 700.0)
        for i, p in enumerate(pairs):
            r = s.compute_raw(p.left, p.right)
            assert np.array_equal(r.disparity_u16, u16[i]), i
            assert np.array_equal(r.depth.view(np.uint32), depth[i].view(np.uint32)), i
