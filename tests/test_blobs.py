"""Marker blob search on raw IR images (depth_metal::MetalStereo::set_blob_params / marker_blobs).

CPU: the restated markers::find_blobs (oracle/sgm_oracle.c) against a direct Python flood fill of
detect.cpp:14-45, and the restated candidate gates on synthetic stickers. GPU: the CUDA search through the
C ABI against the oracle, bit for bit (boxes, pixel counts, peaks, order and the number found), alone and
concurrently with the stereo of a raw frame."""
import numpy as np
import pytest


def _flood_fill_blobs(img, thr):
    """libs/markers/src/detect.cpp:14-45 in Python: (x0, y0, x1, y1, pixels, peak, first pixel) in raster
    order of the first pixel."""
    h, w = img.shape
    label = np.full((h, w), -1, np.int64)
    out = []
    for y in range(h):
        for x in range(w):
            if img[y, x] <= thr or label[y, x] >= 0:
                continue
            b = [x, y, x, y, 0, 0, y * w + x]  # the flood fill starts at the blob's first pixel in raster order
            stack = [(x, y)]
            label[y, x] = len(out)
            while stack:
                px, py = stack.pop()
                b[4] += 1
                b[5] = max(b[5], int(img[py, px]))
                b[0], b[2], b[1], b[3] = min(b[0], px), max(b[2], px), min(b[1], py), max(b[3], py)
                for qx, qy in ((px - 1, py), (px + 1, py), (px, py - 1), (px, py + 1)):
                    if 0 <= qx < w and 0 <= qy < h and label[qy, qx] < 0 and img[qy, qx] > thr:
                        label[qy, qx] = len(out)
                        stack.append((qx, qy))
            out.append(b)
    return np.array(out, np.int64).reshape(-1, 7)


def _marker_image(seed, w=320, h=256, dim=0.55, n=12):
    from open_source_einstar_b200 import synth
    rng = np.random.default_rng(seed)
    base = (rng.random((h, w)) < 0.5).astype(np.float32) * 200.0 + 20.0
    base = np.clip(base * dim, 0, 255).astype(np.uint8)
    return synth.add_markers(base, n_markers=n, seed=seed, radius=(3.0, 8.0), n_glints=4, n_dots=20, margin=20)


# Parameter sets: the reference's defaults, a permissive one (almost every blob, including huge ones whose
# moments wrap), a strict one.
PARAM_SETS = [
    {},
    dict(min_diameter=1, max_diameter=16384, max_aspect=1e6, min_fill=0.0, border=0, max_axis_ratio=1e9, ring_max_bright=1.0,
         max_blobs=65536),
    dict(threshold=200, min_diameter=6, max_diameter=30, max_aspect=2.0, min_fill=0.7, ring_scale=1.6, ring_contrast=0.3,
         ring_max_bright=0.1),
]


def test_find_blobs_restatement_matches_flood_fill(port):
    rng = np.random.default_rng(5)
    for t in range(6):
        img = (rng.random((37 + t, 53)) * 255).astype(np.uint8)
        img[rng.random(img.shape) < 0.3] = 250  # larger connected regions
        for thr in (100, 150, 240):
            want = _flood_fill_blobs(img, thr)
            got = port.find_blobs(img, thr)
            assert np.array_equal(got[:, :7], want), (t, thr)


def test_candidates_include_every_sticker(port):
    for seed in range(3):
        img, lay = _marker_image(seed)
        boxes, found = port.blob_candidates(img)
        assert found == len(boxes)
        for cx, cy, a, b, ang in lay.markers:
            hit = [r for r in boxes if r[0] <= cx <= r[2] and r[1] <= cy <= r[3]]
            assert len(hit) == 1, (seed, cx, cy)
        # every candidate is a blob of the flood fill
        blobs = {tuple(int(v) for v in r[:6]) for r in _flood_fill_blobs(img, 150)}
        assert all(tuple(int(v) for v in r) in blobs for r in boxes)


def _sorted_rows(boxes):
    return np.array(sorted(map(tuple, np.asarray(boxes).tolist())), np.uint32).reshape(-1, 6)


def _rule_images():
    imgs = [_marker_image(seed)[0] for seed in range(6)]
    imgs += [_marker_image(9, dim=1.0)[0], _marker_image(11, dim=0.8, n=30)[0]]  # many blobs; many stickers
    return imgs


@pytest.mark.parametrize("params", PARAM_SETS)
def test_candidate_rule_equals_the_reference_kernels_rule(port, params):
    """The library's candidate rule (ellipse orientation by half-angle formulas with IEEE square roots, a
    constant table of the 16 ring directions) selects the same blobs as the reference GPU kernel's own rule
    (blob_select, stereo_kernels.metal.inc:847-901: atan2 / cos / sin), restated in oracle.metal_blob_candidates.
    The library's rule is the C restatement here, which the GPU test below holds the CUDA output to."""
    from open_source_einstar_b200 import BlobParams
    bp = BlobParams(**params)
    from oracle.oracle import metal_blob_candidates
    compared = 0
    for img in _rule_images():
        ours, n = port.blob_candidates(img, bp, cap=1 << 16)
        theirs = metal_blob_candidates(port, img, params)
        assert np.array_equal(_sorted_rows(ours), theirs)
        compared += len(theirs)
    assert compared > 20


@pytest.mark.gpu
def test_cuda_candidates_equal_the_reference_kernels_rule(cuda, port):
    """The CUDA candidates against the reference kernel's atan2 / cos / sin rule directly."""
    from open_source_einstar_b200 import BlobParams, CudaStereo, SgmParams, StereoParams
    from oracle.oracle import metal_blob_candidates
    with CudaStereo.create(StereoParams(sgm=SgmParams(num_disparities=32)), 64, 48) as s:
        for params in PARAM_SETS:
            bp = BlobParams(**{**params, "max_blobs": 65536})
            s.set_blob_params(bp)
            for img in _rule_images():
                got, found = s.find_blobs(img)
                assert np.array_equal(_sorted_rows(got), metal_blob_candidates(port, img, params))


@pytest.mark.gpu
@pytest.mark.parametrize("params", PARAM_SETS)
def test_find_blobs_bit_exact(cuda, port, params):
    from open_source_einstar_b200 import BlobParams, CudaStereo, SgmParams, StereoParams
    bp = BlobParams(**params)
    with CudaStereo.create(StereoParams(sgm=SgmParams(num_disparities=32)), 64, 48) as s:
        s.set_blob_params(bp)
        imgs = [_marker_image(seed)[0] for seed in range(3)]
        imgs.append(_marker_image(9, dim=1.0)[0])                    # bright speckle: many blobs
        big = np.full((300, 400), 255, np.uint8)                     # one huge component with holes
        big[::7, ::11] = 0
        imgs.append(big)
        # near the percolation threshold: long, branching components across many 32 x 16 tiles and corners
        rng = np.random.default_rng(11)
        imgs.append(np.where(rng.random((203, 333)) < 0.58, 255, 0).astype(np.uint8))
        corners = np.zeros((97, 161), np.uint8)                      # 2 x 2 squares on every tile corner
        for y in range(15, 96, 16):
            for x in range(31, 160, 32):
                corners[y:y + 2, x:x + 2] = 200
        imgs.append(corners)
        for hh, ww in ((5, 7), (17, 33), (16, 32), (31, 65)):        # smaller than a tile; one border row / column
            imgs.append(np.where(rng.random((hh, ww)) < 0.6, 230, 10).astype(np.uint8))
        for k, img in enumerate(imgs):
            got, found = s.find_blobs(img)
            want, n = port.blob_candidates(img, bp)
            assert found == n and n <= bp.max_blobs, (k, found, n)  # (beyond max_blobs, which are kept is unspecified)
            assert np.array_equal(got, want), k
            # a view with a row stride gives the same
            pad = np.zeros((img.shape[0], img.shape[1] + 13), np.uint8)
            pad[:, :img.shape[1]] = img
            got2, _ = s.find_blobs(pad[:, :img.shape[1]])
            assert np.array_equal(got2, want)


@pytest.mark.gpu
def test_blob_capacity_and_errors(cuda, port):
    from open_source_einstar_b200 import BlobParams, CudaStereo, Errc, SgmParams, StereoError, StereoParams
    img = _marker_image(3, dim=1.0)[0]
    with CudaStereo.create(StereoParams(sgm=SgmParams(num_disparities=32)), 64, 48) as s:
        with pytest.raises(StereoError) as e:
            s.find_blobs(img)
        assert e.value.code == Errc.invalid_argument
        with pytest.raises(StereoError) as e:
            s.set_blob_params(BlobParams(max_blobs=0))
        assert e.value.code == Errc.invalid_argument
        with pytest.raises(StereoError) as e:
            s.set_blob_params(BlobParams(min_diameter=9, max_diameter=4))
        assert e.value.code == Errc.invalid_argument
        s.set_blob_params(BlobParams(max_blobs=5))
        got, found = s.find_blobs(img)
        want, n = port.blob_candidates(img, BlobParams(max_blobs=5), cap=1 << 16)
        assert found == n and n > 5 and len(got) == 5
        wanted = {tuple(int(v) for v in r) for r in want}
        assert all(tuple(int(v) for v in r) in wanted for r in got)


@pytest.mark.gpu
def test_compute_raw_blobs_with_stereo(cuda, port):
    """compute_raw with marker_blobs: both raw images searched concurrently with the stereo; the stereo
    outputs equal those of a plain compute_raw."""
    from open_source_einstar_b200 import BlobParams, CudaStereo, RemapTable, SgmParams, StereoParams, synth
    pr = synth.raw_objects_pair(seed=4, width=640, height=512, f=560.0, num_disparities=64, n_objects=8, device="cuda")
    left, _ = synth.add_markers((pr.left * 0.6).astype(np.uint8), n_markers=15, seed=1)
    right, _ = synth.add_markers((pr.right * 0.6).astype(np.uint8), n_markers=15, seed=2)
    (lx, ly), (rx, ry) = pr.maps
    sp = StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity // 2, num_disparities=64))
    with CudaStereo.create(sp, 320, 256) as s:
        s.set_rectification(RemapTable(lx, ly), RemapTable(rx, ry), 640, 512)
        plain = s.compute_raw(left, right)
        s.set_blob_params(BlobParams())
        for _ in range(2):
            r = s.compute_raw(left, right, blobs=True)
            assert np.array_equal(r.disparity.view(np.uint32), plain.disparity.view(np.uint32))
            for side, img in enumerate((left, right)):
                want, n = port.blob_candidates(img)
                assert r.blobs_found[side] == n
                assert np.array_equal(r.blobs[side], want)
            assert len(r.blobs[0]) >= 15
