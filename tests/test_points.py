"""Points, normals, weights (depth::disparity_to_points) and the packed depth layout (DepthPacker).

CPU: the oracle's restatement against known answers (a tilted plane's normal, the depth gates, the
packed layout's round trip). GPU: the CUDA kernels against the oracle, bit for bit, on a full 640x512
frame from the stereo path (the stated tolerances are asserted too).
"""
import numpy as np
import pytest

from conftest import same_bits

POINT_ATOL = 1e-4   # mm, stated tolerance for points (compared bit for bit as well)
NORMAL_ATOL = 1e-6  # unit normals


def _plane(port, h=48, w=64, slope=0.5):
    f, B = 900.0, 60.0
    cx, cy = (w - 1) / 2, (h - 1) / 2
    xs = np.arange(w)[None, :].repeat(h, 0)
    z = 300 + slope * xs
    d = (f * B / z).astype(np.float32)
    return d, (f, cx, cy, B)


def test_points_of_a_tilted_plane(port):
    d, (f, cx, cy, B) = _plane(port)
    pts, nrm, wts = port.points(d, np.ones_like(d), f, cx, cy, B)
    h, w = d.shape
    assert np.all(pts[..., 3] == 1.0) and np.allclose(pts[..., 2], f * B / d.astype(np.float64), rtol=1e-6)
    # interior normals: the plane z = 300 + slope * x_pixel, i.e. z changes by slope * z / f per mm of x
    inner = nrm[1:-1, 1:-1, :3]
    assert np.allclose(np.linalg.norm(inner, axis=-1), 1.0, atol=NORMAL_ATOL)
    assert np.all(inner[..., 2] < 0)  # towards the camera
    assert np.all(nrm[0, :, :3] == 0) and np.all(nrm[:, -1, :3] == 0)  # no normal on the border
    assert np.allclose(wts[0, :], 0.25, atol=1e-7)  # border: edge weight x confidence 1
    assert np.all((wts[1:-1, 1:-1] > 0) & (wts[1:-1, 1:-1] <= 1))


def test_points_gates_and_invalid(port):
    d, (f, cx, cy, B) = _plane(port)
    d[5, 5] = -1e9                      # invalid disparity
    d[6, 6] = f * B / 100.0             # 100 mm: nearer than min_depth
    pts, nrm, wts = port.points(d, None, f, cx, cy, B)
    for y, x in ((5, 5), (6, 6)):
        assert np.all(pts[y, x] == 0) and np.all(nrm[y, x] == 0) and wts[y, x] == 0
    assert np.all(nrm[5, 4, :3] == 0)   # a neighbour is missing: no normal, edge weight
    assert wts[5, 4] == np.float32(0.25)


def test_pack_depth_round_trip(port):
    from open_source_einstar_b200.points import unpack_depth
    d, (f, cx, cy, B) = _plane(port)
    d[3, 7] = -1e9
    pts, _, wts = port.points(d, np.ones_like(d), f, cx, cy, B)
    packed = port.pack_depth(pts, wts)
    h, w = d.shape
    assert packed.size == h * w * 3
    z, conf = unpack_depth(packed, w, h)
    want = np.where(pts[..., 2] > 0, np.clip(np.round(pts[..., 2] * 50.0), 1, 65535) / 50.0, 0.0)
    assert np.array_equal(z, want.astype(np.float32)) and z[3, 7] == 0
    assert np.array_equal(conf, np.clip(np.round(wts * 255.0), 0, 255).astype(np.uint8))


@pytest.mark.gpu
def test_points_and_packing_match_the_oracle(cuda, port):
    import torch
    from open_source_einstar_b200 import (CudaStereo, PointImageParams, RectifiedGeometry, SgmParams, StereoParams,
                                          disparity_to_points, pack_depth, synth)
    pr = synth.plane_sphere_pair(seed=5, width=640, height=512, num_disparities=64, device="cuda")
    h, w = pr.left.shape
    with CudaStereo.create(StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity, num_disparities=64)), w, h) as s:
        res = s.compute(pr.left, pr.right)
    geom = RectifiedGeometry(pr.f, (w - 1) / 2, (h - 1) / 2, pr.baseline, 0.0)
    for params in (PointImageParams(), PointImageParams(max_depth_jump=2.0, edge_weight=0.5, weight_reference_depth=300.0)):
        d = torch.from_numpy(res.disparity).cuda()
        c = torch.from_numpy(res.confidence).cuda()
        got = disparity_to_points(d, c, geom, params)
        packed = pack_depth(got["points"], got["weights"])
        torch.cuda.synchronize()
        pts, nrm, wts = port.points(res.disparity, res.confidence, geom.f, geom.cx, geom.cy, geom.baseline, 0.0,
                                    params.min_depth, params.max_depth, params.max_depth_jump, params.edge_weight,
                                    params.weight_reference_depth)
        gp, gn, gw = (got[k].cpu().numpy() for k in ("points", "normals", "weights"))
        assert (pts[..., 3] > 0).mean() > 0.3
        assert np.allclose(gp, pts, atol=POINT_ATOL) and same_bits(gp, pts)
        assert np.allclose(gn, nrm, atol=NORMAL_ATOL) and same_bits(gn, nrm)
        assert same_bits(gw, wts)
        assert np.array_equal(packed.cpu().numpy(), port.pack_depth(pts, wts))
