"""The sweep kernels (two launches per frame: the vertical path pair, then the horizontal pair with the WTA
and the L-R check) against the reference's own stereo.cpp (oracle/_ref) and the oracle restatement, bit for
bit, at the benchmark configurations' sizes and on random parameters; and a batch with one pair of each
configuration-3 size checked directly against the reference.
"""
import numpy as np
import pytest

from conftest import mismatch_report, same_bits
from oracle.oracle import OracleSgm

pytestmark = pytest.mark.gpu

DEPTH_RTOL = 1e-4


def _sweep_stereo(p: OracleSgm, w, h, shape, median=True, subpixel=True):
    from open_source_einstar_b200 import CudaStereo, SgmParams, StereoParams
    s = CudaStereo.create(StereoParams(sgm=SgmParams(**p.__dict__), median=median, subpixel=subpixel), w, h)
    s.set_kernel_config(shape[0], shape[1], False, 4, 256, 4, True)
    assert s.kernel_config()["fused_pairs"] == 1
    return s


def test_sweep_config2_raw_1280x1024_d128(cuda, ref, port):
    """Configuration 2 (raw 1280x1024, D=128) on the sweep kernels: rectified bytes, disparity after L-R and
    median, and depth equal the reference pipeline's."""
    from open_source_einstar_b200 import RectifiedGeometry, RemapTable, synth
    pair = synth.raw_objects_pair(seed=1, device="cuda")
    (lx, ly), (rx, ry) = pair.maps
    p = OracleSgm(min_disparity=pair.min_disparity, num_disparities=128)
    with _sweep_stereo(p, 1280, 1024, (8, 8)) as s:
        s.set_rectification(RemapTable(lx, ly), RemapTable(rx, ry), 1280, 1024)
        s.set_point_params(RectifiedGeometry(pair.f, 0, 0, pair.baseline, 0.0), 150.0, 700.0)
        r = s.compute_raw(pair.left, pair.right, rectified=True)
    rl, rr = port.remap(pair.left, lx, ly), port.remap(pair.right, rx, ry)
    assert np.array_equal(r.rect_left, rl) and np.array_equal(r.rect_right, rr)
    d = ref.median3(ref.sgm_disparity(rl, rr, p))
    assert same_bits(r.disparity, d), mismatch_report(r.disparity, d)
    z = port.depth(d, pair.f, pair.baseline, 0.0, 150.0, 700.0)
    nz = z > 0
    assert np.array_equal(r.depth > 0, nz) and np.all(np.abs(r.depth[nz] - z[nz]) <= DEPTH_RTOL * z[nz])
    assert same_bits(r.depth, z)
    assert (d > -1e8).mean() > 0.5


@pytest.mark.parametrize("shape", [(8, 4), (6, 8), (8, 8)])
def test_sweep_config1_640x512_d64(cuda, port, shape):
    """Configuration 1 (640x512 plane + sphere, D=64) in each sweep shape that holds 64 disparities."""
    from open_source_einstar_b200 import RectifiedGeometry, synth
    pair = synth.plane_sphere_pair(seed=2)
    p = OracleSgm(min_disparity=pair.min_disparity, num_disparities=64)
    want = port.pipeline(pair.left, pair.right, p, median=True, geometry=(pair.f, pair.baseline, 0.0))
    with _sweep_stereo(p, 640, 512, shape) as s:
        s.set_point_params(RectifiedGeometry(pair.f, 319.5, 255.5, pair.baseline, 0.0), 150.0, 700.0)
        r = s.compute(pair.left, pair.right)
    assert same_bits(r.disparity, want["disparity"]), mismatch_report(r.disparity, want["disparity"])
    assert np.array_equal(r.disparity_u16, want["disparity_u16"])
    assert same_bits(r.depth, want["depth"])


@pytest.mark.parametrize("seed", range(6))
def test_sweep_random_parameters_against_the_reference(cuda, ref, seed):
    """Random SGM parameters within the sweep kernels' range (P1, P2 with 2 (25 + P2) <= 255, adaptive P2 or
    not, slant steps or not, negative or positive min disparity, uniqueness, L-R threshold, subpixel) and
    odd image sizes, in every sweep shape that holds D, against the reference's sgm_disparity + median3."""
    from open_source_einstar_b200 import synth
    rng = np.random.default_rng(500 + seed)
    w, h = int(rng.integers(60, 260)), int(rng.integers(40, 200))
    nd = int(rng.choice([5, 24, 40, 48, 64, 80, 96, 100, 128]))
    pair = synth.plane_sphere_pair(seed=70 + seed, width=w, height=h, f=1.3 * w, num_disparities=nd)
    p1 = int(rng.integers(2, 20))
    p = OracleSgm(min_disparity=int(pair.min_disparity + rng.integers(-30, 10)), num_disparities=nd, p1=p1,
                  p2=int(rng.integers(p1 + 1, 103)), adaptive_p2=bool(rng.integers(2)), slant_steps=bool(rng.integers(2)),
                  uniqueness=float(rng.choice([0.8, 0.9, 0.95])), lr_max_diff=int(rng.integers(1, 3)))
    subpixel = bool(rng.integers(2))
    want = ref.median3(ref.sgm_disparity(pair.left, pair.right, p, subpixel=subpixel))
    for shape in [(6, 4), (8, 4), (6, 8), (8, 8)]:
        if shape[0] * 2 * shape[1] < nd:
            continue
        with _sweep_stereo(p, w, h, shape, subpixel=subpixel) as s:
            got = s.compute(pair.left, pair.right).disparity
        assert same_bits(got, want), f"{w}x{h} D={nd} {p} shape={shape}: {mismatch_report(got, want)}"


def test_sweep_kernels_refuse_frames_they_cannot_run(cuda):
    from open_source_einstar_b200 import CudaStereo, Errc, SgmParams, StereoError, StereoParams
    for sgm, shape in ((SgmParams(num_disparities=64, eight_paths=True), (8, 4)),
                       (SgmParams(num_disparities=64, p2=120), (8, 4)),
                       (SgmParams(num_disparities=24, census_radius_x=3, census_radius_y=3), (6, 4)),
                       (SgmParams(num_disparities=64), (4, 8)),
                       (SgmParams(num_disparities=128), (8, 4))):
        with CudaStereo.create(StereoParams(sgm=sgm), 64, 48) as s:
            with pytest.raises(StereoError) as e:
                s.set_kernel_config(shape[0], shape[1], False, 4, 256, 4, True)
            assert e.value.code == Errc.invalid_argument


def test_batch_of_configuration_sizes_against_the_reference(cuda, ref, port):
    """One batch with a pair of each configuration-3 size and disparity range (640x512 D=64, 960x768 D=96 and
    D=192, 1280x1024 D=128), sweep kernels where they fit: every pair's u16 disparity and depth equal the
    reference's sgm_disparity + median3 and the restated depth, directly (not only per-pair CUDA runs)."""
    import torch
    from open_source_einstar_b200 import PairDesc, RectifiedGeometry, SgmParams, StereoBatch, StereoParams, synth
    specs = [(640, 512, 64, (8, 4)), (960, 768, 96, (6, 8)), (1280, 1024, 128, (8, 8)), (960, 768, 192, None)]
    pairs = [synth.plane_sphere_pair(seed=90 + i, width=w, height=h, f=1.1 * w, num_disparities=d)
             for i, (w, h, d, _) in enumerate(specs)]
    descs, outs, ins = [], [], []
    for (w, h, d, shape), pr in zip(specs, pairs):
        sp = StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity, num_disparities=d))
        k = {"regs_per_lane": shape[0], "lanes_per_line": shape[1], "fused_pairs": 1} if shape else None
        descs.append(PairDesc(w, h, sp, geometry=RectifiedGeometry(pr.f, 0, 0, pr.baseline), kernel=k))
        ins.append((torch.from_numpy(pr.left).cuda(), torch.from_numpy(pr.right).cuda()))
        outs.append({"disparity_u16": torch.empty((h, w), dtype=torch.int16, device="cuda"),
                     "depth": torch.empty((h, w), dtype=torch.float32, device="cuda")})
    with StereoBatch(descs, micro_batch=1, branches=4) as b:
        for i, ((l, r), o) in enumerate(zip(ins, outs)):
            b.bind(i, l, r, o)
        b.run(stream=torch.cuda.current_stream())
        torch.cuda.synchronize()
    for (w, h, d, shape), pr, o in zip(specs, pairs, outs):
        p = OracleSgm(min_disparity=pr.min_disparity, num_disparities=d)
        disp = ref.median3(ref.sgm_disparity(pr.left, pr.right, p))
        u16 = port.encode_u16(disp, p.min_disparity)
        z = port.depth(disp, pr.f, pr.baseline, 0.0, 150.0, 700.0)
        got = o["disparity_u16"].cpu().numpy().view(np.uint16)
        assert np.array_equal(got, u16), f"{w}x{h} D={d}: {mismatch_report(got, u16)}"
        assert same_bits(o["depth"].cpu().numpy(), z), f"{w}x{h} D={d} depth"
