"""The oracle (CPU restatement, oracle/sgm_oracle.c) pinned against the reference.

Pins: the golden fixtures (outputs of the reference's own stereo.cpp, tests/golden/make_golden.py)
and, when oracle/_ref is built, live runs of the reference on further seeded inputs. The remap and
depth restatements (whose reference files need Eigen, absent here) are pinned by known-answer
properties of the reference formulas.
"""
import hashlib

import numpy as np
import pytest

from conftest import mismatch_report, same_bits
from oracle.oracle import INVALID, OracleSgm


def _params(case):
    return OracleSgm(**case["params"])


def test_golden_sgm_disparity(port, golden):
    for name, c in golden.items():
        d = port.sgm_disparity(c["left"], c["right"], _params(c), c["subpixel"])
        if "disparity" in c:
            assert same_bits(d, c["disparity"]), f"{name}: {mismatch_report(d, c['disparity'])}"
        else:
            assert hashlib.sha256(d.tobytes()).hexdigest() == c["disparity_sha256"], name


def test_golden_median3(port, golden):
    for name, c in golden.items():
        if "disparity" not in c:
            continue
        m = port.median3(c["disparity"])
        assert same_bits(m, c["median"]), f"{name}: {mismatch_report(m, c['median'])}"


def test_golden_digest_case_median(port, golden):
    c = golden["plane_sphere_640x512_d64"]
    d = port.sgm_disparity(c["left"], c["right"], _params(c), c["subpixel"])
    assert hashlib.sha256(port.median3(d).tobytes()).hexdigest() == c["median_sha256"]


def test_golden_census(port, golden):
    for name, c in golden.items():
        if "census_left" not in c:
            continue
        p = _params(c)
        cl = port.census(c["left"], p.census_radius_x, p.census_radius_y)
        assert same_bits(cl, c["census_left"]), name


def test_golden_fixture_cover_edge_cases(golden):
    names = set(golden)
    # empty/unmatched regions, ragged sizes, D below and not a multiple of the warp, 8 paths, 64-bit
    # census, 16-bit path values, negative disparities: the reference's parameter space on the path.
    for need in ("unmatched_noise", "tiny_37x29_d5", "d_not_multiple_of_32_d40", "eight_paths", "census_7x7_u64",
                 "census_9x7_wide", "negative_min_disparity", "no_subpixel_uniq08_lr2"):
        assert need in names
    assert golden["unmatched_noise"]["valid_fraction"] < 0.9


@pytest.mark.parametrize("seed", [11, 12, 13])
def test_port_matches_reference_live(port, ref, seed):
    rng = np.random.default_rng(seed)
    w, h = int(rng.integers(20, 90)), int(rng.integers(10, 60))
    nd = int(rng.integers(1, 70))
    p = OracleSgm(min_disparity=int(rng.integers(-20, 20)), num_disparities=nd,
                  census_radius_x=int(rng.integers(0, 5)), census_radius_y=int(rng.integers(0, 4)),
                  p1=int(rng.integers(0, 20)), p2=int(rng.integers(20, 150)), adaptive_p2=bool(rng.integers(0, 2)),
                  eight_paths=bool(rng.integers(0, 2)), slant_steps=bool(rng.integers(0, 2)),
                  uniqueness=float(rng.uniform(0.6, 1.0)), lr_max_diff=int(rng.integers(0, 3)))
    base = (rng.random((h, w + 40)) * 255).astype(np.uint8)
    left = base[:, 20:20 + w].copy()
    right = np.clip(base[:, 14:14 + w].astype(int) + rng.integers(-5, 6, (h, w)), 0, 255).astype(np.uint8)
    a = port.sgm_disparity(left, right, p)
    b = ref.sgm_disparity(left, right, p)
    assert same_bits(a, b), mismatch_report(a, b)
    assert same_bits(port.median3(a), ref.median3(b))
    assert same_bits(port.census(left, p.census_radius_x, p.census_radius_y),
                     ref.census(left, p.census_radius_x, p.census_radius_y))


def test_planted_mistake_is_detected(port, golden):
    """The comparison catches a one-ulp change: planted in an oracle output, on the CPU."""
    c = golden["plane_sphere_160x128"]
    d = port.sgm_disparity(c["left"], c["right"], _params(c), True)
    i = np.flatnonzero(d > -1e8)[7]
    bad = d.copy().ravel()
    bad[i] = np.nextafter(bad[i], np.float32(1e9))
    assert not same_bits(bad.reshape(d.shape), c["disparity"])


def test_stage_composition(port, golden):
    """census -> cost -> aggregate -> wta -> lr_check, called stage by stage, equals sgm_disparity."""
    c = golden["plane_sphere_160x128"]
    p = _params(c)
    cl = port.census(c["left"], 2, 2)
    cr = port.census(c["right"], 2, 2)
    cost = port.cost_volume(cl, cr, p)
    assert cost.max() <= 25
    sums = port.aggregate(cost, c["left"], p)
    disp, rd = port.wta(sums, p, True)
    d = port.lr_check(disp, rd, p.lr_max_diff)
    assert same_bits(d, c["disparity"])


def _numpy_remap(src, mx, my):
    """Independent float32 statement of calib::remap (rectify.cpp:133-148) in numpy."""
    f32 = np.float32
    h, w = mx.shape
    out = np.zeros((h, w), np.uint8)
    for y in range(h):
        for x in range(w):
            sx, sy = f32(mx[y, x]), f32(my[y, x])
            x0, y0 = int(np.floor(sx)), int(np.floor(sy))
            if x0 < 0 or y0 < 0 or x0 + 1 >= src.shape[1] or y0 + 1 >= src.shape[0]:
                continue
            fx, fy = f32(sx - f32(x0)), f32(sy - f32(y0))
            gx, gy = f32(f32(1) - fx), f32(f32(1) - fy)
            a, b = f32(src[y0, x0]), f32(src[y0, x0 + 1])
            c, d = f32(src[y0 + 1, x0]), f32(src[y0 + 1, x0 + 1])
            top = f32(f32(a * gx) + f32(b * fx))
            bot = f32(f32(c * gx) + f32(d * fx))
            v = f32(f32(top * gy) + f32(bot * fy))
            v = min(max(f32(v + f32(0.5)), f32(0)), f32(255))
            out[y, x] = np.uint8(int(v))
    return out


def test_remap_known_answers(port):
    rng = np.random.default_rng(3)
    src = (rng.random((40, 50)) * 255).astype(np.uint8)
    ys, xs = np.mgrid[0:30, 0:40].astype(np.float32)
    # identity and integer shifts reproduce pixels exactly; the last row/column is out of bounds (x0+1 >= w)
    ident = port.remap(src, xs, ys)
    assert np.array_equal(ident, src[:30, :40])
    shifted = port.remap(src, xs + 3, ys + 2)
    assert np.array_equal(shifted, src[2:32, 3:43])
    oob = port.remap(src, xs - 10, ys)
    assert (oob[:, :10] == 0).all()
    # fractional maps: the separately rounded float32 formula
    mx = (xs * 1.13 + rng.random(xs.shape) * 3).astype(np.float32)
    my = (ys * 1.07 + rng.random(ys.shape) * 3 - 1).astype(np.float32)
    assert np.array_equal(port.remap(src, mx, my), _numpy_remap(src, mx, my))


def test_depth_and_u16_known_answers(port):
    d = np.array([[100.0, 150.25, INVALID, -5.0], [60.0, 10.0, 149.984375, 200.0]], np.float32)
    z = port.depth(d, 900.0, 60.0, 0.0, 150.0, 700.0)
    want = np.where(d > -1e8, 900.0 * 60.0 / d.astype(np.float64), 0.0)
    want = np.where((want < 150) | (want > 700) | (d <= 0), 0.0, want).astype(np.float32)
    assert np.array_equal(z, want)
    zo = port.depth(np.array([[-3.0]], np.float32), 900.0, 60.0, 10.0, 0.0, 1e9)  # d + cx_offset > 0
    assert zo[0, 0] == np.float32(900.0 * 60.0 / 7.0)
    u = port.encode_u16(d, 100)
    assert u[0, 0] == 0 and u[0, 1] == round(50.25 * 64) and u[0, 2] == 0xFFFF
    assert u[0, 3] == 0  # below the search range: clamped
    assert u[1, 2] == round(49.984375 * 64)
