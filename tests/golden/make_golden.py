"""Generates the golden fixtures of the stereo hot path from the reference itself.

Outputs come from oracle/_ref/libref_stereo.so: the reference's libs/depth/src/stereo.cpp compiled
unmodified (census_transform, sgm_disparity, median3). Inputs are seeded synthetic speckle pairs
(open_source_einstar_b200.synth) and seeded random images. Run from the repository root, with the
reference tree present:

    make -C oracle all && python tests/golden/make_golden.py

Writes tests/golden/sgm_golden.npz (arrays) and tests/golden/sgm_golden.json (parameters per case).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import OracleSgm, Ref  # noqa: E402
from open_source_einstar_b200 import synth  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def shifted_random(seed, w, h, shift, noise=6):
    rng = np.random.default_rng(seed)
    base = (rng.random((h, w + abs(shift) + 8)) * 255).astype(np.uint8)
    o = 4 + max(0, -shift)
    left = base[:, o:o + w].copy()
    right = np.clip(base[:, o + shift:o + shift + w].astype(int) + rng.integers(-noise, noise + 1, (h, w)), 0, 255)
    return left, right.astype(np.uint8)


def cases():
    small = synth.plane_sphere_pair(seed=1, width=160, height=128, f=225.0, baseline=60.0, num_disparities=24)
    full = synth.plane_sphere_pair(seed=0, width=640, height=512, f=900.0, baseline=60.0, num_disparities=64)
    nl, nr = shifted_random(5, 96, 64, 11)
    ml, mr = shifted_random(6, 80, 56, -5)
    tl, tr = shifted_random(7, 37, 29, 3)
    rl, rr = shifted_random(8, 64, 48, 0, noise=255)
    sm = dict(min_disparity=small.min_disparity, num_disparities=24)
    return [
        ("plane_sphere_160x128", small.left, small.right, OracleSgm(**sm), True),
        ("eight_paths", small.left, small.right, OracleSgm(**sm, eight_paths=True), False),
        ("no_slant_fixed_p2", small.left, small.right, OracleSgm(**sm, slant_steps=False, adaptive_p2=False), False),
        ("census_7x7_u64", small.left, small.right, OracleSgm(**sm, census_radius_x=3, census_radius_y=3, p2=60), True),
        ("census_9x7_wide", small.left, small.right, OracleSgm(**sm, census_radius_x=4, census_radius_y=3, p2=200), False),
        ("no_subpixel_uniq08_lr2", nl, nr, OracleSgm(min_disparity=4, num_disparities=16, uniqueness=0.8, lr_max_diff=2), False),
        ("negative_min_disparity", ml, mr, OracleSgm(min_disparity=-12, num_disparities=20), False),
        ("tiny_37x29_d5", tl, tr, OracleSgm(min_disparity=1, num_disparities=5), True),
        ("unmatched_noise", rl, rr, OracleSgm(min_disparity=0, num_disparities=16), False),
        ("d_not_multiple_of_32_d40", nl, nr, OracleSgm(min_disparity=0, num_disparities=40, p1=5, p2=40), False),
        ("plane_sphere_640x512_d64", full.left, full.right, OracleSgm(min_disparity=full.min_disparity, num_disparities=64), False),
    ]


# Cases whose outputs are kept as SHA-256 digests of the f32 bytes only (the arrays would dominate the
# fixture size); their inputs are stored in full.
DIGEST_ONLY = {"plane_sphere_640x512_d64"}


def main():
    ref = Ref()
    arrays, manifest = {}, {}
    for name, left, right, p, census in cases():
        subpixel = name != "no_subpixel_uniq08_lr2"
        disp = ref.sgm_disparity(left, right, p, subpixel)
        med = ref.median3(disp)
        arrays[f"{name}/left"] = left
        arrays[f"{name}/right"] = right
        manifest[name] = {"params": p.__dict__, "subpixel": subpixel, "shape": list(left.shape),
                          "valid_fraction": float((disp > -1e8).mean())}
        if name in DIGEST_ONLY:
            manifest[name]["disparity_sha256"] = hashlib.sha256(disp.tobytes()).hexdigest()
            manifest[name]["median_sha256"] = hashlib.sha256(med.tobytes()).hexdigest()
        else:
            arrays[f"{name}/disparity"] = disp
            arrays[f"{name}/median"] = med
        if census:
            arrays[f"{name}/census_left"] = ref.census(left, p.census_radius_x, p.census_radius_y)
        print(f"{name:28s} {left.shape} valid {manifest[name]['valid_fraction']:.3f}")
    np.savez_compressed(os.path.join(OUT, "sgm_golden.npz"), **arrays)
    with open(os.path.join(OUT, "sgm_golden.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "oracle": "oracle/_ref (reference libs/depth/src/stereo.cpp)",
                   "cases": manifest}, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
