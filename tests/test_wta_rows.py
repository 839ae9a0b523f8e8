"""The row-sweep WTA (k_wta_rows / kb_wta_rows: 4 paths, byte path values, lane slabs of 64, 96 or 128
disparities) against the reference's own stereo.cpp (oracle/_ref), bit for bit: rows cut into 1 to 32 chunks
with 1 to 5 right-WTA key sets, padding slots (D below the slab), negative and large minimum disparities,
random images full of ties, uniqueness, L-R threshold and subpixel on and off; and one batch launch whose
pairs share a slab width but differ in chunking.
"""
import numpy as np
import pytest

from conftest import mismatch_report, same_bits
from oracle.oracle import OracleSgm

pytestmark = pytest.mark.gpu

# classic path shapes (regs per lane, lanes per line) for each slab width the row-sweep WTA takes
SHAPES = {64: [(4, 8), (2, 16)], 96: [(6, 8), (3, 16)], 128: [(8, 8), (4, 16)]}


def _stereo(p: OracleSgm, w, h, shape, subpixel=True):
    from open_source_einstar_b200 import CudaStereo, SgmParams, StereoParams
    s = CudaStereo.create(StereoParams(sgm=SgmParams(**p.__dict__), median=True, subpixel=subpixel), w, h, tuned=False)
    s.set_kernel_config(shape[0], shape[1], True, 4, 256, 8, False)
    return s


def _pair(rng, w, h, nd, seed, noise):
    from open_source_einstar_b200 import synth
    if noise:
        return rng.integers(0, 256, (h, w), dtype=np.uint8), rng.integers(0, 256, (h, w), dtype=np.uint8), 0
    pr = synth.plane_sphere_pair(seed=seed, width=w, height=h, f=1.3 * w, num_disparities=nd)
    return pr.left, pr.right, pr.min_disparity


@pytest.mark.parametrize("seed", range(10))
def test_row_wta_random_frames_against_the_reference(cuda, ref, seed):
    """Widths from one chunk (9 px) to 32 chunks of a row, every slab width, D up to the slab (padding),
    random SGM parameters within the byte-value range, against sgm_disparity + median3."""
    rng = np.random.default_rng(4100 + seed)
    w = int(rng.choice([9, 40, 70, 130, 333, 1030, 1900]))
    h = int(rng.choice([5, 17, 31]))
    dp = int(rng.choice([64, 96, 128]))
    nd = int(rng.choice([dp, dp, dp - int(rng.integers(1, 30))]))
    noise = bool(rng.integers(3) == 0) or w < 40
    left, right, mind = _pair(rng, w, h, nd, 300 + seed, noise)
    p1 = int(rng.integers(2, 20))
    p = OracleSgm(min_disparity=int(mind + rng.choice([0, -40, 25, min(3 * w // 4, 300)])), num_disparities=nd, p1=p1,
                  p2=int(rng.integers(p1 + 1, 101)), adaptive_p2=bool(rng.integers(2)), slant_steps=bool(rng.integers(2)),
                  uniqueness=float(rng.choice([0.8, 0.9, 0.95])), lr_max_diff=int(rng.integers(1, 3)))
    subpixel = bool(rng.integers(2))
    want = ref.median3(ref.sgm_disparity(left, right, p, subpixel=subpixel))
    for shape in SHAPES[dp]:
        with _stereo(p, w, h, shape, subpixel=subpixel) as s:
            got = s.compute(left, right).disparity
        assert same_bits(got, want), f"{w}x{h} D={nd} slab {dp} {p} shape={shape}: {mismatch_report(got, want)}"


def test_row_wta_batch_with_mixed_chunking_against_the_reference(cuda, ref, port):
    """Four pairs with the same 64-disparity slab in one micro-batch (one kb_wta_rows launch): 1, 4, 16 and
    32 chunks a row, each pair's u16 disparity equal to the reference's."""
    import torch
    from open_source_einstar_b200 import PairDesc, RectifiedGeometry, SgmParams, StereoBatch, StereoParams, synth
    sizes = [(24, 20), (70, 33), (333, 41), (1030, 18)]
    pairs = [synth.plane_sphere_pair(seed=60 + i, width=w, height=h, f=1.3 * w, num_disparities=64)
             for i, (w, h) in enumerate(sizes)]
    kcfg = {"regs_per_lane": 4, "lanes_per_line": 8, "materialize_costs": 1, "fused_pairs": 0}
    descs, outs = [], []
    for (w, h), pr in zip(sizes, pairs):
        sp = StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity, num_disparities=64))
        descs.append(PairDesc(w, h, sp, geometry=RectifiedGeometry(pr.f, 0, 0, pr.baseline), kernel=kcfg))
        outs.append({"disparity_u16": torch.empty((h, w), dtype=torch.int16, device="cuda")})
    ins = [(torch.from_numpy(pr.left).cuda(), torch.from_numpy(pr.right).cuda()) for pr in pairs]  # bound: kept alive
    with StereoBatch(descs, micro_batch=len(descs), branches=1, tuned=False) as b:
        for i, ((l, r), o) in enumerate(zip(ins, outs)):
            b.bind(i, l, r, o)
        for _ in range(2):  # the second run re-uses the volumes the first left behind
            b.run(stream=torch.cuda.current_stream())
        torch.cuda.synchronize()
    for (w, h), pr, o in zip(sizes, pairs, outs):
        p = OracleSgm(min_disparity=pr.min_disparity, num_disparities=64)
        u16 = port.encode_u16(ref.median3(ref.sgm_disparity(pr.left, pr.right, p)), p.min_disparity)
        got = o["disparity_u16"].cpu().numpy().view(np.uint16)
        assert np.array_equal(got, u16), f"{w}x{h}: {mismatch_report(got, u16)}"
