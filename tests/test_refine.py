"""depth::compute_disparity beyond the hot path (pyramid + slanted ZNCC refinement, detail refinement on the
full-resolution pair, occlusion and spike filters, speckle removal) on the GPU against the reference's own
stereo.cpp (oracle/_ref), bit for bit: disparity and confidence. Each stage is switched on alone first, then
the frontend's production setting (SGM one level below, refinement, detail, filters, speckles) runs from
raw images through the remap tables."""
import numpy as np
import pytest

from conftest import mismatch_report, same_bits

pytestmark = pytest.mark.gpu


def _params(**kw):
    from open_source_einstar_b200 import SgmParams, StereoParams
    sgm = kw.pop("sgm")
    return StereoParams(sgm=SgmParams(**sgm), median=False, **kw)


def _scene(w=320, h=256, seed=3):
    from open_source_einstar_b200 import synth
    return synth.plane_sphere_pair(seed=seed, width=w, height=h, f=1.4 * w, num_disparities=64, device="cuda")


def _check(got, want, what):
    gd, gc = got
    wd, wc = want
    assert (wd > -1e8).mean() > 0.2, f"{what}: too few valid pixels for a meaningful check"
    assert same_bits(gd, wd), f"{what} disparity: {mismatch_report(gd, wd)}"
    assert same_bits(gc, wc), f"{what} confidence: {mismatch_report(gc, wc)}"


@pytest.mark.parametrize("stages", [
    dict(filter_occlusion=True), dict(filter_spikes=True), dict(speckle_max_region_size=60),
    dict(filter_occlusion=True, filter_spikes=True, speckle_max_region_size=200)])
def test_filters_and_speckles_at_full_resolution(cuda, ref, stages):
    from open_source_einstar_b200 import CudaStereo
    pr = _scene()
    h, w = pr.left.shape
    sp = _params(sgm=dict(min_disparity=pr.min_disparity, num_disparities=64), **stages)
    with CudaStereo.create(sp, w, h) as s:
        r = s.compute(pr.left, pr.right)
    _check((r.disparity, r.confidence), ref.compute_disparity(pr.left, pr.right, sp), str(stages))


@pytest.mark.parametrize("levels", [1, 2])
def test_pyramid_refinement(cuda, ref, levels):
    from open_source_einstar_b200 import CudaStereo, RefineParams
    pr = _scene(w=320 if levels == 1 else 384, h=256)
    h, w = pr.left.shape
    mind = pr.min_disparity // (1 << levels) - 2
    for refine in (RefineParams(), RefineParams(search_radius=3, zncc_radius=2, min_zncc=0.3, reject_edge_winners=False)):
        sp = _params(sgm=dict(min_disparity=mind, num_disparities=48 // levels), pyramid_levels=levels, refine=refine)
        with CudaStereo.create(sp, w, h) as s:
            r = s.compute(pr.left, pr.right)
            r2 = s.compute(pr.left, pr.right)
        assert same_bits(r.disparity, r2.disparity)
        _check((r.disparity, r.confidence), ref.compute_disparity(pr.left, pr.right, sp), f"levels {levels} {refine}")


def test_production_setting_from_raw_images(cuda, ref, port):
    """The frontend's configuration (libs/pipeline/src/stereo_frontend.cpp:21-34): rectified pair at half the
    raw resolution, SGM a level below, refinement, detail on the full-resolution pair, filters, speckles."""
    from open_source_einstar_b200 import CudaStereo, RemapTable, synth
    pr = synth.raw_objects_pair(seed=11, width=640, height=512, f=560.0, num_disparities=64, n_objects=8, device="cuda")
    (lx, ly), (rx, ry) = pr.maps
    W, H = 640, 512
    w, h = W // 2, H // 2
    sp = _params(sgm=dict(min_disparity=pr.min_disparity // 4 - 2, num_disparities=40), pyramid_levels=1,
                 detail_enabled=True, filter_occlusion=True, filter_spikes=True, speckle_max_region_size=100)
    with CudaStereo.create(sp, w, h) as s:
        s.set_rectification(RemapTable(lx, ly), RemapTable(rx, ry), W, H)
        r = s.compute_raw(pr.left, pr.right)
    fl, fr = port.remap(pr.left, lx, ly), port.remap(pr.right, rx, ry)
    left, right = ref.downsample2(fl), ref.downsample2(fr)
    _check((r.disparity, r.confidence), ref.compute_disparity(left, right, sp, fl, fr), "production")
    # without the detail stage the result differs (the stage ran)
    sp.detail_enabled = False
    d2, _ = ref.compute_disparity(left, right, sp, fl, fr)
    assert not same_bits(r.disparity, d2)


def test_refinement_is_per_frame_only(cuda):
    from open_source_einstar_b200 import Errc, PairDesc, StereoBatch, StereoError
    sp = _params(sgm=dict(num_disparities=32), pyramid_levels=1)
    with pytest.raises(StereoError) as e:
        StereoBatch([PairDesc(64, 48, sp)])
    assert e.value.code == Errc.unsupported
