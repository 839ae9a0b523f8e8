"""The C ABI without a GPU: the library loads, exports exactly what include/*.h declares, and the
host-side validation returns the reference's error codes (no compute call is made here)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include"))) if f.endswith(".h")]


def declared_symbols():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        names |= set(re.findall(r"DS_API\s+[\w\s\*]+?\b(ds_\w+)\s*\(", text))
    return names


@pytest.fixture(scope="module")
def lib():
    from open_source_einstar_b200 import _native
    from open_source_einstar_b200.build import build_native
    build_native()
    return _native.lib()


def test_exports_every_declared_symbol(lib):
    from open_source_einstar_b200.build import LIB
    declared = declared_symbols()
    assert len(declared) >= 14
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = declared - exported
    assert not missing, f"declared but not exported: {missing}"
    extra = {s for s in exported if s.startswith("ds_")} - declared
    assert not extra, f"exported but not declared: {extra}"
    for s in declared:
        getattr(lib, s)


def test_binding_covers_header(lib):
    from open_source_einstar_b200._native import SIGNATURES
    assert set(SIGNATURES) == declared_symbols()


def test_defaults_mirror_reference(lib):
    """ds_default_params == depth::SgmParams defaults (stereo.hpp:26-40) on the hot path."""
    from open_source_einstar_b200._native import StereoParamsC
    p = StereoParamsC()
    lib.ds_default_params(C.byref(p))
    s = p.sgm
    assert (s.min_disparity, s.num_disparities, s.census_radius_x, s.census_radius_y, s.p1, s.p2) == (0, 64, 2, 2, 8, 96)
    assert (s.adaptive_p2, s.eight_paths, s.slant_steps, s.lr_max_diff) == (1, 0, 1, 1)
    assert abs(s.uniqueness - 0.9) < 1e-7
    assert (p.pyramid_levels, p.subpixel, p.median, p.detail_enabled, p.speckle_max_region_size) == (0, 1, 1, 0, 0)


@pytest.mark.parametrize("change,code,msg", [
    (dict(num_disparities=513), 5, "512 disparities"),
    (dict(num_disparities=0), 5, "disparities"),
    (dict(census_radius_x=5), 5, "census window too large"),
    (dict(census_radius_y=4), 5, "census window too large"),
    (dict(p1=-1), 5, "non-negative"),
])
def test_create_rejects_like_metal(lib, change, code, msg):
    """Validation mirrors metal_stereo.cpp:115-120 (Errc::invalid_argument); checked before any device call."""
    from open_source_einstar_b200 import StereoError, StereoParams, SgmParams, CudaStereo
    sp = SgmParams(**change)
    with pytest.raises(StereoError) as e:
        CudaStereo.create(StereoParams(sgm=sp), 64, 48)
    assert int(e.value.code) == code and msg in e.value.message


@pytest.mark.parametrize("change", [dict(pyramid_levels=5), dict(pyramid_levels=-1),
                                    dict(pyramid_levels=1, refine=dict(zncc_radius=0)),
                                    dict(pyramid_levels=1, refine=dict(search_radius=40)),
                                    dict(detail_enabled=True, detail=dict(step=0.0)),
                                    dict(speckle_max_region_size=-3)])
def test_refinement_parameters_are_validated(lib, change):
    """The stages of depth::compute_disparity beyond the hot path are checked before any device call."""
    from open_source_einstar_b200 import CudaStereo, DetailParams, Errc, RefineParams, StereoError, StereoParams
    kw = dict(change)
    if "refine" in kw:
        kw["refine"] = RefineParams(**kw["refine"])
    if "detail" in kw:
        kw["detail"] = DetailParams(**kw["detail"])
    with pytest.raises(StereoError) as e:
        CudaStereo.create(StereoParams(**kw), 64, 48)
    assert e.value.code == Errc.invalid_argument


def test_bad_sizes(lib):
    from open_source_einstar_b200 import CudaStereo, Errc, StereoError, StereoParams
    for w, h in ((0, 10), (10, 0), (20000, 10)):
        with pytest.raises(StereoError) as e:
            CudaStereo.create(StereoParams(), w, h)
        assert e.value.code == Errc.invalid_argument


def test_missing_library_fails_loudly(monkeypatch):
    from open_source_einstar_b200 import _native
    monkeypatch.setattr(_native, "_lib", None)
    monkeypatch.setattr(_native, "LIB", "/nonexistent/libdepth_cuda.so")
    with pytest.raises(ImportError):
        _native.lib()
