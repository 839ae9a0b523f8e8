"""The no-allocation disparity entry point (ds_sgm_disparity_noalloc) against the allocating one.

Some callers cannot allocate device memory when they need a disparity map (a fixed device-memory
budget reserved at start-up, a real-time loop where an allocation may block or fail, a host framework
whose allocator owns the device). ds_sgm_disparity_noalloc serves them from a static device array;
here its output, through the C ABI, must equal ds_compute_device's (median off) bit for bit on two
calls in a row, and a request larger than the static array must be refused with a clear error.
This file is collected last so that a stop-at-first-failure run has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from oracle.oracle import OracleSgm

pytestmark = pytest.mark.gpu

TOLERANCE_ULP = 0  # disparities are compared bit for bit (integer WTA + IEEE float subpixel)


def _noalloc(lib, sgm_c, left, right, out, subpixel=True):
    h, w = left.shape
    return lib.ds_sgm_disparity_noalloc(C.c_void_p(left.data_ptr()), C.c_void_p(right.data_ptr()), w, h,
                                        C.byref(sgm_c), int(subpixel), C.c_void_p(out.data_ptr()), None)


def _allocating(params: OracleSgm, left, right, subpixel=True):
    import torch
    from open_source_einstar_b200 import CudaStereo, SgmParams, StereoParams
    h, w = left.shape
    out = torch.empty((h, w), dtype=torch.float32, device="cuda")
    with CudaStereo.create(StereoParams(sgm=SgmParams(**params.__dict__), subpixel=subpixel, median=False), w, h) as s:
        s.compute_device(left, right, {"disparity": out}, stream=torch.cuda.current_stream())
        torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_matches_allocating_entry_point(cuda, golden):
    import torch
    from open_source_einstar_b200 import SgmParams, StereoParams
    from open_source_einstar_b200._native import lib
    L = lib()
    # u8 and u16 path values (census_9x7_wide), 64-bit census words, 8 paths, D not a multiple of the lane
    # slab, a negative minimum disparity, and D=5 where most lanes are padding
    cases = ["plane_sphere_160x128", "census_7x7_u64", "eight_paths", "d_not_multiple_of_32_d40", "census_9x7_wide",
             "negative_min_disparity", "tiny_37x29_d5"]
    for name in cases:
        c = golden[name]
        p = OracleSgm(**c["params"])
        left = torch.from_numpy(c["left"]).cuda()
        right = torch.from_numpy(c["right"]).cuda()
        want = _allocating(p, left, right, c["subpixel"])
        sgm_c = StereoParams(sgm=SgmParams(**p.__dict__)).c().sgm
        for call in range(2):  # the static scratch keeps the previous call's contents
            out = torch.full(c["left"].shape, 3.0, dtype=torch.float32, device="cuda")
            rc = _noalloc(L, sgm_c, left, right, out, c["subpixel"])
            assert rc == 0, L.ds_last_global_error().decode()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            diff = np.abs(got.view(np.int32).astype(np.int64) - want.view(np.int32).astype(np.int64))
            assert diff.max() <= TOLERANCE_ULP, f"{name} call {call}: {int((diff > 0).sum())} pixels differ"
            assert np.array_equal(got.view(np.uint32), c["disparity"].view(np.uint32)), f"{name} call {call} vs golden"


def test_noalloc_rejects_requests_beyond_its_scratch(cuda):
    import torch
    from open_source_einstar_b200 import SgmParams, StereoParams
    from open_source_einstar_b200._native import lib
    L = lib()
    left = torch.zeros((1024, 1280), dtype=torch.uint8, device="cuda")
    out = torch.zeros((1024, 1280), dtype=torch.float32, device="cuda")
    sgm_c = StereoParams(sgm=SgmParams(num_disparities=128)).c().sgm
    rc = _noalloc(L, sgm_c, left, left, out)
    assert rc == 5  # DS_INVALID_ARGUMENT
    msg = L.ds_last_global_error().decode()
    assert "scratch" in msg and "bytes" in msg


SCRATCH_BYTES = 16 << 20  # the documented limit of the static array


def _scratch_need(w, h, nd, census_window=25, paths=4, wide=False):
    """The bytes the entry point needs (its documented sizing): two census images of 4-byte words (8 for
    windows of more than 32 neighbours) and the path values of all directions with the lane slabs of the
    library's default shape for nd, each part rounded up to 256 bytes."""
    a256 = lambda v: (v + 255) // 256 * 256
    dp = next(seg * 2 * r for lim, r, seg in ((32, 1, 16), (64, 2, 16), (96, 3, 16), (128, 4, 16), (192, 3, 32),
                                              (256, 4, 32), (384, 6, 32), (512, 8, 32)) if nd <= lim)
    cw = 8 if census_window - 1 > 32 else 4
    return 2 * a256(w * h * cw) + a256(w * h * dp * paths * (2 if wide else 1))


def test_noalloc_limit_boundary(cuda):
    """The documented example (320 x 240 at 32 disparities, 4 paths) fits; at 320 columns and 32 disparities
    the tallest image that fits is accepted and one row more is refused with the bytes it would need."""
    import torch
    from open_source_einstar_b200 import SgmParams, StereoParams
    from open_source_einstar_b200._native import lib
    L = lib()
    sgm_c = StereoParams(sgm=SgmParams(num_disparities=32)).c().sgm
    assert _scratch_need(320, 240, 32) <= SCRATCH_BYTES
    h_max = max(h for h in range(1, 2000) if _scratch_need(320, h, 32) <= SCRATCH_BYTES)
    for h, ok in ((240, True), (h_max, True), (h_max + 1, False)):
        img = torch.zeros((h, 320), dtype=torch.uint8, device="cuda")
        out = torch.zeros((h, 320), dtype=torch.float32, device="cuda")
        rc = _noalloc(L, sgm_c, img, img, out)
        torch.cuda.synchronize()
        if ok:
            assert rc == 0, (h, L.ds_last_global_error().decode())
        else:
            assert rc == 5, h
            assert str(_scratch_need(320, h, 32)) in L.ds_last_global_error().decode()
