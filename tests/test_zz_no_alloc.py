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
    cases = ["plane_sphere_160x128", "census_7x7_u64", "eight_paths", "d_not_multiple_of_32_d40"]
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
