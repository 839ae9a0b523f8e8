"""B200-native stereo-depth hot path of the Einstar scanner pipeline.

rectify -> census -> Hamming cost -> multi-path SGM -> WTA + subpixel -> L-R check -> 3x3 median ->
depth, as hand-written sm_100a CUDA behind the C ABI in include/depth_cuda.h (libdepth_cuda.so).
The Python classes mirror the reference's stereo-matcher interface (depth_metal::MetalStereo).
"""
from .stereo import (  # noqa: F401
    BLOB_FIELDS,
    INVALID_DISPARITY,
    BlobParams,
    CudaStereo,
    DetailParams,
    Errc,
    RectifiedGeometry,
    RefineParams,
    RemapTable,
    SgmParams,
    StereoError,
    StereoParams,
    StereoResult,
    StereoTimings,
    valid_disparity,
)
from .batch import PairDesc, StereoBatch  # noqa: F401,E402
from .points import PointImageParams, disparity_to_points, pack_depth  # noqa: F401,E402
