"""sensemap_b200 — B200-native PatchMatch multi-view-stereo depth-map engine.

Drop-in for SenseMap's per-reference-view depth-map stage
(sensemap::mvs::PatchMatchACMMCuda). The compute lives in ``libsmvs.so``
(hand-written sm_100a CUDA behind the C ABI in include/smvs.h); this package
marshals arguments and provides the reference-shaped Python API.
"""
from ._native import NativeLibraryError, SmvsError, STORE_F16, STORE_F32, STORE_U8  # noqa: F401
from .patch_match import PatchMatchACMMCuda, PatchMatchOptions, Problem, View  # noqa: F401
from .cross_filter import CrossFilterCuda  # noqa: F401
from .mat_io import read_mat, write_depth_map, write_normal_map, encode_normal_map, decode_normal_map  # noqa: F401

__all__ = ["PatchMatchACMMCuda", "CrossFilterCuda", "PatchMatchOptions", "Problem", "View", "SmvsError", "NativeLibraryError",
           "read_mat", "write_depth_map", "write_normal_map", "encode_normal_map", "decode_normal_map",
           "STORE_U8", "STORE_F16", "STORE_F32"]
