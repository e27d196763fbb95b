"""SenseMap map files through the C ABI: Mat<T> ("W&H&D&" + little-endian
payload, src/util/mat.h:179-215) and NormalMap's uint32 encoding
(src/mvs/normal_map.cc:137-181)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


def write_depth_map(path: str, depth: np.ndarray) -> None:
    d = np.ascontiguousarray(depth, dtype=np.float32)
    h, w = d.shape[-2:]
    depth_slices = 1 if d.ndim == 2 else d.shape[0]
    N.check(N.lib().smvs_write_mat_f32(path.encode(), d.ctypes.data, w, h, depth_slices))


def encode_normal_map(normal: np.ndarray) -> np.ndarray:
    n = np.ascontiguousarray(normal, dtype=np.float32)
    _, h, w = n.shape
    out = np.empty((h, w), np.uint32)
    N.check(N.lib().smvs_encode_normal_map(n.ctypes.data, w, h, out.ctypes.data))
    return out


def decode_normal_map(code: np.ndarray) -> np.ndarray:
    c = np.ascontiguousarray(code, dtype=np.uint32)
    h, w = c.shape
    out = np.empty((3, h, w), np.float32)
    N.check(N.lib().smvs_decode_normal_map(c.ctypes.data, w, h, out.ctypes.data))
    return out


def write_normal_map(path: str, normal: np.ndarray) -> None:
    code = encode_normal_map(normal)
    h, w = code.shape
    N.check(N.lib().smvs_write_mat_u32(path.encode(), code.ctypes.data, w, h, 1))


def read_mat(path: str, dtype=np.float32) -> np.ndarray:
    """Read a Mat file; returns D x H x W (or H x W when D == 1)."""
    dtype = np.dtype(dtype)
    w, h, d = C.c_int(), C.c_int(), C.c_int()
    N.check(N.lib().smvs_read_mat(path.encode(), None, 0, dtype.itemsize, C.byref(w), C.byref(h), C.byref(d)))
    out = np.empty((d.value, h.value, w.value), dtype)
    N.check(N.lib().smvs_read_mat(path.encode(), out.ctypes.data, out.nbytes, dtype.itemsize, C.byref(w),
                                  C.byref(h), C.byref(d)))
    return out[0] if d.value == 1 else out
