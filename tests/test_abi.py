"""C-ABI library: loads, exports every declared symbol, option handling and
file formats (no GPU needed; no compute calls)."""
import ctypes as C
import math
import re
from pathlib import Path

import numpy as np
import pytest

from sensemap_b200 import _native as N
from sensemap_b200 import mat_io
from sensemap_b200.patch_match import PatchMatchOptions

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        names += re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(smvs_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = N.lib()
    decl = declared_functions()
    assert len(decl) >= 20
    missing = [n for n in decl if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    # The Python binding covers every declared entry point too.
    assert set(decl) <= set(N.exported_symbols())


def test_defaults_match_reference():
    o = N.smvs_options()
    N.check(N.lib().smvs_options_default(C.byref(o)))
    # PatchMatchOptions defaults, patch_match_options.h:42-304
    assert o.window_radius == 5 and o.window_step == 2 and o.sigma_spatial == 5.0
    assert abs(o.sigma_color - 0.2) < 1e-6 and o.num_samples == 15 and o.num_iterations == 5
    assert o.geom_consistency == 1 and o.init_depth_random == 0 and o.thk == 4
    assert abs(o.random_angle1_range - math.radians(20)) < 1e-6
    assert abs(o.geom_consistency_regularizer - 0.3) < 1e-6 and abs(o.geom_consistency_max_cost - 3.0) < 1e-6
    py = PatchMatchOptions()
    for name, _ in N.smvs_options._fields_:
        assert abs(float(getattr(py, name)) - float(getattr(o, name))) < 1e-6, name


@pytest.mark.parametrize("field,value", [("window_radius", 6), ("window_step", 3), ("thk", 5), ("thk", 0),
                                         ("depth_min", -1.0), ("propagate_depth", True), ("image_storage", 7),
                                         ("num_samples", 0)])
def test_options_check_rejects(field, value):
    o = PatchMatchOptions(depth_min=1.0, depth_max=10.0)
    o.check()
    setattr(o, field, value)
    with pytest.raises(N.SmvsError) as ei:
        o.check()
    assert ei.value.status == N.SMVS_EINVAL
    assert N.last_error()


def test_prior_option_combinations():
    """has_prior_depth alone is valid; propagate_depth needs given maps
    (init_depth_random = 0) and no geometric pass, and excludes has_prior_depth
    (patch_match_cuda.cu:946-947)."""
    o = PatchMatchOptions(depth_min=1.0, depth_max=10.0, has_prior_depth=True)
    o.check()
    o = PatchMatchOptions(depth_min=1.0, depth_max=10.0, propagate_depth=True, geom_consistency=False,
                          init_depth_random=False)
    o.check()
    for bad in (dict(has_prior_depth=True), dict(init_depth_random=True), dict(geom_consistency=True)):
        q = PatchMatchOptions(depth_min=1.0, depth_max=10.0, propagate_depth=True, geom_consistency=False,
                              init_depth_random=False)
        for k, v in bad.items():
            setattr(q, k, v)
        with pytest.raises(N.SmvsError):
            q.check()


def test_mat_roundtrip(tmp_path):
    rng = np.random.default_rng(0)
    d = rng.random((7, 9)).astype(np.float32)
    p = str(tmp_path / "x.bin")
    mat_io.write_depth_map(p, d)
    raw = Path(p).read_bytes()
    assert raw.startswith(b"9&7&1&")
    assert len(raw) == len(b"9&7&1&") + 4 * 63
    np.testing.assert_array_equal(mat_io.read_mat(p), d)


def _encode_py(n):
    # NormalMap::Encode, src/mvs/normal_map.cc:159-181, restated in numpy float32.
    s = ((1 - n[0].astype(np.float64)) * 0.5).astype(np.float32)
    m = (np.float32(1.0) / np.sqrt(np.float32(1) - s)).astype(np.float32)
    q1 = (n[1].astype(np.float64) * 0.5 * m).astype(np.float32)
    q2 = (n[2].astype(np.float64) * 0.5 * m).astype(np.float32)
    q1 = np.clip(q1, np.float32(-0.999999), np.float32(0.999999))
    q2 = np.clip(q2, np.float32(-0.999999), np.float32(0.999999))
    iq1 = ((q1 + np.float32(1)) * np.float32(32767)).astype(np.uint32)
    iq2 = ((q2 + np.float32(1)) * np.float32(32767)).astype(np.uint32)
    return (iq1 << 16) | iq2


def test_normal_encoding_matches_reference_formula(tmp_path):
    rng = np.random.default_rng(1)
    n = rng.normal(size=(3, 13, 17)).astype(np.float32)
    n /= np.linalg.norm(n, axis=0, keepdims=True)
    n[:, 0, 0] = 0  # filtered pixel
    code = mat_io.encode_normal_map(n)
    np.testing.assert_array_equal(code, _encode_py(n))
    dec = mat_io.decode_normal_map(code)
    valid = np.ones(n.shape[1:], bool)
    valid[0, 0] = False
    cosang = (dec * n).sum(0)[valid]
    assert cosang.min() > 0.9999
    p = str(tmp_path / "n.bin")
    mat_io.write_normal_map(p, n)
    np.testing.assert_array_equal(mat_io.read_mat(p, np.uint32), code)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setenv("SMVS_LIBRARY", str(tmp_path / "nope.so"))
    monkeypatch.setattr(N, "_LIB", None)
    with pytest.raises(N.NativeLibraryError):
        N.lib()


def test_cpp_wrapper_compiles_and_links(tmp_path):
    """include/smvs.hpp (the C++ shape of the reference operator) compiles
    against the C ABI and links the in-tree library; only GPU-free calls run."""
    import shutil
    import subprocess
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    src = tmp_path / "use.cpp"
    src.write_text('''
#include "smvs.hpp"
#include <cstdio>
int main() {
  smvs_options o = smvs::DefaultOptions();
  o.depth_min = 1; o.depth_max = 10; o.window_step = 1;
  smvs::Check(smvs_options_check(&o));
  o.window_radius = 6;
  try { smvs::Check(smvs_options_check(&o)); return 1; } catch (const smvs::Error& e) {
    std::printf("%d %s\\n", e.status, e.what());
  }
  return 0;
}
''')
    lib = N.library_path()
    exe = tmp_path / "use"
    res = subprocess.run([gxx, "-std=c++17", f"-I{ROOT / 'include'}", str(src), str(lib), f"-Wl,-rpath,{lib.parent}",
                          "-o", str(exe)], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True)
    assert run.returncode == 0 and run.stdout.startswith("1 "), (run.stdout, run.stderr)
