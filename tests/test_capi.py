"""The C ABI library: it loads and exports every symbol include/gsj.h declares; no GPU needed."""
import ctypes
import os
import re

import numpy as np

import gsj
from gsj._build import lib_path

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "gsj.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gsj_[a-z0-9_]+)\s*\(", src)) - {"gsj_join_sink", "gsj_points_sink", "gsj_pairs_sink"})


def test_exports_every_declared_symbol():
    lib = ctypes.CDLL(lib_path("libgsj.so"))
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(gsj.SIGNATURES), set(names) - set(gsj.SIGNATURES)


def test_de9im_helpers_without_gpu():
    code = 1 | 3 << 12 | 2 << 14 | 3 << 16
    assert gsj.de9im_str(code) == "0FFFFF212"
    assert gsj.de9im_transpose(gsj.de9im_transpose(code)) == code
    assert gsj.de9im_match(code, "0********") and not gsj.de9im_match(code, "F********")


def test_defaults_match_reference_refine_params():
    p = gsj.refine_params()
    assert (p.tol_rel, p.eps_par, p.tol_abs, p.want_area, p.want_relate, p.snap_half_ulp) == (1e-12, 1e-7, 1e-11, 1, 0, 0)


def test_errors_are_status_codes_not_exits():
    """Without a usable device (CPU container) context creation fails with a status, it does not abort."""
    import torch
    if torch.cuda.is_available():
        return
    h = ctypes.c_void_p()
    rc = gsj.lib().gsj_ctx_create(0, ctypes.byref(h))
    assert rc != 0 and not h.value
    assert gsj.lib().gsj_join(None, None, None, None, None, gsj.JOIN_SINK(lambda *a: 0), None, None) == 1


def test_result_types_construct_without_gpu():
    r = gsj.JoinResult(np.zeros((0, 2), np.uint32), None, None, {"candidates": 0})
    assert len(r.pairs) == 0 and r.stats["candidates"] == 0


def test_sink_copy_out_matches_source():
    """The binding's copy of a sink's rows out of library-owned host memory (sliced across threads above 8 MiB)."""
    import ctypes

    import numpy as np

    import gsj
    rng = np.random.default_rng(3)
    for n, dt in ((0, np.uint32), (7, np.float64), (3_000_001, np.uint32), (1_500_007, np.float64)):
        src = rng.integers(0, 2**31, n).astype(dt)
        ptr = src.ctypes.data_as(ctypes.POINTER(np.ctypeslib.as_ctypes_type(dt)))
        out = gsj._copy_out(ptr, n, dt)
        assert out.dtype == dt and np.array_equal(out, src) and out.ctypes.data != src.ctypes.data


def test_headers_are_plain_c(tmp_path):
    """include/gsj.h and include/gsjd.h compile as C99 (what a cgo / FFI binding or the reference's C callers see)."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        import pytest
        pytest.skip("no C compiler")
    inc = os.path.join(ROOT, "include")
    src = tmp_path / "h.c"
    src.write_text('#include "gsj.h"\n#include "gsjd.h"\nint main(void) { gsj_refine_shape s = {4, 32, 128, 32}; gsj_tune_result t;\n'
                   '  (void)t; return s.run + GSJ_TUNE_KEEP_RUNS + GSJ_REFINE_FILTERED_FP32; }\n')
    r = subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", inc, "-c", str(src), "-o", str(tmp_path / "h.o")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
