"""CPU-side checks of the C ABI: the library loads and exports every symbol that
include/*.h declares, and host logic that needs no GPU behaves like the reference."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "grid-mg-bench_b200", "libgmg_b200.so")


def declared_symbols():
    syms = set()
    for name in os.listdir(os.path.join(ROOT, "include")):
        if not name.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", name)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(gmg_\w+)\s*\(", text):
            syms.add(m.group(1))
    return syms


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        import sys
        sys.path.insert(0, os.path.join(ROOT, "grid-mg-bench_b200"))
        import build
        build.build()
    return ctypes.CDLL(LIB)


def test_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert len(syms) > 20
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if l.strip()}
    missing = sorted(s for s in syms if s not in exported)
    assert not missing, missing
    for s in syms:
        getattr(lib, s)


def test_point_map_matches_oracle(lib):
    for ndim in (4, 5):
        for faster in (0, 1):
            dirs, disps = orc.geometry(ndim, faster)
            for p in range(9):
                assert lib.gmg_point_from_dir_disp(ndim, faster, dirs[p], disps[p]) == p
    assert lib.gmg_point_from_dir_disp(4, 1, 0, 2) == -1


@pytest.mark.parametrize("mask_kind", [-1, 0, 3, 4, 7, 9, 10])
def test_lut_bit_exact_vs_oracle(lib, mask_kind):
    fd, cd = (8, 4, 8, 4), (2, 2, 2, 1)
    b = [f // c for f, c in zip(fd, cd)]
    bv = int(np.prod(b))
    Vc, Vf = int(np.prod(cd)), int(np.prod(fd))
    l = np.zeros((Vc, bv), np.int32)
    s = np.zeros(Vc, np.int32)
    r = np.zeros(Vf, np.int32)
    i4 = lambda d: (ctypes.c_int * 4)(*d)
    st = lib.gmg_lut_build(i4(fd), i4(cd), mask_kind, l.ctypes.data_as(ctypes.c_void_p),
                           s.ctypes.data_as(ctypes.c_void_p), r.ctypes.data_as(ctypes.c_void_p))
    assert st == 0
    if mask_kind == -1:
        mask = None
    elif mask_kind < 8:
        mask = orc.outer_mask(fd, cd, mask_kind)
    else:
        mask = orc.parity_mask(fd, cd, mask_kind - 9)
    lo, so, ro = orc.lut(fd, cd, mask)
    assert np.array_equal(l, lo) and np.array_equal(s, so) and np.array_equal(r, ro)


def test_bad_arguments_return_status(lib):
    lib.gmg_last_error.restype = ctypes.c_char_p
    h = ctypes.c_void_p()
    bad = (ctypes.c_int * 4)(4, 4, 0, 4)
    assert lib.gmg_coarse_create(bad, 8, 0, ctypes.byref(h)) == 2  # GMG_ERR_SHAPE
    assert b"extent" in lib.gmg_last_error()
    ok = (ctypes.c_int * 4)(4, 4, 4, 4)
    assert lib.gmg_coarse_create(ok, 7, 0, ctypes.byref(h)) == 1  # odd nbasis
    assert lib.gmg_lut_build(ok, (ctypes.c_int * 4)(3, 4, 4, 4), -1, None, None, None) == 1


def test_mg_params_layout_and_defaults(lib, tmp_path):
    # the Python binding's gmg_mg_params matches the C layout field by field,
    # and the defaults carry MultiGridParams' refinement defaults
    # (MultigridParams.h:99, :105: setupRefinementIter {0, 0},
    # setupRecursiveUpdates true)
    import sys
    sys.path.insert(0, os.path.join(ROOT, "grid-mg-bench_b200"))
    import gmg
    fields = [f[0] for f in gmg.MGParams._fields_]
    src = tmp_path / "layout.c"
    body = "".join(f'  printf("%zu\\n", offsetof(gmg_mg_params, {f}));\n' for f in fields)
    src.write_text('#include <stdio.h>\n#include "gmg.h"\nint main(void) {\n'
                   '  printf("%zu\\n", sizeof(gmg_mg_params));\n' + body + "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(gmg.MGParams)] + [getattr(gmg.MGParams, f).offset for f in fields]
    assert got == want
    p = gmg.MGParams()
    lib.gmg_mg_params_default.argtypes = [ctypes.c_void_p]
    assert lib.gmg_mg_params_default(ctypes.addressof(p)) == 0
    assert list(p.refine_iters) == [0, 0] and p.recursive_updates == 1
    assert p.nlevels == 3 and list(p.nvec) == [12, 16] and p.graph == 1
    # the refinement checks its handle before touching the device
    assert lib.gmg_mg_refine(None, None) != 0
