"""The C-ABI boundary: the library loads, exports every entry point that
include/conan_pm.h declares, and rejects bad arguments with an error code
and message before touching a GPU (the reference throws a string,
src/base/main.cc:101-116)."""
import ctypes
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT


def header_functions():
    src = (ROOT / "include" / "conan_pm.h").read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"\b(conan_[a-z0-9_]+)\s*\(", src))
    names -= {"conan_step_cb"}
    return sorted(names)


def test_library_exports_every_declared_symbol(conan):
    lib = conan._lib.lib()
    names = header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(conan._lib.LIB_PATH)], capture_output=True, text=True)
    exported = set(re.findall(r"\bT (conan_[a-z0-9_]+)", out.stdout))
    assert set(names) <= exported


def test_binding_declares_exactly_the_header(conan):
    assert set(conan._lib.SIGNATURES) == set(header_functions())


def test_library_links_cufft_and_builds_for_sm100a():
    lib = ROOT / "conan_b200" / "lib" / "libconan_pm.so"
    ldd = subprocess.run(["ldd", str(lib)], capture_output=True, text=True).stdout
    assert "libcufft" in ldd
    from conan_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)


def test_version_and_error_strings(conan):
    lib = conan._lib.lib()
    assert b"sm_100a" in lib.conan_version()


def _pm(**kw):
    from conan_b200 import _lib as L
    p = L.PMParams()
    p.dim, p.n_mass, p.f, p.size, p.H0, p.Omega_m, p.Omega_L = 3, 16, 1, 10.0, 68.5, 1.0, 0.0
    for k, v in kw.items():
        setattr(p, k, v)
    return p


@pytest.mark.parametrize("kw,msg", [({"dim": 4}, "dimensions"), ({"dim": 0}, "dimensions"),
                                    ({"n_mass": 12}, "power of two"), ({"f": 3}, "power of two"),
                                    ({"size": -1.0}, "size"), ({"precision": 7}, "precision"),
                                    ({"gradient": 9}, "gradient"), ({"n_mass": 2048, "f": 2}, "exceeds")])
def test_pm_create_rejects_bad_parameters(conan, kw, msg):
    lib = conan._lib.lib()
    p = _pm(**kw)
    h = lib.conan_pm_create(ctypes.byref(p))
    assert not h
    assert msg in conan._lib.last_error()


def test_null_handles_and_pointers(conan):
    lib = conan._lib.lib()
    assert lib.conan_pm_kick(None, 0.1, 0.01) == conan._lib.ERR_ARG
    assert "null" in conan._lib.last_error()
    assert lib.conan_pm_create(None) is None
    assert lib.conan_diff_create(None) is None
    assert lib.conan_ens_create(None, 0, None) is None
    lib.conan_pm_destroy(None)  # no-op


@pytest.mark.parametrize("kw,code", [({"dim": 5}, 7), ({"mbits": 0}, 1), ({"size": 0.0}, 1), ({"precision": 3}, 1)])
def test_ic_rejects_bad_parameters(conan, kw, code):
    from conan_b200 import _lib as L
    p = L.ICParams()
    p.dim, p.mbits, p.size, p.scale, p.sigma = 3, 4, 10.0, 8.0, 0.83
    for k, v in kw.items():
        setattr(p, k, v)
    out = np.empty(16 ** 3)
    assert L.lib().conan_ic_generate(ctypes.byref(p), None, L.ptr(out)) == code


def test_python_api_raises(conan):
    with pytest.raises(conan.ConanError, match="power of two"):
        conan.Gravity(3, 12, 1, 10.0)
    with pytest.raises(conan.ConanError):
        conan.generate_random_field({"dim": 7, "mbits": 3})
