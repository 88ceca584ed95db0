"""ctypes wrappers of liboracle.so (FP64 CPU restatement; test infrastructure).

Arrays follow the reference layout: meshes flat with axis 0 fastest,
particle vectors (n, dim). Functions cite the reference code they restate in
conan_oracle.cc.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
_d = C.c_double
_lib = None


def build():
    """Builds liboracle.so (and _ref/ when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB))
        _lib.oracle_adot.restype = C.c_double
    return _lib


def P(a):
    return a.ctypes.data_as(C.c_void_p)


def noise_mt19937(seed: int, n: int) -> np.ndarray:
    out = np.empty(n)
    lib().oracle_noise_mt19937(C.c_ulong(seed), C.c_size_t(n), P(out))
    return out


def dft(a: np.ndarray, dim: int, N: int, sign: int = -1) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.complex128)
    out = np.empty_like(a)
    lib().oracle_dft(dim, N, P(a), P(out), sign)
    return out


def grf_scale_free(dim, mbits, L, ns, smooth, scale, sigma, noise) -> np.ndarray:
    noise = np.ascontiguousarray(noise, dtype=np.float64)
    out = np.empty_like(noise)
    lib().oracle_grf_scale_free(dim, mbits, _d(L), _d(ns), int(smooth), _d(scale), _d(sigma), P(noise), P(out))
    return out


def grf_cdm(dim, mbits, L, Omega0, H0, ns, noise) -> np.ndarray:
    noise = np.ascontiguousarray(noise, dtype=np.float64)
    out = np.empty_like(noise)
    lib().oracle_grf_cdm(dim, mbits, _d(L), _d(Omega0), _d(H0), _d(ns), P(noise), P(out))
    return out


def potential(dim, mbits, L, dens) -> np.ndarray:
    out = np.array(dens, dtype=np.float64, copy=True)
    lib().oracle_potential(dim, mbits, _d(L), P(out))
    return out


def displacement(dim, mbits, L, pot) -> np.ndarray:
    pot = np.ascontiguousarray(pot, dtype=np.float64)
    out = np.empty((pot.size, dim))
    lib().oracle_displacement(dim, mbits, _d(L), P(pot), P(out))
    return out


def zeldovich(dim, Nm, L, phi, a_pos, a_mom):
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    X = np.empty((phi.size, dim))
    Pm = np.empty((phi.size, dim))
    lib().oracle_zeldovich(dim, Nm, _d(L), P(phi), _d(a_pos), _d(a_mom), P(X), P(Pm))
    return X, Pm


def md_cic(dim, N, L, X, m=1.0) -> np.ndarray:
    X = np.ascontiguousarray(X, dtype=np.float64)
    out = np.empty(N ** dim)
    lib().oracle_md_cic(dim, N, _d(L), P(X), C.c_size_t(X.size // dim), _d(m), P(out))
    return out


def cic(dim, N, L, f, s, X) -> np.ndarray:
    """The `cic` tool's density of a snapshot (cic_run, src/cic/cic.hh:49-81)."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    out = np.empty((N * f) ** dim)
    lib().oracle_cic(dim, N, _d(L), f, s, P(X), P(out))
    return out


def poisson(dim, N, L, G, a, delta_plus_one) -> np.ndarray:
    out = np.array(delta_plus_one, dtype=np.float64, copy=True)
    lib().oracle_poisson(dim, N, _d(L), _d(G), _d(a), P(out))
    return out


def interp_gradient(dim, N, L, phi, X) -> np.ndarray:
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    X = np.ascontiguousarray(X, dtype=np.float64)
    out = np.empty_like(X)
    lib().oracle_interp_gradient(dim, N, _d(L), P(phi), P(X), C.c_size_t(X.size // dim), P(out))
    return out


def adot(H0, Om, OL, a) -> float:
    return lib().oracle_adot(_d(H0), _d(Om), _d(OL), _d(a))


def kick(dim, Nm, f, L, H0, Om, OL, X, Pm, a, da, want_phi=False):
    phi = np.empty((Nm * f) ** dim) if want_phi else None
    lib().oracle_kick(dim, Nm, f, _d(L), _d(H0), _d(Om), _d(OL), P(X), P(Pm), _d(a), _d(da),
                      P(phi) if want_phi else None)
    return phi


def drift(dim, Nm, H0, Om, OL, X, Pm, a, da):
    lib().oracle_drift(dim, Nm, _d(H0), _d(Om), _d(OL), P(X), P(Pm), _d(a), _d(da))


def run(dim, Nm, f, L, H0, Om, OL, phi, a0, da, n):
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    X = np.empty((Nm ** dim, dim))
    Pm = np.empty((Nm ** dim, dim))
    lib().oracle_run(dim, Nm, f, _d(L), _d(H0), _d(Om), _d(OL), P(phi), _d(a0), _d(da), C.c_uint(n), P(X), P(Pm))
    return X, Pm


def power_spectrum(dim, N, L, delta, nbins=None):
    nb = nbins or N // 2 + 1
    delta = np.ascontiguousarray(delta, dtype=np.float64)
    k, p, c = np.empty(nb), np.empty(nb), np.empty(nb)
    lib().oracle_power_spectrum(dim, N, _d(L), P(delta), nb, P(k), P(p), P(c))
    return k, p, c


def diff_forward(dim, mbits, f, L, ns, smooth, scale, sigma, a0, da, n, noise, H0=68.5, Om=1.0, OL=0.0):
    """Final CIC density contrast of the differentiable model (FP64 CPU)."""
    noise = np.ascontiguousarray(noise, dtype=np.float64)
    out = np.empty(((1 << mbits) * f) ** dim)
    lib().oracle_diff_forward(dim, mbits, f, _d(L), _d(ns), int(smooth), _d(scale), _d(sigma), _d(H0), _d(Om),
                              _d(OL), _d(a0), _d(da), C.c_uint(n), P(noise), P(out))
    return out


def diff_adjoint(dim, mbits, f, L, ns, smooth, scale, sigma, a0, da, n, noise, deltabar, H0=68.5, Om=1.0,
                 OL=0.0):
    """(final density contrast, dL/dnoise) for dL/d(density) = deltabar (FP64 CPU adjoint)."""
    noise = np.ascontiguousarray(noise, dtype=np.float64)
    deltabar = np.ascontiguousarray(deltabar, dtype=np.float64)
    dens = np.empty(deltabar.size)
    gb = np.empty_like(noise)
    lib().oracle_diff_adjoint(dim, mbits, f, _d(L), _d(ns), int(smooth), _d(scale), _d(sigma), _d(H0), _d(Om),
                              _d(OL), _d(a0), _d(da), C.c_uint(n), P(noise), P(deltabar), P(dens), P(gb))
    return dens, gb


def fof(dim, L, ll, X):
    """Friends-of-friends tags and group count (fof_run, src/fof/fof.cc:164-231)."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    n = X.size // dim
    tags = np.empty(n, dtype=np.uint64)
    f = lib().oracle_fof
    f.restype = C.c_ulonglong
    ng = f(dim, C.c_size_t(n), _d(L), _d(ll), P(X), P(tags))
    return tags, int(ng)


def _ref_modulus(a, b):
    """modulus(double, double), src/base/misc.hh:144-148 (truncating casts)."""
    return a - int(a / b - 1) * b if a < 0 else a - int(a / b) * b


def fof_report(X, tags, L) -> str:
    """The text fof_run writes after the header and history (src/fof/fof.cc:
    233-279), from the tags: groups of at least 10 particles with the first
    member's wrapped position, mass and 0-based number; two newlines; every
    group's members in index order with random_colour(t) = srand(t);
    rand() % 1022 (libc's own generator). Doubles as std::ostream prints them
    (%g)."""
    libc = C.CDLL(None)
    X = np.asarray(X, dtype=np.float64)
    tags = np.asarray(tags, dtype=np.int64)
    dim = X.shape[1]
    ng = int(tags.max()) if tags.size else 0
    order = np.argsort(tags, kind="stable")
    mass = np.bincount(tags - 1, minlength=ng)
    first = np.full(ng, -1, dtype=np.int64)
    first[tags[order[np.r_[0, np.cumsum(mass)[:-1]]]] - 1] = order[np.r_[0, np.cumsum(mass)[:-1]]]
    vec = lambda x: "".join("%g " % v for v in x)  # noqa: E731
    out = []
    for t in range(ng):
        if mass[t] < 10:
            continue
        out.append(vec([_ref_modulus(float(v), L) for v in X[first[t]]]) + " %d %d\n" % (mass[t], t))
    out.append("\n\n")
    colour = []
    for t in range(ng):
        libc.srand(C.c_uint(t))
        colour.append(libc.rand() % 1022)
    for i in order:
        out.append(vec(X[i]) + " %d\n" % colour[tags[i] - 1])
    return "".join(out)


def fof_text_body(text: str) -> str:
    """The part of a fof output file after its header and history blocks."""
    lines = text.split("\n")
    h = lines.index("# history")
    e = lines.index("", h)
    return "\n".join(lines[e + 1:])
