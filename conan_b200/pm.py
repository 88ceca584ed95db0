"""Python mirror of the reference's `ic` and `run` interfaces over libconan_pm.so.

Names and argument meaning follow the reference:
  generate_random_field(H) / compute_potential(H, D) / compute_displacement(H, D)
      src/ic/ic.hh:14-17 (H: the `ic` header keys dim, mbits, size, ns,
      smooth, scale-free, scale, sigma, seed, Omega0, H0)
  Gravity (a Solver: init / kick / drift / save_snapshot)
      src/run/leapfrog.hh:6-15, src/run/nbody.hh:53-219
  LeapFrog(a0, da, n).run(solver)   src/run/leapfrog.hh:23-47
  Cosmology(H0, Omega_m, Omega_L)   src/run/cosmology.hh:6-28

Meshes are flat float64 arrays with axis 0 fastest (reshape with
``order="F"``); particle arrays are (N^dim, dim) like mVector<double,R>.
Every call runs on the GPU; errors raise ConanError with the library's
message (the reference throws strings, src/base/main.cc:101-116).
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Dict, Optional

import numpy as np

from . import _lib as L

_PREC = {"fp32": L.FP32, "float32": L.FP32, "fp64": L.FP64, "float64": L.FP64}
_GRAD = {"fd4": L.GRAD_FD4, "spectral": L.GRAD_SPECTRAL}


def _truthy(v) -> bool:
    if isinstance(v, str):
        return v.strip() not in ("", "0", "false", "False")
    return bool(v)


def ic_params(H: Dict, precision: str = "fp64", device: int = 0) -> L.ICParams:
    """ICParams from `ic` options / header keys (defaults of src/ic/main.cc:15-65)."""
    g = lambda k, d: H.get(k, d)  # noqa: E731
    p = L.ICParams()
    p.dim = int(g("dim", 3))
    p.mbits = int(g("mbits", 8))
    p.size = float(g("size", 100.0))
    p.seed = int(g("seed", 0))
    p.ns = float(g("ns", 0.96))
    p.smooth = int(_truthy(g("smooth", False)))
    p.scale_free = int(_truthy(g("scale-free", g("scale_free", False))))
    p.scale = float(g("scale", 8.0))
    p.sigma = float(g("sigma", 0.83))
    p.Omega0 = float(g("Omega0", 0.32))
    p.H0 = float(g("H0", 69.0))
    p.precision = _PREC[precision]
    p.device = device
    return p


def _ncells(p: L.ICParams) -> int:
    return (1 << p.mbits) ** p.dim


def white_noise(H: Dict, device: int = 0) -> np.ndarray:
    """Philox white noise of the GPU generator (N^dim unit normals)."""
    p = ic_params(H, device=device)
    out = np.empty(_ncells(p))
    L.check(L.lib().conan_ic_noise(C.byref(p), L.ptr(out)))
    return out


def generate_random_field(H: Dict, noise: Optional[np.ndarray] = None, precision: str = "fp64",
                          device: int = 0) -> np.ndarray:
    """Conan::generate_random_field. `noise` (N^dim unit normals in memory
    order) replaces the GPU Philox noise, e.g. with the reference's mt19937
    sequence for bit-level parity."""
    p = ic_params(H, precision, device)
    out = np.empty(_ncells(p))
    nz = None if noise is None else np.ascontiguousarray(noise, dtype=np.float64)
    if nz is not None and nz.size != out.size:
        raise ValueError("noise has the wrong size")
    L.check(L.lib().conan_ic_generate(C.byref(p), L.ptr(nz), L.ptr(out)))
    return out


def compute_potential(H: Dict, data: np.ndarray, precision: str = "fp64", device: int = 0) -> np.ndarray:
    """Conan::compute_potential (returns the potential; the input is kept)."""
    p = ic_params(H, precision, device)
    out = np.array(data, dtype=np.float64, copy=True).ravel()
    L.check(L.lib().conan_ic_potential(C.byref(p), L.ptr(out)))
    return out


def compute_displacement(H: Dict, potential: np.ndarray, precision: str = "fp64",
                         device: int = 0) -> np.ndarray:
    """Conan::compute_displacement record, shape (N^dim, dim)."""
    p = ic_params(H, precision, device)
    pot = np.ascontiguousarray(potential, dtype=np.float64).ravel()
    out = np.empty((_ncells(p), p.dim))
    L.check(L.lib().conan_ic_displacement(C.byref(p), L.ptr(pot), L.ptr(out)))
    return out


def cic(X: np.ndarray, dim: int, n_mass: int, L_box: float, f: int = 2, sub_sample: int = 1,
        device: int = 0) -> np.ndarray:
    """The `cic` tool, cic_run<R> (src/cic/cic.hh:49-81): density of a
    snapshot's positions X (n_mass^dim x dim, absolute) on the (f n_mass)^dim
    mesh, optionally from a sub_sample-times finer interpolated grid."""
    p = L.CicParams()
    p.dim, p.n_mass, p.f, p.size, p.sub_sample, p.device = dim, n_mass, f, float(L_box), sub_sample, device
    x = np.ascontiguousarray(X, dtype=np.float64)
    if x.size != n_mass ** dim * dim:
        raise ValueError(f"expected {n_mass ** dim} x {dim} positions, got {x.shape}")
    out = np.empty((n_mass * f) ** dim)
    L.check(L.lib().conan_cic(C.byref(p), L.ptr(x), L.ptr(out)))
    return out


def _fof_params(dim, n, L_box, linking_length, device):
    p = L.FofParams()
    p.dim, p.n_particles, p.size, p.linking_length, p.device = dim, n, float(L_box), float(linking_length), device
    return p


def fof(X: np.ndarray, dim: int, L_box: float, linking_length: float, device: int = 0):
    """The `fof` tool's groups, fof_run<R> (src/fof/fof.cc:164-231): returns
    (tags, n_groups) for the positions X (n x dim, not wrapped); tags[i] is
    particle i's group, numbered from 1 in the order of the groups' lowest
    particle index, as the reference's tags."""
    x = np.ascontiguousarray(X, dtype=np.float64)
    if x.size % dim:
        raise ValueError(f"positions of shape {x.shape} are not n x {dim}")
    n = x.size // dim
    tags = np.empty(n, dtype=np.uint64)
    ng = C.c_ulonglong(0)
    L.check(L.lib().conan_fof(C.byref(_fof_params(dim, n, L_box, linking_length, device)), L.ptr(x),
                              tags.ctypes.data_as(C.c_void_p), C.byref(ng)))
    return tags, int(ng.value)


class FoF:
    """Friends-of-friends with the device buffers kept between calls
    (conan_fof_create / conan_fof_run / conan_fof_run_device)."""

    def __init__(self, dim: int, n: int, L_box: float, linking_length: float, device: int = 0):
        self.dim, self.n = dim, n
        self.h = L.lib().conan_fof_create(C.byref(_fof_params(dim, n, L_box, linking_length, device)))
        if not self.h:
            raise L.ConanError(L.ERR_ALLOC, L.last_error())

    def __call__(self, X: np.ndarray):
        x = np.ascontiguousarray(X, dtype=np.float64)
        if x.size != self.n * self.dim:
            raise ValueError(f"expected {self.n} x {self.dim} positions, got {x.shape}")
        tags = np.empty(self.n, dtype=np.uint64)
        ng = C.c_ulonglong(0)
        L.check(L.lib().conan_fof_run(self.h, L.ptr(x), tags.ctypes.data_as(C.c_void_p), C.byref(ng)))
        return tags, int(ng.value)

    def run_device(self, x_ptr: int, tags_ptr: int, stream: int = 0) -> int:
        """Device pointers (n x dim doubles in, n uint64 tags out); returns the group count."""
        ng = C.c_ulonglong(0)
        L.check(L.lib().conan_fof_run_device(self.h, C.c_void_p(x_ptr), C.c_void_p(tags_ptr), C.byref(ng),
                                             C.c_void_p(stream)))
        return int(ng.value)

    def close(self):
        if getattr(self, "h", None):
            L.lib().conan_fof_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: the module's globals may be gone
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Cosmology:
    """src/run/cosmology.hh:6-28."""

    def __init__(self, H0: float = 68.5, Omega_m: float = 1.0, Omega_L: float = 0.0):
        self.H0, self.Omega_m, self.Omega_L = H0, Omega_m, Omega_L
        self.Omega_k = 1 - Omega_m - Omega_L
        self.grav_cst = 3.0 / 2 * Omega_m * H0 * H0

    def __call__(self, a: float) -> float:
        return self.H0 * a * np.sqrt(self.Omega_L + self.Omega_m * a ** -3.0 + self.Omega_k * a ** -2.0)

    def G(self) -> float:
        return self.grav_cst


class Gravity:
    """The PM solver: the reference's Gravity<R> on the GPU."""

    def __init__(self, dim: int, n_mass: int, f: int, L_box: float, cosmology: Cosmology = None,
                 precision: str = "fp32", gradient: str = "fd4", periodic_gather: bool = False,
                 device: int = 0):
        c = cosmology or Cosmology()
        p = L.PMParams()
        p.dim, p.n_mass, p.f, p.size = dim, n_mass, f, L_box
        p.H0, p.Omega_m, p.Omega_L = c.H0, c.Omega_m, c.Omega_L
        p.precision = _PREC[precision]
        p.gradient = _GRAD[gradient]
        p.periodic_gather = int(periodic_gather)
        p.device = device
        self.params = p
        self.dim, self.n_mass, self.f, self.L = dim, n_mass, f, L_box
        self.np = n_mass ** dim
        self.ncells = (n_mass * f) ** dim
        h = L.lib().conan_pm_create(C.byref(p))
        if not h:
            raise L.ConanError(L.ERR_ARG, L.last_error())
        self._h = h
        self._cb = None

    # -- Solver interface -------------------------------------------------
    def init(self, phi: np.ndarray, a_pos: float, a_mom: float):
        phi = np.ascontiguousarray(phi, dtype=np.float64).ravel()
        if phi.size != self.np:
            raise ValueError("potential must have N^dim values")
        L.check(L.lib().conan_pm_init(self._h, L.ptr(phi), a_pos, a_mom))

    def kick(self, a: float, da: float):
        L.check(L.lib().conan_pm_kick(self._h, a, da))

    def drift(self, a: float, da: float):
        L.check(L.lib().conan_pm_drift(self._h, a, da))

    def run(self, phi: Optional[np.ndarray], a0: float, da: float, n: int,
            callback: Optional[Callable[[int, float], Optional[bool]]] = None, every: int = 1):
        """LeapFrog::run from phi (None: continue from the current state)."""
        ph = None if phi is None else np.ascontiguousarray(phi, dtype=np.float64).ravel()
        L.check(L.lib().conan_pm_set_callback_interval(self._h, every))
        if callback is None:
            cb = L.STEP_CB()
        else:
            def _cb(h, step, a, user):
                r = callback(int(step), float(a))
                return 1 if r is False else 0
            cb = L.STEP_CB(_cb)
        self._cb = cb
        L.check(L.lib().conan_pm_run(self._h, L.ptr(ph), a0, da, n, cb, None))

    # -- state ----------------------------------------------------------------
    def state(self):
        X = np.empty((self.np, self.dim))
        P = np.empty((self.np, self.dim))
        L.check(L.lib().conan_pm_get_state(self._h, L.ptr(X), L.ptr(P)))
        return X, P

    def state_into(self, X: np.ndarray, P: np.ndarray):
        """Absolute state into caller-owned (e.g. pinned) float64 arrays of
        shape (N^dim, dim); either may be None."""
        for a in (X, P):
            if a is not None and (a.dtype != np.float64 or a.size != self.np * self.dim
                                  or not a.flags.c_contiguous):
                raise ValueError("state arrays must be C-contiguous float64 of N^dim x dim")
        L.check(L.lib().conan_pm_get_state(self._h, L.ptr(X), L.ptr(P)))

    def set_state(self, X, P, a_pos: float, a_mom: float):
        X = np.ascontiguousarray(X, dtype=np.float64)
        P = np.ascontiguousarray(P, dtype=np.float64)
        L.check(L.lib().conan_pm_set_state(self._h, L.ptr(X), L.ptr(P), a_pos, a_mom))

    def scale_factors(self):
        a, b = C.c_double(), C.c_double()
        L.check(L.lib().conan_pm_scale_factors(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def density(self) -> np.ndarray:
        out = np.empty(self.ncells)
        L.check(L.lib().conan_pm_density(self._h, L.ptr(out)))
        return out

    def potential(self) -> np.ndarray:
        out = np.empty(self.ncells)
        L.check(L.lib().conan_pm_potential(self._h, L.ptr(out)))
        return out

    def power_spectrum(self, nbins: Optional[int] = None):
        nb = nbins or (self.n_mass * self.f) // 2 + 1
        k, P, c = np.empty(nb), np.empty(nb), np.empty(nb)
        L.check(L.lib().conan_pm_power_spectrum(self._h, nb, L.ptr(k), L.ptr(P), L.ptr(c)))
        return k, P, c

    # -- profiling ------------------------------------------------------------
    def set_profiling(self, on: bool = True):
        L.check(L.lib().conan_pm_set_profiling(self._h, int(on)))

    def profile(self) -> Dict[str, tuple]:
        out = {}
        i = 0
        name = C.create_string_buffer(64)
        n = C.c_int()
        ms = C.c_double()
        while L.lib().conan_pm_profile_entry(self._h, i, name, C.byref(n), C.byref(ms)) == L.OK:
            out[name.value.decode()] = (n.value, ms.value)
            i += 1
        return out

    def profile_reset(self):
        L.check(L.lib().conan_pm_profile_reset(self._h))

    def device_bytes(self) -> int:
        b = C.c_size_t()
        L.check(L.lib().conan_pm_device_bytes(self._h, C.byref(b)))
        return b.value

    def sync(self):
        L.check(L.lib().conan_pm_sync(self._h))

    @property
    def deposit_mode(self) -> str:
        """"sorted" (counting sort + tiled reduction) or "lagrangian"
        (lattice tiles into shared-memory windows, FP32)."""
        m = C.c_int()
        L.check(L.lib().conan_pm_get_deposit(self._h, C.byref(m)))
        return "lagrangian" if m.value == L.DEPOSIT_LAGRANGIAN else "sorted"

    @deposit_mode.setter
    def deposit_mode(self, mode: str):
        L.check(L.lib().conan_pm_set_deposit(self._h, {"sorted": L.DEPOSIT_SORTED,
                                                       "lagrangian": L.DEPOSIT_LAGRANGIAN}[mode]))

    def autotune(self, a: float, da: float) -> list:
        """Times the deposit and gradient-mesh variants over leapfrog steps
        from the current state (scale factor a of the next drift, step da)
        and keeps the fastest; the state is left as it was. Returns the
        timings: [{knob, value, ms_per_step, chosen}, ...]."""
        import json
        buf = C.create_string_buffer(16384)
        L.check(L.lib().conan_pm_autotune(self._h, a, da, buf, len(buf)))
        return json.loads(buf.value.decode())

    def stream_ptr(self) -> int:
        """The handle's cudaStream_t as an integer (torch.cuda.ExternalStream)."""
        s = C.c_void_p()
        L.check(L.lib().conan_pm_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def close(self):
        if getattr(self, "_h", None):
            L.lib().conan_pm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class LeapFrog:
    """src/run/leapfrog.hh:23-47 over any object with init/kick/drift."""

    def __init__(self, a0: float, da: float, n: int):
        self.a0, self.da, self.n = a0, da, n

    def run(self, solver, phi=None, save_snapshot=None):
        solver.init(phi, self.a0, self.a0 + self.da / 2)
        a = self.a0
        for i in range(self.n):
            solver.drift(a, self.da)
            solver.kick(a + self.da / 2, self.da)
            a += self.da
            if save_snapshot:
                save_snapshot(i, a)
