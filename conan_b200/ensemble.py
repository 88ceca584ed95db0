"""Batched ensembles of independent PM boxes with uneven mesh sizes.

    ens = Ensemble.standard()        # the 96-box ensemble: 32 x 32^3, 32 x 64^3, 32 x 128^3
    ens.init()                       # ICs on the GPU, targets, autotuned deposit tiles
    ens.run()                        # all members, all steps: one CUDA graph launch
    loss = ens.forward_adjoint()     # forward + adjoint of every member
    k, P = ens.mean_power_spectrum(32)

Across GPUs the members are independent: `shard(members, rank, world)`
assigns members round-robin, each rank runs its share with no collective on
the data path, and `allreduce_mean_pk` combines the per-member spectra
(torch.distributed, any backend) into the ensemble mean.
"""
from __future__ import annotations

import ctypes as C
import json
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib as L


def standard_members(n_per_class: int = 32, sizes=(5, 6, 7), L_box: float = 100.0,
                     ns_choices=(-2.5, -2.0, -1.5, -1.0), rng_seed: int = 6, seed0: int = 1000):
    """Members of the 96-box ensemble: n_per_class boxes per mesh size
    (2^5, 2^6, 2^7 per side), L = 100, spectral index drawn uniformly from
    ns_choices with numpy default_rng(6), seeds 1000 + i."""
    rng = np.random.default_rng(rng_seed)
    out = []
    i = 0
    for mb in sizes:
        for _ in range(n_per_class):
            out.append((mb, L_box, float(rng.choice(ns_choices)), seed0 + i))
            i += 1
    return out


def shard(members: Sequence, rank: int, world: int) -> List:
    """Round-robin share of the members for one rank (no data exchange)."""
    return list(members[rank::world])


def allreduce_mean_pk(P: np.ndarray, count: np.ndarray, dist=None) -> np.ndarray:
    """Ensemble-mean power spectrum from per-member spectra of this rank:
    P[m, bin] and the number of members per bin; sums across ranks with
    torch.distributed when `dist` is given (the only collective)."""
    s = np.asarray(P, dtype=np.float64).sum(axis=0)
    c = np.asarray(count, dtype=np.float64)
    if dist is not None:
        import torch
        t = torch.tensor(np.concatenate([s, c]), dtype=torch.float64)
        dist.all_reduce(t)
        v = t.numpy()
        s, c = v[: s.size], v[s.size:]
    return np.where(c > 0, s / np.maximum(c, 1), 0.0)


class Ensemble:
    def __init__(self, members: Sequence[Tuple[int, float, float, int]], dim: int = 3, a0: float = 0.05,
                 a_end: float = 1.0, steps: int = 40, H0: float = 68.5, Omega_m: float = 1.0,
                 Omega_L: float = 0.0, sigma: float = 0.83, scale: float = 8.0, precision: str = "fp32",
                 device: int = 0, autotune: bool = True):
        p = L.EnsParams()
        p.dim, p.H0, p.Omega_m, p.Omega_L = dim, H0, Omega_m, Omega_L
        p.sigma, p.scale, p.a0, p.da, p.n = sigma, scale, a0, (a_end - a0) / steps, steps
        p.precision = {"fp32": L.FP32, "fp64": L.FP64}[precision]
        p.device, p.autotune = device, int(autotune)
        arr = (L.EnsMember * len(members))()
        for i, (mb, Lb, ns, seed) in enumerate(members):
            arr[i].mbits, arr[i].size, arr[i].ns, arr[i].seed = mb, Lb, ns, seed
        self.members = list(members)
        self.dim = dim
        h = L.lib().conan_ens_create(C.byref(p), len(members), arr)
        if not h:
            raise L.ConanError(L.ERR_ARG, L.last_error())
        self._h = h

    @classmethod
    def standard(cls, **kw):
        return cls(standard_members(), **kw)

    def init(self):
        L.check(L.lib().conan_ens_init(self._h))

    def run(self) -> float:
        L.check(L.lib().conan_ens_run(self._h))
        return self.last_ms()[0]

    def forward_adjoint(self) -> np.ndarray:
        loss = np.empty(len(self.members))
        L.check(L.lib().conan_ens_forward_adjoint(self._h, L.ptr(loss)))
        return loss

    def last_ms(self):
        r, a = C.c_double(), C.c_double()
        L.check(L.lib().conan_ens_last_ms(self._h, C.byref(r), C.byref(a)))
        return r.value, a.value

    def total_particles(self) -> int:
        n = C.c_size_t()
        L.check(L.lib().conan_ens_total_particles(self._h, C.byref(n)))
        return n.value

    def describe(self) -> dict:
        buf = C.create_string_buffer(65536)
        L.check(L.lib().conan_ens_describe(self._h, buf, len(buf)))
        return json.loads(buf.value.decode())

    def power_spectrum(self, member: int, nbins: Optional[int] = None):
        nb = nbins or (1 << self.members[member][0]) // 2 + 1
        k, P, c = np.empty(nb), np.empty(nb), np.empty(nb)
        L.check(L.lib().conan_ens_power_spectrum(self._h, member, nb, L.ptr(k), L.ptr(P), L.ptr(c)))
        return k, P, c

    def state(self, member: int):
        n = (1 << self.members[member][0]) ** self.dim
        X, P = np.empty((n, self.dim)), np.empty((n, self.dim))
        L.check(L.lib().conan_ens_state(self._h, member, L.ptr(X), L.ptr(P)))
        return X, P

    def member_fields(self, member: int, gradient: bool = True):
        """(white noise, target density, d loss / d noise) of a member; the
        gradient is that of the last forward_adjoint (None if gradient=False)."""
        n = (1 << self.members[member][0]) ** self.dim
        noise, target = np.empty(n), np.empty(n)
        g = np.empty(n) if gradient else None
        L.check(L.lib().conan_ens_member_fields(self._h, member, L.ptr(noise), L.ptr(target),
                                                L.ptr(g) if gradient else None))
        return noise, target, g

    def mean_power_spectrum(self, nbins: int, dist=None):
        """Mean P(k) over the members (and ranks), bins of width 2 pi / L."""
        Ps, cnt = [], np.zeros(nbins)
        k = None
        for i in range(len(self.members)):
            kk, P, c = self.power_spectrum(i, nbins)
            Ps.append(P)
            cnt += (c > 0)
            k = kk if k is None else np.where(c > 0, kk, k)
        return k, allreduce_mean_pk(np.array(Ps), cnt, dist)

    def close(self):
        if getattr(self, "_h", None):
            L.lib().conan_ens_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
