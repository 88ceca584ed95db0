"""torch.autograd binding of the differentiable PM model (conan_diff_*).

    model = DiffPM(dim=3, mbits=7, L=100.0, ns=-2.0, a0=0.05, da=0.0296875, n=32)
    delta = model(noise)            # noise: (N^dim,) CUDA tensor, float32/float64
    loss = ((delta - target) ** 2).mean()
    loss.backward()                 # noise.grad via the hand-written adjoint

The forward runs the initial conditions (scale-free Gaussian random field,
potential, Zel'dovich start), n leapfrog steps and the final CIC deposit on
the GPU; backward runs the adjoint of all of it (reversible leapfrog with an
exact checkpoint every `checkpoint_every` steps). Tensors are flat with axis
0 fastest, the reference's mesh layout. One model holds the state of its last
forward: call backward before the next forward of the same model.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib as L


class DiffPM:
    def __init__(self, dim: int = 3, mbits: int = 7, L_box: float = 100.0, ns: float = -2.0,
                 smooth: bool = False, scale: float = 8.0, sigma: float = 0.83, a0: float = 0.05,
                 da: float = 0.0296875, n: int = 32, checkpoint_every: int = 8, f: int = 1,
                 precision: str = "fp32", H0: float = 68.5, Omega_m: float = 1.0, Omega_L: float = 0.0,
                 periodic_gather: bool = False, device: int = 0):
        p = L.DiffParams()
        prec = {"fp32": L.FP32, "fp64": L.FP64}[precision]
        p.ic.dim, p.ic.mbits, p.ic.size, p.ic.ns = dim, mbits, L_box, ns
        p.ic.smooth, p.ic.scale_free, p.ic.scale, p.ic.sigma = int(smooth), 1, scale, sigma
        p.ic.Omega0, p.ic.H0, p.ic.precision, p.ic.device = 0.32, 69.0, prec, device
        p.pm.dim, p.pm.n_mass, p.pm.f, p.pm.size = dim, 1 << mbits, f, L_box
        p.pm.H0, p.pm.Omega_m, p.pm.Omega_L = H0, Omega_m, Omega_L
        p.pm.precision, p.pm.gradient, p.pm.periodic_gather, p.pm.device = prec, L.GRAD_FD4, int(periodic_gather), device
        p.a0, p.da, p.n, p.checkpoint_every = a0, da, n, checkpoint_every
        self.params = p
        self.dtype = torch.float32 if precision == "fp32" else torch.float64
        self.device = torch.device("cuda", device)
        self.nnoise = (1 << mbits) ** dim
        self.ncells = ((1 << mbits) * f) ** dim
        h = L.lib().conan_diff_create(C.byref(p))
        if not h:
            raise L.ConanError(L.ERR_ARG, L.last_error())
        self._h = h

    def _check(self, t, n, name):
        if t.dtype != self.dtype or t.device != self.device or t.numel() != n or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous {self.dtype} tensor of {n} values on {self.device}")

    def forward_raw(self, noise: torch.Tensor, out: torch.Tensor):
        self._check(noise, self.nnoise, "noise")
        self._check(out, self.ncells, "density")
        s = torch.cuda.current_stream(self.device).cuda_stream
        L.check(L.lib().conan_diff_forward(self._h, C.c_void_p(noise.data_ptr()), C.c_void_p(out.data_ptr()),
                                           C.c_void_p(s)))

    def backward_raw(self, gdens: torch.Tensor, gnoise: torch.Tensor):
        self._check(gdens, self.ncells, "density gradient")
        self._check(gnoise, self.nnoise, "noise gradient")
        s = torch.cuda.current_stream(self.device).cuda_stream
        L.check(L.lib().conan_diff_backward(self._h, C.c_void_p(gdens.data_ptr()), C.c_void_p(gnoise.data_ptr()),
                                            C.c_void_p(s)))

    def __call__(self, noise: torch.Tensor) -> torch.Tensor:
        return PMDensity.apply(noise, self)

    def close(self):
        if getattr(self, "_h", None):
            L.lib().conan_diff_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PMDensity(torch.autograd.Function):
    """delta_final = PM(noise); backward = the hand-written adjoint."""

    @staticmethod
    def forward(ctx, noise, model: DiffPM):
        noise = noise.detach().contiguous()
        out = torch.empty(model.ncells, dtype=model.dtype, device=model.device)
        model.forward_raw(noise, out)
        ctx.model = model
        return out

    @staticmethod
    def backward(ctx, g):
        model = ctx.model
        gn = torch.empty(model.nnoise, dtype=model.dtype, device=model.device)
        model.backward_raw(g.contiguous(), gn)
        return gn, None


def benchmark_adjoint_ratio(device: int = 0, mbits: int = 7, steps: int = 32, repeat: int = 3):
    """Forward and adjoint time of the differentiable 128^3 box (L=100,
    n_s=-2, 32 steps a=0.05..1, checkpoint every 8), FP32, CUDA events."""
    torch.cuda.set_device(device)
    da = 0.95 / steps
    m = DiffPM(dim=3, mbits=mbits, L_box=100.0, ns=-2.0, a0=0.05, da=da, n=steps, checkpoint_every=8,
               device=device)
    g = torch.Generator(device="cuda").manual_seed(4)
    noise = torch.randn(m.nnoise, device=m.device, dtype=m.dtype, generator=g)
    out = torch.empty(m.ncells, device=m.device, dtype=m.dtype)
    gn = torch.empty_like(noise)
    gd = torch.randn(m.ncells, device=m.device, dtype=m.dtype, generator=g) * 1e-6
    m.forward_raw(noise, out)
    m.backward_raw(gd, gn)
    fw, bw = [], []
    for _ in range(repeat):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        e[0].record()
        m.forward_raw(noise, out)
        e[1].record()
        m.backward_raw(gd, gn)
        e[2].record()
        torch.cuda.synchronize()
        fw.append(e[0].elapsed_time(e[1]))
        bw.append(e[1].elapsed_time(e[2]))
    m.close()
    f, b = min(fw), min(bw)
    return {"forward_ms": f, "adjoint_ms": b, "adjoint_over_forward": b / f,
            "config": f"3D {1 << mbits}^3 particles/mesh, L=100, ns=-2, {steps} steps a=0.05->1, checkpoint 8, FP32"}
