"""The benchmark configurations at their full sizes (seeded synthetic fields).

* 2D PM, 256^2 particles on 256^2 cells, L = 50, P(k) ~ k^-1, Zel'dovich at
  a = 0.02, 100 steps to a = 1, FP64: positions and final P(k) against the
  FP64 CPU oracle on the same mt19937 noise; FP32 against the same oracle.
* 3D PM, 128^3 on 128^3, L = 100, P(k) ~ k^-2 smoothed at one cell, 50 steps
  from a = 0.02: FP32 (lattice index + displacement) against FP64 on the GPU,
  final P(k) within 1e-3 and the position RMS in cells.
* The 96-box ensemble: ensemble-mean P(k) in FP32 against FP64.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pk_err(P, Pr, c):
    m = (c > 0) & (np.arange(len(c)) > 0)
    return float(np.max(np.abs(P[m] - Pr[m]) / Pr[m]))


def _dx_cells(X, Xr, cell, L):
    d = (X - Xr) / cell
    n = L / cell
    return (d + n / 2) % n - n / 2  # minimum image


def test_2d_256_fp64_and_fp32_against_the_oracle(gpu, conan, oracle):
    dim, mbits, L, ns = 2, 8, 50.0, -1.0
    N = 1 << mbits
    noise = oracle.noise_mt19937(1, N ** dim)
    dens = oracle.grf_scale_free(dim, mbits, L, ns, False, 8.0, 0.83, noise)
    phi = oracle.potential(dim, mbits, L, dens)
    a0, da, n = 0.02, 0.0098, 100
    Xr, Pr = oracle.run(dim, N, 1, L, 68.5, 1.0, 0.0, phi, a0, da, n)
    cell = L / N
    kr, Pkr, cr = oracle.power_spectrum(dim, N, L, oracle.md_cic(dim, N, L, Xr) - 1.0)
    for prec in ("fp64", "fp32"):
        g = conan.Gravity(dim, N, 1, L, precision=prec)
        g.run(phi, a0, da, n)
        X, P = g.state()
        k, Pk, c = g.power_spectrum(len(cr))
        g.close()
        dx = _dx_cells(X, Xr, cell, L)
        rms = float(np.sqrt(np.mean(dx ** 2)))
        err = _pk_err(Pk, Pkr, cr)
        print(f"2D 256^2 {prec}: position rms {rms:.2e} max {np.abs(dx).max():.2e} cells, P(k) max rel err {err:.2e}")
        if prec == "fp64":
            assert np.abs(dx).max() < 1e-6 and err < 1e-8
        else:
            assert rms < 0.05 and err < 1e-3


def test_3d_128_fp32_against_fp64(gpu, conan, oracle):
    dim, mbits, L = 3, 7, 100.0
    N = 1 << mbits
    H = {"dim": dim, "mbits": mbits, "size": L, "ns": -2.0, "smooth": 1, "scale-free": 1, "scale": 0.78125,
         "sigma": 0.83, "seed": 2}
    noise = oracle.noise_mt19937(2, N ** dim)
    dens = conan.generate_random_field(H, noise=noise)
    phi = conan.compute_potential(H, dens)
    out = {}
    for prec in ("fp64", "fp32"):
        g = conan.Gravity(dim, N, 1, L, precision=prec)
        g.run(phi, 0.02, 0.0196, 50)
        out[prec] = (*g.state(), *g.power_spectrum())
        g.close()
    X64, _, k, P64, c = out["fp64"]
    X32, _, _, P32, _ = out["fp32"]
    dx = _dx_cells(X32, X64, L / N, L)
    rms = float(np.sqrt(np.mean(dx ** 2)))
    err = _pk_err(P32, P64, c)
    print(f"3D 128^3 FP32 vs FP64: position rms {rms:.2e} cells, P(k) max rel err {err:.2e}")
    assert err < 1e-3 and rms < 0.05


def test_ensemble_mean_pk_fp32_against_fp64(gpu, conan):
    from conan_b200.ensemble import Ensemble, standard_members
    members = standard_members(n_per_class=4)
    pk = {}
    for prec in ("fp32", "fp64"):
        e = Ensemble(members, precision=prec)
        e.init()
        e.run()
        pk[prec] = e.mean_power_spectrum(17)
        e.close()
    k, P32 = pk["fp32"]
    _, P64 = pk["fp64"]
    m = (P64 > 0) & (np.arange(len(P64)) > 0)  # bin 0 is the k = 0 mode, zero up to rounding
    err = float(np.max(np.abs(P32[m] - P64[m]) / P64[m]))
    print(f"ensemble (12 boxes, 32^3..128^3, 40 steps) mean P(k) FP32 vs FP64: max rel err {err:.2e}")
    assert err < 1e-3
