"""The benchmark configurations at their full sizes (seeded synthetic fields).

* 2D PM, 256^2 particles on 256^2 cells, L = 50, P(k) ~ k^-1, Zel'dovich at
  a = 0.02, 100 steps to a = 1, FP64: positions and final P(k) against the
  FP64 CPU oracle on the same mt19937 noise; FP32 against the same oracle.
* 3D PM, 128^3 on 128^3, L = 100, P(k) ~ k^-2 smoothed at one cell, 50 steps
  from a = 0.02: FP32 (lattice index + displacement) and FP64 on the GPU,
  each against the FP64 CPU oracle run on the same mt19937 noise and
  potential: position RMS (minimum image, cells) and the final P(k) per
  shell, FP32 within 1e-3.
* The 96-box ensemble: ensemble-mean P(k) in FP32 against FP64 on the GPU,
  and its 32^3 class (32 boxes) against the FP64 CPU oracle run on the same
  white noise, per member and as the class mean.
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


def test_3d_128_fp32_against_the_oracle(gpu, conan, oracle):
    """ic -d 3 -b 7 -L 100 --scale-free -n -2 --smooth --scale 0.78125 --seed 2;
    run -f 1 -a0 0.02 -da 0.0196 -n 50 (LeapFrog::run, src/run/leapfrog.hh:
    33-46, over Gravity<3>, src/run/nbody.hh:97-133)."""
    dim, mbits, L = 3, 7, 100.0
    N = 1 << mbits
    noise = oracle.noise_mt19937(2, N ** dim)
    dens = oracle.grf_scale_free(dim, mbits, L, -2.0, True, 0.78125, 0.83, noise)
    phi = oracle.potential(dim, mbits, L, dens)
    a0, da, n = 0.02, 0.0196, 50
    Xr, _ = oracle.run(dim, N, 1, L, 68.5, 1.0, 0.0, phi, a0, da, n)
    kr, Pkr, cr = oracle.power_spectrum(dim, N, L, oracle.md_cic(dim, N, L, Xr) - 1.0)
    m = (cr > 0) & (np.arange(len(cr)) > 0)
    res = {}
    for prec in ("fp64", "fp32"):
        g = conan.Gravity(dim, N, 1, L, precision=prec)
        g.run(phi, a0, da, n)
        X, _ = g.state()
        _, Pk, _ = g.power_spectrum(len(cr))
        g.close()
        dx = _dx_cells(X, Xr, L / N, L)
        ratio = Pk[m] / Pkr[m]
        res[prec] = (float(np.sqrt(np.mean(dx ** 2))), float(np.abs(dx).max()), float(np.max(np.abs(ratio - 1))))
        print(f"C2 3D 128^3 {prec} vs oracle: position rms {res[prec][0]:.2e} max {res[prec][1]:.2e} cells; "
              f"P(k) ratio per shell: max |r - 1| {res[prec][2]:.2e}, shells 1..{m.sum()} "
              f"[{ratio.min():.8f}, {ratio.max():.8f}]")
    assert res["fp64"][1] < 1e-6 and res["fp64"][2] < 1e-9
    assert res["fp32"][2] < 1e-3 and res["fp32"][0] < 0.05


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


def test_ensemble_32_class_against_the_oracle(gpu, conan, oracle):
    """The 32 boxes of 32^3 of the 96-box ensemble (spectral indices from
    default_rng(6), seeds 1000 + i, L = 100, 40 steps a = 0.05 -> 1, FP32,
    run batched in one graph launch) against FP64 CPU oracle runs on the same
    white noise: every member's P(k) and the class mean within 1e-3."""
    from conan_b200.ensemble import Ensemble, standard_members
    members = standard_members()[:32]
    assert all(mb == 5 for mb, _, _, _ in members)
    nb, steps = 17, 40
    e = Ensemble(members, precision="fp32")
    e.init()
    e.run()
    gpu_pk = np.array([e.power_spectrum(i, nb)[1] for i in range(len(members))])
    e.close()
    ref_pk = []
    for mb, L, ns, seed in members:
        N = 1 << mb
        noise = conan.white_noise({"dim": 3, "mbits": mb, "seed": seed})
        phi = oracle.potential(3, mb, L, oracle.grf_scale_free(3, mb, L, ns, False, 8.0, 0.83, noise))
        X, _ = oracle.run(3, N, 1, L, 68.5, 1.0, 0.0, phi, 0.05, 0.95 / steps, steps)
        ref_pk.append(oracle.power_spectrum(3, N, L, oracle.md_cic(3, N, L, X) - 1.0, nb)[1])
    ref_pk = np.array(ref_pk)
    sel = np.arange(nb) > 0
    per = np.abs(gpu_pk[:, sel] / ref_pk[:, sel] - 1)
    mean_err = float(np.max(np.abs(gpu_pk.mean(0)[sel] / ref_pk.mean(0)[sel] - 1)))
    print(f"C5 32^3 class (32 boxes, 40 steps) FP32 vs oracle: mean P(k) max rel err {mean_err:.2e}; "
          f"worst member {per.max():.2e}, median member {np.median(per.max(1)):.2e}")
    assert mean_err < 1e-3 and per.max() < 1e-3


def test_ensemble_gradient_against_the_cpu_adjoint(gpu, conan, oracle):
    """The batched forward + adjoint of the ensemble (two 32^3 members of
    the 96-box set, L = 100, 40 steps a = 0.05 -> 1, FP32, checkpoint 8):
    each member's loss (mean squared difference to its target density) and
    its gradient with respect to the white noise against the FP64 CPU model
    and adjoint run on the same noise and target."""
    from conan_b200.ensemble import Ensemble, standard_members
    members = standard_members()[:2]
    steps = 40
    e = Ensemble(members, precision="fp32", steps=steps)
    e.init()
    loss = e.forward_adjoint()
    fields = [e.member_fields(i) for i in range(len(members))]
    e.close()
    for i, (mb, L, ns, seed) in enumerate(members):
        noise, target, g = fields[i]
        args = (3, mb, 1, L, ns, False, 8.0, 0.83, 0.05, 0.95 / steps, steps, noise)
        dref = oracle.diff_forward(*args)
        lref = float(np.mean((dref - target) ** 2))
        _, gref = oracle.diff_adjoint(*args, 2 * (dref - target) / dref.size)
        scale = np.max(np.abs(gref))
        rel_max = float(np.max(np.abs(g - gref)) / scale)
        big = np.abs(gref) > 1e-2 * scale
        rel = np.abs(g - gref)[big] / np.abs(gref)[big]
        lerr = abs(loss[i] - lref) / lref
        print(f"ensemble member {i} (32^3, 40 steps) FP32 vs FP64 CPU adjoint: loss rel err {lerr:.2e}; "
              f"max |dg| / max |g| {rel_max:.2e}; median rel (components above 1%) {np.median(rel):.2e}")
        # measured on a B200: loss 1.3e-6, max 1.1e-4 of the largest component, median 3.7e-5
        assert lerr < 1e-5 and rel_max < 1e-3 and np.median(rel) < 2e-4


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
