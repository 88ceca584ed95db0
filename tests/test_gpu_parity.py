"""GPU parity of every kernel of the path against the FP64 CPU oracle.

Tolerances: FP64 GPU vs FP64 oracle 1e-11 relative to the field's maximum
(FFT rounding, summation order); FP32 GPU vs FP64 oracle 2e-5 relative
(single-precision arithmetic). Integer work (cell ids, counts) is exact.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EdS = dict(H0=68.5, Om=1.0, OL=0.0)


def rel(a, b):
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300)


def _H(dim, mbits, L, ns, smooth, scale, seed, scale_free=True):
    return {"dim": dim, "mbits": mbits, "size": L, "ns": ns, "smooth": smooth, "scale-free": scale_free,
            "scale": scale, "sigma": 0.83, "seed": seed}


@pytest.mark.parametrize("dim,mbits,L,ns,smooth,scale", [
    (2, 6, 50.0, -1.0, False, 8.0), (3, 5, 100.0, -2.0, True, 0.78125 * 4), (2, 5, 20.0, -1.5, True, 2.0)])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-11), ("fp32", 2e-5)])
def test_grf_potential_displacement(gpu, conan, oracle, dim, mbits, L, ns, smooth, scale, prec, tol):
    H = _H(dim, mbits, L, ns, smooth, scale, 7)
    noise = oracle.noise_mt19937(7, (1 << mbits) ** dim)
    ref = oracle.grf_scale_free(dim, mbits, L, ns, smooth, scale, 0.83, noise)
    got = conan.generate_random_field(H, noise=noise, precision=prec)
    assert rel(got, ref) < tol
    pref = oracle.potential(dim, mbits, L, ref)
    pgot = conan.compute_potential(H, ref, precision=prec)
    assert rel(pgot, pref) < tol
    dref = oracle.displacement(dim, mbits, L, pref)
    dgot = conan.compute_displacement(H, pref, precision=prec)
    assert rel(dgot, dref) < tol * 10


def test_grf_cdm_branch(gpu, conan, oracle):
    H = _H(3, 5, 200.0, 0.96, False, 8.0, 11, scale_free=False)
    H.update(Omega0=0.32, H0=69.0)
    noise = oracle.noise_mt19937(11, 32 ** 3)
    ref = oracle.grf_cdm(3, 5, 200.0, 0.32, 69.0, 0.96, noise)
    got = conan.generate_random_field(H, noise=noise, precision="fp64")
    assert rel(got, ref) < 1e-11


def test_philox_noise_statistics(gpu, conan):
    z = conan.white_noise({"dim": 3, "mbits": 6, "seed": 5})
    assert abs(z.mean()) < 5 / np.sqrt(z.size)
    assert abs(z.var() - 1) < 5 * np.sqrt(2 / z.size)
    z2 = conan.white_noise({"dim": 3, "mbits": 6, "seed": 5})
    assert np.array_equal(z, z2)
    assert not np.array_equal(z, conan.white_noise({"dim": 3, "mbits": 6, "seed": 6}))


def _particles(dim, Nm, f, L, amp, seed):
    rng = np.random.default_rng(seed)
    q = np.stack(np.meshgrid(*[np.arange(Nm)] * dim, indexing="ij"), -1)
    q = q.reshape(-1, dim)[:, ::-1] if dim > 1 else q.reshape(-1, 1)  # axis 0 fastest
    X = q * (L / Nm) + rng.uniform(-amp, amp, size=q.shape) * (L / (Nm * f))
    Pm = rng.normal(0, 1, size=q.shape) * (L / (Nm * f))
    return np.ascontiguousarray(X), np.ascontiguousarray(Pm)


@pytest.mark.parametrize("dim,Nm,f", [(2, 64, 1), (3, 32, 1), (3, 16, 2), (2, 32, 2), (3, 8, 2), (1, 64, 1),
                                      (2, 32, 1), (1, 1024, 1), (1, 512, 4), (3, 64, 1)])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-11), ("fp32", 1e-5)])
def test_deposit_matches_md_cic(gpu, conan, oracle, dim, Nm, f, prec, tol):
    L = 40.0
    X, Pm = _particles(dim, Nm, f, L, 3.0, 1)
    g = conan.Gravity(dim, Nm, f, L, precision=prec)
    g.set_state(X, Pm, 0.1, 0.1)
    got = g.density()
    ref = oracle.md_cic(dim, Nm * f, L, X, float(f) ** dim) - 1.0
    assert np.max(np.abs(got - ref)) < tol * max(1.0, np.max(np.abs(ref)))
    # bit-identical on repeat (integer accumulation)
    assert np.array_equal(got, g.density())
    g.close()


@pytest.mark.parametrize("dim,Nm,f,amp", [(3, 32, 1, 3.0), (3, 64, 1, 12.0), (3, 16, 2, 3.0), (3, 8, 2, 6.0),
                                          (2, 64, 1, 20.0), (2, 32, 2, 3.0), (2, 16, 1, 2.0), (1, 1024, 1, 50.0),
                                          (1, 128, 2, 9.0), (3, 32, 1, 400.0), (2, 64, 1, 5000.0)])
def test_lagrangian_deposit_equals_sorted_bit_for_bit(gpu, conan, dim, Nm, f, amp):
    """Both FP32 deposits sum the same integer corner weights, so the
    densities are identical, also for tiles stretched far beyond their
    shared-memory window (amp in force cells: particles leave the window,
    cross the periodic boundary, or land anywhere in the box)."""
    X, Pm = _particles(dim, Nm, f, 40.0, amp, 7)
    g = conan.Gravity(dim, Nm, f, 40.0, precision="fp32")
    assert g.deposit_mode == "lagrangian"
    g.set_state(X, Pm, 0.1, 0.1)
    lag = g.density()
    g.deposit_mode = "sorted"
    srt = g.density()
    assert np.array_equal(lag, srt)
    g.deposit_mode = "lagrangian"
    assert np.array_equal(lag, g.density())  # the accumulator was cleared
    g.close()


def test_deposit_modes_give_identical_runs(gpu, conan, oracle):
    dim, mbits, L = 3, 5, 64.0
    Nm = 1 << mbits
    noise = oracle.noise_mt19937(11, Nm ** dim)
    phi = oracle.potential(dim, mbits, L, oracle.grf_scale_free(dim, mbits, L, -2, True, 2.0, 0.83, noise))
    out = []
    for mode in ("lagrangian", "sorted"):
        g = conan.Gravity(dim, Nm, 1, L)
        g.deposit_mode = mode
        g.run(phi, 0.05, 0.0475, 8)
        out.append(g.state())
        g.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    # switching between steps: the sorted deposit must not reuse stale ranks
    g = conan.Gravity(dim, Nm, 1, L)
    conan.LeapFrog(0.05, 0.0475, 4).run(g, phi)
    g.deposit_mode = "sorted"
    for i in range(4, 8):
        a = 0.05 + i * 0.0475
        g.drift(a, 0.0475)
        g.kick(a + 0.0475 / 2, 0.0475)
        g.deposit_mode = "lagrangian" if i % 2 else "sorted"
    X, P = g.state()
    assert np.array_equal(X, out[0][0]) and np.array_equal(P, out[0][1])
    g.close()
    g = conan.Gravity(dim, Nm, 1, L, precision="fp64")
    assert g.deposit_mode == "sorted"
    with pytest.raises(conan.ConanError):
        g.deposit_mode = "lagrangian"
    g.close()


@pytest.mark.parametrize("dim,Nm,f", [(2, 64, 1), (3, 32, 1), (3, 16, 2), (1, 64, 2), (3, 64, 1), (3, 32, 2)])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("fp32", 3e-4)])
def test_kick_and_drift_match_reference(gpu, conan, oracle, dim, Nm, f, prec, tol):
    L = 50.0
    X, Pm = _particles(dim, Nm, f, L, 2.5, 2)
    a, da = 0.3, 0.02
    g = conan.Gravity(dim, Nm, f, L, precision=prec)
    g.set_state(X, Pm, a, a)
    g.kick(a, da)
    Xg, Pg = g.state()
    Xr, Pr = X.copy(), Pm.copy()
    oracle.kick(dim, Nm, f, L, 68.5, 1.0, 0.0, Xr, Pr, a, da)
    assert np.allclose(Xg, X, rtol=0, atol=1e-12 * L if prec == "fp64" else 1e-5 * L)
    assert rel(Pg - Pm, Pr - Pm) < tol
    g.drift(a, da)
    Xg2, _ = g.state()
    oracle.drift(dim, Nm, 68.5, 1.0, 0.0, Xr, Pr, a, da)
    assert np.max(np.abs(Xg2 - Xr)) < (1e-10 if prec == "fp64" else 2e-4) * L / (Nm * f)
    assert g.scale_factors() == (a, a)
    g.close()


def test_negative_coordinates_use_reference_truncation(gpu, conan, oracle):
    # particles near the origin with negative unwrapped coordinates: the
    # reference gather extrapolates (truncating cast); periodic mode differs.
    dim, Nm, L = 2, 32, 32.0
    X, Pm = _particles(dim, Nm, 1, L, 1.5, 3)
    phi = np.sin(np.arange(Nm ** dim) * 0.37)
    ref = oracle.interp_gradient(dim, Nm, L, phi, X)
    assert np.any(X < 0)
    out = {}
    for periodic in (False, True):
        g = conan.Gravity(dim, Nm, 1, L, precision="fp64", periodic_gather=periodic)
        g.set_state(X, np.zeros_like(X), 0.5, 0.5)
        g.kick(0.5, 0.01)
        _, P = g.state()
        out[periodic] = P
        g.close()
    adot = oracle.adot(68.5, 1.0, 0.0, 0.5)
    # quirk mode equals the reference interpolation of the solver's own phi
    g = conan.Gravity(dim, Nm, 1, L, precision="fp64")
    g.set_state(X, np.zeros_like(X), 0.5, 0.5)
    g.kick(0.5, 0.01)
    phi_gpu = g.potential()
    ref = oracle.interp_gradient(dim, Nm, L, phi_gpu, X)
    assert rel(-out[False] / (0.01 / adot), ref) < 1e-11
    neg = np.any(X < 0, axis=1) & np.any(np.abs(X / (L / Nm) - np.round(X / (L / Nm))) > 1e-9, axis=1)
    assert np.max(np.abs(out[False][neg] - out[True][neg])) > 0
    g.close()


@pytest.mark.parametrize("dim,mbits,f,prec,tol", [(2, 6, 1, "fp64", 1e-9), (3, 4, 2, "fp64", 1e-9),
                                                  (2, 6, 1, "fp32", 2e-3)])
def test_leapfrog_run_matches_oracle(gpu, conan, oracle, dim, mbits, f, prec, tol):
    Nm, L = 1 << mbits, 50.0
    noise = oracle.noise_mt19937(3, Nm ** dim)
    dens = oracle.grf_scale_free(dim, mbits, L, -1.0, False, 8.0, 0.83, noise)
    phi = oracle.potential(dim, mbits, L, dens)
    a0, da, n = 0.02, 0.049, 20
    Xr, Pr = oracle.run(dim, Nm, f, L, 68.5, 1.0, 0.0, phi, a0, da, n)
    g = conan.Gravity(dim, Nm, f, L, precision=prec)
    g.run(phi, a0, da, n)
    Xg, Pg = g.state()
    cell = L / (Nm * f)
    assert np.max(np.abs(Xg - Xr)) / cell < tol * (1e3 if prec == "fp32" else 1)
    assert rel(Pg, Pr) < tol * (10 if prec == "fp32" else 1e2)
    a_pos, a_mom = g.scale_factors()
    assert abs(a_pos - (a0 + (n - 1) * da)) < 1e-12 and abs(a_mom - (a0 + (n - 1) * da + da / 2)) < 1e-12
    g.close()


def test_run_equals_separate_drift_kick_calls(gpu, conan, oracle):
    # the graph-captured fused loop is bit-identical to the unfused API calls
    dim, mbits, L = 3, 5, 64.0
    Nm = 1 << mbits
    noise = oracle.noise_mt19937(9, Nm ** dim)
    phi = oracle.potential(dim, mbits, L, oracle.grf_scale_free(dim, mbits, L, -2, True, 2.0, 0.83, noise))
    a0, da, n = 0.05, 0.0475, 6
    g1 = conan.Gravity(dim, Nm, 1, L)
    g1.run(phi, a0, da, n)
    X1, P1 = g1.state()
    g2 = conan.Gravity(dim, Nm, 1, L)
    conan.LeapFrog(a0, da, n).run(g2, phi)
    X2, P2 = g2.state()
    assert np.array_equal(X1, X2) and np.array_equal(P1, P2)
    g3 = conan.Gravity(dim, Nm, 1, L)
    seen = []
    g3.run(phi, a0, da, n, callback=lambda i, a: seen.append((i, a)), every=2)
    X3, _ = g3.state()
    assert np.array_equal(X1, X3)
    assert [s[0] for s in seen] == [1, 3, 5]
    for g in (g1, g2, g3):
        g.close()


def test_power_spectrum_matches_oracle(gpu, conan, oracle):
    dim, Nm, L = 3, 32, 100.0
    X, Pm = _particles(dim, Nm, 1, L, 2.0, 4)
    g = conan.Gravity(dim, Nm, 1, L, precision="fp64")
    g.set_state(X, Pm, 0.5, 0.5)
    k, P, c = g.power_spectrum()
    delta = oracle.md_cic(dim, Nm, L, X) - 1.0
    kr, Pr, cr = oracle.power_spectrum(dim, Nm, L, delta)
    assert np.array_equal(c, cr)
    m = cr > 0
    m[0] = False  # the k = 0 shell is the (vanishing) mean
    assert abs(P[0]) < 1e-20
    assert np.max(np.abs(P[m] - Pr[m]) / Pr[m]) < 1e-10
    assert np.max(np.abs(k[m] - kr[m]) / kr[m]) < 1e-12
    g.close()


def test_spectral_gradient_runs_and_is_close_to_fd4(gpu, conan, oracle):
    dim, mbits, L = 3, 5, 100.0
    Nm = 1 << mbits
    noise = oracle.noise_mt19937(1, Nm ** dim)
    phi = oracle.potential(dim, mbits, L, oracle.grf_scale_free(dim, mbits, L, -2, True, 3.0, 0.83, noise))
    out = []
    for grad in ("fd4", "spectral"):
        g = conan.Gravity(dim, Nm, 1, L, precision="fp64", gradient=grad)
        g.run(phi, 0.02, 0.0196, 5)
        out.append(g.state()[0])
        g.close()
    cell = L / Nm
    d = np.max(np.abs(out[0] - out[1])) / cell
    assert 0 < d < 0.05


@pytest.mark.parametrize("dim,Nm,f,s", [(3, 16, 2, 1), (3, 16, 1, 2), (3, 8, 2, 4), (2, 32, 2, 2), (2, 64, 1, 1),
                                        (1, 128, 2, 4), (3, 32, 1, 1)])
def test_cic_tool_matches_oracle(gpu, conan, oracle, dim, Nm, f, s):
    """conan_cic against the oracle's cic_run (positions anywhere, wrapped)."""
    L = 30.0
    X, _ = _particles(dim, Nm, f, L, 6.0, 11)
    got = conan.cic(X, dim, Nm, L, f=f, sub_sample=s)
    ref = oracle.cic(dim, Nm, L, f, s, X)
    assert np.max(np.abs(got - ref)) <= 1e-11 * np.max(np.abs(ref))
    # total mass: N^dim unit masses, but (f N)^dim when sub-sampled, since
    # the reference weights the (s N)^dim points by (s N / f N)^-dim
    total = Nm ** dim if s == 1 else (Nm * f) ** dim
    assert abs(got.sum() - total) < 1e-9 * total
    assert np.array_equal(got, conan.cic(X, dim, Nm, L, f=f, sub_sample=s))  # order-independent sums


@pytest.mark.parametrize("Nm,f", [(64, 1), (128, 1), (64, 2), (256, 1), (64, 8), (64, 16)])
def test_plane_transforms_and_z_pass_give_the_3d_potential(gpu, conan, Nm, f):
    """FP32 3D meshes of 64..1024 cells solve Poisson as 2D transforms of the
    z planes around the shared-memory z pass; the potential equals the FP64
    solve (3D transforms) on the same particles to FP32 rounding."""
    L = 100.0
    X, Pm = _particles(3, Nm, f, L, 2.0, 9)
    phis = {}
    for prec in ("fp32", "fp64"):
        g = conan.Gravity(3, Nm, f, L, precision=prec)
        g.set_state(X, Pm, 0.4, 0.4)
        g.kick(0.4, 0.01)
        phis[prec] = g.potential()
        g.close()
    assert rel(phis["fp32"], phis["fp64"]) < 2e-5


@pytest.mark.parametrize("Nm,f", [(64, 1), (32, 2), (128, 1)])
def test_gradient_mesh_kernels_give_the_same_kick(gpu, conan, monkeypatch, Nm, f):
    """The gradient-mesh kernels the autotuner chooses between (one thread
    per cell, z-marching tiles) do the same arithmetic: the kicked momenta
    agree bit for bit."""
    L = 100.0
    X, Pm = _particles(3, Nm, f, L, 2.0, 11)
    out = {}
    for kern in ("cell", "zm"):
        monkeypatch.setenv("CONAN_GRAD_KERNEL", kern)
        g = conan.Gravity(3, Nm, f, L, precision="fp32")
        g.set_state(X, Pm, 0.4, 0.4)
        g.kick(0.4, 0.01)
        out[kern] = g.state()[1]
        g.close()
    assert np.array_equal(out["cell"], out["zm"])


@pytest.mark.parametrize("Nm,f,columns,mode", [(256, 1, 16, "1"), (64, 8, 16, "1"), (128, 2, 16, "1"),
                                               (64, 8, 32, "1"), (128, 2, 32, "1"), (64, 8, 32, "2")])
def test_cluster_plane_pass_matches_cufft_planes(gpu, conan, monkeypatch, Nm, f, columns, mode):
    """256^3 and 512^3 FP32 meshes transform their z planes in thread-block
    clusters (the forward pass reading the integer deposit directly); the
    potential and the kicked momenta equal those of cuFFT's plane transforms
    to FP32 rounding."""
    L = 100.0
    X, Pm = _particles(3, Nm, f, L, 2.0, 9)
    out = {}
    monkeypatch.setenv("CONAN_PLANE_COLUMNS", str(columns))
    for on in ("0", mode):  # mode 2: the cluster forward pass, cuFFT's inverse
        monkeypatch.setenv("CONAN_PLANE_PASS", on)
        g = conan.Gravity(3, Nm, f, L, precision="fp32")
        g.set_state(X, Pm, 0.4, 0.4)
        g.set_profiling(True)
        g.kick(0.4, 0.01)
        kernels = set(g.profile())
        assert ("plane_r2c" in kernels) == (on != "0") and ("plane_c2r" in kernels) == (on == "1"), kernels
        out[on] = (g.potential(), g.state()[1])
        g.close()
    assert rel(out[mode][0], out["0"][0]) < 2e-6
    assert rel(out[mode][1], out["0"][1]) < 2e-6
