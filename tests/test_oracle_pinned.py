"""The CPU oracle is pinned to the unmodified reference.

The golden fixtures were written by the reference's own `conan ic` / `conan
run` binary and its md_cic / LinearInterpolation<Gradient> templates
(tests/golden/make_golden.py). The reference ships no known-answer tests of
its own (every unit test prints and returns true), so these goldens are the
parity anchor. The oracle restates the same algorithm with the same FFT, so
agreement is to rounding.
"""
import numpy as np
import pytest

from conftest import GOLDEN as GOLDEN_DIR, load_golden

EdS = (68.5, 1.0, 0.0)


def _args(s):
    toks = str(s).split()
    out = {}
    i = 0
    while i < len(toks):
        t = toks[i]
        if i + 1 < len(toks) and not toks[i + 1].startswith("--") and not (
                toks[i + 1].startswith("-") and not toks[i + 1][1:].replace(".", "").isdigit()):
            out[t.lstrip("-")] = toks[i + 1]
            i += 2
        else:
            out[t.lstrip("-")] = "1"
            i += 1
    return out


def _ic(g):
    a = _args(g["ic_args"])
    dim, mbits, L = int(a["d"]), int(a["b"]), float(a["L"])
    return a, dim, mbits, L


@pytest.mark.parametrize("name", ["c1s", "c2s", "c3s"])
def test_oracle_grf_potential_displacement(oracle, name):
    g = load_golden(name)
    a, dim, mbits, L = _ic(g)
    noise = oracle.noise_mt19937(int(a["seed"]), (1 << mbits) ** dim)
    dens = oracle.grf_scale_free(dim, mbits, L, float(a["n"]), "smooth" in a, float(a.get("scale", 8.0)), 0.83,
                                 noise)
    assert np.max(np.abs(dens - g["density"])) <= 1e-13 * np.max(np.abs(g["density"]))
    pot = oracle.potential(dim, mbits, L, dens)
    assert np.max(np.abs(pot - g["potential"])) <= 1e-13 * np.max(np.abs(g["potential"]))
    if "displacement" in g:
        disp = oracle.displacement(dim, mbits, L, pot)
        assert np.max(np.abs(disp - g["displacement"])) <= 1e-13 * np.max(np.abs(g["displacement"]))


def test_oracle_cdm_branch(oracle):
    g = load_golden("c4s")
    a, dim, mbits, L = _ic(g)
    noise = oracle.noise_mt19937(4, (1 << mbits) ** dim)
    dens = oracle.grf_cdm(dim, mbits, L, 0.3, 70.0, 0.96, noise)
    assert np.max(np.abs(dens - g["density"])) <= 1e-13 * np.max(np.abs(g["density"]))


@pytest.mark.parametrize("name,f,cosmo", [("c1s", 1, EdS), ("c2s", 1, EdS), ("c3s", 2, EdS),
                                          ("c4s", 2, (68.5, 0.31, 0.69))])
def test_oracle_run_matches_reference_snapshots(oracle, name, f, cosmo):
    g = load_golden(name)
    a, dim, mbits, L = _ic(g)
    r = _args(g["run_args"])
    a0, da = float(r["a0"]), float(r["da"])
    Nm = 1 << mbits
    for snap in (1, 2):
        if f"pos{snap}" not in g:
            continue
        X, P = oracle.run(dim, Nm, f, L, *cosmo, g["potential"], a0, da, 10 * snap)
        cell = L / (Nm * f)
        assert np.max(np.abs(X - g[f"pos{snap}"])) < 1e-9 * cell
        assert np.max(np.abs(P - g[f"mom{snap}"])) < 1e-9 * np.max(np.abs(g[f"mom{snap}"]))
        a = a0
        for _ in range(10 * snap - 1):
            a += da
        assert abs(float(g[f"apos{snap}"]) - a) < 1e-4  # header keeps 6 significant digits


@pytest.mark.parametrize("name", ["c1s", "c2s", "c3s", "c4s"])
def test_oracle_cic_matches_reference_cic_tool(oracle, name):
    """The `cic` tool of the reference (plain and sub-sampled) on its own snapshots."""
    g = load_golden(name)
    _, dim, mbits, L = _ic(g)
    N = 1 << mbits
    keys = [k for k in g if k.startswith("rho") and not k.startswith("rhohdr")]
    assert keys
    for k in keys:
        snap, f, s = k[3:].split("_")
        rho = oracle.cic(dim, N, L, int(f[1:]), int(s[1:]), g[f"pos{snap}"])
        assert np.max(np.abs(rho - g[k])) <= 1e-12 * np.max(np.abs(g[k])), k


@pytest.mark.parametrize("dim,N,L", [(2, 16, 10.0), (3, 8, 5.0), (1, 32, 7.0)])
def test_oracle_kernels_match_reference_templates(oracle, dim, N, L):
    g = load_golden("kernels")
    X = g[f"X_{dim}d"]
    cic = oracle.md_cic(dim, N, L, X)
    assert np.max(np.abs(cic - g[f"cic_{dim}d"])) < 1e-13
    grad = oracle.interp_gradient(dim, N, L, g[f"phi_{dim}d"], X)
    assert np.max(np.abs(grad - g[f"interp_{dim}d"])) < 1e-12 * np.max(np.abs(g[f"interp_{dim}d"]))


@pytest.mark.parametrize("dim,N", [(1, 64), (2, 16), (3, 8)])
def test_fft_shim_matches_numpy(oracle, dim, N):
    rng = np.random.default_rng(dim)
    a = rng.normal(size=(N,) * dim) + 1j * rng.normal(size=(N,) * dim)
    f = oracle.dft(a.ravel(), dim, N, -1).reshape(a.shape)
    assert np.max(np.abs(f - np.fft.fftn(a))) < 1e-12 * np.max(np.abs(f))
    b = oracle.dft(f.ravel(), dim, N, +1).reshape(a.shape) / N ** dim
    assert np.max(np.abs(b - a)) < 1e-13 * np.max(np.abs(a)) * 10


def test_oracle_power_spectrum_of_single_mode(oracle):
    N, L = 16, 10.0
    x = np.arange(N)
    delta = np.cos(2 * np.pi * 3 * x / N)[None, :] * np.ones((N, 1))  # axis 0 fastest: mode n = 3
    k, P, c = oracle.power_spectrum(2, N, L, delta.ravel())
    assert np.argmax(P) == 3
    assert 2.5 * 2 * np.pi / L <= k[3] < 3.5 * 2 * np.pi / L
    # |delta_hat|^2 = (N^2/2)^2 on each of the modes (+-3, 0), averaged over
    # the c[3] modes of the shell, times L^2/N^4
    assert abs(P[3] - 2 * (N * N / 2) ** 2 / c[3] * L ** 2 / N ** 4) < 1e-9
    assert np.all(P[np.arange(len(P)) != 3] < 1e-20)


def _fof_case(name):
    g = load_golden("fof")
    snap = str(g[f"{name}_snapshot"])
    if ":" in snap:
        f, k = snap.split(":")
        X = np.load(GOLDEN_DIR / f)[k]
    else:
        X = g[snap]
    return (X, int(g[f"{name}_dim"]), float(g[f"{name}_L"]), float(str(g[f"{name}_ll"])),
            str(g[f"{name}_text"]))


@pytest.mark.parametrize("name", [str(c) for c in load_golden("fof")["cases"]])
def test_oracle_fof_matches_reference_fof_tool(oracle, name):
    """The `fof` tool of the reference on snapshots of its own runs: the
    oracle's groups, written in the reference's text format, give the
    reference's output file byte for byte after the header and history."""
    X, dim, L, ll, text = _fof_case(name)
    tags, ng = oracle.fof(dim, L, ll, X)
    assert ng == int(tags.max())
    assert oracle.fof_report(X, tags, L) == oracle.fof_text_body(text)


def test_oracle_fof_cell_list_equals_all_pairs(oracle):
    """The oracle's cell list finds the same friends as testing every pair
    (positions outside the box, both cell-list regimes)."""
    rng = np.random.default_rng(3)
    for dim, n, L, ll in [(3, 400, 10.0, 0.9), (3, 300, 10.0, 4.0), (2, 500, 7.0, 0.3), (2, 200, 7.0, 3.0)]:
        X = rng.uniform(-0.6 * L, 1.6 * L, size=(n, dim))
        X[n // 2:] = X[:n // 2] + rng.normal(0, ll / 2, size=(n - n // 2, dim))  # close pairs
        tags, ng = oracle.fof(dim, L, ll, X)
        # all pairs with the reference's predicate, groups by union-find with min-index roots
        par = np.arange(n)

        def find(a):
            while par[a] != a:
                a = par[a]
            return a
        for i in range(n):
            e = X - X[i]
            d = np.where(e > L / 2, e - L, np.where(e < -L / 2, e + L, e))
            v = np.zeros(n)
            for k in range(dim):
                v = v + d[:, k] * d[:, k]
            for j in np.nonzero(v <= ll * ll)[0]:
                a, b = find(i), find(j)
                if a != b:
                    par[max(a, b)] = min(a, b)
        roots = np.array([find(i) for i in range(n)])
        _, first = np.unique(roots, return_index=True)
        number = {roots[f]: k + 1 for k, f in enumerate(sorted(first))}
        assert ng == len(first)
        assert np.array_equal(tags, np.array([number[r] for r in roots], dtype=np.uint64))
