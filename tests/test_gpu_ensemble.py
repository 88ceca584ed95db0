"""Batched ensembles: batching changes indexing only, so every member of a
mixed-size ensemble reproduces, bit for bit, the same member run alone; the
graph-captured run is repeatable; the autotuner picks one of its variants;
forward+adjoint gives the single-member losses."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MEMBERS = [(5, 100.0, -2.0, 1000), (4, 60.0, -1.5, 1001), (5, 100.0, -1.0, 1002), (4, 60.0, -2.5, 1003),
           (5, 100.0, -1.5, 1004)]


def _ens(members, **kw):
    from conan_b200.ensemble import Ensemble
    e = Ensemble(members, steps=12, **kw)
    e.init()
    return e


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_members_match_single_runs(gpu, conan, prec):
    e = _ens(MEMBERS, precision=prec)
    e.run()
    for i, m in enumerate(MEMBERS):
        X, P = e.state(i)
        s = _ens([m], precision=prec, autotune=False)
        s.run()
        Xs, Ps = s.state(0)
        assert np.array_equal(X, Xs) and np.array_equal(P, Ps), f"member {i}"
        k, Pk, c = e.power_spectrum(i)
        k2, Pk2, c2 = s.power_spectrum(0)
        assert np.array_equal(Pk, Pk2)
        s.close()
    e.close()


def test_graph_run_repeats_and_autotuner_reports(gpu, conan):
    e = _ens(MEMBERS)
    e.run()
    X1, _ = e.state(2)
    ms = e.run()
    X2, _ = e.state(2)
    assert np.array_equal(X1, X2)
    assert ms > 0
    d = e.describe()
    assert len(d["classes"]) == 2
    for c in d["classes"]:
        assert c["deposit"] in ("sorted", "lagrangian")
        assert c["tuned_at_a"] > 0.05  # timed on the state half way through the run
        knobs = {t["knob"] for t in c["tuning"]}
        assert knobs == {"deposit", "gradient"}
        for k in knobs:  # one chosen value per knob, the fastest timed
            ts = [t for t in c["tuning"] if t["knob"] == k]
            chosen = [t for t in ts if t["chosen"]]
            assert len(chosen) == 1 and chosen[0]["ms_per_step"] == min(t["ms_per_step"] for t in ts)
    assert e.total_particles() == 3 * 32 ** 3 + 2 * 16 ** 3
    e.close()


def test_forward_adjoint_losses_match_single_members(gpu, conan):
    e = _ens(MEMBERS)
    loss = e.forward_adjoint()
    assert np.all(loss > 0)
    for i, m in enumerate(MEMBERS[:2]):
        s = _ens([m], autotune=False)
        l1 = s.forward_adjoint()
        assert abs(l1[0] - loss[i]) <= 1e-6 * loss[i]
        s.close()
    r, a = e.last_ms()
    assert a > 0
    e.close()


def test_ensemble_mean_pk_is_finite(gpu, conan):
    e = _ens(MEMBERS)
    e.run()
    k, P = e.mean_power_spectrum(8)
    assert np.all(np.isfinite(P)) and np.all(P[1:] > 0)
    e.close()


def test_single_box_autotuner_keeps_state_and_results(gpu, conan):
    """The solver's autotuner on a clustered 64^3 state: every knob reports
    its candidates, the state comes back unchanged, and the run after tuning
    gives the density of an untuned solver (the deposit variants sum the same
    integers, the gradient variants do the same arithmetic; the sorted and
    Lagrangian paths gather in different kernels, so FP32 rounding of the
    later steps may differ)."""
    n, L = 64, 64.0
    H = {"dim": 3, "mbits": 6, "size": L, "ns": -2.0, "smooth": 0, "scale-free": 1, "scale": 8.0, "sigma": 0.83,
         "seed": 9}
    phi = conan.compute_potential(H, conan.generate_random_field(H))
    a0, da = 0.05, 0.05
    out = []
    for tuned in (False, True):
        g = conan.Gravity(3, n, 1, L, precision="fp32")
        g.run(phi, a0, da, 8)
        X0, P0 = g.state()
        if tuned:
            rep = g.autotune(a0 + 8 * da, da)
            X1, P1 = g.state()
            assert np.array_equal(X0, X1) and np.array_equal(P0, P1)
            knobs = {r["knob"] for r in rep}
            assert knobs == {"deposit", "gradient", "z pass"}  # a 64^3 mesh solves Poisson with the z pass
            assert sum(r["chosen"] for r in rep) == len(knobs)
        g.run(None, a0 + 8 * da, da, 4)
        out.append(g.density())
        g.close()
    assert np.max(np.abs(out[0] - out[1])) <= 1e-5 * max(1.0, np.max(np.abs(out[0])))



def test_batched_members_through_the_cluster_plane_pass(gpu, conan, monkeypatch):
    """Two 256^3 members batched in one size class, 12 steps to a = 1: the
    cluster plane passes (one cluster per z plane and member) give the states
    of cuFFT's plane transforms to FP32 rounding (measured on a B200:
    position rms 1.2e-5 and 1.4e-5 cells, P(k) within 7e-7; the largest
    single difference, 0.05 cells, is a particle in a caustic), and each
    member equals itself run alone bit for bit."""
    members = [(8, 200.0, -1.5, 7), (8, 200.0, -2.0, 8)]
    out, pk = {}, {}
    for mode in ("0", "1"):
        monkeypatch.setenv("CONAN_PLANE_PASS", mode)
        e = _ens(members, autotune=False)
        e.run()
        out[mode] = [e.state(i)[0] for i in range(len(members))]
        pk[mode] = [e.power_spectrum(i, 64)[1] for i in range(len(members))]
        e.close()
    cell = 200.0 / 256
    for i in range(len(members)):
        d = np.abs(out["1"][i] - out["0"][i]) / cell
        rms = float(np.sqrt(np.mean(d ** 2)))
        perr = float(np.max(np.abs(pk["1"][i][1:] / pk["0"][i][1:] - 1)))
        print(f"member {i}: position rms {rms:.2e} cells, max {d.max():.2e} cells; P(k) max rel diff {perr:.2e}")
        assert rms < 1e-4 and perr < 1e-4, f"member {i}"
    monkeypatch.setenv("CONAN_PLANE_PASS", "1")
    s = _ens(members[1:], autotune=False)
    s.run()
    assert np.array_equal(s.state(0)[0], out["1"][1])
    s.close()
