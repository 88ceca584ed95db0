"""GPU friends-of-friends (conan_fof) against the oracle and the reference's
own `fof` output files. Group tags are integers: the bar is exact equality."""
import numpy as np
import pytest

from conftest import GOLDEN, load_golden

pytestmark = pytest.mark.gpu


def _clustered(dim, n, L, seed, shift=True):
    """Blobs of several sizes over a uniform background; coordinates left
    unwrapped (some shifted by -L, +L, +1.7 L) as snapshots hold them."""
    rng = np.random.default_rng(seed)
    nb = n // 4
    X = rng.uniform(0, L, size=(n, dim))
    centres = rng.uniform(0, L, size=(64, dim))
    which = rng.integers(0, 64, size=n - nb)
    widths = np.geomspace(L / 400, L / 20, 64)
    X[nb:] = centres[which] + rng.normal(size=(n - nb, dim)) * widths[which, None]
    if shift:
        k = rng.integers(0, 5, size=(n, dim))
        X += np.choose(k, [0.0, 0.0, -L, L, 1.7 * L])
    return np.ascontiguousarray(X)


def _golden_case(name):
    g = load_golden("fof")
    snap = str(g[f"{name}_snapshot"])
    if ":" in snap:
        f, k = snap.split(":")
        X = np.load(GOLDEN / f)[k]
    else:
        X = g[snap]
    return X, int(g[f"{name}_dim"]), float(g[f"{name}_L"]), float(str(g[f"{name}_ll"])), str(g[f"{name}_text"])


@pytest.mark.parametrize("name", [str(c) for c in load_golden("fof")["cases"]])
def test_fof_reproduces_reference_groups(gpu, conan, oracle, name):
    """GPU tags on the reference's snapshots give the reference's fof file body."""
    X, dim, L, ll, text = _golden_case(name)
    tags, ng = conan.fof(X, dim, L, ll)
    ref, ngr = oracle.fof(dim, L, ll, X)
    assert ng == ngr
    assert np.array_equal(tags, ref)
    assert oracle.fof_report(X, tags, L) == oracle.fof_text_body(text)


@pytest.mark.parametrize("dim,n,L,ll", [
    (3, 200_000, 100.0, 0.2), (3, 200_000, 100.0, 0.05), (3, 50_000, 100.0, 1.5), (2, 200_000, 50.0, 0.03),
    (2, 100_000, 50.0, 0.2), (3, 5_000, 10.0, 3.5), (2, 3_000, 10.0, 4.0), (3, 20_000, 10.0, 10.0),
    (3, 1, 10.0, 1.0), (2, 2, 10.0, 1.0)])
def test_fof_matches_oracle(gpu, conan, oracle, dim, n, L, ll):
    """Clustered and uniform particles, unwrapped coordinates; linking lengths
    from far below the mean spacing to beyond L / 3 (one cell) and L (one
    group)."""
    X = _clustered(dim, n, L, 100 * dim + n % 97)
    ref, ngr = oracle.fof(dim, L, ll, X)
    for _ in range(4):  # the union-find runs concurrently: every run must give the same tags
        tags, ng = conan.fof(X, dim, L, ll)
        assert ng == ngr
        assert np.array_equal(tags, ref)
    if ll >= L:
        assert ng == 1


def test_fof_links_at_exactly_the_linking_length(gpu, conan, oracle):
    """A lattice whose spacing is exactly the linking length (dyadic values,
    so d^2 == ll^2 exactly) is one group; a hair less and every point is alone."""
    L, m = 16.0, 32
    q = np.stack(np.meshgrid(*[np.arange(m)] * 3, indexing="ij"), -1).reshape(-1, 3) * (L / m)
    tags, ng = conan.fof(q, 3, L, L / m)
    assert ng == 1
    tags, ng = conan.fof(q, 3, L, np.nextafter(L / m, 0))
    assert ng == m ** 3 and np.array_equal(tags, np.arange(1, m ** 3 + 1, dtype=np.uint64))
    ref, _ = oracle.fof(3, L, np.nextafter(L / m, 0), q)
    assert np.array_equal(tags, ref)


def test_fof_engine_reuse_and_device_pointers(gpu, conan, oracle):
    """One engine over several snapshots, host and device entry points alike."""
    import torch
    dim, n, L, ll = 3, 100_000, 50.0, 0.12
    eng = conan.FoF(dim, n, L, ll)
    for seed in (1, 2):
        X = _clustered(dim, n, L, seed)
        ref, ngr = oracle.fof(dim, L, ll, X)
        tags, ng = eng(X)
        assert ng == ngr and np.array_equal(tags, ref)
        xd = torch.from_numpy(X).cuda()
        td = torch.empty(n, dtype=torch.int64, device="cuda")
        ng2 = eng.run_device(xd.data_ptr(), td.data_ptr(), torch.cuda.current_stream().cuda_stream)
        assert ng2 == ngr and np.array_equal(td.cpu().numpy().astype(np.uint64), ref)
    eng.close()


def test_fof_rejects_bad_arguments(gpu, conan):
    X = np.zeros((10, 3))
    for dim, L, ll in [(1, 10.0, 1.0), (4, 10.0, 1.0), (3, 0.0, 1.0), (3, 10.0, 0.0), (3, 10.0, float("nan"))]:
        with pytest.raises(conan.ConanError):
            conan.fof(X.reshape(-1)[: 10 * dim] if dim <= 3 else np.zeros((10, 4)), dim, L, ll)


@pytest.mark.parametrize("m_row", [2_000, 10_000])
def test_fof_long_rows(gpu, conan, oracle, m_row):
    """One transverse cell holding a column of m_row particles along x: a row
    sorted in shared memory (up to 4096 particles) and one that takes the
    radix-sort path (longer)."""
    rng = np.random.default_rng(m_row)
    L, ll, n = 100.0, 0.8, 30_000
    X = rng.uniform(0, L, size=(n, 3))
    X[:m_row, 0] = rng.uniform(0, L, m_row)
    X[:m_row, 1] = rng.uniform(50.5, 50.7, m_row)  # transverse cell (63, 25) of side 0.8
    X[:m_row, 2] = rng.uniform(20.1, 20.3, m_row)
    ref, ngr = oracle.fof(3, L, ll, X)
    for _ in range(2):
        tags, ng = conan.fof(X, 3, L, ll)
        assert ng == ngr
        assert np.array_equal(tags, ref)
