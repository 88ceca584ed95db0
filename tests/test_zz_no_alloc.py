"""conan_deposit_static, the deposit entry point that allocates nothing,
checked through the C ABI against conan_pm_density (the handle's own FP32
deposit) on the same particles, two calls in a row with different inputs so
that the second call also shows the shared accumulator was cleared.

This file is collected last on purpose: it runs after every other test in a
full run, and it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TOL = 1e-5  # the FP32 deposit tolerance of the parity tests (relative to max(1, |delta|))


def _particles(dim, n, f, amp, seed):
    """Displacements (dim, n^dim) FP32 in force cells and the matching
    absolute positions for a box of L = n f (one force cell = 1)."""
    rng = np.random.default_rng(seed)
    d = rng.uniform(-amp, amp, size=(dim, n ** dim)).astype(np.float32)
    q = np.stack(np.meshgrid(*[np.arange(n)] * dim, indexing="ij"), -1).reshape(-1, dim)[:, ::-1]
    X = np.ascontiguousarray(q * f + d.T.astype(np.float64))
    return d, X


def _static(lib, dim, n, f, d, stream):
    dt = torch.from_numpy(d).cuda()
    out = torch.empty((n * f) ** dim, dtype=torch.float32, device="cuda")
    ptr = [dt[k].data_ptr() if k < dim else None for k in range(3)]
    rc = lib.conan_deposit_static(dim, n, f, ptr[0], ptr[1], ptr[2], out.data_ptr(), stream)
    return rc, dt, out


# fine meshes (3D f = 4 and 8, 2D f = 8: 128^3 and 1024^2 cells) take the
# two-cell window, where every corner goes to the accumulator directly
@pytest.mark.parametrize("dim,n,f,amp", [(3, 32, 1, 3.0), (3, 64, 2, 12.0), (3, 8, 2, 40.0), (2, 256, 1, 30.0),
                                         (2, 32, 4, 5.0), (1, 1024, 2, 300.0), (3, 32, 4, 6.0), (3, 16, 8, 20.0),
                                         (2, 128, 8, 10.0)])
def test_static_deposit_matches_pm_density(gpu, conan, dim, n, f, amp):
    from conan_b200 import _lib as L
    lib = L.lib()
    stream = torch.cuda.current_stream().cuda_stream
    g = conan.Gravity(dim, n, f, float(n * f), precision="fp32")
    for call, seed in enumerate((21, 22)):  # two calls in a row, different particles
        d, X = _particles(dim, n, f, amp, seed)
        g.set_state(X, np.zeros_like(X), 0.5, 0.5)
        ref = g.density()
        rc, dt, out = _static(lib, dim, n, f, d, stream)
        assert rc == L.OK, L.last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy().astype(np.float64)
        err = np.max(np.abs(got - ref))
        assert err <= TOL * max(1.0, np.max(np.abs(ref))), f"call {call}: max difference {err}"
    g.close()


def test_static_deposit_rejects_meshes_beyond_its_array(gpu, conan):
    from conan_b200 import _lib as L
    lib = L.lib()
    d = torch.zeros((3, 8), dtype=torch.float32, device="cuda")
    out = torch.zeros(8, dtype=torch.float32, device="cuda")
    # 256^3 = 2^24 cells > 2^21: refused before any device work
    rc = lib.conan_deposit_static(3, 128, 2, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), out.data_ptr(), None)
    assert rc == L.ERR_ARG and "at most 2097152 cells" in L.last_error()
    rc = lib.conan_deposit_static(4, 8, 1, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), out.data_ptr(), None)
    assert rc == L.ERR_UNSUPPORTED
    rc = lib.conan_deposit_static(3, 4, 1, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), out.data_ptr(), None)
    assert rc == L.ERR_UNSUPPORTED  # below the smallest lattice tile
