"""Failure detection on the GPU without a fault: a bounded wait that nothing
completes runs out, the host reads CONAN_ERR_TIMEOUT from the error word,
and the context stays usable for the next calls."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_reports_a_timeout(gpu, conan):
    from conan_b200 import _lib as L
    lib = L.lib()
    for _ in range(2):
        rc = lib.conan_selftest_bounded_wait(2000, None)
        assert rc == L.ERR_TIMEOUT, L.last_error()
        assert "bounded wait" in L.last_error()
    # the device still works: a deposit through the handle afterwards
    n = 16
    g = conan.Gravity(3, n, 1, float(n), precision="fp32")
    q = np.stack(np.meshgrid(*[np.arange(n)] * 3, indexing="ij"), -1).reshape(-1, 3)[:, ::-1].astype(np.float64)
    g.set_state(q + 0.25, np.zeros_like(q), 0.5, 0.5)
    d = g.density()
    g.close()
    assert abs(d.mean()) < 1e-6 and np.all(np.abs(d) < 1e-5)  # a uniform lattice: delta = 0
