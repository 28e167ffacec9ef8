"""The batched and served workloads' generators (CPU): sizes drawn
log-uniformly within the stated range, 1-4 shells per system, both element
mixes, dense mesh tags, walls on every shell, and the host form of the rigid
motion (the bits the device's k_rigid produces)."""
import numpy as np

from tioga_b200 import cases
from tioga_b200.serving import apply_rigid, rigid


def test_batch_distribution():
    systems = cases.config2(2, nsys=16, nmin=3e3, nmax=3e4)
    assert len(systems) == 16
    shells = [len(s.blocks) - 1 for s in systems]
    assert min(shells) >= 1 and max(shells) <= 4
    mixed = [s.meta["mixed"] for s in systems]
    assert any(mixed) and not all(mixed)
    for s in systems:
        assert [b.tag for b in s.blocks] == list(range(1, len(s.blocks) + 1))
        assert len(s.blocks[0].wbc) == 0
        assert all(len(b.wbc) > 0 and len(b.obc) > 0 for b in s.blocks[1:])
        nvs = {nv for b in s.blocks for nv, _ in b.cells}
        assert nvs == {8} if not s.meta["mixed"] else len(nvs) > 1
        # the node budget lands within a factor of the target range
        assert 1e3 < s.nnodes < 1e5
    # reproducible from the seed
    again = cases.config2(2, nsys=16, nmin=3e3, nmax=3e4)
    assert all(np.array_equal(a.blocks[1].x, b.blocks[1].x) for a, b in zip(systems, again))


def test_rigid_motion_keeps_distances():
    rng = np.random.default_rng(5)
    x = rng.normal(size=(500, 3))
    A, b = rigid(rng, x.mean(axis=0), max_deg=2.0, max_shift=0.1)
    assert np.allclose(A @ A.T, np.eye(3), atol=1e-14)
    y = apply_rigid(x.copy(), A, b)
    d0 = np.linalg.norm(x[1:] - x[:-1], axis=1)
    d1 = np.linalg.norm(y[1:] - y[:-1], axis=1)
    assert np.allclose(d0, d1, rtol=1e-13)
    # component k is ((A[k,0] x + A[k,1] y) + A[k,2] z) + b[k], in that order
    k = 1
    want = ((A[k, 0] * x[:, 0] + A[k, 1] * x[:, 1]) + A[k, 2] * x[:, 2]) + b[k]
    assert np.array_equal(y[:, k].view(np.int64), want.view(np.int64))
