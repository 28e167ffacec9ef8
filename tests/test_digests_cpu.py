"""The digest fixtures of the benchmarked sizes, on the CPU: the digests see
single-bit changes, and the oracle's restatement reproduces the compiled
reference's digests on the smallest systems of the batched workload."""
import os

import numpy as np
import pytest

from tioga_b200 import cases
from tioga_b200.capi import run_system
from tests.golden import digest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def test_record_hashes_see_one_bit():
    f = np.load(os.path.join(GOLD, "cfg1_small_s1.npz"))
    rec, ind, frac = f["receptors_2"], f["indices_2"], f["frac_2"]
    h = digest.record_hashes(rec, ind, frac)
    assert h.size == rec.shape[0] and np.unique(h).size == h.size
    f2 = frac.copy()
    f2[7] = np.nextafter(f2[7], 2.0)
    assert (digest.record_hashes(rec, ind, f2) != h).sum() == 1
    i2 = ind.copy()
    i2[-1] += 1  # the last record's donor cell
    h2 = digest.record_hashes(rec, i2, frac)
    assert (h2 != h).sum() == 1 and h2[-1] != h[-1]
    r2 = rec.copy()
    r2[0, 1] += 1  # the first record's receptor node
    assert (digest.record_hashes(r2, ind, frac) != h).sum() == 1


def test_chunk_hashes_see_one_value():
    q = np.random.default_rng(0).uniform(-1, 1, 3 * digest.Q_CHUNK + 17)
    h = digest.chunk_hashes(q)
    assert h.size == 4
    q[digest.Q_CHUNK + 5] = np.nextafter(q[digest.Q_CHUNK + 5], 2.0)
    assert (digest.chunk_hashes(q) != h).tolist() == [False, True, False, False]


@pytest.mark.parametrize("k", [2, 12])
def test_oracle_matches_reference_digests_cfg2(oracle_lib, k):
    """Systems 2 and 12 of the batched workload (30 k and 39 k nodes)."""
    fix = np.load(os.path.join(GOLD, "cfg2_16.npz"))
    system = cases.config2(2, nsys=k + 1)[k]
    assert digest.input_digest(system) == str(fix[f"input_digest_s{k}"])
    q0 = cases.fields(system, nvar=5, seed=200 + k)
    out = run_system(oracle_lib, system, q_blocks=q0, nvar=5, itype="row")
    res = digest.compare(fix, system, out, prefix=f"s{k}_")
    assert res["blocks"] == len(system.blocks)
    assert res["iblank"] == 0 and res["records"] == 0 and res["q_chunks"] == 0, res
