"""The oracle (C restatement of the reference, oracle/tioga_oracle.c) against
golden fixtures produced by the compiled reference (tests/golden/).  Bar:
bit-identical iblank, receptor lists, donor indices, weights and updated
fields.  Runs on the CPU."""
import os

import numpy as np
import pytest

from tests.golden import make_golden as mg
from tests.conftest import REF_LIB

GOLDEN = os.path.dirname(mg.__file__)


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def check_against_golden(lib, name):
    g = load(name)
    system, q, out = mg.run_case(lib, name)
    assert str(g["digest"]) == mg.digest(system), "the seeded mesh generator changed"
    for b, q0 in zip(system.blocks, q):
        t = b.tag
        np.testing.assert_array_equal(out["iblank"][t], g[f"iblank_{t}"].astype(np.int32))
        rec, ind, frac = out["donors"][t]
        np.testing.assert_array_equal(rec, g[f"receptors_{t}"])
        np.testing.assert_array_equal(ind, g[f"indices_{t}"])
        assert np.array_equal(frac.view(np.int64), g[f"frac_{t}"].view(np.int64))
        changed = np.nonzero(out["q"][t] != q0)[0]
        np.testing.assert_array_equal(changed, g[f"qidx_{t}"])
        assert np.array_equal(out["q"][t][changed].view(np.int64), g[f"qval_{t}"].view(np.int64))


@pytest.mark.parametrize("name", list(mg.CASES))
def test_oracle_matches_reference_fixtures(name, oracle_lib):
    check_against_golden(oracle_lib, name)


@pytest.mark.parametrize("name", list(mg.CASES))
def test_compiled_reference_reproduces_fixtures(name):
    if not os.path.exists(REF_LIB):
        pytest.skip("the compiled reference needs the reference sources (make -C oracle ref)")
    check_against_golden(REF_LIB, name)


def test_fixtures_exercise_every_state():
    """The fixtures hold holes, receptors, several cell types and cancellations."""
    g = load("cfg1_small_s1")
    ibl = np.concatenate([g[k] for k in g.files if k.startswith("iblank_")])
    assert (ibl == 0).sum() > 0 and (ibl == -1).sum() > 0 and (ibl == 1).sum() > 0
    nw = np.concatenate([g[k][:, 3] for k in g.files if k.startswith("receptors_")])
    assert set(np.unique(nw)) >= {4, 5, 6, 8}


# Seeds beyond the fixtures: the restatement against the compiled reference
# run in the same process, on every observable (CPU, seconds).
LIVE_CASES = [
    ("small_config0", 3, {}),
    ("small_config0", 4, dict(isym=0, nfringe=2)),
    ("small_config1", 3, {}),
    ("small_config1", 4, dict(mexclude=1)),
    ("small_config1_seam", 3, dict(nfringe=2)),
]


@pytest.mark.parametrize("factory,seed,settings", LIVE_CASES)
def test_oracle_matches_compiled_reference_on_more_seeds(factory, seed, settings, oracle_lib):
    if not os.path.exists(REF_LIB):
        pytest.skip("the compiled reference needs the reference sources (make -C oracle ref)")
    from tioga_b200 import cases
    from tioga_b200.capi import run_system
    system = getattr(cases, factory)(seed)
    q = cases.fields(system, nvar=3, seed=100 + seed)
    ref = run_system(REF_LIB, system, q_blocks=q, nvar=3, **settings)
    got = run_system(oracle_lib, system, q_blocks=q, nvar=3, **settings)
    for b in system.blocks:
        t = b.tag
        np.testing.assert_array_equal(got["iblank"][t], ref["iblank"][t])
        for x, y in zip(got["donors"][t], ref["donors"][t]):
            assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8))
        assert np.array_equal(got["q"][t].view(np.int64), ref["q"][t].view(np.int64))
    ibl = np.concatenate([ref["iblank"][b.tag] for b in system.blocks])
    assert (ibl == -1).sum() > 0
