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
