"""getReceptorInfo (src/tioga.C:572-671) with cell global ids: the fixtures
made by the compiled reference (tests/golden/*_gid.npz, through the C++
class by oracle/ref_gid_shim.C) against the reference's own donor lists, the
compiled reference against the fixtures, and the B200 library against both.
Bar: identical int32 rows."""
import os

import numpy as np
import pytest

from tests.conftest import REF_LIB
from tests.golden import make_golden as mg
from tioga_b200 import library_path
from tioga_b200.capi import TiogaLibrary, run_system

GOLDEN = os.path.dirname(mg.__file__)


def _fixture(name):
    return np.load(os.path.join(GOLDEN, name + "_gid.npz"))


def _donor_fixture(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    system = mg.CASES[name][0]()
    donors = {}
    for b in system.blocks:
        t = b.tag
        donors[t] = (g[f"receptors_{t}"], g[f"indices_{t}"], g[f"frac_{t}"])
    return system, donors


@pytest.mark.parametrize("name", mg.GID_CASES)
def test_fixture_agrees_with_reference_donor_lists(name):
    """The reference's getReceptorInfo rows are its getDonorInfo records,
    donor blocks in registration order, with the cell ids mapped to global
    ids (both from the compiled reference)."""
    g = _fixture(name)
    system, donors = _donor_fixture(name)
    assert str(g["digest"]) == mg.digest(system)
    gids = mg.cell_gids(system, 500 + mg.CASES[name][4])
    want = mg.receptor_info_from_donors(system, donors, gids)
    assert len(want) > 0
    np.testing.assert_array_equal(g["receptorinfo"], want)
    # the ids use their high words, so the two-word packing is exercised
    assert (g["receptorinfo"][:, 3] != 0).all()


@pytest.mark.parametrize("name", mg.GID_CASES)
def test_compiled_reference_reproduces_fixture(name):
    if not os.path.exists(REF_LIB):
        pytest.skip("the compiled reference needs the reference sources (make -C oracle ref)")
    system, gids, out = mg.run_gid_case(REF_LIB, name)
    np.testing.assert_array_equal(out["receptorinfo"], _fixture(name)["receptorinfo"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", mg.GID_CASES)
def test_b200_matches_fixture(name):
    system, gids, out = mg.run_gid_case(library_path(), name)
    np.testing.assert_array_equal(out["receptorinfo"], _fixture(name)["receptorinfo"])


@pytest.mark.gpu
def test_b200_full_cfg0_agrees_with_its_donor_lists():
    """Full-size cfg0: the rows equal those derived from the library's own
    getdonorinfo lists."""
    from tioga_b200 import cases
    system = cases.config0(0)
    gids = mg.cell_gids(system, 77)
    out = run_system(library_path(), system, cell_gids=gids)
    want = mg.receptor_info_from_donors(system, out["donors"], gids)
    assert len(want) > 1000
    np.testing.assert_array_equal(out["receptorinfo"], want)


@pytest.mark.gpu
def test_b200_missing_ids_is_an_error():
    """A donating block without cell ids reports an error (the reference
    would read through a null pointer)."""
    from tioga_b200 import cases, extras
    system = cases.small_config0(0)
    t = TiogaLibrary(library_path())
    extras(t.lib)
    t.init()
    t.register_system(system)
    t.preprocess_grids()
    t.performconnectivity()
    assert t.lib.tioga_b200_last_error() == 0
    rows = t.getreceptorinfo()
    assert rows.shape == (0, 4)
    assert t.lib.tioga_b200_last_error() != 0
    t.delete()
