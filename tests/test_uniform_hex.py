"""The uniform-hex fast path (tioga::set_uniform_hex_flag, src/tioga.h:195-201;
MeshBlock::check_for_uniform_hex and create_hex_cell_map, src/MeshBlock.C:
1249-1409; MeshBlock::search_uniform_hex, src/search.C:271-341): a block of
identical rectangular hexahedra is searched by index lookup instead of its
tree.  The reference offers the switch only through its C++ class; the
compiled reference gets it through the test shim (oracle/ref_gid_shim.C).

CPU: the oracle's restatement against the compiled reference.  GPU: the
library (tioga_b200_set_uniform_hex_flag_) against the compiled reference,
in both precision forms.  The shell carries the flag too in one case: it is
not uniform, so its check fails and it keeps the tree search."""
import ctypes as C
import os

import numpy as np
import pytest

from tioga_b200 import cases
from tioga_b200.capi import run_system
from tests.compare import diff_runs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libtioga_ref.so")

CASES = [(0, (1,)), (1, (1,)), (2, (1, 2))]  # seed, tags flagged


def _flags(kind, tags):
    def setup(t):
        for tag in tags:
            if kind == "ref":
                t.lib.refshim_set_uniform_hex_flag_(C.byref(C.c_int(tag)), C.byref(C.c_int(1)))
            elif kind == "oracle":
                t.lib.tioga_oracle_set_uniform_hex_flag(C.c_int(tag), C.c_int(1))
            else:
                t.lib.tioga_b200_set_uniform_hex_flag_(C.byref(C.c_int(tag)), C.byref(C.c_int(1)))
    return setup


def _combine(*fns):
    def setup(t):
        for f in fns:
            f(t)
    return setup


@pytest.mark.skipif(not os.path.exists(REF), reason="needs the compiled reference (make -C oracle ref)")
@pytest.mark.parametrize("seed,tags", CASES)
def test_oracle_uniform_hex_matches_reference(oracle_lib, seed, tags):
    system = cases.small_config0_uniform(seed)
    q = cases.fields(system, nvar=3, seed=40 + seed)
    ref = run_system(REF, system, q_blocks=q, nvar=3, setup=_flags("ref", tags))
    orc = run_system(oracle_lib, system, q_blocks=q, nvar=3, setup=_flags("oracle", tags),
                     after=lambda t: [t.lib.tioga_oracle_uniform_hex(C.c_int(b.tag)) for b in system.blocks])
    assert orc["after"] == [1, 0]  # the box is found uniform, the shell is not
    assert not diff_runs(system, ref, orc)
    assert ref["donors"][1][0].shape[0] > 0  # the box donates
    # the lookup takes a cell by index, without the tree's containment order,
    # so donors on shared faces differ from the tree search's: the case is live
    plain = run_system(REF, system, q_blocks=q, nvar=3)
    assert diff_runs(system, plain, ref)


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF), reason="needs the compiled reference (make -C oracle ref)")
@pytest.mark.parametrize("seed,tags", CASES)
@pytest.mark.parametrize("precision", [1, 0])
def test_gpu_uniform_hex_matches_reference(seed, tags, precision):
    """Shifted box: no face coincidences, every output exact and no tie."""
    import tioga_b200 as tb
    system = cases.small_config0_uniform(seed, shift=0.0173)
    q = cases.fields(system, nvar=3, seed=40 + seed)
    ref = run_system(REF, system, q_blocks=q, nvar=3, setup=_flags("ref", tags))

    def prec(t):
        tb.set_int(t.lib, "tioga_b200_set_precision_", precision)

    gpu = run_system(tb.library_path(), system, q_blocks=q, nvar=3,
                     setup=_combine(_flags("gpu", tags), prec),
                     after=lambda t: (tb.extras(t.lib).tioga_b200_last_error(), tb.stats(t.lib)["nties"]))
    assert gpu["after"] == (0, 0)  # no error, no order-dependent tie
    assert not diff_runs(system, ref, gpu)


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF), reason="needs the compiled reference (make -C oracle ref)")
@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("precision", [1, 0])
def test_gpu_uniform_hex_on_faces(seed, precision):
    """Unshifted box: the shell's seam and pole nodes lie on box faces, where
    the lookup decides (the box's donor records must equal the reference's);
    the box's lattice nodes lie on the shell's seam faces, where two shell
    cells accept and the reference's tree order decides.  There the library
    takes the lowest cell id and counts the query as a tie: the shell's
    records may differ only at counted ties."""
    import tioga_b200 as tb
    system = cases.small_config0_uniform(seed)
    q = cases.fields(system, nvar=3, seed=40 + seed)
    ref = run_system(REF, system, q_blocks=q, nvar=3, setup=_flags("ref", (1,)))

    def prec(t):
        tb.set_int(t.lib, "tioga_b200_set_precision_", precision)

    gpu = run_system(tb.library_path(), system, q_blocks=q, nvar=3, setup=_combine(_flags("gpu", (1,)), prec),
                     after=lambda t: (tb.extras(t.lib).tioga_b200_last_error(), tb.stats(t.lib)["nties"]))
    err, nties = gpu["after"]
    assert err == 0
    box, shell = system.blocks[0].tag, system.blocks[1].tag
    for t in (box, shell):
        assert np.array_equal(ref["iblank"][t], gpu["iblank"][t])
    for a, b in zip(ref["donors"][box], gpu["donors"][box]):
        assert np.array_equal(a, b)
    ra, ia, _ = ref["donors"][shell]
    rb, ib, _ = gpu["donors"][shell]
    assert np.array_equal(ra, rb)  # the same receptors
    pos = np.concatenate([[0], np.cumsum(ra[:, 3] + 1)])
    differ = sum(not np.array_equal(ia[pos[k]:pos[k + 1]], ib[pos[k]:pos[k + 1]]) for k in range(ra.shape[0]))
    assert differ <= nties, (differ, nties)
