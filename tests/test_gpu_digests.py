"""Parity at the benchmarked sizes: the B200 library against digests of the
compiled reference's outputs (tests/golden/make_digests.py).

  cfg1_full  the 18.5 M-node mixed-element system the benchmark times
  cfg2_16    16 systems of the batched workload, connected in one instance
  cfg4_full  the high-order workload (linear connectivity and the
             degree-3 path)

Every iblank, every getdonorinfo record (receptor row, donor nodes and cell,
weights as bit patterns) and every updated field value must equal the
reference's: the digests count mismatches per node, per record and per 4096
field values, and the tests require zero.  Both the split-precision form
and the FP64 form are checked.
"""
import os

import numpy as np
import pytest

from tioga_b200 import cases
from tioga_b200.capi import TiogaLibrary, run_batch
from tests.golden import digest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")

pytestmark = pytest.mark.gpu


def _lib():
    import tioga_b200 as tb
    lib = TiogaLibrary(tb.library_path())
    tb.extras(lib.lib)
    return lib, tb


def _fixture(name):
    return np.load(os.path.join(GOLD, name + ".npz"))


def _zero(res):
    return res["iblank"] == 0 and res["records"] == 0 and res["q_chunks"] == 0 and res["blocks"] > 0


def connect_and_digest(lib, tb, system, q0, precision, nvar=5):
    """One connectivity call at `precision` on a registered system, then its
    donors and a data update on fresh copies of q0."""
    tb.set_int(lib.lib, "tioga_b200_set_precision_", precision)
    lib.performconnectivity()
    assert lib.lib.tioga_b200_last_error() == 0
    out = {"iblank": {}, "donors": {}, "q": {}}
    for b in system.blocks:
        out["iblank"][b.tag] = lib.iblank(b.tag).copy()
        out["donors"][b.tag] = lib.getdonorinfo(b.tag)
    qs = [np.array(q, dtype=np.float64, copy=True) for q in q0]
    for b, q in zip(system.blocks, qs):
        lib.registersolution(b.tag, q)
    lib.dataupdate_mb(nvar, "row")
    for b, q in zip(system.blocks, qs):
        out["q"][b.tag] = q
    return out, tb.stats(lib.lib)


def test_cfg1_full_matches_reference_digests():
    fix = _fixture("cfg1_full")
    system = cases.config1(1)
    assert digest.input_digest(system) == str(fix["input_digest"]), "mesh generator changed"
    q0 = cases.fields(system, nvar=5, seed=21)
    lib, tb = _lib()
    lib.init()
    lib.register_system(system)
    lib.preprocess_grids()
    for precision in (1, 0):
        out, st = connect_and_digest(lib, tb, system, q0, precision)
        res = digest.compare(fix, system, out)
        assert _zero(res), (precision, res)
        assert st["nties"] == 0
        assert st["nreceptor"] == sum(int(fix[f"counts_{b.tag}"][0]) for b in system.blocks)
    lib.delete()


def test_cfg2_batch_matches_reference_digests():
    fix = _fixture("cfg2_16")
    systems = cases.config2(2, nsys=16)
    for k, s in enumerate(systems):
        assert digest.input_digest(s) == str(fix[f"input_digest_s{k}"]), "mesh generator changed"
    q_sets = [cases.fields(s, nvar=5, seed=200 + k) for k, s in enumerate(systems)]
    import tioga_b200 as tb
    for precision in (1, 0):
        outs = run_batch(tb.library_path(), systems, q_sets=q_sets, nvar=5, itype="row",
                         setup=lambda t, p=precision: tb.set_int(t.lib, "tioga_b200_set_precision_", p))
        for k, (s, out) in enumerate(zip(systems, outs)):
            res = digest.compare(fix, s, out, prefix=f"s{k}_")
            assert _zero(res), (precision, k, res)


def test_cfg4_full_matches_digests():
    """Linear connectivity against the compiled reference; the high-order path
    against the oracle's restatement (the reference's callbacks carry no block
    id, so the reference cannot run it with both blocks active)."""
    from tests.ho_harness import run_highorder
    fix = _fixture("cfg4_full")
    system, ho = cases.config4(4)
    assert digest.input_digest(system) == str(fix["input_digest"]), "mesh generator changed"
    qlin = cases.fields(system, nvar=5, seed=5)
    lib, tb = _lib()
    lib.init()
    lib.register_system(system)
    lib.preprocess_grids()
    for precision in (1, 0):
        out, _ = connect_and_digest(lib, tb, system, qlin, precision)
        res = digest.compare(fix, system, out, prefix="lin_")
        assert _zero(res), (precision, res)
    lib.delete()
    qdof = cases.dof_fields(ho, 5, seed=5)
    for precision in (1, 0):
        hout = run_highorder(tb.library_path(), system, ho, 5, qdof, "gpu",
                             setup=lambda t, p=precision: tb.set_int(t.lib, "tioga_b200_set_precision_", p))
        for b in system.blocks:
            t = b.tag
            assert np.array_equal(hout["iblank"][t].astype(np.int8), fix[f"iblank_ho_{t}"]), (precision, t)
            assert np.array_equal(hout["cells"][t].astype(np.int8), fix[f"cells_ho_{t}"]), (precision, t)
            rec, w = hout["points"][t]
            assert np.array_equal(digest.point_hashes(rec, w), fix[f"points_ho_{t}"]), (precision, t)
            assert np.array_equal(digest.chunk_hashes(hout["q"][t]), fix[f"qhash_ho_{t}"]), (precision, t)
