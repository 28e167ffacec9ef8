"""Digest fixtures of the compiled TIOGA reference at the benchmarked sizes.

    make -C oracle ref oracle && python tests/golden/make_digests.py [cfg1 cfg2 cfg4]

The reference (oracle/_ref/libtioga_ref.so, built from the reference's own
sources) runs the full call sequence on the workloads the benchmark times:

  cfg1_full   config1(seed 1): the 257^3 mixed-element background and three
              65x65x129 shells (18.5 M nodes), 5 fields ~ U(-1,1)
  cfg2_16     the first 16 systems of config2(seed 2) (the batched workload),
              each connected alone as the reference runs independent systems
  cfg4_full   config4(seed 4): the linear connectivity by the compiled
              reference ("lin" digests), and the high-order path by the
              oracle's restatement driven by the Lagrange callbacks ("ho"
              digests).  The reference's callbacks carry no block id, so it
              cannot run the high-order path with both blocks active; the
              restatement is pinned against it where it can
              (tests/test_highorder_oracle.py).

Each fixture stores digests (tests/golden/digest.py), not the outputs, plus
the input digest and the reference's wall time per call on one core.
"""
from __future__ import annotations

import ctypes as C
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tioga_b200 import cases  # noqa: E402
from tioga_b200.capi import TiogaLibrary  # noqa: E402
from tests.golden import digest  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "libtioga_ref.so")
ORACLE = os.path.join(ROOT, "oracle", "_ref", "liboracle.so")
CFG2_SYSTEMS = 16
NVAR = 5
FIELD_SEED = {"cfg1_full": 21, "cfg2_16": 200, "cfg4_full": 5}


def run_timed(lib_path, system, q0, nvar=NVAR):
    """The reference's call sequence with the calls timed.  Returns the
    run_system-style result and (preprocess s, connectivity s, data update s)."""
    t = TiogaLibrary(lib_path)
    t.init()
    t.register_system(system)
    t0 = time.perf_counter()
    t.preprocess_grids()
    t1 = time.perf_counter()
    t.performconnectivity()
    t2 = time.perf_counter()
    out = {"iblank": {}, "donors": {}, "q": {}}
    for b in system.blocks:
        out["iblank"][b.tag] = t.iblank(b.tag).copy()
        out["donors"][b.tag] = t.getdonorinfo(b.tag)
    qs = [np.array(q, dtype=np.float64, copy=True) for q in q0]
    for b, q in zip(system.blocks, qs):
        t.registersolution(b.tag, q)
    t3 = time.perf_counter()
    t.dataupdate_mb(nvar, "row")
    t4 = time.perf_counter()
    for b, q in zip(system.blocks, qs):
        out["q"][b.tag] = q
    t.delete()
    return out, (t1 - t0, t2 - t1, t4 - t3)


def query_count(system) -> int:
    """Q (the metric's unit) from the oracle's query lists, which equal the
    reference's nsearch lists."""
    t = TiogaLibrary(ORACLE)
    t.init()
    t.register_system(system)
    t.preprocess_grids()
    t.performconnectivity()
    ns, nd, tot = C.c_int(), C.c_int(), 0
    for b in system.blocks:
        t.lib.tioga_oracle_searchstats(C.c_int(b.tag), C.byref(ns), C.byref(nd))
        tot += ns.value
    t.delete()
    return tot


def make_cfg1():
    name = "cfg1_full"
    system = cases.config1(1)
    q0 = cases.fields(system, nvar=NVAR, seed=FIELD_SEED[name])
    out, (tp, tc, tu) = run_timed(REF, system, q0)
    arrs = digest.make(system, out, q0)
    arrs["input_digest"] = np.array(digest.input_digest(system))
    arrs["ref_seconds"] = np.array([tp, tc, tu])
    arrs["query_points"] = np.array([query_count(system)])
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrs)
    print(name, "saved: preprocess %.1f s, connectivity %.1f s, update %.2f s" % (tp, tc, tu), flush=True)


def make_cfg2():
    name = "cfg2_16"
    systems = cases.config2(2, nsys=CFG2_SYSTEMS)
    arrs, secs, qs = {}, [], []
    for k, system in enumerate(systems):
        q0 = cases.fields(system, nvar=NVAR, seed=FIELD_SEED[name] + k)
        out, s = run_timed(REF, system, q0)
        arrs.update(digest.make(system, out, q0, prefix=f"s{k}_"))
        arrs[f"input_digest_s{k}"] = np.array(digest.input_digest(system))
        secs.append(s)
        qs.append(query_count(system))
        print(name, k, system.name, "connectivity %.1f s" % s[1], flush=True)
    arrs["ref_seconds"] = np.array(secs)
    arrs["query_points"] = np.array(qs)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrs)
    print(name, "saved", flush=True)


def make_cfg4():
    from tests.ho_harness import run_highorder
    name = "cfg4_full"
    system, ho = cases.config4(4)
    qlin = cases.fields(system, nvar=NVAR, seed=FIELD_SEED[name])
    out, s = run_timed(REF, system, qlin)
    arrs = digest.make(system, out, qlin, prefix="lin_")
    qdof = cases.dof_fields(ho, NVAR, seed=FIELD_SEED[name])
    t0 = time.perf_counter()
    hout = run_highorder(ORACLE, system, ho, NVAR, qdof, "hook")
    tho = time.perf_counter() - t0
    for b in system.blocks:
        t = b.tag
        arrs[f"iblank_ho_{t}"] = hout["iblank"][t].astype(np.int8)
        arrs[f"cells_ho_{t}"] = hout["cells"][t].astype(np.int8)
        rec, w = hout["points"][t]
        arrs[f"points_ho_{t}"] = digest.point_hashes(rec, w)
        arrs[f"qhash_ho_{t}"] = digest.chunk_hashes(hout["q"][t])
    arrs["input_digest"] = np.array(digest.input_digest(system))
    arrs["ref_seconds"] = np.array([s[0], s[1], s[2], tho])
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrs)
    print(name, "saved: reference connectivity %.1f s, oracle high-order run %.1f s" % (s[1], tho), flush=True)


if __name__ == "__main__":
    if not (os.path.exists(REF) and os.path.exists(ORACLE)):
        sys.exit("build the compiled reference and the oracle first: make -C oracle ref oracle")
    which = sys.argv[1:] or ["cfg1", "cfg2", "cfg4"]
    for w in which:
        {"cfg1": make_cfg1, "cfg2": make_cfg2, "cfg4": make_cfg4}[w]()
