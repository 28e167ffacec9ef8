"""Serving form on the GPU: requests (time steps with rigid motions of the
shells) of several systems run through the request loop.  Each result must be
the same, bit for bit, alone (one system, one slot) and in the mix (all
systems, several slots, a budget small enough to evict and re-admit
systems), and the last step of every system must equal the oracle run on the
moved meshes (the reference's per-step sequence on the same inputs)."""
import numpy as np
import pytest

from tioga_b200 import cases
from tioga_b200.capi import run_system
from tioga_b200.serving import Server, apply_rigid, rigid
from tests.compare import diff_runs

pytestmark = pytest.mark.gpu

NSTEPS = 3
NVAR = 5


def _workload():
    systems = cases.small_config2(7, nsys=5)
    steps = []  # steps[s][k] = [(tag, A, b)]
    for s, sysm in enumerate(systems):
        rng = np.random.default_rng(100 + s)
        cur = [b.x.copy() for b in sysm.blocks]
        st = []
        for k in range(NSTEPS):
            mv = []
            for i, b in enumerate(sysm.blocks[1:], start=1):
                A, bb = rigid(rng, cur[i].mean(axis=0), max_deg=2.0, max_shift=0.02)
                apply_rigid(cur[i], A, bb)
                mv.append((b.tag, A, bb))
            st.append(mv)
        steps.append(st)
    return systems, steps


def _fields(system, s, k):
    return cases.fields(system, nvar=NVAR, seed=1000 * s + k)


def _run(server, systems, steps, order):
    """Submit the (system, step) requests in `order`, each with its own
    output arrays; returns {(s, k): (iblanks, q)}."""
    tickets, outs = [], {}
    for s, k in order:
        sysm = systems[s]
        q = [a.copy() for a in _fields(sysm, s, k)]
        ibl = [np.zeros(b.nnodes, dtype=np.int32) for b in sysm.blocks]
        tickets.append(((s, k), server.submit(s, steps[s][k], q=q, nvar=NVAR, ibl_out=ibl)))
        outs[(s, k)] = (ibl, q)
    for key, t in tickets:
        info = server.wait(t)
        assert info["rc"] == 0, (key, info)
        assert info["nquery"] > 0
    return outs


@pytest.mark.timeout(600)
def test_same_alone_and_in_the_mix(oracle_lib):
    systems, steps = _workload()
    alone, held = {}, []
    for s, sysm in enumerate(systems):
        srv = Server(budget_bytes=8 << 30, nslots=1)
        srv.add_system(s, sysm)
        alone.update(_run(srv, systems, steps, [(s, k) for k in range(NSTEPS)]))
        held.append(srv.stats()["bytes"])
        srv.close()
    # the mix: every system at once, three slots, room for about half of them
    # (so systems are evicted and admitted again between their steps)
    budget = int(max(1.2 * max(held), 0.5 * sum(held)))
    srv = Server(budget_bytes=budget, nslots=3)
    for s, sysm in enumerate(systems):
        srv.add_system(s, sysm)
    order = [(s, k) for k in range(NSTEPS) for s in range(len(systems))]
    mix = _run(srv, systems, steps, order)
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(order)
    assert st["evictions"] > 0, st
    for key in alone:
        ia, qa = alone[key]
        ib, qb = mix[key]
        for a, b in zip(ia, ib):
            assert np.array_equal(a, b), f"iblank differs for {key}"
        for a, b in zip(qa, qb):
            assert np.array_equal(a.view(np.int64), b.view(np.int64)), f"fields differ for {key}"
    # the last step against the oracle on the moved meshes
    for s, sysm in enumerate(systems):
        moved = cases.System([cases.Block(b.tag, b.x.copy(), b.cells, b.wbc, b.obc, b.name) for b in sysm.blocks],
                             sysm.name, sysm.meta)
        for k in range(NSTEPS):
            for tag, A, bb in steps[s][k]:
                blk = [b for b in moved.blocks if b.tag == tag][0]
                apply_rigid(blk.x, A, bb)
        ref = run_system(oracle_lib, moved, q_blocks=_fields(sysm, s, NSTEPS - 1), nvar=NVAR)
        ibl, q = alone[(s, NSTEPS - 1)]
        got = {"iblank": {b.tag: ibl[i] for i, b in enumerate(sysm.blocks)},
               "donors": ref["donors"], "q": {b.tag: q[i] for i, b in enumerate(sysm.blocks)}}
        problems = diff_runs(moved, ref, got)
        assert not problems, f"system {s}:\n" + "\n".join(problems)


@pytest.mark.timeout(300)
def test_device_fields_equal_host_fields():
    """A request whose fields live on the device (a GPU solver's arrays)
    updates them exactly as the host form updates host arrays."""
    import torch
    systems, steps = _workload()
    s, sysm = 1, systems[1]
    out = {}
    for form in ("host", "device"):
        srv = Server(budget_bytes=8 << 30, nslots=1)
        srv.add_system(s, sysm)
        res = []
        for k in range(NSTEPS):
            q = [a.copy() for a in _fields(sysm, s, k)]
            ibl = [np.zeros(b.nnodes, dtype=np.int32) for b in sysm.blocks]
            if form == "host":
                info = srv.wait(srv.submit(s, steps[s][k], q=q, nvar=NVAR, ibl_out=ibl))
            else:
                dq = [torch.from_numpy(a).cuda() for a in q]
                info = srv.wait(srv.submit(s, steps[s][k], q_device=dq, nvar=NVAR, ibl_out=ibl))
                torch.cuda.synchronize()
                q = [t.cpu().numpy() for t in dq]
            assert info["rc"] == 0, info
            res.append((ibl, q))
        srv.close()
        out[form] = res
    for (ia, qa), (ib, qb) in zip(out["host"], out["device"]):
        for a, b in zip(ia, ib):
            assert np.array_equal(a, b)
        for a, b in zip(qa, qb):
            assert np.array_equal(a.view(np.int64), b.view(np.int64))


@pytest.mark.timeout(300)
def test_pool_reserved_and_not_grown():
    """The server's memory pool is reserved at creation and serves every
    request of a moving-mesh stream without growing (a growth holds the
    pool's lock and stalls every slot)."""
    systems, steps = _workload()
    srv = Server(budget_bytes=4 << 30, nslots=3)
    for s, sysm in enumerate(systems):
        srv.add_system(s, sysm)
    st0 = srv.stats()
    assert st0["pool_reserved_at_create"] > 0
    assert st0["pool_bytes"] >= st0["pool_reserved_at_create"]
    order = [(s, k) for k in range(NSTEPS) for s in range(len(systems))]
    _run(srv, systems, steps, order)
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(order)
    assert st["peak_bytes"] <= st["pool_reserved_at_create"]
    assert st["pool_bytes"] == st0["pool_bytes"], (st0, st)
