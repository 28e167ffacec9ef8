"""Generate the golden fixtures from the compiled TIOGA reference.

    make -C oracle ref && python tests/golden/make_golden.py

The reference (oracle/_ref/libtioga_ref.so, compiled from the reference's own
sources with a single-rank MPI shim) is driven through its C API on small
seeded systems; its outputs are stored as compressed .npz files next to this
script together with a digest of the inputs.  The CPU tests check the C
restatement in oracle/ against these files, and the GPU tests check the B200
library against them, so parity is pinned to the reference itself.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tioga_b200 import cases  # noqa: E402
from tioga_b200.capi import run_system  # noqa: E402


def user_resolutions(system, seed):
    """Seeded user node/cell resolutions for the first block."""
    rng = np.random.default_rng(seed)
    b = system.blocks[0]
    nres = rng.uniform(0.5, 1.5, b.nnodes) * 1e-2
    cres = rng.uniform(0.5, 1.5, b.ncells) * 1e-2
    return {b.tag: (nres, cres)}


def shell_resolutions(system, seed):
    """Seeded user resolutions for every block but the first, spread widely
    enough that coincident seam nodes differ and their merged (max)
    resolution changes donor choices."""
    rng = np.random.default_rng(seed)
    return {b.tag: (rng.uniform(0.02, 0.6, b.nnodes), rng.uniform(0.02, 0.6, b.ncells))
            for b in system.blocks[1:]}


# name -> (system factory, settings, nvar, itype, field seed)
CASES = {
    "cfg0_small_s0": (lambda: cases.small_config0(0), {}, 5, "row", 11),
    "cfg1_small_s1": (lambda: cases.small_config1(1), {}, 5, "row", 12),
    "cfg0_small_s1_opts": (lambda: cases.small_config0(1), dict(isym=0, nfringe=2, mexclude=1), 3, "column", 13),
    "cfg1_small_s2_userres": (lambda: cases.small_config1(2), "userres", 2, "row", 14),
    # duplicated phi seams: coincident query points, merged by uniqNodesTree
    "cfg1_small_s1_seam": (lambda: cases.small_config1_seam(1), {}, 5, "row", 15),
    "cfg0_small_s2_seam_shellres": (lambda: cases.small_config0_seam(2), "shellres", 4, "row", 16),
    # tioga_reduce_fringes_ after the connectivity (tioga.C:737-885)
    "cfg0_small_s0_reduce": (lambda: cases.small_config0(0), "reduce", 5, "row", 17),
    "cfg1_small_s1_reduce_nf2": (lambda: cases.small_config1(1), "reduce_nf2", 5, "row", 18),
    "cfg1_small_s1_seam_reduce": (lambda: cases.small_config1_seam(1), "reduce", 5, "row", 19),
}


def _reduce(t):
    t.lib.tioga_reduce_fringes_()


# cases rerun with cell global ids on every block, for getReceptorInfo
# (tioga.C:572-671); stored as <name>_gid.npz
GID_CASES = ("cfg0_small_s0", "cfg1_small_s1", "cfg1_small_s1_reduce_nf2")


def cell_gids(system, seed):
    """Seeded, distinct uint64 cell ids per block, with high words in use."""
    rng = np.random.default_rng(seed)
    out = []
    for b in system.blocks:
        perm = rng.permutation(b.ncells).astype(np.uint64)
        out.append((np.uint64(b.tag) << np.uint64(40)) + perm * np.uint64(1000003) + np.uint64(7))
    return out


def receptor_info_from_donors(system, donors, gids):
    """getReceptorInfo restated from getDonorInfo's lists (dataUpdate.C:121-178):
    per donor block in registration order, per live record, (receptor node,
    mesh tag of the receptor block, donor cell id's global id as two int32
    words, low first)."""
    tags = [b.tag for b in system.blocks]
    rows = []
    for k, b in enumerate(system.blocks):
        rec, ind, _ = donors[b.tag]
        pos = 0
        for r in rec:
            nw = int(r[3])
            cell = int(ind[pos + nw])
            pos += nw + 1
            g = int(gids[k][cell])
            rows.append([int(r[1]), tags[int(r[2])], np.int64(g & 0xffffffff).astype(np.int32),
                         np.int64(g >> 32).astype(np.int32)])
    return np.array(rows, dtype=np.int32).reshape(-1, 4)


def run_gid_case(lib, name):
    fac, _, nvar, itype, fseed = CASES[name]
    system = fac()
    gids = cell_gids(system, 500 + fseed)
    out = run_system(lib, system, nvar=nvar, itype=itype, cell_gids=gids, **settings_for(name, system))
    return system, gids, out


def digest(system):
    h = hashlib.sha256()
    for b in system.blocks:
        h.update(np.ascontiguousarray(b.x).tobytes())
        for nv, c in b.cells:
            h.update(np.int32(nv).tobytes())
            h.update(np.ascontiguousarray(c, dtype=np.int32).tobytes())
        h.update(np.ascontiguousarray(b.wbc, dtype=np.int32).tobytes())
        h.update(np.ascontiguousarray(b.obc, dtype=np.int32).tobytes())
    return h.hexdigest()


def settings_for(name, system):
    s = CASES[name][1]
    if s == "userres":
        return {"resolutions": user_resolutions(system, 99)}
    if s == "shellres":
        return {"resolutions": shell_resolutions(system, 98)}
    if s == "reduce":
        return {"after": _reduce}
    if s == "reduce_nf2":
        return {"after": _reduce, "nfringe": 2}
    return dict(s)


def run_case(lib, name):
    fac, _, nvar, itype, fseed = CASES[name]
    system = fac()
    q = cases.fields(system, nvar=nvar, seed=fseed)
    out = run_system(lib, system, q_blocks=q, nvar=nvar, itype=itype, **settings_for(name, system))
    return system, q, out


def save(name, system, q, out):
    arrs = {"digest": np.array(digest(system))}
    for b, q0 in zip(system.blocks, q):
        t = b.tag
        arrs[f"iblank_{t}"] = out["iblank"][t].astype(np.int8)
        rec, ind, frac = out["donors"][t]
        arrs[f"receptors_{t}"] = rec
        arrs[f"indices_{t}"] = ind
        arrs[f"frac_{t}"] = frac
        changed = np.nonzero(out["q"][t] != q0)[0]
        arrs[f"qidx_{t}"] = changed.astype(np.int32)
        arrs[f"qval_{t}"] = out["q"][t][changed]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrs)


if __name__ == "__main__":
    lib = os.path.join(ROOT, "oracle", "_ref", "libtioga_ref.so")
    if not os.path.exists(lib):
        sys.exit("build the compiled reference first: make -C oracle ref")
    names = sys.argv[1:] or list(CASES) + [n + "_gid" for n in GID_CASES]
    for name in names:
        if name.endswith("_gid"):
            system, gids, out = run_gid_case(lib, name[:-4])
            np.savez_compressed(os.path.join(HERE, name + ".npz"), digest=np.array(digest(system)),
                                receptorinfo=out["receptorinfo"])
        else:
            system, q, out = run_case(lib, name)
            save(name, system, q, out)
        print(name, "saved")
