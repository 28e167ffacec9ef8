"""Compact digests of a connectivity result, for parity at the benchmarked sizes.

At full size (cfg1: 18.5 M nodes, about 0.4 M interpolation records) the
reference's outputs are too large to store, so a fixture keeps:

  iblank      every node's iblank (int8, compressed: it is mostly 1)
  records     one 32-bit hash per getdonorinfo record (dataUpdate.C:136-159):
              its receptor row (4 ints), donor indices (nw+1 ints, the last
              the donor cell id) and weights (nw+1 doubles, as bit patterns)
  q           one 32-bit hash per 4096 values of the updated fields (ROW layout)
  counts      dcount, fcount and the number of updated values per block

Mismatches are then counted exactly for iblanks and per record for donors
(a record whose hash differs is a mismatch; two different records collide
with probability 2^-32), and per chunk for the updated fields.

The hash is a sum over a record's words of splitmix64(word + position key),
so it is vectorised with numpy and independent of how records are chunked.
"""
from __future__ import annotations

import hashlib

import numpy as np

Q_CHUNK = 4096
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_G = np.uint64(0x9E3779B97F4A7C15)


def _key(c: int) -> np.uint64:
    """c times the golden-ratio constant, modulo 2^64 (a column key)."""
    return np.uint64((c * 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF)


def _mix(z: np.ndarray) -> np.ndarray:
    """splitmix64's finaliser, elementwise on uint64 (wrapping arithmetic)."""
    z = z.astype(np.uint64, copy=True)
    z ^= z >> np.uint64(30)
    z *= _M1
    z ^= z >> np.uint64(27)
    z *= _M2
    z ^= z >> np.uint64(31)
    return z


def _segment_sum(vals: np.ndarray, starts: np.ndarray, n: int) -> np.ndarray:
    out = np.zeros(n, dtype=np.uint64)
    if n == 0 or vals.size == 0:
        return out
    nonempty = starts < vals.size
    out[nonempty] = np.add.reduceat(vals, starts[nonempty])
    return out


def record_hashes(rec: np.ndarray, ind: np.ndarray, frac: np.ndarray) -> np.ndarray:
    """uint32 hash per getdonorinfo record.  rec is (dcount, 4) with the
    weight count in column 3; ind and frac hold nw+1 entries per record."""
    rec = np.asarray(rec, dtype=np.int64).reshape(-1, 4)
    d = rec.shape[0]
    if d == 0:
        return np.zeros(0, dtype=np.uint32)
    nw1 = rec[:, 3] + 1
    starts = np.zeros(d, dtype=np.int64)
    np.cumsum(nw1[:-1], out=starts[1:])
    total = int(nw1.sum())
    if total != len(ind) or total != len(frac):
        raise ValueError(f"record lengths {total} do not match indices {len(ind)} / weights {len(frac)}")
    pos = (np.arange(total, dtype=np.int64) - np.repeat(starts, nw1)).astype(np.uint64)
    iw = np.asarray(ind, dtype=np.int64).astype(np.uint64)
    fw = np.ascontiguousarray(frac, dtype=np.float64).view(np.uint64)
    h_i = _mix(iw + (pos + np.uint64(16)) * _G)
    h_f = _mix(fw ^ ((pos + np.uint64(48)) * _G))
    h = _segment_sum(h_i + h_f, starts, d)
    for c in range(4):
        h += _mix(rec[:, c].astype(np.uint64) + _key(c + 1))
    return (h >> np.uint64(32)).astype(np.uint32)


def chunk_hashes(values: np.ndarray, chunk: int = Q_CHUNK) -> np.ndarray:
    """uint32 hash per `chunk` consecutive FP64 values (their bit patterns)."""
    w = np.ascontiguousarray(values, dtype=np.float64).view(np.uint64)
    n = (w.size + chunk - 1) // chunk
    pos = np.arange(w.size, dtype=np.uint64) % np.uint64(chunk)
    h = _mix(w ^ ((pos + np.uint64(1)) * _G))
    starts = np.arange(n, dtype=np.int64) * chunk
    return (_segment_sum(h, starts, n) >> np.uint64(32)).astype(np.uint32)


def point_hashes(rec: np.ndarray, w: np.ndarray) -> np.ndarray:
    """uint32 hash per high-order point donor: its 4-int record and its
    weight row (bit patterns, trailing zeros included)."""
    rec = np.asarray(rec, dtype=np.int64).reshape(-1, 4)
    n = rec.shape[0]
    if n == 0:
        return np.zeros(0, dtype=np.uint32)
    ww = np.ascontiguousarray(w, dtype=np.float64).reshape(n, -1).view(np.uint64)
    pos = np.arange(ww.shape[1], dtype=np.uint64)[None, :]
    h = _mix(ww ^ ((pos + np.uint64(64)) * _G)).sum(axis=1, dtype=np.uint64)
    for c in range(4):
        h += _mix(rec[:, c].astype(np.uint64) + _key(c + 1))
    return (h >> np.uint64(32)).astype(np.uint32)


def input_digest(system) -> str:
    """SHA-256 of every input array of a system (coordinates, connectivity,
    wall and overset-boundary nodes), so a fixture names the mesh it was
    made from."""
    h = hashlib.sha256()
    for b in system.blocks:
        h.update(np.ascontiguousarray(b.x).tobytes())
        for nv, c in b.cells:
            h.update(np.int32(nv).tobytes())
            h.update(np.ascontiguousarray(c, dtype=np.int32).tobytes())
        h.update(np.ascontiguousarray(b.wbc, dtype=np.int32).tobytes())
        h.update(np.ascontiguousarray(b.obc, dtype=np.int32).tobytes())
    return h.hexdigest()


def make(system, out, q0=None, prefix: str = "") -> dict:
    """Digest arrays of one run_system-style result (iblank, donors, q)."""
    arrs = {}
    for k, b in enumerate(system.blocks):
        t = b.tag
        p = f"{prefix}{t}"
        arrs[f"iblank_{p}"] = np.asarray(out["iblank"][t]).astype(np.int8)
        rec, ind, frac = out["donors"][t]
        arrs[f"rechash_{p}"] = record_hashes(rec, ind, frac)
        arrs[f"counts_{p}"] = np.array([rec.shape[0], len(ind)], dtype=np.int64)
        if q0 is not None and t in out.get("q", {}):
            q = out["q"][t]
            arrs[f"qhash_{p}"] = chunk_hashes(q)
            arrs[f"qchanged_{p}"] = np.array([int((q != q0[k]).sum())], dtype=np.int64)
    return arrs


def compare(fix, system, out, prefix: str = "") -> dict:
    """Mismatch counts of a result against a fixture's digests:
    iblank nodes, donor records (by hash, or every record of a block whose
    counts differ) and updated-field chunks."""
    res = {"iblank": 0, "records": 0, "record_total": 0, "q_chunks": 0, "blocks": 0}
    for b in system.blocks:
        t = b.tag
        p = f"{prefix}{t}"
        if f"iblank_{p}" not in fix:
            continue
        res["blocks"] += 1
        ib_ref = fix[f"iblank_{p}"].astype(np.int32)
        ib = np.asarray(out["iblank"][t], dtype=np.int32)
        res["iblank"] += int((ib_ref != ib).sum()) if ib.shape == ib_ref.shape else int(ib_ref.size)
        rec, ind, frac = out["donors"][t]
        ref_h = fix[f"rechash_{p}"]
        res["record_total"] += int(ref_h.size)
        try:
            h = record_hashes(rec, ind, frac)
        except ValueError:
            h = np.zeros(0, dtype=np.uint32)
        if h.size == ref_h.size:
            res["records"] += int((h != ref_h).sum())
        else:
            res["records"] += max(int(h.size), int(ref_h.size))
        if f"qhash_{p}" in fix and t in out.get("q", {}):
            qh = chunk_hashes(out["q"][t])
            ref_q = fix[f"qhash_{p}"]
            res["q_chunks"] += int((qh != ref_q).sum()) if qh.size == ref_q.size else int(ref_q.size)
    return res
