"""Comparison of two TIOGA runs (see tioga_b200.capi.run_system)."""
import numpy as np


def diff_runs(system, a, b, exact_q=True):
    """Return a list of human-readable mismatches (empty when identical).
    iblank, receptor lists and donor indices must match exactly; weights and
    updated fields bit for bit (the FP64 arithmetic follows the same order)."""
    out = []
    for blk in system.blocks:
        t = blk.tag
        ia, ib = a["iblank"][t], b["iblank"][t]
        if not np.array_equal(ia, ib):
            bad = np.nonzero(ia != ib)[0]
            out.append(f"tag {t}: iblank differs at {len(bad)} nodes, first {bad[:5].tolist()} "
                       f"a={ia[bad[:5]].tolist()} b={ib[bad[:5]].tolist()}")
        ra, xa, fa = a["donors"][t]
        rb, xb, fb = b["donors"][t]
        if ra.shape != rb.shape or not np.array_equal(ra, rb):
            out.append(f"tag {t}: receptor lists differ ({ra.shape[0]} vs {rb.shape[0]})")
        else:
            if not np.array_equal(xa, xb):
                out.append(f"tag {t}: donor indices differ at {(xa != xb).sum()} entries")
            if not np.array_equal(fa.view(np.int64), fb.view(np.int64)):
                d = np.abs(fa - fb)
                out.append(f"tag {t}: weights differ at {(fa != fb).sum()} entries, max {d.max():.3e}")
        if t in a["q"] and t in b["q"]:
            qa, qb = a["q"][t], b["q"][t]
            if exact_q and not np.array_equal(qa.view(np.int64), qb.view(np.int64)):
                out.append(f"tag {t}: q differs at {(qa != qb).sum()} entries, max {np.abs(qa - qb).max():.3e}")
    return out
