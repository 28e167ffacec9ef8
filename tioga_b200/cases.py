"""Seeded synthetic overset systems.

The reference ships no benchmark meshes for its connectivity path, so every
workload here is generated from a seed: a Cartesian hex background box and
one or more spherical-shell near-body meshes (wall nodes on the inner sphere,
overset-boundary nodes on the outer sphere).  Vertex orderings follow the
reference's cell conventions so that signed cell volumes are positive
(src/math.c:298-330 face tables, src/cellVolume.f90:62-91) and the Newton
parameterisations match (src/math.c:199-287):

  hex      v0..v3 bottom face counter-clockwise, v4..v7 above them
  prism    v0,v1,v2 bottom triangle, v3,v4,v5 above them
  pyramid  v0..v3 base, normal towards the apex v4
  tet      v3 above the counter-clockwise triangle v0,v1,v2

Shell meshes share their pole nodes and their phi seam so the wall is closed
and no coincident query points exist.  Pole-adjacent cells are degenerate hexes
(two collapsed edges), exactly as a structured spherical grid gives them.

Block arrays are 0-based here; the C-API wrappers add the 1-based offset that
TIOGA expects (src/codetypes.h:36).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

NV_HEX, NV_PRISM, NV_PYR, NV_TET = 8, 6, 5, 4


@dataclass
class Block:
    """One mesh block: one TIOGA ``registergrid_data`` call."""

    tag: int
    x: np.ndarray                      # (N, 3) float64
    cells: list                        # [(nv, conn (nc, nv) int32 0-based)]
    wbc: np.ndarray                    # wall-boundary node ids, 0-based int32
    obc: np.ndarray                    # overset-boundary node ids, 0-based int32
    name: str = ""

    @property
    def nnodes(self) -> int:
        return int(self.x.shape[0])

    @property
    def ncells(self) -> int:
        return int(sum(c.shape[0] for _, c in self.cells))


@dataclass
class System:
    """An overset system: the blocks registered in one TIOGA instance."""

    blocks: list
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def nnodes(self) -> int:
        return sum(b.nnodes for b in self.blocks)

    @property
    def ncells(self) -> int:
        return sum(b.ncells for b in self.blocks)


# ---------------------------------------------------------------------------
# Cartesian background
# ---------------------------------------------------------------------------
def hex_box(n: int, lo: float = -5.0, hi: float = 5.0, perturb: float = 0.0,
            rng: np.random.Generator | None = None, split_prism_zneg: bool = False):
    """n^3 nodes on [lo,hi]^3; interior nodes jittered by U(-p,p)*h per axis.

    With ``split_prism_zneg`` every hex whose cell centre has z<0 becomes two
    prisms whose triangles lie on the x-faces (the diagonal v0-v7 of the x=i
    face), which keeps neighbouring splits face-conforming.
    Returns (x, cells) with node id = i + n*(j + n*k).
    """
    h = (hi - lo) / (n - 1)
    g = lo + h * np.arange(n, dtype=np.float64)
    z, y, xx = np.meshgrid(g, g, g, indexing="ij")
    x = np.stack([xx.ravel(), y.ravel(), z.ravel()], axis=1)
    if perturb > 0.0:
        assert rng is not None
        idx = np.arange(n)
        inner = (idx > 0) & (idx < n - 1)
        mask = (inner[None, None, :] & inner[None, :, None] & inner[:, None, None]).ravel()
        d = rng.uniform(-perturb * h, perturb * h, size=(int(mask.sum()), 3))
        x[mask] += d
    m = n - 1
    i, j, k = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    # iterate with i fastest: build in (k, j, i) order
    i = i.transpose(2, 1, 0).ravel(); j = j.transpose(2, 1, 0).ravel(); k = k.transpose(2, 1, 0).ravel()

    def nid(a, b, c):
        return (a + n * (b + n * c)).astype(np.int32)

    h0 = nid(i, j, k); h1 = nid(i + 1, j, k); h2 = nid(i + 1, j + 1, k); h3 = nid(i, j + 1, k)
    h4 = nid(i, j, k + 1); h5 = nid(i + 1, j, k + 1); h6 = nid(i + 1, j + 1, k + 1); h7 = nid(i, j + 1, k + 1)
    hexes = np.stack([h0, h1, h2, h3, h4, h5, h6, h7], axis=1)
    if not split_prism_zneg:
        return x, [(NV_HEX, hexes)]
    zc = lo + h * (k + 0.5)
    neg = zc < 0.0
    keep = hexes[~neg]
    s = hexes[neg]
    pa = s[:, [0, 3, 7, 1, 2, 6]]
    pb = s[:, [0, 7, 4, 1, 6, 5]]
    prisms = np.empty((2 * s.shape[0], 6), dtype=np.int32)
    prisms[0::2] = pa
    prisms[1::2] = pb
    return x, [(NV_HEX, keep), (NV_PRISM, prisms)]


# ---------------------------------------------------------------------------
# Spherical shell
# ---------------------------------------------------------------------------
def _radii(nr: int, r0: float, r1: float, ratio: float) -> np.ndarray:
    if ratio == 1.0:
        return np.linspace(r0, r1, nr)
    dr = np.power(ratio, np.arange(nr - 1, dtype=np.float64))
    dr *= (r1 - r0) / dr.sum()
    r = np.concatenate([[r0], r0 + np.cumsum(dr)])
    r[-1] = r1
    return r


def sphere_shell(nr: int, nt: int, nphi: int, r0: float, r1: float,
                 ratio: float = 1.1, center=(0.0, 0.0, 0.0), perturb: float = 0.0,
                 rng: np.random.Generator | None = None, split_layers: int = 0,
                 seam_copy: bool = False):
    """Structured spherical shell: nr radii x nt polar angles x nphi azimuths.

    Poles (t=0, t=nt-1) are single nodes per radius and phi=2*pi is the phi=0
    seam, so the layer holds 2 + (nt-2)*(nphi-1) distinct nodes.  With
    ``seam_copy`` the phi=2*pi side gets nodes of its own instead (an O-grid
    with a duplicated seam, appended after each layer's nodes): each lies
    within about 1e-16 of its phi=0 twin, so the twins are coincident query
    points for a donor mesh.  Cell vertex
    order maps (u, v, w) to (r, theta, phi), a right-handed frame, so hex
    volumes are positive.  Cells of the first ``split_layers`` radial layers
    that do not touch a pole are split into 5 tets, 2 prisms or 3 pyramids,
    the kind chosen per cell from ``rng``.

    Returns (x, cells, wall_nodes, outer_nodes, cell_kind) where cell_kind is
    the per-cell split code (0 hex, 1 tets, 2 prisms, 3 pyramids).
    """
    r = _radii(nr, r0, r1, ratio)
    th = np.linspace(0.0, np.pi, nt)
    ph = np.linspace(0.0, 2.0 * np.pi, nphi)
    npl = nphi - 1
    L = 2 + (nt - 2) * npl
    # node coordinates in spherical index space (interior theta only)
    R = np.repeat(r, L)
    T = np.empty(nr * L); P = np.empty(nr * L)
    layer_t = np.concatenate([[0.0], np.repeat(th[1:-1], npl), [np.pi]])
    layer_p = np.concatenate([[0.0], np.tile(ph[:-1], nt - 2), [0.0]])
    T[:] = np.tile(layer_t, nr)
    P[:] = np.tile(layer_p, nr)
    if perturb > 0.0:
        assert rng is not None
        dr = np.diff(r)
        drl = np.minimum(dr[:-1], dr[1:])                       # interior radii
        dth = th[1] - th[0]
        dph = ph[1] - ph[0]
        for i in range(1, nr - 1):
            sl = slice(i * L + 1, i * L + L - 1)                # skip both poles
            cnt = L - 2
            R[sl] += rng.uniform(-perturb, perturb, cnt) * drl[i - 1]
            T[sl] += rng.uniform(-perturb, perturb, cnt) * dth
            P[sl] += rng.uniform(-perturb, perturb, cnt) * dph
    c = np.asarray(center, dtype=np.float64)
    nseam = (nt - 2) if seam_copy else 0
    if seam_copy:  # the twin of every interior phi=0 node, at phi + 2*pi
        lay = np.arange(nr * L).reshape(nr, L)
        twin = lay[:, 1:1 + (nt - 2) * npl].reshape(nr, nt - 2, npl)[:, :, 0]
        R = np.concatenate([R.reshape(nr, L), R[twin]], axis=1).ravel()
        T = np.concatenate([T.reshape(nr, L), T[twin]], axis=1).ravel()
        P = np.concatenate([P.reshape(nr, L), P[twin] + 2.0 * np.pi], axis=1).ravel()
    Lx = L + nseam
    st = np.sin(T)
    x = np.stack([R * st * np.cos(P), R * st * np.sin(P), R * np.cos(T)], axis=1) + c

    def nid(i, t, p):
        base = i * Lx
        out = base + 1 + (t - 1) * npl + (p % npl)
        if seam_copy:
            out = np.where(p == npl, base + L + (t - 1), out)
        out = np.where(t == 0, base, out)
        out = np.where(t == nt - 1, base + L - 1, out)
        return out.astype(np.int32)

    i, t, p = np.meshgrid(np.arange(nr - 1), np.arange(nt - 1), np.arange(nphi - 1), indexing="ij")
    i = i.ravel(); t = t.ravel(); p = p.ravel()
    v = [nid(i, t, p), nid(i + 1, t, p), nid(i + 1, t + 1, p), nid(i, t + 1, p),
         nid(i, t, p + 1), nid(i + 1, t, p + 1), nid(i + 1, t + 1, p + 1), nid(i, t + 1, p + 1)]
    hexes = np.stack(v, axis=1)
    wall = np.arange(0, Lx, dtype=np.int32)
    outer = np.arange((nr - 1) * Lx, nr * Lx, dtype=np.int32)
    kind = np.zeros(hexes.shape[0], dtype=np.int8)
    if split_layers <= 0:
        return x, [(NV_HEX, hexes)], wall, outer, kind
    assert rng is not None
    splittable = (i < split_layers) & (t > 0) & (t < nt - 2)
    kind[splittable] = rng.integers(1, 4, size=int(splittable.sum())).astype(np.int8)
    hx = hexes[kind == 0]
    s1 = hexes[kind == 1]
    s2 = hexes[kind == 2]
    s3 = hexes[kind == 3]
    tets = np.concatenate([s1[:, [0, 1, 3, 4]], s1[:, [1, 2, 3, 6]], s1[:, [3, 6, 7, 4]],
                           s1[:, [1, 5, 6, 4]], s1[:, [1, 6, 3, 4]]], axis=0) if len(s1) else np.zeros((0, 4), np.int32)
    prisms = np.concatenate([s2[:, [0, 1, 2, 4, 5, 6]], s2[:, [0, 2, 3, 4, 6, 7]]], axis=0) if len(s2) else np.zeros((0, 6), np.int32)
    pyrs = np.concatenate([s3[:, [1, 5, 6, 2, 0]], s3[:, [3, 2, 6, 7, 0]], s3[:, [4, 7, 6, 5, 0]]], axis=0) if len(s3) else np.zeros((0, 5), np.int32)
    cells = [(NV_HEX, hx)]
    for nv, cc in ((NV_PRISM, prisms), (NV_PYR, pyrs), (NV_TET, tets)):
        if len(cc):
            cells.append((nv, cc.astype(np.int32)))
    return x, cells, wall, outer, kind


# ---------------------------------------------------------------------------
# The workloads
# ---------------------------------------------------------------------------
def _empty_i32():
    return np.zeros(0, dtype=np.int32)


def config0(seed: int = 0, nbg: int = 65, nr: int = 33, nt: int = 33, nphi: int = 65,
            perturb: float = 0.05, seam_copy: bool = False, bg_perturb: float | None = None,
            bg_shift: float = 0.0) -> System:
    """Plain all-hex case: 65^3 background box on [-5,5]^3 plus one shell
    (r 0.5 -> 2.0, radial ratio 1.1) at the origin; interior nodes jittered
    by +-5% of the local spacing (the background by bg_perturb when given:
    0 leaves it a uniform Cartesian box, shifted by bg_shift on every axis)."""
    rng = np.random.default_rng(seed)
    pb = perturb if bg_perturb is None else bg_perturb
    xb, cb = hex_box(nbg, -5.0 + bg_shift, 5.0 + bg_shift, pb, rng if pb > 0 else None)
    xs, cs, wall, outer, _ = sphere_shell(nr, nt, nphi, 0.5, 2.0, 1.1, (0.0, 0.0, 0.0), perturb, rng,
                                          seam_copy=seam_copy)
    bg = Block(1, xb, cb, _empty_i32(), _empty_i32(), name="background")
    sh = Block(2, xs, cs, wall, outer, name="shell")
    return System([bg, sh], name=f"cfg0(nbg={nbg},shell={nr}x{nt}x{nphi},seed={seed})",
                  meta={"seed": seed})


def shell_centres(rng: np.random.Generator, nshell: int, rwall: np.ndarray, router: np.ndarray,
                  box: float = 3.0, margin: float = 0.05, tries: int = 10000,
                  domain: float = 4.9) -> np.ndarray:
    """Random centres in [-box, box]^3 such that every shell lies inside the
    background box [-domain, domain]^3 and no wall sphere lies inside another
    shell (walls stay out of every other mesh's donor region)."""
    c = np.zeros((nshell, 3))
    for a in range(nshell):
        for _ in range(tries):
            cand = rng.uniform(-box, box, 3)
            ok = bool(np.all(np.abs(cand) + router[a] <= domain))
            for b in range(a):
                d = np.linalg.norm(cand - c[b])
                if d < max(router[a] + rwall[b], router[b] + rwall[a]) + margin:
                    ok = False
                    break
            if ok:
                c[a] = cand
                break
        else:
            raise RuntimeError("could not place shells")
    return c


def config1(seed: int = 1, nbg: int = 257, nshell: int = 3, nr: int = 65, nt: int = 65,
            nphi: int = 129, split_layers: int = 4, seam_copy: bool = False) -> System:
    """Mixed-element case: 257^3 background whose z<0 hexes are split into
    two prisms each, plus three shells (wall radius U(0.3,0.6), outer radius
    4x wall) at random centres within |x|<=3, 65x65x129 nodes each, whose
    first four radial layers are split per cell into 5 tets, 2 prisms or 3
    pyramids.  No jitter, so every split is face-conforming."""
    rng = np.random.default_rng(seed)
    xb, cb = hex_box(nbg, -5.0, 5.0, 0.0, None, split_prism_zneg=True)
    blocks = [Block(1, xb, cb, _empty_i32(), _empty_i32(), name="background")]
    rwall = rng.uniform(0.3, 0.6, nshell)
    router = 4.0 * rwall
    centres = shell_centres(rng, nshell, rwall, router)
    for s in range(nshell):
        xs, cs, wall, outer, _ = sphere_shell(nr, nt, nphi, rwall[s], router[s], 1.1,
                                              centres[s], 0.0, rng, split_layers, seam_copy)
        blocks.append(Block(2 + s, xs, cs, wall, outer, name=f"shell{s}"))
    return System(blocks, name=f"cfg1(nbg={nbg},{nshell}x{nr}x{nt}x{nphi},seed={seed})",
                  meta={"seed": seed, "centres": centres.tolist(), "rwall": rwall.tolist()})


# ---------------------------------------------------------------------------
# High-order workload: Lagrange hexahedra described by their degrees of
# freedom (element-major, tensor order i fastest, reference cube [0,1]^3 with
# node (i, j, k) at (i/p, j/p, k/p)), registered through their corners
# ---------------------------------------------------------------------------
@dataclass
class HighOrder:
    """Degree and DOF coordinates (ncells, (p+1)^3, 3) of one block's cells."""

    p: int
    xdof: np.ndarray


HEX_TO_TENSOR = [0, 1, 3, 2, 4, 5, 7, 6]  # hex vertex order -> tensor (i fastest) order


def shell_q(ne_r: int, ne_t: int, ne_p: int, p: int, r0: float, r1: float, ratio: float,
            theta0: float, theta1: float, center, perturb: float, rng: np.random.Generator,
            cap_obc: bool = True):
    """Curved band of a spherical shell, theta in [theta0, theta1], phi periodic,
    as ne_r x ne_t x ne_p Lagrange hexahedra of degree p.  Every DOF is a point
    of one global (ne_r p + 1) x (ne_t p + 1) x (ne_p p) lattice in (r, theta,
    phi), so neighbouring elements share their face DOFs bit for bit; DOFs
    inside an element are moved by +-``perturb`` of the local lattice spacing.
    Returns (corner coordinates, hex cells, wall nodes, overset-boundary nodes,
    DOF coordinates (ncells, (p+1)^3, 3))."""
    nr, nt, npp = ne_r * p + 1, ne_t * p + 1, ne_p * p
    # element corner radii graded by `ratio`; the DOF radii equispaced inside each element
    rc = _radii(ne_r + 1, r0, r1, ratio)
    r = np.concatenate([rc[e] + (rc[e + 1] - rc[e]) * np.arange(p) / p for e in range(ne_r)] + [rc[-1:]])
    th = np.linspace(theta0, theta1, nt)
    ph = np.linspace(0.0, 2.0 * np.pi, npp + 1)[:-1]
    c = np.asarray(center, dtype=np.float64)

    def xyz(R, T, P):
        st = np.sin(T)
        return np.stack([R * st * np.cos(P), R * st * np.sin(P), R * np.cos(T)], axis=-1) + c

    # element (a, b, d) = (r, theta, phi) index; DOF (i, j, k) along (r, theta, phi)
    a, b, d = np.meshgrid(np.arange(ne_r), np.arange(ne_t), np.arange(ne_p), indexing="ij")
    a = a.ravel(); b = b.ravel(); d = d.ravel()
    n1 = p + 1
    k, j, i = np.meshgrid(np.arange(n1), np.arange(n1), np.arange(n1), indexing="ij")
    i = i.ravel(); j = j.ravel(); k = k.ravel()
    ri = a[:, None] * p + i[None, :]
    ti = b[:, None] * p + j[None, :]
    pi = (d[:, None] * p + k[None, :]) % npp
    R = r[ri].copy(); T = th[ti].copy(); P = ph[pi].copy()
    if perturb > 0.0:
        inner = ((i > 0) & (i < p) & (j > 0) & (j < p) & (k > 0) & (k < p))[None, :].repeat(len(a), 0)
        dr = (r[np.minimum(ri + 1, nr - 1)] - r[np.maximum(ri - 1, 0)]) * 0.5
        R[inner] += rng.uniform(-perturb, perturb, int(inner.sum())) * dr[inner]
        T[inner] += rng.uniform(-perturb, perturb, int(inner.sum())) * (th[1] - th[0])
        P[inner] += rng.uniform(-perturb, perturb, int(inner.sum())) * (ph[1] - ph[0])
    xdof = xyz(R, T, P)
    # registered corner mesh: lattice points with indices multiple of p
    nrc, ntc, npc = ne_r + 1, ne_t + 1, ne_p

    def nid(ia, ib, id_):
        return ((id_ % npc) * ntc + ib) * nrc + ia

    ia, ib, id_ = np.meshgrid(np.arange(nrc), np.arange(ntc), np.arange(npc), indexing="ij")
    corner = np.zeros((nrc * ntc * npc, 3))
    corner[nid(ia, ib, id_).ravel()] = xyz(r[ia.ravel() * p], th[ib.ravel() * p], ph[id_.ravel() * p])
    # hex vertex order (u, v, w) = (r, theta, phi): right-handed, positive volume
    tensor = np.stack([nid(a + di, b + dj, d + dk) for dk in (0, 1) for dj in (0, 1) for di in (0, 1)], axis=1)
    hexes = tensor[:, [0, 1, 3, 2, 4, 5, 7, 6]].astype(np.int32)
    wall = np.flatnonzero(np.isin(np.arange(len(corner)), nid(0, ib, id_).ravel())).astype(np.int32)
    rim = np.zeros(len(corner), bool)
    edge = (ia.ravel() == nrc - 1)
    if cap_obc:  # the theta caps are overset boundaries too
        edge = edge | (ib.ravel() == 0) | (ib.ravel() == ntc - 1)
    rim[nid(ia, ib, id_).ravel()[edge]] = True
    return corner, [(NV_HEX, hexes)], wall, np.flatnonzero(rim).astype(np.int32), xdof


def config4(seed: int = 4, nbg: int = 97, ne_r: int = 24, ne_t: int = 24, ne_p: int = 48, p: int = 3,
            perturb: float = 0.02, wall: bool = True, cap_obc: bool = True):
    """High-order case: a degree-1 background box (nbg^3 nodes on [-5,5]^3)
    and a curved band of a spherical shell (r 0.5 -> 2.0, theta in
    [pi/4, 3pi/4]) of ne_r x ne_t x ne_p degree-p Lagrange hexahedra whose
    inner DOFs are moved by +-2% of the spacing.  Returns the System of the
    registered corner meshes and each block's HighOrder description."""
    rng = np.random.default_rng(seed)
    xb, cb = hex_box(nbg, -5.0, 5.0, 0.0, None)
    hx = cb[0][1]
    bg_dof = xb[hx[:, HEX_TO_TENSOR]]                       # (ncells, 8, 3)
    xs, cs, wn, on, sh_dof = shell_q(ne_r, ne_t, ne_p, p, 0.5, 2.0, 1.1, np.pi / 4, 3 * np.pi / 4,
                                     (0.1, -0.2, 0.05), perturb, rng, cap_obc)
    bg = Block(1, xb, cb, _empty_i32(), _empty_i32(), name="background")
    sh = Block(2, xs, cs, wn if wall else _empty_i32(), on, name=f"shell-q{p}")
    system = System([bg, sh], name=f"cfg4(nbg={nbg},q{p} {ne_r}x{ne_t}x{ne_p},seed={seed})", meta={"seed": seed})
    return system, [HighOrder(1, bg_dof), HighOrder(p, sh_dof)]


def small_config4(seed: int = 4, wall: bool = True):
    """config4 geometry at test size (17^3 box, 2 x 4 x 8 cubic elements)."""
    return config4(seed, nbg=17, ne_r=2, ne_t=4, ne_p=8, p=3, wall=wall)


def dof_fields(ho: list, nvar: int, seed: int = 5) -> list:
    """Element-major DOF values (ncells * (p+1)^3 * nvar, ROW) of a seeded
    cubic polynomial in x, y, z per variable."""
    rng = np.random.default_rng(seed)
    out = []
    coef = rng.uniform(-1.0, 1.0, (nvar, 20))
    for h in ho:
        X = h.xdof.reshape(-1, 3)
        x, y, z = X[:, 0], X[:, 1], X[:, 2]
        mono = np.stack([np.ones_like(x), x, y, z, x * x, y * y, z * z, x * y, y * z, z * x,
                         x ** 3, y ** 3, z ** 3, x * x * y, x * x * z, y * y * x, y * y * z, z * z * x,
                         z * z * y, x * y * z], axis=1)
        out.append((mono @ coef.T).reshape(-1).astype(np.float64))
    return out


def fields(system: System, nvar: int = 5, seed: int = 7) -> list:
    """Per-block solution arrays q (ROW layout, nnodes*nvar) ~ U(-1, 1)."""
    rng = np.random.default_rng(seed)
    return [rng.uniform(-1.0, 1.0, b.nnodes * nvar) for b in system.blocks]


def linear_fields(system: System, nvar: int = 5) -> list:
    """q = x + y + z for every variable (the reference driver's exactness
    check, driver/testTioga.f90:97-107)."""
    out = []
    for b in system.blocks:
        s = b.x.sum(axis=1)
        out.append(np.repeat(s, nvar).astype(np.float64))
    return out


def batch_system(rng: np.random.Generator, nnodes: float, nshell: int, mixed: bool, name: str = "") -> System:
    """One system of the batched workload: a background box on [-5,5]^3 plus
    ``nshell`` shells built as in config0 (radial ratio 1.1, outer radius 4x
    the wall radius U(0.3, 0.6), centres within |x|<=3), about ``nnodes``
    nodes in all (60% background, the rest shared by the shells).  All-hex
    systems get config0's +-5% jitter; mixed-element ones split the
    background's z<0 hexes into prisms and the shells' first radial layers
    into tets, prisms or pyramids (config1), without jitter."""
    nbg = max(9, int(round((0.6 * nnodes) ** (1.0 / 3.0))))
    nt = max(5, int(round((0.4 * nnodes / nshell / 2.0) ** (1.0 / 3.0))))
    nr, nphi = nt, 2 * nt - 1
    perturb = 0.0 if mixed else 0.05
    xb, cb = hex_box(nbg, -5.0, 5.0, perturb, rng if perturb > 0 else None, split_prism_zneg=mixed)
    blocks = [Block(1, xb, cb, _empty_i32(), _empty_i32(), name="background")]
    rwall = rng.uniform(0.3, 0.6, nshell)
    router = 4.0 * rwall
    centres = shell_centres(rng, nshell, rwall, router)
    split = min(4, max(1, nr // 4)) if mixed else 0
    for a in range(nshell):
        xs, cs, wall, outer, _ = sphere_shell(nr, nt, nphi, rwall[a], router[a], 1.1, centres[a], perturb, rng,
                                              split)
        blocks.append(Block(2 + a, xs, cs, wall, outer, name=f"shell{a}"))
    return System(blocks, name=name or f"batch(nbg={nbg},{nshell}x{nr}x{nt}x{nphi},mixed={mixed})",
                  meta={"centres": centres.tolist(), "rwall": rwall.tolist(), "mixed": mixed})


def config2(seed: int = 2, nsys: int = 64, nmin: float = 5e4, nmax: float = 2e6) -> list:
    """Batched workload: ``nsys`` independent overset systems, each a
    background box plus 1-4 shells (batch_system), with node counts drawn
    log-uniformly in [nmin, nmax] and all-hex or mixed-element with
    probability 0.5, from one seed."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(nsys):
        n = float(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        nshell = int(rng.integers(1, 5))
        mixed = bool(rng.uniform() < 0.5)
        out.append(batch_system(rng, n, nshell, mixed, name=f"cfg2[{k}](n~{int(n)},{nshell} shells,"
                                f"{'mixed' if mixed else 'hex'})"))
    return out


def small_config2(seed: int = 2, nsys: int = 6) -> list:
    """The batched workload at test size: systems of 3e3 to 2e4 nodes."""
    return config2(seed, nsys=nsys, nmin=3e3, nmax=2e4)


CONFIGS = {
    "cfg0": config0,
    "cfg1": config1,
}


def small_config0(seed: int = 0) -> System:
    """cfg0 geometry at test size (17^3 box, 9x9x17 shell)."""
    return config0(seed, nbg=17, nr=9, nt=9, nphi=17)


def small_config0_uniform(seed: int = 0, nbg: int = 17, shift: float = 0.0) -> System:
    """small_config0 with an unjittered background: a uniform Cartesian hex
    box, the case of the reference's uniform-hex search (search.C:271-341).
    Unshifted, the box's lattice planes hold the shell's unjittered seam and
    pole nodes (they lie on box faces, where the lookup and the tree search
    pick different cells) and its lattice nodes lie on the shell's seam faces
    (tied shell cells); a shift off the origin removes both."""
    return config0(seed, nbg=nbg, nr=9, nt=9, nphi=17, bg_perturb=0.0, bg_shift=shift)


def small_config0_seam(seed: int = 0) -> System:
    """small_config0 with the shell's phi seam duplicated (coincident query points)."""
    return config0(seed, nbg=17, nr=9, nt=9, nphi=17, seam_copy=True)


def small_config1_seam(seed: int = 1) -> System:
    """small_config1 with every shell's phi seam duplicated (coincident query points)."""
    return config1(seed, nbg=33, nshell=3, nr=9, nt=9, nphi=17, split_layers=2, seam_copy=True)


def small_config1(seed: int = 1) -> System:
    """cfg1 geometry at test size (33^3 box, three 9x9x17 shells)."""
    return config1(seed, nbg=33, nshell=3, nr=9, nt=9, nphi=17, split_layers=2)
