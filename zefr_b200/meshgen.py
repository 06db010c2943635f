"""Synthetic gmsh 2.2 meshes for the DFR residual workloads.

ZEFR reads gmsh 2.2 ASCII meshes (reference ``src/geometry.cpp:307-957``):
``$PhysicalNames`` maps boundary names to conditions, ``$Nodes`` must be
numbered 1..N in order (the reader discards the ids, ``src/geometry.cpp:418-444``),
and ``$Elements`` carries the physical id as the first tag.  The generators here
build the mesh shapes the workloads are defined on and write them in that format,
so the same file feeds this library's reader and the reference solver.

Node orderings follow gmsh: 4-node quad counter-clockwise; 9-node quad corners,
edge midpoints (0-1, 1-2, 2-3, 3-0), centre; 8-node hex bottom face
counter-clockwise then top face; triangles counter-clockwise.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, List, Sequence, Tuple

import numpy as np

# gmsh element type ids used here
GMSH_LINE2, GMSH_TRI3, GMSH_QUAD4, GMSH_HEX8, GMSH_LINE3, GMSH_QUAD9 = 1, 2, 3, 5, 8, 10

ETYPE_OF_GMSH = {GMSH_TRI3: "tri", GMSH_QUAD4: "quad", GMSH_QUAD9: "quad", GMSH_HEX8: "hex"}


@dataclasses.dataclass
class Mesh:
    """An unstructured mesh of one element type.

    ``nodes``: (N, 3) float64; ``elements``: (E, nn) int64 zero-based node ids;
    ``bnd_faces``: list of (gmsh face type, zero-based node ids, boundary name).
    """

    ndims: int
    nodes: np.ndarray
    gmsh_type: int
    elements: np.ndarray
    bnd_faces: List[Tuple[int, Tuple[int, ...], str]]

    @property
    def etype(self) -> str:
        return ETYPE_OF_GMSH[self.gmsh_type]

    @property
    def n_elements(self) -> int:
        return int(self.elements.shape[0])

    def boundary_names(self) -> List[str]:
        seen: List[str] = []
        for _, _, name in self.bnd_faces:
            if name not in seen:
                seen.append(name)
        return seen


def write_gmsh(mesh: Mesh, path: str) -> None:
    """Write ``mesh`` as gmsh 2.2 ASCII with a FLUID volume group."""
    names = mesh.boundary_names()
    phys = {name: i + 1 for i, name in enumerate(names)}
    fluid_id = len(names) + 1
    lines: List[str] = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$PhysicalNames"]
    lines.append(str(len(names) + 1))
    for name in names:
        lines.append(f'{mesh.ndims - 1} {phys[name]} "{name}"')
    lines.append(f'{mesh.ndims} {fluid_id} "FLUID"')
    lines.append("$EndPhysicalNames")
    lines.append("$Nodes")
    lines.append(str(mesh.nodes.shape[0]))
    for i, (x, y, z) in enumerate(mesh.nodes.tolist()):
        lines.append(f"{i + 1} {x!r} {y!r} {z!r}")
    lines.append("$EndNodes")
    lines.append("$Elements")
    lines.append(str(len(mesh.bnd_faces) + mesh.n_elements))
    eid = 1
    for ftype, fnodes, name in mesh.bnd_faces:
        p = phys[name]
        lines.append(f"{eid} {ftype} 2 {p} {p} " + " ".join(str(n + 1) for n in fnodes))
        eid += 1
    for ele in mesh.elements:
        lines.append(f"{eid} {mesh.gmsh_type} 2 {fluid_id} {fluid_id} " + " ".join(str(int(n) + 1) for n in ele))
        eid += 1
    lines.append("$EndElements")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def read_gmsh(path: str) -> Mesh:
    """Read a gmsh 2.2 ASCII mesh of one volume element type (test helper)."""
    with open(path) as f:
        text = f.read().split("\n")
    it = iter(range(len(text)))
    names: Dict[int, Tuple[int, str]] = {}
    nodes = None
    eles: List[List[int]] = []
    etype = None
    bnd: List[Tuple[int, Tuple[int, ...], int]] = []
    i = 0
    ndims = 0
    while i < len(text):
        line = text[i].strip()
        if line == "$PhysicalNames":
            n = int(text[i + 1])
            for k in range(n):
                parts = text[i + 2 + k].split()
                names[int(parts[1])] = (int(parts[0]), parts[2].strip('"'))
            i += n + 2
        elif line == "$Nodes":
            n = int(text[i + 1])
            nodes = np.array([[float(v) for v in text[i + 2 + k].split()[1:4]] for k in range(n)])
            i += n + 2
        elif line == "$Elements":
            n = int(text[i + 1])
            rows = [text[i + 2 + k].split() for k in range(n)]
            i += n + 2
            vol_dim = max(d for d, _ in names.values())
            ndims = vol_dim
            for r in rows:
                t, ntag = int(r[1]), int(r[2])
                tag = int(r[3])
                nd = [int(v) - 1 for v in r[3 + ntag:]]
                if names.get(tag, (vol_dim, ""))[0] == vol_dim:
                    etype = t
                    eles.append(nd)
                else:
                    bnd.append((t, tuple(nd), tag))
        else:
            i += 1
    assert nodes is not None and etype is not None
    faces = [(t, nd, names[tag][1]) for t, nd, tag in bnd]
    return Mesh(ndims=ndims, nodes=nodes, gmsh_type=etype, elements=np.array(eles, dtype=np.int64), bnd_faces=faces)


def box_quads(nx: int, ny: int, x0: float = -5.0, x1: float = 5.0, y0: float = -5.0, y1: float = 5.0,
              bnd="PERIODIC") -> Mesh:
    """Structured nx-by-ny 4-node quads on [x0,x1]x[y0,y1], all sides tagged
    ``bnd``, or, for a 4-tuple, the sides x0, x1, y0, y1 tagged in that order.

    Elements are ordered x fastest; each quad is counter-clockwise.
    """
    b_x0, b_x1, b_y0, b_y1 = (bnd,) * 4 if isinstance(bnd, str) else tuple(bnd)
    xs = np.linspace(x0, x1, nx + 1)
    ys = np.linspace(y0, y1, ny + 1)
    X, Y = np.meshgrid(xs, ys)  # (ny+1, nx+1)
    nodes = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], axis=1)

    def nid(i: int, j: int) -> int:
        return j * (nx + 1) + i

    eles = np.array([[nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)]
                     for j in range(ny) for i in range(nx)], dtype=np.int64)
    faces: List[Tuple[int, Tuple[int, ...], str]] = []
    for i in range(nx):
        faces.append((GMSH_LINE2, (nid(i, 0), nid(i + 1, 0)), b_y0))
        faces.append((GMSH_LINE2, (nid(i + 1, ny), nid(i, ny)), b_y1))
    for j in range(ny):
        faces.append((GMSH_LINE2, (nid(nx, j), nid(nx, j + 1)), b_x1))
        faces.append((GMSH_LINE2, (nid(0, j + 1), nid(0, j)), b_x0))
    return Mesh(2, nodes, GMSH_QUAD4, eles, faces)


def box_hexes(nx: int, ny: int, nz: int, lo: Sequence[float] = (0.0, 0.0, 0.0),
              hi: Sequence[float] = (2 * math.pi, 2 * math.pi, 2 * math.pi), bnd: str = "PERIODIC") -> Mesh:
    """Structured 8-node hexes on the box [lo, hi], all sides tagged ``bnd`` (x fastest)."""
    xs = np.linspace(lo[0], hi[0], nx + 1)
    ys = np.linspace(lo[1], hi[1], ny + 1)
    zs = np.linspace(lo[2], hi[2], nz + 1)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    nodes = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    sx, sy = 1, nx + 1
    sz = (nx + 1) * (ny + 1)
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    i, j, k = (a.transpose(2, 1, 0).ravel() for a in (i, j, k))  # x fastest
    base = k * sz + j * sy + i * sx
    eles = np.stack([base, base + sx, base + sx + sy, base + sy,
                     base + sz, base + sz + sx, base + sz + sx + sy, base + sz + sy], axis=1).astype(np.int64)

    def n(ii, jj, kk):
        return kk * sz + jj * sy + ii * sx

    faces: List[Tuple[int, Tuple[int, ...], str]] = []
    for jj in range(ny):
        for ii in range(nx):
            faces.append((GMSH_QUAD4, (n(ii, jj, 0), n(ii, jj + 1, 0), n(ii + 1, jj + 1, 0), n(ii + 1, jj, 0)), bnd))
            faces.append((GMSH_QUAD4, (n(ii, jj, nz), n(ii + 1, jj, nz), n(ii + 1, jj + 1, nz), n(ii, jj + 1, nz)), bnd))
    for kk in range(nz):
        for ii in range(nx):
            faces.append((GMSH_QUAD4, (n(ii, 0, kk), n(ii + 1, 0, kk), n(ii + 1, 0, kk + 1), n(ii, 0, kk + 1)), bnd))
            faces.append((GMSH_QUAD4, (n(ii, ny, kk), n(ii, ny, kk + 1), n(ii + 1, ny, kk + 1), n(ii + 1, ny, kk)), bnd))
    for kk in range(nz):
        for jj in range(ny):
            faces.append((GMSH_QUAD4, (n(0, jj, kk), n(0, jj, kk + 1), n(0, jj + 1, kk + 1), n(0, jj + 1, kk)), bnd))
            faces.append((GMSH_QUAD4, (n(nx, jj, kk), n(nx, jj + 1, kk), n(nx, jj + 1, kk + 1), n(nx, jj, kk + 1)), bnd))
    return Mesh(3, nodes, GMSH_HEX8, eles, faces)


def jitter_interior(mesh: Mesh, amount: float, seed: int) -> Mesh:
    """Move every node not on a boundary face by U(-amount, amount) per coordinate.

    Boundary nodes stay fixed so periodic faces keep matching centroids
    (the reference pairs them at 1e-6, ``src/geometry.cpp:1159-1255``).
    """
    rng = np.random.default_rng(seed)
    on_bnd = np.zeros(mesh.nodes.shape[0], dtype=bool)
    for _, fn, _ in mesh.bnd_faces:
        on_bnd[list(fn)] = True
    d = rng.uniform(-amount, amount, size=mesh.nodes.shape)
    d[:, mesh.ndims:] = 0.0
    d[on_bnd] = 0.0
    return dataclasses.replace(mesh, nodes=mesh.nodes + d)


def box_tris(n: int, x0: float = 0.0, x1: float = 1.0, seed: int = 0, jitter: float = 0.15,
             bnd: str = "PERIODIC") -> Mesh:
    """n-by-n quad box on [x0,x1]^2 with each quad split along a seed-chosen diagonal,
    interior nodes jittered by U(-jitter*h, jitter*h)."""
    q = box_quads(n, n, x0, x1, x0, x1, bnd)
    rng = np.random.default_rng(seed)
    choice = rng.integers(2, size=q.n_elements)
    tris = []
    for (a, b, c, d), ch in zip(q.elements, choice):
        if ch == 0:
            tris += [[a, b, c], [a, c, d]]
        else:
            tris += [[a, b, d], [b, c, d]]
    m = Mesh(2, q.nodes, GMSH_TRI3, np.array(tris, dtype=np.int64), q.bnd_faces)
    h = (x1 - x0) / n
    return jitter_interior(m, jitter * h, seed + 1) if jitter > 0 else m


def cylinder_omesh(nr: int = 48, nt: int = 96, r0: float = 0.5, r1: float = 20.0, stretch: float = 1.1,
                   wall_amp: Sequence[float] = (), wall_name: str = "WALL", far_name: str = "FARFIELD") -> Mesh:
    """O-mesh of nr radial x nt circumferential 9-node quads around a circle.

    Radial spacing is geometric with ratio ``stretch`` from r0 to r1; the wall
    (r = r0) is displaced radially by sum_k a_k cos(k theta) / sin(k theta) terms
    given in ``wall_amp`` (pairs), the displacement decaying linearly to zero at
    r1.  Each element is counter-clockwise in (r, theta); the wall is boundary
    ``wall_name`` and the outer circle ``far_name``.
    """
    # radial node positions for 2*nr+1 levels (corner + mid levels)
    if stretch == 1.0:
        rc = np.linspace(r0, r1, nr + 1)
    else:
        dr0 = (r1 - r0) * (stretch - 1.0) / (stretch ** nr - 1.0)
        rc = r0 + dr0 * (stretch ** np.arange(nr + 1) - 1.0) / (stretch - 1.0)
    rl = np.empty(2 * nr + 1)
    rl[0::2] = rc
    rl[1::2] = 0.5 * (rc[:-1] + rc[1:])
    th = np.linspace(0.0, 2 * math.pi, 2 * nt + 1)[:-1]
    amps = list(wall_amp)

    def wall_disp(t):
        d = np.zeros_like(t)
        for k in range(len(amps) // 2):
            d = d + amps[2 * k] * np.cos((k + 1) * t) + amps[2 * k + 1] * np.sin((k + 1) * t)
        return d

    R, T = np.meshgrid(rl, th, indexing="ij")  # (2nr+1, 2nt)
    frac = (r1 - R) / (r1 - r0)
    Rd = R + frac * wall_disp(T)
    nodes = np.stack([Rd * np.cos(T), Rd * np.sin(T), np.zeros_like(R)], axis=-1).reshape(-1, 3)
    ntl = 2 * nt

    def nid(ir, it):
        return ir * ntl + (it % ntl)

    eles = []
    for i in range(nr):
        for j in range(nt):
            r_, t_ = 2 * i, 2 * j
            eles.append([nid(r_, t_), nid(r_ + 2, t_), nid(r_ + 2, t_ + 2), nid(r_, t_ + 2),
                         nid(r_ + 1, t_), nid(r_ + 2, t_ + 1), nid(r_ + 1, t_ + 2), nid(r_, t_ + 1),
                         nid(r_ + 1, t_ + 1)])
    faces: List[Tuple[int, Tuple[int, ...], str]] = []
    for j in range(nt):
        faces.append((GMSH_LINE3, (nid(0, 2 * j + 2), nid(0, 2 * j), nid(0, 2 * j + 1)), wall_name))
        faces.append((GMSH_LINE3, (nid(2 * nr, 2 * j), nid(2 * nr, 2 * j + 2), nid(2 * nr, 2 * j + 1)), far_name))
    return Mesh(2, nodes, GMSH_QUAD9, np.array(eles, dtype=np.int64), faces)
