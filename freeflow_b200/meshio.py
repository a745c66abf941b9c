"""Medit ``.mesh`` reading and surface extraction for the fluid step.

The reference reads Medit files with ``MeshLoader2D`` / ``MeshLoader3D``
(``src/io/MeshLoader.cpp:19-146``, ``:147-271``):

- a header line ``MeshVersionFormatted <v>``;
- a header line ``Dimension <d>``;
- blocks ``Vertices``, ``Edges`` (2D files) and ``Triangles``, or ``Vertices``, ``Triangles`` and
  ``Tetrahedra`` (3D files): the keyword, a count line, then one entry per line. Indices are 1-based;
  trailing reference tags are ignored.
- Unknown lines are skipped with a warning.

Two differences, both more lenient: block keywords are matched after stripping white space (the
reference compares the whole line, so a CRLF file loses its blocks there), and ``End`` ends the
file (the reference skips it as an unknown line, with the same result on a well-formed file).

The fluid step only sees a solid's surface:

- 2D: the boundary segments of the triangle mesh;
- 3D: the boundary triangles of the tetrahedral mesh, or the ``Triangles`` block when there are no tetrahedra.

``surface_of`` extracts that surface. ``place`` applies a solid's scale, rotation and
translation from its JSON block.
"""
from __future__ import annotations

import math
import warnings
from dataclasses import dataclass

import numpy as np


@dataclass
class MeditMesh:
    dimension: int
    vertices: np.ndarray                  # (nv, dim) float64
    triangles: np.ndarray                 # (nt, 3) int64, 0-based
    tetrahedra: np.ndarray                # (ntet, 4) int64, 0-based
    edges: np.ndarray = None              # (ned, 2) int64, 0-based (2D files only)


def load_medit(path: str, dimension: int | None = None) -> MeditMesh:
    """Reads a Medit file; raises ValueError on a malformed header or block."""
    with open(path) as f:
        lines = f.read().splitlines()
    it = iter(lines)

    def header(keyword):
        line = next(it, "")
        parts = line.split()
        if not parts or parts[0] != keyword or len(parts) < 2:
            raise ValueError(f"{path}: expected '{keyword}', got '{line}'")
        return parts[1]

    header("MeshVersionFormatted")
    dim = int(header("Dimension"))
    if dimension is not None and dim != dimension:
        raise ValueError(f"{path}: a {dimension}D mesh was expected, the file is {dim}D")
    verts, tris, tets, edges = [], [], [], []
    blocks = ("Vertices", "Edges", "Triangles") if dim == 2 else ("Vertices", "Triangles", "Tetrahedra")
    for line in it:
        key = line.strip()
        if not key:
            continue
        if key in blocks:
            count = int(next(it).strip())
            width = {"Vertices": dim, "Edges": 2, "Triangles": 3, "Tetrahedra": 4}[key]
            rows = []
            for _ in range(count):
                vals = next(it).split()
                if len(vals) < width:
                    raise ValueError(f"{path}: short {key} entry '{' '.join(vals)}'")
                rows.append(vals[:width])
            if key == "Vertices":
                verts = np.array(rows, dtype=np.float64).reshape(-1, dim)
            elif key == "Edges":
                edges = np.array(rows, dtype=np.int64).reshape(-1, 2) - 1
            elif key == "Triangles":
                tris = np.array(rows, dtype=np.int64).reshape(-1, 3) - 1
            else:
                tets = np.array(rows, dtype=np.int64).reshape(-1, 4) - 1
        elif key == "End":
            break
        else:
            warnings.warn(f"{path}: unknown keyword '{key}' skipped")
    return MeditMesh(dim, np.asarray(verts, np.float64).reshape(-1, dim),
                     np.asarray(tris, np.int64).reshape(-1, 3), np.asarray(tets, np.int64).reshape(-1, 4),
                     np.asarray(edges, np.int64).reshape(-1, 2))


def boundary_edges(triangles: np.ndarray) -> np.ndarray:
    """Edges used by exactly one triangle, oriented as in that triangle."""
    e = np.concatenate([triangles[:, [0, 1]], triangles[:, [1, 2]], triangles[:, [2, 0]]], axis=0)
    key = np.sort(e, axis=1)
    _, inv, cnt = np.unique(key, axis=0, return_inverse=True, return_counts=True)
    return e[cnt[inv.reshape(-1)] == 1]


def boundary_faces(tetrahedra: np.ndarray) -> np.ndarray:
    """Faces used by exactly one tetrahedron."""
    t = tetrahedra
    f = np.concatenate([t[:, [0, 2, 1]], t[:, [0, 1, 3]], t[:, [0, 3, 2]], t[:, [1, 2, 3]]], axis=0)
    key = np.sort(f, axis=1)
    _, inv, cnt = np.unique(key, axis=0, return_inverse=True, return_counts=True)
    return f[cnt[inv.reshape(-1)] == 1]


def surface_of(mesh: MeditMesh):
    """(vertices, elements, vertex ids) of the surface, renumbered compactly;
    vertex ids map surface vertices back to mesh vertices."""
    if mesh.dimension == 2:
        el = boundary_edges(mesh.triangles)
    elif len(mesh.tetrahedra):
        el = boundary_faces(mesh.tetrahedra)
    else:
        el = mesh.triangles
    ids, inv = np.unique(el.reshape(-1), return_inverse=True)
    return mesh.vertices[ids].copy(), inv.reshape(el.shape).astype(np.uint32), ids


def place(vertices: np.ndarray, translate, rotate, scale) -> np.ndarray:
    """The reference's initial transform of a solid: scale, then rotate, then translate.

    - 2D (``Mesh2D::applyInitialTransform``, ``src/fem/DeformableMesh.cpp:403-423``): `rotate` is in
      degrees. The rotation matrix there is built with glm's column-major constructor from
      (cos, -sin, sin, cos), which turns points by -rotate. That is reproduced here, with the
      reference's roundings: the arithmetic is double, but scale and translate pass through float,
      and the angle is glm::radians of float(rotate) in float (float(rotate) times the float of
      pi/180), so a 180-degree turn leaves sin = -8.74e-8, not 0. Each coordinate is formed as
      there, c * x + s * y with two roundings and no fused multiply-add.
    - 3D (``Mesh3D::applyInitialTransform``, ``:158-185``): ``eulerAngleYXZ`` of (rotate[1], rotate[0],
      rotate[2]) degrees, i.e. R = Ry(rotate[1]) Rx(rotate[0]) Rz(rotate[2]). The reference forms it
      in float (glm::mat4); here it is double, so coordinates can differ from it by a float ulp.
    """
    if np.asarray(vertices).shape[1] == 2:
        f32 = np.float32
        v = np.asarray(vertices, np.float64) * np.asarray(scale, f32).astype(np.float64)
        a = float(f32(f32(float(rotate)) * f32(math.pi / 180.0)))
        c, s = math.cos(a), math.sin(a)
        t = np.asarray(translate, f32).astype(np.float64)
        x, y = v[:, 0], v[:, 1]
        return np.stack([c * x + s * y + t[0], -s * x + c * y + t[1]], axis=1)
    v = np.asarray(vertices, np.float64) * np.asarray(scale, np.float64)
    ax, ay, az = (math.radians(float(r)) for r in rotate)
    Rx = np.array([[1, 0, 0], [0, math.cos(ax), -math.sin(ax)], [0, math.sin(ax), math.cos(ax)]])
    Ry = np.array([[math.cos(ay), 0, math.sin(ay)], [0, 1, 0], [-math.sin(ay), 0, math.cos(ay)]])
    Rz = np.array([[math.cos(az), -math.sin(az), 0], [math.sin(az), math.cos(az), 0], [0, 0, 1]])
    R = Ry @ Rx @ Rz
    return v @ R.T + np.asarray(translate, np.float64)


def write_medit(path: str, vertices: np.ndarray, triangles=None, tetrahedra=None):
    """Writes a Medit file (1-based indices, zero reference tags)."""
    v = np.asarray(vertices)
    with open(path, "w") as f:
        f.write("MeshVersionFormatted 1\n")
        f.write(f"Dimension {v.shape[1]}\n")
        f.write("Vertices\n")
        f.write(f"{len(v)}\n")
        for row in v:
            f.write(" ".join(repr(float(x)) for x in row) + " 0\n")
        for name, arr in (("Triangles", triangles), ("Tetrahedra", tetrahedra)):
            if arr is None:
                continue
            a = np.asarray(arr) + 1
            f.write(f"{name}\n{len(a)}\n")
            for row in a:
                f.write(" ".join(str(int(x)) for x in row) + " 0\n")
        f.write("End\n")
