"""Generate the golden fixtures under tests/golden/ from the reference's own
test data (run once in a container that has the reference checkout; the
fixtures are committed, so tests never read the reference at run time).

Fixtures:
  cavity_hex_polymesh.npz -- test/grids/OF_cavity_hex/polyMesh (OpenFOAM ASCII),
                             parsed into points/faces/owner/neighbour/patches.
                             Pins the mesh counts of test/test_mesh_conversion.jl:49-57.
  laplace_3by3.json       -- expected_A_matrix / expected_b_vector of
                             test/unit_test_laplace.jl:112-127, with the cell
                             centroids of the 3x3 unit-square mesh they refer to.
  pitzdaily_polymesh.npz  -- examples/0_GRIDS/OF_pitzDaily/polyMesh (counts pinned by
                             test/0_TEST_CASES/2d_incompressible_pitzdaily_Smagorinsky.jl:14-16).

Usage: python tests/golden/make_fixtures.py [/path/to/XCALibre.jl]
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _strip_foam(text: str) -> str:
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    text = re.sub(r"FoamFile\s*\{.*?\}", "", text, flags=re.S)
    return text


def _list_body(text: str):
    """Return (count, body) of the first top-level 'N ( ... )' list."""
    m = re.search(r"(\d+)\s*\(", text)
    n = int(m.group(1))
    depth, i0 = 0, m.end() - 1
    for i in range(i0, len(text)):
        if text[i] == "(":
            depth += 1
        elif text[i] == ")":
            depth -= 1
            if depth == 0:
                return n, text[i0 + 1:i]
    raise ValueError("unterminated list")


def read_polymesh(d: str) -> dict:
    rd = lambda f: _strip_foam(open(os.path.join(d, f)).read())
    n, body = _list_body(rd("points"))
    pts = np.array([[float(v) for v in t.split()] for t in re.findall(r"\(([^()]*)\)", body)])
    assert pts.shape == (n, 3)
    n, body = _list_body(rd("faces"))
    faces = [[int(v) for v in t.split()] for t in re.findall(r"\d+\s*\(([^()]*)\)", body)]
    assert len(faces) == n
    n, body = _list_body(rd("owner"))
    owner = np.array([int(v) for v in body.split()], dtype=np.int32)
    n, body = _list_body(rd("neighbour"))
    neigh = np.array([int(v) for v in body.split()], dtype=np.int32)
    btxt = rd("boundary")
    names, sizes, starts = [], [], []
    for m in re.finditer(r"(\w+)\s*\{([^}]*)\}", btxt):
        nf = re.search(r"nFaces\s+(\d+)", m.group(2))
        sf = re.search(r"startFace\s+(\d+)", m.group(2))
        if nf and sf:
            names.append(m.group(1))
            sizes.append(int(nf.group(1)))
            starts.append(int(sf.group(1)))
    offs = np.zeros(len(faces) + 1, dtype=np.int32)
    offs[1:] = np.cumsum([len(f) for f in faces])
    return dict(points=pts, face_offsets=offs, face_nodes=np.array([v for f in faces for v in f], dtype=np.int32),
                owner=owner, neighbour=neigh, patch_names=np.array(names), patch_sizes=np.array(sizes, dtype=np.int32),
                patch_starts=np.array(starts, dtype=np.int32))


def laplace_expected(path: str) -> dict:
    txt = open(path).read()
    mA = re.search(r"expected_A_matrix\s*=\s*\[(.*?)\]", txt, flags=re.S)
    rows = [r.strip() for r in mA.group(1).strip().split(";") if r.strip()]
    A = [[float(v) for v in r.split()] for r in rows]
    mb = re.search(r"expected_b_vector\s*=\s*\[(.*?)\]", txt, flags=re.S)
    b = [float(v) for v in mb.group(1).split(",")]
    # cell k (1-based) of laplace_unit_3by3.unv: column (k-1)//3 from the
    # left wall, row (k-1)%3 from the top (cells 1-3 touch left_wall, cells
    # 3,6,9 touch bottom_wall -- read off the Dirichlet entries of b)
    cent = [[((k // 3) + 0.5) / 3.0, ((2 - k % 3) + 0.5) / 3.0] for k in range(9)]
    return dict(A=A, b=b, centroids=cent, atol_A=0.1,
                source="test/unit_test_laplace.jl:112-130")


def main(ref: str) -> None:
    pm = read_polymesh(os.path.join(ref, "test/grids/OF_cavity_hex/polyMesh"))
    np.savez_compressed(os.path.join(HERE, "cavity_hex_polymesh.npz"), **pm)
    pz = read_polymesh(os.path.join(ref, "examples/0_GRIDS/OF_pitzDaily/polyMesh"))
    np.savez_compressed(os.path.join(HERE, "pitzdaily_polymesh.npz"), **pz)
    with open(os.path.join(HERE, "laplace_3by3.json"), "w") as f:
        json.dump(laplace_expected(os.path.join(ref, "test/unit_test_laplace.jl")), f, indent=1)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
