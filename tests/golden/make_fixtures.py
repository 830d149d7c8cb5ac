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
  smoother_5x5.json       -- the 5x5 system of test/test_smoothers.jl:31-46 (i, j, v, b;
                             50 Jacobi sweeps with omega 1 from zero must reach A\\b to 0.1).
  bfs_10mm_unv.npz        -- examples/0_GRIDS/backwardFacingStep_10mm.unv (the mesh of
                             test/0_TEST_CASES/2d_incompressible_laminar_BFS.jl), parsed by
                             the small reader below into points, elements and groups.
  bfs_5mm_unv.npz         -- examples/0_GRIDS/backwardFacingStep_5mm.unv (the mesh of
                             test/0_TEST_CASES/2d_incompressible_transient_KOmega_BFS_lowRe.jl),
                             parsed the same way.
  cavity_hex_unv3.npz     -- test/grids/OF_cavity_hex/cavity_hex.unv (hex cells; counts pinned by
                             test/test_mesh_conversion.jl:43-61), 3D parse below.
  streamtube_unv3.npz     -- examples/0_GRIDS/3d_streamtube_1.0x0.1x0.1_0.08mm.unv (tetrahedra).

Usage: python tests/golden/make_fixtures.py /path/to/XCALibre.jl
       (or XCAL_REFERENCE_DIR=/path/to/XCALibre.jl python tests/golden/make_fixtures.py)
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


def smoother_system(path: str) -> dict:
    txt = open(path).read()

    def vec(name):
        return re.search(name + r"\s*=\s*\[(.*?)\]", txt).group(1).split(",")

    # entries such as 200*500: products of integers
    b = [float(np.prod([int(f) for f in t.split("*")])) for t in vec(r"\bb")]
    return dict(i=[int(v) for v in vec(r"\bi")], j=[int(v) for v in vec(r"\bj")], v=[float(v) for v in vec(r"\bv")],
                b=b, loops=50, omega=1.0, atol=0.1, source="test/test_smoothers.jl:31-46")


def read_unv_raw(path: str) -> dict:
    """Datasets 2411 (points), 2412 (elements: 6-field header ending in the
    vertex count, then the vertex line; beam orientation lines skipped) and
    2467 (groups) of a .unv file, with 1-based labels as in the file."""
    pts, ecount, eidx, everts, gnames, gelems = [], [], [], [], [], []
    ds, inblock = None, False
    hdr = None
    for line in open(path):
        s = line.split()
        if not s:
            continue
        if s[0] == "-1":
            inblock, ds = not inblock, None
            continue
        if inblock and ds is None:
            ds = s[0]
            continue
        if ds == "2411" and "." in s[0]:
            pts.append([float(v) for v in s[:3]])
        elif ds == "2412":
            if len(s) == 6:
                hdr = (int(s[0]), int(s[-1]))
            elif s[0] != "0" and hdr is not None and len(s) == hdr[1]:
                eidx.append(hdr[0])
                ecount.append(hdr[1])
                everts.extend(int(v) for v in s)
                hdr = None
        elif ds == "2467":
            if len(s) == 8 and s[1] == "0":
                gelems.append([])
            elif not s[0].lstrip("-").isdigit():
                gnames.append(s[0])
            else:
                gelems[-1].append(int(s[1]))
                if len(s) >= 6:
                    gelems[-1].append(int(s[5]))
    goff = np.zeros(len(gelems) + 1, dtype=np.int64)
    goff[1:] = np.cumsum([len(g) for g in gelems])
    return dict(points=np.array(pts), elem_index=np.array(eidx, dtype=np.int32),
                elem_count=np.array(ecount, dtype=np.int32), elem_vertices=np.array(everts, dtype=np.int32),
                group_names=np.array(gnames), group_offsets=goff,
                group_elements=np.array([e for g in gelems for e in g], dtype=np.int32))


def read_unv3_raw(path: str) -> dict:
    """Datasets 2411 (3-field point lines), 2412 (edges skipped; faces 41/44
    and cells 111/112/115 with their node lines) and 2467 (group name lines,
    then entity lines whose element labels, less the edge count, are face
    positions) of a 3D .unv file; labels stay 1-based."""
    pts, fcount, fverts, ccount, cverts, gnames, gelems = [], [], [], [], [], [], []
    n_edge = 0
    lines = [ln.strip() for ln in open(path)]
    i, ds = 0, ""
    while i < len(lines):
        ln = lines[i]
        i += 1
        if not ln:
            continue
        if ln == "-1":
            if ds == "":
                ds = lines[i]
                i += 1
                ds = "" if ds == "-1" else ds
            else:
                ds = ""
            continue
        t = ln.split()
        if ds == "2411" and len(t) == 3:
            pts.append([float(v.replace("D", "e")) for v in t])
        elif ds == "2412" and len(t) == 6:
            etype, nn = int(t[1]), int(t[5])
            if nn == 2 or etype == 11:
                n_edge += 1
                i += 1
            elif etype in (41, 44):
                fv = [int(v) for v in lines[i].split()]
                i += 1
                fcount.append(len(fv))
                fverts.extend(fv)
            elif etype in (111, 112, 115):
                cv = []
                while len(cv) < nn:
                    cv.extend(int(v) for v in lines[i].split())
                    i += 1
                ccount.append(len(cv))
                cverts.extend(cv)
        elif ds == "2467":
            if len(t) == 1 and not t[0].lstrip("-").isdigit():
                gnames.append(t[0])
                gelems.append([])
            elif gelems and len(t) in (4, 8) and t[1] != "0":
                gelems[-1].append(int(t[1]) - n_edge)
                if len(t) == 8:
                    gelems[-1].append(int(t[5]) - n_edge)
    goff = np.zeros(len(gelems) + 1, dtype=np.int64)
    goff[1:] = np.cumsum([len(g) for g in gelems])
    return dict(points=np.array(pts), face_count=np.array(fcount, dtype=np.int32),
                face_vertices=np.array(fverts, dtype=np.int32), cell_count=np.array(ccount, dtype=np.int32),
                cell_vertices=np.array(cverts, dtype=np.int32), group_names=np.array(gnames),
                group_offsets=goff, group_faces=np.array([e for g in gelems for e in g], dtype=np.int32))


def main(ref: str) -> None:
    pm = read_polymesh(os.path.join(ref, "test/grids/OF_cavity_hex/polyMesh"))
    np.savez_compressed(os.path.join(HERE, "cavity_hex_polymesh.npz"), **pm)
    pz = read_polymesh(os.path.join(ref, "examples/0_GRIDS/OF_pitzDaily/polyMesh"))
    np.savez_compressed(os.path.join(HERE, "pitzdaily_polymesh.npz"), **pz)
    with open(os.path.join(HERE, "laplace_3by3.json"), "w") as f:
        json.dump(laplace_expected(os.path.join(ref, "test/unit_test_laplace.jl")), f, indent=1)
    with open(os.path.join(HERE, "smoother_5x5.json"), "w") as f:
        json.dump(smoother_system(os.path.join(ref, "test/test_smoothers.jl")), f, indent=1)
    np.savez_compressed(os.path.join(HERE, "cavity_hex_unv3.npz"),
                        **read_unv3_raw(os.path.join(ref, "test/grids/OF_cavity_hex/cavity_hex.unv")))
    np.savez_compressed(os.path.join(HERE, "streamtube_unv3.npz"),
                        **read_unv3_raw(os.path.join(ref, "examples/0_GRIDS/3d_streamtube_1.0x0.1x0.1_0.08mm.unv")))
    for mm in (10, 5):
        np.savez_compressed(os.path.join(HERE, "bfs_%dmm_unv.npz" % mm),
                            **read_unv_raw(os.path.join(ref, "examples/0_GRIDS/backwardFacingStep_%dmm.unv" % mm)))
    print("fixtures written to", HERE)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("XCAL_REFERENCE_DIR", "")
    if not ref:
        sys.exit("usage: make_fixtures.py /path/to/XCALibre.jl (or set XCAL_REFERENCE_DIR)")
    main(ref)
