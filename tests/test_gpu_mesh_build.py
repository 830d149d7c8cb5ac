"""The polyMesh importer's GPU geometry (xcal_foam_mesh_build_device)
against the host build: every array identical (the same operations in the
same order), on generated meshes (permuted numbering, skewed interior
points, a 2D slab, a periodic box) and the reference's pitzDaily polyMesh
(committed fixture); and the time of both on the 128^3 channel."""
import time

import numpy as np
import pytest

from test_oracle_golden import _polymesh

pytestmark = pytest.mark.gpu

ARRAYS = ("face_owner", "face_neigh", "face_centre", "face_normal", "face_e", "face_area", "face_delta",
          "face_weight", "cell_centre", "cell_volume", "cell_faces_offset", "cell_faces", "cell_nsign",
          "cell_neighbours", "boundary_cellsID", "patch_start", "patch_count")


def _meshes(x):
    yield "channel", x.channel_polymesh(20, 12, 10, seed=3)
    yield "skewed", x.box_polymesh(14, 9, 8, lengths=(2.0, 1.0, 1.0), seed=5, skew=0.25, skew_seed=5,
                                   patches=[("inlet", ["xmin"]), ("outlet", ["xmax"]),
                                            ("walls", ["ymin", "ymax", "zmin", "zmax"])])
    yield "cavity", x.cavity_polymesh(24, seed=2)
    yield "periodic", x.periodic_box_polymesh(10, seed=4)
    yield "pitzdaily", _polymesh(x, "pitzdaily_polymesh.npz")


def test_device_build_identical(x, ctx):
    for name, pm in _meshes(x):
        a = x.build_mesh3(pm)
        b = x.build_mesh3(pm, device=0)
        for k in ARRAYS:
            assert np.array_equal(getattr(a, k), getattr(b, k)), (name, k)


def test_device_build_large(x, ctx):
    pm = x.channel_polymesh(128, 128, 128, seed=0)
    t0 = time.perf_counter()
    a = x.build_mesh3(pm)
    t1 = time.perf_counter()
    b = x.build_mesh3(pm, device=0)
    t2 = time.perf_counter()
    for k in ARRAYS:
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    print(f"128^3 channel: host build {t1 - t0:.2f} s, device build {t2 - t1:.2f} s")
