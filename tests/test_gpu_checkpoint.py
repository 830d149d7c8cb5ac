"""Checkpoint / restart of the product and result output from run_.

* A case run N iterations, checkpointed (Case.checkpoint, saved to .npz and
  loaded back) and restored into a fresh case gives the results of 2N
  uninterrupted iterations bit for bit: SIMPLE in FP64 and mixed precision,
  PISO (periodic LES) in graph mode.
* run_ with write_interval writes the reference's result files (VTK
  iteration_<k>.vtu, or an OpenFOAM case) holding the fields of those
  iterations, and writing does not change the results."""
import os
import xml.etree.ElementTree as ET

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["simple-fp64", "simple-mixed", "piso-graph"])
def test_restart_bit_identical(x, ctx, tmp_path, mode):
    A = x.api
    if mode.startswith("simple"):
        mesh = x.build_mesh3(x.channel_polymesh(12, 6, 6, seed=3, length=2.0))
        mk = lambda: x.cases.channel_case(mesh, iterations=10, precision=mode.split("-")[1])
        pref, N = None, 4
    else:
        mesh = x.build_mesh3(x.periodic_box_polymesh(8, seed=5))
        U0 = x.cases.fourier_field(mesh, seed=5)
        mk = lambda: x.cases.periodic_les_case(mesh, steps=6, U0=U0, precision="mixed")
        pref, N = 0.0, 3

    def new_case():
        model, config = mk()
        cfg, keep = x.build_config(model, config, pref=pref)
        dm = A.DeviceMesh(ctx, mesh)
        c = A.Case(dm, cfg)
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
        if mode == "piso-graph":
            c.set_graph_mode(True)
        return c, (dm, keep)

    def run(c, n):
        return c.simple_iterate(n)[0] if mode.startswith("simple") else c.piso_step(n)[0]

    a, ka = new_case()
    ra = run(a, 2 * N)
    b, kb = new_case()
    rb = run(b, N)
    path = str(tmp_path / "ck.npz")
    x.save_checkpoint(b.checkpoint(), path)
    c, kc = new_case()
    c.restore(x.load_checkpoint(path))
    rc = run(c, N)
    assert np.array_equal(np.vstack([rb, rc]), ra)
    for f in (x._abi.FIELD_U, x._abi.FIELD_P, x._abi.FIELD_MDOTF):
        assert np.array_equal(c.get_field(f), a.get_field(f))


def _vtu_fields(path):
    root = ET.parse(path).getroot()
    return {da.get("Name"): np.array(da.text.split(), dtype=np.float64)
            for da in root.iter("DataArray") if da.get("Name") in ("U", "p")}


@pytest.mark.parametrize("fmt", ["vtk", "openfoam"])
def test_run_writes_results(x, tmp_path, fmt):
    mesh = x.build_mesh3(x.cavity_polymesh(12, seed=2))
    plain_model, plain_cfg = x.cases.cavity_case(mesh, iterations=4)
    r0 = x.run_(plain_model, plain_cfg, pref=0.0)
    model, config = x.cases.cavity_case(mesh, iterations=4)
    config.runtime.write_interval = 2
    out = x.VTK() if fmt == "vtk" else x.OpenFOAM()
    r1 = x.run_(model, config, pref=0.0, output=out, output_dir=str(tmp_path))
    for k in r0:
        assert np.array_equal(r0[k], r1[k]), k
    assert np.array_equal(plain_model.momentum.U, model.momentum.U)
    if fmt == "vtk":
        assert sorted(os.listdir(tmp_path)) == ["iteration_2.vtu", "iteration_4.vtu"]
        last = _vtu_fields(str(tmp_path / "iteration_4.vtu"))
        assert np.array_equal(last["U"].reshape(-1, 3), np.asarray(model.momentum.U).T)
        assert np.array_equal(last["p"], model.momentum.p)
    else:
        from importlib import import_module
        W = import_module(x.__name__ + ".writers")
        assert {"2", "4", "constant", "XCALibre.foam"} <= set(os.listdir(tmp_path))
        assert np.array_equal(W._read_foam_internal(str(tmp_path / "4" / "U")), np.asarray(model.momentum.U).T)
        assert np.array_equal(W._read_foam_internal(str(tmp_path / "4" / "p")), model.momentum.p)
