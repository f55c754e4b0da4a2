"""The C-ABI boundary without a GPU: the library loads, exports every entry
point include/z4c_b200.h declares, reports the reference's defaults, builds
block coordinates bit for bit as the reference does, and rejects bad input
and a missing device with error codes."""
import ctypes as C
import json
import os
import re

import numpy as np
import pytest

import z4c_b200 as Z
import z4c_oracle as O
from z4c_testlib import ROOT, Case

HEADER = os.path.join(ROOT, "include", "z4c_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(z4c_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_entry_point():
    lib = C.CDLL(Z.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(Z.EXPORTS)


def test_defaults_match_reference():
    p = Z.default_params()
    ref = O.default_params()
    for name, _ in Z.Params._fields_:
        assert getattr(p, name) == getattr(ref, name), name
    assert p.r_max_con == float("inf")


@pytest.mark.parametrize("name", ["ops_gw1", "ops_punc2", "ops_rs2", "ops_somm2", "evol_gw16",
                                  "evol_punc4", "evol_somm4"])
def test_block_coordinates_bitwise(name):
    c = Case(name)
    m = c.mesh
    mesh = Z.Mesh(m["nb"], m["nx"], m["xmin"], m["xmax"], m["bc"])
    for g, grid_b in enumerate(c.order):
        xs, dxs = mesh.block_coords(grid_b)
        assert np.array_equal(np.concatenate(xs), c.rec["xf"][g])
        assert np.array_equal(np.array(dxs), c.rec["dx"][g])


@pytest.mark.parametrize("name", ["ops_gw1", "ops_punc2", "ops_rs2", "ops_somm2", "evol_gw16",
                                  "evol_punc4", "evol_somm4"])
def test_time_step_matches_reference(name):
    """NewBlockTimeStep + Mesh::NewTimeStep with the decks' Courant number 0.25
    give the reference's dt bit for bit."""
    c = Case(name)
    m = c.mesh
    mesh = Z.Mesh(m["nb"], m["nx"], m["xmin"], m["xmax"], m["bc"])
    assert mesh.new_dt(0.25) == c.rec["time_dt"][1]


def test_create_errors_without_device_or_with_bad_mesh():
    bad = Z.Mesh((1, 1, 1), (4, 8, 8), (0, 0, 0), (1, 1, 1))
    with pytest.raises(Z.Z4cError) as e:
        Z.Z4c(bad)
    assert e.value.code in (-1, -7)  # EINVAL (nx < 2*ng), or ENODEV first
    half = Z.Mesh((1, 1, 1), (8, 8, 8), (0, 0, 0), (1, 1, 1), bc=[0, 1, 0, 0, 0, 0])
    with pytest.raises(Z.Z4cError):
        Z.Z4c(half)
    with pytest.raises(Z.Z4cError) as e:
        Z.Z4c(Z.Mesh((1, 1, 1), (8, 8, 8), (0, 0, 0), (1, 1, 1)), integrator="rk4")
        pytest.skip("a CUDA device is present")
    assert e.value.code == -7


@pytest.mark.parametrize("name", ["evol_gw16", "evol_punc4", "evol_somm4"])
def test_initial_data_pipeline_matches_reference(name):
    """Host initial data (restated problem generators) taken through the
    oracle's ADMToZ4c, ghost exchange and ghost-only AlgConstr reproduces the
    reference's initialised state bit for bit."""
    from z4c_b200 import initial_data as ID
    c = Case(name)
    m = c.mesh
    mesh = Z.Mesh(m["nb"], m["nx"], m["xmin"], m["xmax"], m["bc"])
    p = O.default_params(**c.params)
    if "gw" in name:
        adm = ID.gauge_wave1(mesh, amplitude=0.01)
    else:
        adm = ID.punctures(mesh, p, masses=(1.0,), centres=((0.0, 0.0, 0.0),))
    adm = c.from_grid(adm)
    blocks = c.blocks()
    u = np.stack([O.adm_to_z4c(b, p, adm[g]) for g, b in enumerate(blocks)])
    u = c.from_grid(O.mesh_exchange(c.nb, c.nx, m["bc"], c.to_grid(u)))
    u = np.stack([O.algconstr(b, p, u[g], ghosts_only=True) for g, b in enumerate(blocks)])
    assert np.array_equal(u, c.rec["u_init"])
