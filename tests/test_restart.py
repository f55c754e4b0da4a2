"""Reference restart files (outputs/restart.cpp) through the C ABI.

The fixture is the restart file the stock reference driver wrote at the end
of the evol_track4 run (a puncture tracker, 2x2x1 MeshBlocks): its bytes
before the MeshBlock data are stored, the data section is that run's final
state.  The reader must recover state, time, dt, cycle and tracker; the
writer must reproduce the file byte for byte, except for padding bytes that
the reference copies from uninitialised memory; when the reference build is
present, the reference must continue from a file this library wrote exactly
as it continues from its own."""
import os
import subprocess
import sys

import numpy as np
import pytest

import z4c_b200 as Z
from z4c_testlib import GOLDEN, ROOT, Case

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "athena_ref")


def _reference_file(tmp_path):
    z = np.load(os.path.join(GOLDEN, "restart_track4.npz"))
    c = Case("evol_track4")
    path = tmp_path / "golden.final.rst"
    path.write_bytes(z["prefix"].tobytes() + c.rec["u_final"].astype("<f8").tobytes())
    return str(path), c


def test_reader_recovers_the_reference_state(tmp_path):
    path, c = _reference_file(tmp_path)
    info = Z.restart_info(path)
    assert info["nb"] == (2, 2, 1) and info["block_nx"] == (8, 8, 8)
    assert info["ncycle"] == int(c.rec["nlim"])
    row = c.rec["tracker"][-1]  # iter, time, x, y, z, betax, betay, betaz (16 digits)
    assert info["time"] == pytest.approx(row[1], rel=1e-15)
    assert info["dt"] == c.rec["time_dt"][1]
    np.testing.assert_allclose(info["trackers"][0], row[2:8], rtol=1e-15, atol=0)
    mesh = Z.Mesh.from_restart(path)
    assert mesh.bc == (Z.BC_OUTFLOW,) * 6 and mesh.xmin == (-4.0, -4.0, -2.0)
    info2, u = Z.restart_read(path)
    assert np.array_equal(u, c.to_grid(c.rec["u_final"]))
    assert Z.restart_text(path).endswith("<par_end>\n")


def _same_but_padding(a, b, text_bytes, ntrk, nblocks):
    """Byte equality outside the padding of RegionSize (4 bytes after its
    three ints) and of each LogicalLocation (4 bytes after its level)."""
    if len(a) != len(b):
        return False
    a, b = bytearray(a), bytearray(b)
    pads = [text_bytes + 92 + q for q in range(4)]
    ids = text_bytes + 124 + 48 * ntrk
    pads += [ids + 40 * n + 28 + q for n in range(nblocks) for q in range(4)]
    for p in pads:
        a[p] = b[p] = 0
    return a == b


def test_writer_reproduces_the_reference_file(tmp_path):
    path, c = _reference_file(tmp_path)
    info, u = Z.restart_read(path)
    out = tmp_path / "ours.rst"
    text = Z.restart_text(path)
    Z.restart_write(str(out), text, Z.Mesh.from_restart(path), u, info["time"], info["dt"],
                    info["ncycle"], info["trackers"])
    assert _same_but_padding(out.read_bytes(), open(path, "rb").read(), len(text), 1, 4)


def test_reader_rejects_other_files(tmp_path):
    bad = tmp_path / "x.rst"
    bad.write_bytes(b"not a restart file")
    with pytest.raises(Z.Z4cError):
        Z.restart_info(str(bad))
    path, _ = _reference_file(tmp_path)
    raw = open(path, "rb").read()
    (tmp_path / "cut.rst").write_bytes(raw[:-1000])
    with pytest.raises(Z.Z4cError):
        Z.restart_read(str(tmp_path / "cut.rst"))


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference build (oracle/_ref) absent")
def test_reference_restarts_from_our_file(tmp_path):
    """The reference runs 3 more steps from a file written here (its own
    3-step state, read and re-written by this library) and lands bit for bit
    where it lands from its own restart file."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden as M
    from z4cio import read_records
    case = dict(M.EVOL["track4"])

    def run(tag, nlim, extra="", restart=None):
        d = tmp_path / tag
        d.mkdir()
        inp = d / "case.inp"
        inp.write_text(M.deck(case, "unused", nlim=nlim, dump_final=str(d / "final.rec")) + extra)
        cmd = [REF_BIN, "-r", str(restart)] if restart else [REF_BIN, "-i", str(inp)]
        if restart:
            cmd += [f"time/nlim={nlim}", f"problem/dump_final={d / 'final.rec'}"]
        subprocess.run(cmd, cwd=d, check=True, stdout=subprocess.DEVNULL)
        return d, read_records(str(d / "final.rec"))["u"]

    d3, _ = run("first", 3, M.RST_DECK)
    _, u_own = run("own", 6, restart=d3 / "golden.final.rst")
    info, u = Z.restart_read(str(d3 / "golden.final.rst"))
    ours = tmp_path / "ours.rst"
    Z.restart_write(str(ours), Z.restart_text(str(d3 / "golden.final.rst")),
                    Z.Mesh.from_restart(str(d3 / "golden.final.rst")), u, info["time"], info["dt"],
                    info["ncycle"], info["trackers"])
    _, u_rest = run("second", 6, restart=ours)
    assert np.array_equal(u_rest, u_own)


@pytest.mark.gpu
def test_context_load_evolve_save(tmp_path):
    """The reference's restart state loaded into a context, saved back
    unchanged (bytes equal), then evolved on the device with its tracker."""
    path, c = _reference_file(tmp_path)
    mesh = Z.Mesh.from_restart(path)
    ctx = Z.Z4c(mesh, Z.default_params(**c.params), "rk4")
    info = ctx.restart_load(path)
    assert np.array_equal(ctx.download(Z.REG_U), c.to_grid(c.rec["u_final"]))
    pos, beta = ctx.tracker(0)
    np.testing.assert_array_equal(np.concatenate([pos, beta]), info["trackers"][0])
    out = tmp_path / "saved.rst"
    text = Z.restart_text(path)
    ctx.restart_save(str(out), text, info["time"], info["dt"], info["ncycle"])
    assert _same_but_padding(out.read_bytes(), open(path, "rb").read(), len(text), 1, 4)
    ctx.evolve(info["dt"], 2)
    assert ctx.check_finite()
    assert np.linalg.norm(ctx.tracker(0)[0] - pos) > 0
    ctx.close()


def _reference_ml_file(tmp_path):
    """The reference's restart file of the two-level mesh with an
    integer-hash state in its data section (blocks in gid order)."""
    z = np.load(os.path.join(GOLDEN, "restart_ml.npz"))
    g, n, k, j, i = np.meshgrid(np.arange(15), np.arange(22), np.arange(17), np.arange(17),
                                np.arange(17), indexing="ij")
    u = ((g * 131 + n * 31 + k * 7 + j * 3 + i) % 1009) / 1009.0 - 0.5
    assert u.nbytes == int(z["data_bytes"])
    path = tmp_path / "golden.final.rst"
    path.write_bytes(z["prefix"].tobytes() + u.astype("<f8").tobytes())
    return str(path), u


def test_refined_mesh_file_is_read():
    """The ID list of a refined mesh's restart file: levels and locations
    of the 15 blocks, the root grid from the <meshblock> size."""
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        from pathlib import Path
        path, _ = _reference_ml_file(Path(d))
        info = Z.restart_info(path)
        assert info["nlevels"] == 2 and info["nbtotal"] == 15
        assert info["nb"] == (2, 2, 2) and info["block_nx"] == (8, 8, 8)
        mesh = Z.Mesh.from_restart(path)
        ml = np.load(os.path.join(GOLDEN, "ml_exchange_outflow.npz"))
        assert np.array_equal(mesh.locs, ml["meta"][:, 1:5])
        assert mesh.nblocks == 15 and mesh.root_level == 1


@pytest.mark.gpu
def test_refined_context_load_save(tmp_path):
    """A refined context restarts from the reference's file (state in gid
    order) and writes it back byte for byte except for padding."""
    path, u = _reference_ml_file(tmp_path)
    mesh = Z.Mesh.from_restart(path)
    ctx = Z.Z4c(mesh, Z.default_params(chi_div_floor=1e-5), "rk4")
    info = ctx.restart_load(path)
    assert np.array_equal(ctx.download(Z.REG_U), u)
    out = tmp_path / "saved.rst"
    text = Z.restart_text(path)
    ctx.restart_save(str(out), text, info["time"], info["dt"], info["ncycle"])
    assert _same_but_padding(out.read_bytes(), open(path, "rb").read(), len(text), 0, 15)
    ctx.close()
