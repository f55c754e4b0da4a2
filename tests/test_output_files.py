"""History and puncture-tracker files in the reference's formats: the text
this package writes from the reference's own numbers is the text the
reference writes (run here when its build is present)."""
import os
import subprocess
import sys

import numpy as np
import pytest

from z4c_testlib import ROOT

from z4c_b200.outputs import HistoryOutput, TrackerOutput

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "athena_ref")


def _run_reference(tmp_path, case_name, nlim, hst_format=None):
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden as M
    case = dict(M.EVOL[case_name])
    text = M.deck(case, "unused", nlim=nlim, hst=hst_format is not None)
    if hst_format is not None:
        text = text.replace("data_format = %.17e", f"data_format = {hst_format}")
    (tmp_path / "case.inp").write_text(text)
    subprocess.run([REF_BIN, "-i", "case.inp"], cwd=tmp_path, check=True,
                   stdout=subprocess.DEVNULL)


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("fmt", ["%.17e", "%12.5e"])
def test_history_file_matches_reference_text(tmp_path, fmt):
    _run_reference(tmp_path, "gw16", 3, hst_format=fmt)
    ref = (tmp_path / "golden.hst").read_text().splitlines()
    rows = [[float(x) for x in line.split()] for line in ref if not line.startswith("#")]
    ours = tmp_path / "ours.hst"
    h = HistoryOutput(str(ours), data_format=fmt)
    for r in rows:
        h.write(r[0], r[1], int(r[2]), r[3:11])
    got = ours.read_text().splitlines()
    assert got[1:] == ref[1:]  # the first line carries the build's own tag
    assert got[0].startswith("# GR-Athena++ (") and got[0].endswith(") history data")


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference build (oracle/_ref) absent")
def test_tracker_file_matches_reference_text(tmp_path):
    _run_reference(tmp_path, "track4", 3)
    ref = (tmp_path / "golden.puncture_0.txt").read_text().splitlines()
    t = TrackerOutput("golden", 0, directory=str(tmp_path / "ours"))
    os.makedirs(tmp_path / "ours")
    for line in ref[1:]:
        v = line.split()
        t.write(int(v[0]), float(v[1]), [float(x) for x in v[2:5]], [float(x) for x in v[5:8]])
    assert (tmp_path / "ours" / "golden.puncture_0.txt").read_text().splitlines() == ref


def test_history_rows_round_trip(tmp_path):
    h = HistoryOutput(str(tmp_path / "a.hst"), data_format="%.17e")
    vals = np.random.default_rng(3).random(8)
    h.write(0.25, 0.125, 512, vals)
    h.write(0.5, 0.125, 512, vals * 2)
    lines = (tmp_path / "a.hst").read_text().splitlines()
    assert len(lines) == 4 and lines[1].startswith("# [1]=time [2]=dt [3]=N_MeshBlock [4]=H-norm2")
    back = np.array([float(x) for x in lines[3].split()])
    assert back[2] == 512 and np.array_equal(back[3:], vals * 2)
