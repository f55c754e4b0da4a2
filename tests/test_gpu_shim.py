"""The reference-side shim (oracle/ref/z4c_b200_shim.hpp) inside the
reference's own operator driver: built with -DZ4C_SHIM, the driver calls
Z4cRHS, AlgConstr and Z4cToADM through the adapter and the B200 library,
while everything else (mesh set-up, initial data, ghost exchange, boundary
conditions, stage algebra, constraints) stays the reference's code.  Its
records must reproduce the reference's own (the ops_* fixtures) to the RHS
parity bound, normwise relative 1e-12 per register."""
import os
import subprocess

import pytest

from z4c_testlib import ROOT, Case, rel_err

pytestmark = pytest.mark.gpu
SHIM_BIN = os.path.join(ROOT, "oracle", "_ref", "z4c_ops_shim")
TOL = 1e-12
RECORDS = ["rhs0", "alg0", "adm0", "con0", "s1_rhs", "s1_alg", "s2_alg", "s3_alg", "s4_alg",
           "s4_adm", "s4_con"]


@pytest.mark.skipif(not os.path.exists(SHIM_BIN), reason="shim driver (oracle/_ref) absent")
@pytest.mark.parametrize("name", ["gw1", "punc2", "rs2", "somm2"])
def test_reference_driver_with_the_shim_reproduces_the_reference(name, tmp_path):
    import make_golden as G
    from z4cio import read_records
    rec_path = os.path.join(tmp_path, "shim.rec")
    inp = os.path.join(tmp_path, "case.inp")
    with open(inp, "w") as f:
        f.write(G.deck(G.CASES[name], rec_path))
    subprocess.run([SHIM_BIN, "-i", inp], cwd=tmp_path, check=True, stdout=subprocess.DEVNULL)
    got = read_records(rec_path)
    ref = Case(f"ops_{name}").rec
    assert (got["u0"] == ref["u0"]).all(), "same initial state"
    for r in RECORDS:
        if r not in ref:
            continue
        e = rel_err(got[r], ref[r])
        print(f"{name} {r}: {e:.2e}")
        assert e <= TOL, r
