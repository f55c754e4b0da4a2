"""The FP64 operation count behind the roofline figure of bench.py: the
reference algorithm's operations per interior vertex per stage, counted by
running the oracle (which follows the reference operation by operation) with
a counting number type."""
import json
import os
import subprocess

from z4c_testlib import ROOT


def test_fp64_operation_count_matches_bench_constant():
    exe = os.path.join(ROOT, "oracle", "_build", "count_ops")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    out = json.loads(subprocess.run([exe, "16"], capture_output=True, text=True,
                                    check=True).stdout)
    assert out["interior_vertices"] == 17 ** 3
    import bench
    assert round(out["rhs"]["total"]) + out["stage"]["total"] == bench.FP64_OPS_PER_POINT_STAGE
    # nearly all of it is separately rounded adds and multiplies: the FP64
    # pipe sees one instruction per operation
    assert out["rhs"]["div"] < 3 and out["rhs"]["fn"] < 10
    # PrepareZ4cDerivatives + Z4cWeyl, the psi4 diagnostics figure
    assert round(out["weyl"]["total"]) == bench.FP64_OPS_PER_POINT_WEYL
