"""An adaptive run on the device against the reference's own adaptive run
of the same deck (fixture amr_bbh_amr.npz): Brill-Lindquist punctures on a
4-level mesh refined by the reference's Linf_box_in_box criterion around the
two puncture trackers, 60 rk4 cycles with one refinement and one
derefinement regrid (z4c_b200.amr.AdaptiveEvolution: the host replays the
reference's tree rules, the device steps, tracks, regrids and finalises).

Checked every cycle: the MeshBlock list (gid order) and dt exactly, the
tracker positions, and the history norms; at the end the final state on four
MeshBlocks and per-variable sums over all of them.  The run starts from the
reference's own initialised state (the reference build, run here for zero
cycles, dumps it), so both sides start from the same bits; the device's own
initial data (the host's Brill-Lindquist data, ADMToZ4c and the ghost
finalisation) are checked against that state first, at the bounds of the
initial-data parity tests (CUDA's and glibc's cube root differ by an ulp, and
the outflow extrapolation amplifies that on the outer planes).

Tolerances.  As in the configuration tests, the device and the reference
differ per step only where CUDA's and glibc's pow round differently, but this
run samples the fields a fraction of a cell from two punctures, where psi is
about 10 and the constraint terms are large differences: fields within a
normwise relative 1e-10, history norms within 1e-6 relative, tracker
positions within 1e-12.  The reference's history row of a cycle that
regridded is NaN: its new MeshBlocks enter ADMConstraints with a zero ADM
interior (FinalizeZ4cADMGhosts converts the ghosts only, skip_physical, and
the Main AMR group carries storage.u alone), so those rows are checked for
the reference's NaN and the device's finite value.
"""
import json
import os
import subprocess

import numpy as np
import pytest

from z4c_testlib import GOLDEN, NG, ROOT, rel_err, var_rel_err

pytestmark = pytest.mark.gpu
FIX = os.path.join(GOLDEN, "amr_bbh_amr.npz")
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "athena_ref")
FIELD_TOL = 1e-10
HST_TOL = 1e-6
TRACK_TOL = 1e-12


def reference_initial_state(tmp_path):
    """The reference's initialised state of the AMR case (gid order): the
    stock driver run for zero cycles, its final dump."""
    import make_golden as G
    from z4cio import read_records
    case = G.AMR["bbh_amr"]
    out = os.path.join(tmp_path, "init.rec")
    inp = os.path.join(tmp_path, "case.inp")
    with open(inp, "w") as f:
        f.write(G.deck(case, "unused", nlim=0, dump_final=out, threads=os.cpu_count() or 1))
    subprocess.run([REF_BIN, "-i", inp], cwd=tmp_path, check=True, stdout=subprocess.DEVNULL)
    rec = read_records(out)
    return rec["u"], rec["meta"]


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference build (oracle/_ref) absent")
def test_adaptive_run_matches_reference(tmp_path):
    import z4c_b200 as Z
    from z4c_b200 import amr as A
    from z4c_b200 import initial_data as ID
    import make_golden as G
    fx = np.load(FIX)
    mesh_d = json.loads(str(fx["mesh"]))
    amr = json.loads(str(fx["amr"]))
    prob = json.loads(str(fx["problem"]))
    ex = json.loads(str(fx["extra"]))
    params = Z.default_params(**json.loads(str(fx["params"])))
    start = [tuple(ex[f"bh_{n}_{c}"] for c in "xyz") for n in range(ex["npunct"])]
    masses = [prob[f"bl_m_{n}"] for n in range(ex["npunct"])]
    shift = (prob.get("shift_x", 0.0), prob.get("shift_y", 0.0), prob.get("shift_z", 0.0))
    ref = A.Refinement(mesh_d["nb"], mesh_d["nx"], mesh_d["xmin"], mesh_d["xmax"],
                       mesh_d["bc"], amr["numlevel"], amr["derefine_count"], prob["par_b"])

    integ = json.loads(str(fx["integrator"]))
    blocks, cycles, trk, hst = fx["blocks"], fx["cycles"], fx["trackers"], fx["hst"]
    s = int(fx["stride"])

    def ref_list(c):
        rows = blocks[blocks[:, 0] == c]
        return rows[:, 2:6].astype(np.int64)

    u_ref, meta = reference_initial_state(str(tmp_path))
    assert np.array_equal(meta, fx["init_meta"])
    assert np.array_equal(G.state_sums(u_ref), fx["u_init_sums"])

    # the device's own initial data on the mesh its initial loop builds
    def initial(mesh):
        return ID.punctures(mesh, params, masses=masses, centres=start, shift=shift)

    own = A.AdaptiveEvolution(A.Refinement(
        mesh_d["nb"], mesh_d["nx"], mesh_d["xmin"], mesh_d["xmax"], mesh_d["bc"],
        amr["numlevel"], amr["derefine_count"], prob["par_b"]), params, integ, initial, start)
    assert np.array_equal(own.mesh.locs, ref_list(0))
    u0 = own.ctx.download(Z.REG_U)
    own.close()
    nn = u0.shape[2]
    I = (slice(None), slice(None), slice(NG, nn - NG - 1), slice(NG, nn - NG - 1),
         slice(NG, nn - NG - 1))
    e_int, e_all = rel_err(u0[I], u_ref[I]), rel_err(u0, u_ref)
    print(f"initial data: interior {e_int:.2e}, whole register {e_all:.2e}")
    assert e_int <= 1e-14 and e_all <= 1e-7
    del u0

    # the run, from the reference's initial state
    run = A.AdaptiveEvolution(ref, params, integ, lambda ctx: ctx.upload(Z.REG_U, u_ref),
                              start, load=True)
    assert np.array_equal(run.mesh.locs, ref_list(0))
    del u_ref

    def hst_row(t):
        rows = np.flatnonzero(np.isclose(hst[:, 0], t, rtol=0, atol=1e-9))
        assert rows.size, t
        return hst[rows[0]]

    got0 = run.ctx.hst_norms()
    row = hst_row(0.0)
    assert np.max(np.abs(got0 - row[3:11]) / np.maximum(np.abs(row[3:11]), 1e-300)) <= HST_TOL
    worst_h, worst_t, regrids = 0.0, 0.0, []
    nlim = int(fx["nlim"])
    for c in range(nlim):
        assert run.dt == cycles[c, 2], c
        pos = np.array(run.trackers())
        worst_t = max(worst_t, float(np.abs(pos - trk[c]).max()))
        if run.step():
            regrids.append(c + 1)
        assert np.array_equal(run.mesh.locs, ref_list(c + 1)), f"cycle {c + 1}"
        row = hst_row(cycles[c + 1, 1])
        assert int(row[2]) == run.mesh.nblocks
        got = run.ctx.hst_norms()
        if c + 1 in regrids:
            assert np.isnan(row[3]) and np.all(np.isfinite(got)), c + 1
            continue
        d = np.max(np.abs(got - row[3:11]) / np.maximum(np.abs(row[3:11]), 1e-300))
        worst_h = max(worst_h, float(d))
    pos = np.array(run.trackers())
    worst_t = max(worst_t, float(np.abs(pos - trk[nlim]).max()))
    print(f"regrids at cycles {regrids}, worst history {worst_h:.2e}, tracker {worst_t:.2e}")
    assert len(regrids) == 2
    assert worst_t <= TRACK_TOL
    assert worst_h <= HST_TOL

    u = run.ctx.download(Z.REG_U)
    run.close()
    sample = u[fx["final_sample_blocks"]][:, :, ::s, ::s, ::s]
    e_reg = rel_err(sample, fx["u_final_sample"])
    e_var = var_rel_err(sample, fx["u_final_sample"])
    print(f"final state sample normwise {e_reg:.2e}, worst variable {e_var:.2e}")
    assert e_reg <= FIELD_TOL and e_var <= 100 * FIELD_TOL
    sums, ref_sums = G.state_sums(u), fx["u_final_sums"]
    scale = np.abs(ref_sums[:, 2]).max()
    assert np.all(np.abs(sums[:, 2] - ref_sums[:, 2]) <= FIELD_TOL * scale)
