"""The benchmark configurations at their stated sizes and lengths, on the
device, against the reference's own runs of them (fixtures scale_*.npz made by
tests/golden/make_golden.py with the reference build):

  scale_gw48     the gauge-wave benchmark as written: 48^3 cells in one
                 periodic MeshBlock, harmonic-like lapse, zero shift,
                 A = 0.01, KO 0.02, kappa1 0.02, 1000 rk4 steps
  scale_punc512  the single-puncture benchmark: 128^3 cells as 512
                 MeshBlocks of 16^3, outflow faces, 40 rk4 steps
  scale_rs512    the robust-stability benchmark: Minkowski plus
                 U(-1e-10, 1e-10) on all 22 variables, periodic, 40 steps

The reference's state is too large to store (1.4 GB per register on the
512-block mesh), so each fixture keeps the history norms of every step,
per-variable sums of the final state, and the final state at every other
vertex of six MeshBlocks (every fourth of the 48^3 block).  The initial state
is the reference's own: the reference build (oracle/_ref) runs the same deck
for zero steps on this machine and dumps it, so both sides start from the
same bits.

Tolerances, stated per quantity.  The device evaluates every expression in
the reference's order without contraction, so a step differs from the
reference's only where CUDA's and glibc's pow/cbrt round differently by an
ulp (AlgConstr's pow(det, -1/3) and the lapse's pow): the fields stay within
a normwise relative 1e-11 of the reference's after 1000 steps.  The history
norms are sums of squared constraints, which are differences of nearly equal
second-derivative terms (on the robust-stability state a norm of 1e-12 is
built from terms of order 1e-8), so the same ulp differences move them by up
to 1e-6 relative; that is the bound on them.
"""
import json
import os
import subprocess

import numpy as np
import pytest

from z4c_testlib import GOLDEN, NG, ROOT, rel_err, var_rel_err

pytestmark = pytest.mark.gpu
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "athena_ref")
needs_ref = pytest.mark.skipif(not os.path.exists(REF_BIN),
                               reason="reference build (oracle/_ref) absent")
FIELD_TOL = 1e-11  # normwise relative, whole register
VAR_TOL = 1e-9     # worst variable, measured against 1e-10 of the largest
HST_TOL = 1e-6     # history norms, relative


def reference_initial_state(name, tmp_path):
    """The reference's initialised state of a SCALE case (gid order): the
    stock driver run for zero steps, its final dump."""
    import make_golden as G
    from z4cio import read_records, write_records
    case = G.SCALE[name]
    out = os.path.join(tmp_path, "init.rec")
    text = G.deck(case, "unused", nlim=0, dump_final=out, threads=os.cpu_count() or 1)
    if case["test"] == "inject":
        inj = os.path.join(tmp_path, "inject.rec")
        write_records(inj, {"u": G.noise_state_gid(case)})
        text = text.replace("<driver>", f"inject_file = {inj}\n<driver>")
    inp = os.path.join(tmp_path, "case.inp")
    with open(inp, "w") as f:
        f.write(text)
    subprocess.run([REF_BIN, "-i", inp], cwd=tmp_path, check=True, stdout=subprocess.DEVNULL)
    rec = read_records(out)
    os.remove(out)
    return rec["u"], rec["meta"]


@needs_ref
@pytest.mark.parametrize("name", ["gw48", "punc512", "rs512"])
def test_config_against_reference_run(name, tmp_path):
    import z4c_b200 as Z
    import make_golden as G
    fx = np.load(os.path.join(GOLDEN, f"scale_{name}.npz"))
    mesh_d = json.loads(str(fx["mesh"]))
    params = json.loads(str(fx["params"]))
    integ = json.loads(str(fx["integrator"]))
    nlim = int(fx["nlim"])
    dt = float(fx["time_dt"][1])
    u_gid, meta = reference_initial_state(name, str(tmp_path))
    assert np.array_equal(meta, fx["meta"])
    # the initial state is the one the fixture's run started from
    assert np.array_equal(G.state_sums(u_gid), fx["u_init_sums"])
    nb = mesh_d["nb"]
    order = [int(m[2] + nb[0] * (m[3] + nb[1] * m[4])) for m in meta]
    u_grid = np.empty_like(u_gid)
    u_grid[order] = u_gid
    del u_gid

    mesh = Z.Mesh(nb, mesh_d["nx"], mesh_d["xmin"], mesh_d["xmax"], mesh_d["bc"])
    ctx = Z.Z4c(mesh, Z.default_params(**params), integ)
    ctx.upload(Z.REG_U, u_grid)
    del u_grid
    hst_ref = fx["hst"]
    times = hst_ref[:, 0]
    worst_hst = 0.0
    for n in range(1, nlim + 1):
        ctx.evolve(dt, 1, with_constraints=True)
        row = np.flatnonzero(np.isclose(times, n * dt, rtol=0, atol=1e-9 * dt))
        assert row.size, f"no history row at step {n}"
        ref = hst_ref[row[0], 3:11]
        got = ctx.hst_norms()
        d = np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300))
        worst_hst = max(worst_hst, float(d))
    u = ctx.download(Z.REG_U)
    con = ctx.download(Z.REG_CON)
    ctx.close()
    print(f"{name}: worst history norm difference {worst_hst:.2e}")
    assert worst_hst <= HST_TOL, worst_hst

    # final state: the sampled MeshBlocks at every stride-th vertex
    s = int(fx["stride"])
    sample = u[fx["sample_blocks"]][:, :, ::s, ::s, ::s]
    ref = fx["u_final_sample"]
    e_reg, e_var = rel_err(sample, ref), var_rel_err(sample, ref)
    print(f"{name}: final state sample normwise {e_reg:.2e}, worst variable {e_var:.2e}")
    assert e_reg <= FIELD_TOL
    assert e_var <= VAR_TOL
    # and per-variable sums over every interior vertex of every block
    sums = G.state_sums(u)
    ref_sums = fx["u_final_sums"]
    scale = np.abs(ref_sums[:, 2]).max()
    assert np.all(np.abs(sums[:, 2] - ref_sums[:, 2]) <= FIELD_TOL * scale)  # max |u|
    npts = mesh.nblocks * np.prod([n + 1 for n in mesh.nx])
    assert np.all(np.abs(sums[:, 0] - ref_sums[:, 0]) <= FIELD_TOL * scale * npts)
    csum = G.state_sums(con)
    np.testing.assert_allclose(csum[:, 1], fx["con_final_sums"][:, 1], rtol=HST_TOL, atol=0)
