"""The contracted path (z4c_set_contract: fused multiply-adds; advection,
Kreiss-Oliger and the stage update in one per-variable column pass after the
main pass) against the reference's own outputs.  Its right-hand side is not the
reference's bit for bit, so every check is a bound:

  right-hand side      normwise relative 1e-12 per register (the FP64
                       agreement bound per RHS evaluation) on the operator
                       fixtures, relative to the larger of the right-hand
                       side and the scale of the terms it is made of (the
                       state times the second-derivative stencil's weight
                       sum, 1088 / (180 dx^2)); the gr_sommerfeld case keeps
                       the exact path and stays bit for bit.  Where the
                       right-hand side is far below its terms, as on the
                       robust-stability state (Minkowski plus 1e-10 noise: a
                       stencil on g ~ 1 sums terms of 100 to 1e-8), the
                       reference's own rounding of those terms is what
                       contraction changes, so the difference is measured
                       against them; on the other states it is also within
                       1e-12 of the right-hand side itself.  (Per variable
                       the difference can reach 1e-10 of that variable's
                       own size for the same reason.)
  one RK4 step         every stage's state within 1e-12 of the reference's
                       on the interior (ghosts: see GHOST_TOL)
  evolution            the history norms of the 12-step puncture run within
                       1e-9 relative, as for the exact path; its final state
                       within 1e-10 on the interior
"""
import numpy as np
import pytest

from z4c_testlib import Case, rel_err, var_rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-12
# whole register, ghosts included: on outflow faces the fifth-order
# extrapolation (u_g = 5u_1 - 10u_2 + 10u_3 - 5u_4 + u_5, axis after axis)
# multiplies the interior's round-off differences by up to ~10^3 per axis
GHOST_TOL = 1e-8
OPS = ["ops_gw1", "ops_punc2", "ops_rs2", "ops_somm2"]


def make_ctx(c):
    import z4c_b200 as Z
    m = c.mesh
    mesh = Z.Mesh(m["nb"], m["nx"], m["xmin"], m["xmax"], m["bc"])
    ctx = Z.Z4c(mesh, Z.default_params(**c.params), c.integrator)
    ctx.set_contract(True)
    assert ctx.get_contract()
    return Z, ctx


@pytest.mark.parametrize("name", OPS)
def test_contracted_rhs_within_bound(name):
    c = Case(name)
    Z, ctx = make_ctx(c)
    I = c.interior()
    ctx.upload(Z.REG_U, c.to_grid(c.rec["u0"]))
    ctx.Z4cRHS(Z.REG_U, Z.REG_RHS)
    rhs = c.from_grid(ctx.download(Z.REG_RHS))
    ref = c.rec["rhs0"]
    scale = np.abs(c.rec["u0"]).max() * 1088.0 / (180.0 * float(np.min(c.rec["dx"])) ** 2)
    e = float(np.abs(rhs[I] - ref[I]).max()) / max(float(np.abs(ref[I]).max()), scale)
    print(f"{name}: normwise {rel_err(rhs[I], ref[I]):.2e} of the right-hand side, {e:.2e} "
          f"of the term scale, worst variable {var_rel_err(rhs[I], ref[I]):.2e}")
    assert e <= TOL
    if "rs" not in name:  # right-hand sides of the size of their terms
        assert rel_err(rhs[I], ref[I]) <= TOL
    if "somm" in name:  # exact path kept on gr_sommerfeld meshes
        Zx, ex = make_ctx(c)
        ex.set_contract(False)
        ex.upload(Z.REG_U, c.to_grid(c.rec["u0"]))
        ex.Z4cRHS(Z.REG_U, Z.REG_RHS)
        assert np.array_equal(ex.download(Z.REG_RHS), ctx.download(Z.REG_RHS))
        ex.close()
    ctx.close()


@pytest.mark.parametrize("name", OPS)
def test_contracted_step_within_bound(name):
    c = Case(name)
    Z, ctx = make_ctx(c)
    dt = c.rec["time_dt"][1]
    I = c.interior()
    ctx.upload(Z.REG_U, c.to_grid(c.rec["u0"]))
    for s in range(1, 5):
        ctx.stage(s, dt)
        u = c.from_grid(ctx.download(Z.REG_U))
        ref = c.rec[f"s{s}_alg"]
        assert rel_err(u[I], ref[I]) <= TOL, f"stage {s}"
        assert rel_err(u, ref) <= GHOST_TOL, f"stage {s}"
    # the captured step takes the same path
    ctx.upload(Z.REG_U, c.to_grid(c.rec["u0"]))
    ctx.evolve(dt, 1)
    u = c.from_grid(ctx.download(Z.REG_U))
    assert rel_err(u[I], c.rec["s4_alg"][I]) <= TOL
    ctx.close()


def test_contracted_evolution_history():
    c = Case("evol_punc4")
    Z, ctx = make_ctx(c)
    dt = c.rec["time_dt"][1]
    nlim = int(c.rec["nlim"])
    ctx.upload(Z.REG_U, c.to_grid(c.rec["u_init"]))
    ctx.evolve(dt, nlim, with_constraints=True)
    hst = ctx.hst_norms()
    np.testing.assert_allclose(hst, c.rec["hst"][nlim, 3:11], rtol=1e-9, atol=1e-30)
    u = c.from_grid(ctx.download(Z.REG_U))
    # after 12 steps the extrapolated outer vertex planes have fed their
    # amplified round-off back into the interior: 1e-10
    I = c.interior()
    assert rel_err(u[I], c.rec["u_final"][I]) <= 1e-10
    assert rel_err(u, c.rec["u_final"]) <= GHOST_TOL
    ctx.close()


def test_contract_switch_keeps_exact_path_exact():
    """Switching the contracted path off again restores the exact path's
    bits (the flag only selects the launch sequence)."""
    c = Case("ops_punc2")
    Z, ctx = make_ctx(c)
    u0 = c.to_grid(c.rec["u0"])
    ctx.upload(Z.REG_U, u0)
    ctx.Z4cRHS(Z.REG_U, Z.REG_RHS)
    fast = ctx.download(Z.REG_RHS)
    ctx.set_contract(False)
    ctx.Z4cRHS(Z.REG_U, Z.REG_RHS)
    exact = ctx.download(Z.REG_RHS)
    ctx.close()
    m = c.mesh
    fresh = Z.Z4c(Z.Mesh(m["nb"], m["nx"], m["xmin"], m["xmax"], m["bc"]),
                  Z.default_params(**c.params), c.integrator)
    fresh.upload(Z.REG_U, u0)
    fresh.Z4cRHS(Z.REG_U, Z.REG_RHS)
    assert np.array_equal(exact, fresh.download(Z.REG_RHS))
    assert not np.array_equal(fast, exact)  # the contracted path did run
    fresh.close()


@pytest.mark.parametrize("contract", [False, True])
@pytest.mark.parametrize("threads", [64, 128])
def test_register_budget_changes_no_bits(contract, threads):
    """The 168-register instances of the heavy passes compute the same
    values as the 255-register ones (register allocation only), on 16^3
    MeshBlocks where they apply."""
    import z4c_b200 as Z
    from z4c_b200 import initial_data as ID
    mesh = Z.Mesh((2, 2, 2), (16, 16, 16), (-4.0,) * 3, (4.0,) * 3, "outflow")
    params = Z.default_params(diss=0.02, chi_div_floor=1e-5, damp_kappa1=0.02, shift_eta=2.0,
                              r_max_con=1e300)
    ctx = Z.Z4c(mesh, params, "rk4")
    ctx.set_contract(contract)
    ID.load_adm(ctx, ID.punctures(mesh, params, masses=(1.0,), centres=((0.1, 0.05, 0.02),)))
    ctx.evolve(0.05, 2)  # a state with nonzero shift and curvature
    out = []
    for regs in (0, 168):
        ctx.set_tile(threads, 128, 0)
        ctx.set_point_regs(regs)
        assert ctx.get_point_regs() == regs
        ctx.Z4cRHS(Z.REG_U, Z.REG_RHS)
        out.append(ctx.download(Z.REG_RHS))
    ctx.close()
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("nb,lim,steps", [
    ((2, 2, 2), (4.0, 4.0, 4.0), (6, 4)),
    ((3, 2, 2), (6.0, 4.0, 4.0), (3, 3)),  # a merged grid of 48 x 32 x 32 cells
    # the benchmark's mesh: 512 blocks of 16^3, whose merged 128^3 grid runs
    # the compile-time-geometry instances of the passes
    ((8, 8, 8), (16.0, 16.0, 16.0), (2, 2))])
def test_merged_grid_evolution_matches_blocks(nb, lim, steps):
    """On a uniform outflow mesh the contracted path's z4c_evolve runs on one
    vertex grid holding every block; against the block-by-block evolution
    (set_merged(False)) the state, the ADM and constraint registers, the
    history norms and the tracker agree to round-off.  The blocks' shared
    vertices hold one value in the merged grid where the block evolution
    averages its owners' copies; those differences are ~1 ulp and grow at the
    outflow faces like every round-off difference here (3e-12 of the interior
    after these 10 steps)."""
    import z4c_b200 as Z
    from z4c_b200 import initial_data as ID
    mesh = Z.Mesh(nb, (16, 16, 16), tuple(-v for v in lim), lim, "outflow")
    params = Z.default_params(diss=0.02, chi_div_floor=1e-5, damp_kappa1=0.02, shift_eta=2.0,
                              r_max_con=1e300)
    adm = ID.punctures(mesh, params, masses=(1.0,), centres=((0.3, 0.15, -0.1),))
    runs = []
    for merged in (True, False):
        ctx = Z.Z4c(mesh, params, "rk4")
        ctx.set_contract(True)
        ctx.set_merged(merged)
        assert ctx.get_merged() == merged
        ID.load_adm(ctx, adm)
        ctx.add_tracker((0.3, 0.15, -0.1))
        dt = 0.25 * float(np.min(ctx.dx()))
        ctx.evolve(dt, steps[0])
        ctx.evolve(dt, steps[1], with_constraints=True)
        runs.append(dict(u=ctx.download(Z.REG_U), adm=ctx.download(Z.REG_ADM),
                         con=ctx.download(Z.REG_CON), hst=ctx.hst_norms(),
                         trk=np.array(ctx.tracker(0)[0])))
        ctx.close()
    m, b = runs
    I = (slice(None), slice(None), slice(4, 21), slice(4, 21), slice(4, 21))
    # the interior bound of the 12-step evolution test above: round-off
    # amplified at the outflow faces feeds back into the interior
    assert rel_err(m["u"][I], b["u"][I]) <= 1e-10
    # ghosts: the corner ghosts take three extrapolation cascades (x, y, z)
    # of the interior's differences, up to ~1e4 times (3e-8 here)
    assert rel_err(m["u"], b["u"]) <= 1e-6
    assert rel_err(m["adm"][I], b["adm"][I]) <= 1e-10
    assert rel_err(m["con"][I], b["con"][I]) <= 1e-8  # constraints: differences of O(1) terms
    np.testing.assert_allclose(m["hst"], b["hst"], rtol=1e-9, atol=1e-30)
    np.testing.assert_allclose(m["trk"], b["trk"], rtol=0, atol=1e-13)


def test_merged_grid_on_a_periodic_mesh():
    """Periodic meshes merge too: the merged grid is one block exchanging
    with itself.  Gauge wave on 2^3 blocks of 16^3, against the blocks."""
    import z4c_b200 as Z
    from z4c_b200 import initial_data as ID
    mesh = Z.Mesh((2, 2, 2), (16, 16, 16), (-0.5,) * 3, (0.5,) * 3, "periodic")
    params = Z.default_params(lapse_harmonic=1.0, lapse_harmonicf=0.0, lapse_oplog=0.0,
                              lapse_advect=0.0, shift_Gamma=0.0, shift_eta=0.0, shift_advect=0.0,
                              diss=0.02, damp_kappa1=0.02, r_max_con=1e300, eps_floor=-1.0)
    adm = ID.gauge_wave1(mesh, amplitude=0.05)
    out = []
    for merged in (True, False):
        ctx = Z.Z4c(mesh, params, "rk4")
        ctx.set_contract(True)
        ctx.set_merged(merged)
        assert ctx.get_merged() == merged
        ID.load_adm(ctx, adm)
        dt = 0.25 * float(np.min(ctx.dx()))
        ctx.evolve(dt, 8, with_constraints=True)
        out.append((ctx.download(Z.REG_U), ctx.hst_norms()))
        ctx.close()
    assert rel_err(out[0][0], out[1][0]) <= 1e-12
    # the gauge wave satisfies the constraints: its norms (1e-14 and below)
    # are sums of round-off, so they agree to round-off of round-off
    np.testing.assert_allclose(out[0][1], out[1][1], rtol=1e-5, atol=1e-22)


def test_merged_grid_only_where_it_applies():
    """Mixed face kinds, the exact path and the per-block loop keep the blocks."""
    import z4c_b200 as Z
    params = Z.default_params(diss=0.02)
    mix = Z.Z4c(Z.Mesh((2, 2, 2), (8, 8, 8), (-1.0,) * 3, (1.0,) * 3,
                       bc=[0, 0, 1, 1, 1, 1]), params, "rk4")
    mix.set_contract(True)
    assert not mix.get_merged()
    mix.close()
    ctx = Z.Z4c(Z.Mesh((2, 2, 2), (8, 8, 8), (-1.0,) * 3, (1.0,) * 3, "outflow"), params, "rk4")
    assert not ctx.get_merged()  # exact path
    ctx.set_contract(True)
    assert ctx.get_merged()
    ctx.set_per_block(True)
    assert not ctx.get_merged()
    ctx.close()
