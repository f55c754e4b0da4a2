"""Full-size checks on the benchmark mesh (512 MeshBlocks of 16^3): the
batched launch against the per-block launch loop and against the CPU oracle
on sampled blocks, graph replay against stage-by-stage stepping, and
size-independent properties (periodic translation symmetry, convergence
order of the gauge wave)."""
import numpy as np
import pytest

import z4c_oracle as O
from z4c_testlib import rel_err

pytestmark = pytest.mark.gpu
PUNC = dict(diss=0.02, chi_div_floor=1e-5, damp_kappa1=0.02, damp_kappa2=0.0, shift_eta=2.0,
            r_max_con=1e300)


def mesh_ctx(bc, nb=(8, 8, 8), nx=(16, 16, 16), lim=16.0, integ="rk4", **kw):
    import z4c_b200 as Z
    mesh = Z.Mesh(nb, nx, (-lim,) * 3, (lim,) * 3, bc)
    p = Z.default_params(**{**PUNC, **kw})
    return Z, Z.Z4c(mesh, p, integ)


def puncture_state(Z, ctx):
    from z4c_b200 import initial_data as ID
    adm = ID.punctures(ctx.mesh, ctx.params, masses=(0.5, 0.5),
                       centres=((1.5, 0.3, 0.1), (-1.5, -0.2, 0.0)))
    ID.load_adm(ctx, adm)
    return ctx.download(Z.REG_U)


def test_batched_equals_per_block_and_oracle_on_full_mesh():
    Z, ctx = mesh_ctx("outflow")
    u = puncture_state(Z, ctx)
    ctx.Z4cRHS(Z.REG_U, Z.REG_RHS, -1)
    batched = ctx.download(Z.REG_RHS)
    ctx.upload(Z.REG_RHS, np.zeros_like(batched))
    for b in range(ctx.nblocks):
        ctx.Z4cRHS(Z.REG_U, Z.REG_RHS, b)
    per_block = ctx.download(Z.REG_RHS)
    assert np.array_equal(batched, per_block)
    p = O.default_params(**PUNC)
    I = (slice(None), slice(4, 21), slice(4, 21), slice(4, 21))
    for b in (0, 73, 219, 292, 511):  # corners, faces and the punctures' blocks
        xs, dxs = ctx.mesh.block_coords(b)
        ref = O.rhs(O.Block(ctx.mesh.nx, dxs, xs), p, u[b])
        assert rel_err(batched[b][I], ref[I]) <= 1e-12, b
    ctx.close()


def test_graph_steps_equal_stage_calls_and_per_block_path():
    Z, ctx = mesh_ctx("outflow")
    u0 = puncture_state(Z, ctx)
    dx = ctx.dx()
    dt = 0.25 * float(dx.min())
    for s in range(1, 5):
        ctx.stage(s, dt)
    for s in range(1, 5):
        ctx.stage(s, dt)
    by_stage = ctx.download(Z.REG_U)
    ctx.upload(Z.REG_U, u0)
    ctx.evolve(dt, 2)
    assert np.array_equal(ctx.download(Z.REG_U), by_stage)
    ctx.upload(Z.REG_U, u0)
    ctx.set_per_block(True)
    ctx.evolve(dt, 2)
    assert np.array_equal(ctx.download(Z.REG_U), by_stage)
    assert ctx.check_finite()
    ctx.close()


def test_noise_state_periodic_translation_symmetry():
    """Shifting a periodic state by whole blocks permutes the blocks of the
    result exactly: the exchange and the RHS do not depend on where a block
    sits."""
    from z4c_b200 import initial_data as ID
    Z, ctx = mesh_ctx("periodic", nb=(4, 4, 4))
    u = ID.noise_state(ctx.mesh, amplitude=1e-10, seed=5)
    ID.load_z4c(ctx, u)
    dt = 0.25 * float(ctx.dx().min())
    u0 = ctx.download(Z.REG_U)
    ctx.evolve(dt, 1)
    a = ctx.download(Z.REG_U).reshape(4, 4, 4, *u0.shape[1:])
    shifted = u0.reshape(4, 4, 4, *u0.shape[1:])
    shifted = np.roll(shifted, 1, axis=2).reshape(u0.shape)
    ctx.upload(Z.REG_U, shifted)
    ctx.evolve(dt, 1)
    b = ctx.download(Z.REG_U).reshape(4, 4, 4, *u0.shape[1:])
    assert np.array_equal(np.roll(a, 1, axis=2), b)
    ctx.close()


def test_gauge_wave_convergence_order():
    """The benchmark gauge wave converges at the scheme's order: the error of
    the physical g_xx against the exact wave 1 - A sin(2 pi (x - t))."""
    import z4c_b200 as Z
    from z4c_b200 import initial_data as ID
    errs = []
    for nx in (16, 32):
        mesh = Z.Mesh((1, 1, 1), (nx,) * 3, (-0.5,) * 3, (0.5,) * 3, "periodic")
        p = Z.default_params(lapse_harmonic=1.0, lapse_harmonicf=0.0, lapse_oplog=0.0,
                             lapse_advect=0.0, shift_Gamma=0.0, shift_eta=0.0,
                             shift_advect=0.0, diss=0.0, damp_kappa1=0.02, r_max_con=1e300)
        ctx = Z.Z4c(mesh, p, "rk4")
        ID.load_adm(ctx, ID.gauge_wave1(mesh, amplitude=0.01))
        dt = 0.25 / nx
        nsteps = nx * 2  # t = 0.5
        ctx.evolve(dt, nsteps, with_constraints=True)
        adm = ctx.download(Z.REG_ADM)[0]
        x = ctx.coords(0)[0]
        t = dt * nsteps
        exact = 1 - 0.01 * np.sin(2 * np.pi * (x - t))
        g = adm[Z.ADM_GXX, 4:-4, 4:-4, 4:-4]
        errs.append(np.sqrt(np.mean((g - exact[None, None, 4:-4]) ** 2)))
        ctx.close()
    order = np.log2(errs[0] / errs[1])
    assert order > 3.5, (errs, order)


def test_launch_shapes_and_autotuner_leave_results_unchanged():
    """Every launch shape the autotuner can pick gives the same bits; the
    autotuner leaves u untouched and picks a supported shape."""
    Z, ctx = mesh_ctx("outflow", nb=(4, 4, 4))
    u0 = puncture_state(Z, ctx)
    dt = 0.25 * float(ctx.dx().min())
    ref = None
    for shape in [(128, 256, 2), (64, 128, 0), (256, 512, 1), (128, 512, 3), (128, 128, 4)]:
        ctx.set_tile(*shape)
        assert ctx.get_tile() == shape
        ctx.upload(Z.REG_U, u0)
        ctx.evolve(dt, 1)
        out = ctx.download(Z.REG_U)
        if ref is None:
            ref = out
        assert np.array_equal(out, ref), shape
    ctx.upload(Z.REG_U, u0)
    shape, ms = ctx.autotune(reps=2)
    assert shape[0] in (64, 128, 256) and shape[1] in (128, 256, 512) and 0 <= shape[2] <= 4
    assert ms > 0
    assert np.array_equal(ctx.download(Z.REG_U), u0)
    ctx.evolve(dt, 1)
    assert np.array_equal(ctx.download(Z.REG_U), ref)
    with pytest.raises(Z.Z4cError):
        ctx.set_tile(100, 256, 2)
    ctx.close()
