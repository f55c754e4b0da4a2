"""z4c_evolve_jobs: independent states evolved from host memory, with the
copies of one job overlapping the evolution of the next.

Every job must give what the sequential calls give (upload, z4c_evolve with
the constraints, z4c_hst_norms, download) bit for bit: the pipeline changes
where the copies run, not the arithmetic.  Five jobs exercise the reuse of
the two staging slots; page-locked and pageable host buffers both run, and
so does a call that downloads the norms only.
"""
import ctypes as C

import numpy as np
import pytest

import z4c_b200 as Z


def test_rejects_bad_arguments_without_a_context():
    """Argument checks come before any device work (no GPU needed)."""
    arr = (C.c_void_p * 1)(0x1000)
    h = np.empty(8)
    rc = Z.lib().z4c_evolve_jobs(None, 1, arr, arr, h.ctypes.data_as(C.POINTER(C.c_double)),
                                 0.1, 1)
    assert rc != 0 and b"null context" in Z.lib().z4c_last_error()


def _states(mesh, params, ctx, ID):
    out = []
    for m, x in ((1.0, 0.0), (0.8, 0.3), (0.6, -0.45), (1.1, 0.15), (0.9, -0.2)):
        ID.load_adm(ctx, ID.punctures(mesh, params, masses=(m,), centres=((x, 0.1, -0.05),)))
        out.append(ctx.download(Z.REG_U))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("pinned", [True, False])
def test_jobs_match_sequential_calls(pinned):
    import torch
    from z4c_b200 import initial_data as ID
    params = Z.default_params(diss=0.02, chi_div_floor=1e-5, damp_kappa1=0.02, shift_eta=2.0,
                              r_max_con=1e300)
    mesh = Z.Mesh((2, 2, 2), (16, 16, 16), (-4.0,) * 3, (4.0,) * 3, "outflow")
    ctx = Z.Z4c(mesh, params, "rk4")
    ctx.set_contract(True)
    dt = 0.25 * float(np.min(ctx.dx()))
    states = _states(mesh, params, ctx, ID)
    nsteps = 3

    expect, expect_hst = [], []
    for s in states:
        ctx.upload(Z.REG_U, s)
        ctx.evolve(dt, nsteps, with_constraints=True)
        expect_hst.append(ctx.hst_norms())
        expect.append(ctx.download(Z.REG_U))

    def buf(a=None):
        t = torch.empty(a.shape if a is not None else states[0].shape, dtype=torch.float64)
        if pinned:
            t = t.pin_memory()
        n = t.numpy()
        if a is not None:
            n[...] = a
        return n

    inputs = [buf(s) for s in states]
    outputs = [buf() for _ in states]
    for o in outputs:
        o.fill(np.nan)
    for calls in range(2):  # a second call reuses the staging of the first
        hst = ctx.evolve_jobs(inputs, outputs, dt, nsteps)
        for j in range(len(states)):
            assert np.array_equal(outputs[j], expect[j]), f"job {j}, call {calls}"
            assert np.array_equal(hst[j], expect_hst[j]), f"job {j}, call {calls}"
    # u holds the last job's state
    assert np.array_equal(ctx.download(Z.REG_U), expect[-1])
    # a single job
    hst = ctx.evolve_jobs(inputs[1:2], outputs[:1], dt, nsteps)
    assert np.array_equal(outputs[0], expect[1]) and np.array_equal(hst[0], expect_hst[1])
    # the norms only
    hst = ctx.evolve_jobs(inputs, None, dt, nsteps)
    for j in range(len(states)):
        assert np.array_equal(hst[j], expect_hst[j]), f"job {j}, norms only"
    ctx.close()


@pytest.mark.gpu
def test_norms_only_jobs_on_three_block_layers():
    """With the norms only and three or more block layers in z, the library
    uploads only the vertex planes the merged grid reads of the blocks off
    the z faces; the norms are still those of the separate calls, bit for
    bit."""
    import torch
    from z4c_b200 import initial_data as ID
    params = Z.default_params(diss=0.02, chi_div_floor=1e-5, damp_kappa1=0.02, shift_eta=2.0,
                              r_max_con=1e300)
    mesh = Z.Mesh((2, 2, 3), (16, 16, 16), (-4.0, -4.0, -6.0), (4.0, 4.0, 6.0), "outflow")
    ctx = Z.Z4c(mesh, params, "rk4")
    ctx.set_contract(True)
    assert ctx.get_merged()
    dt = 0.25 * float(np.min(ctx.dx()))
    states = _states(mesh, params, ctx, ID)[:4]
    expect_hst = []
    for st in states:
        ctx.upload(Z.REG_U, st)
        ctx.evolve(dt, 2, with_constraints=True)
        expect_hst.append(ctx.hst_norms())
    inputs = []
    for st in states:
        t = torch.from_numpy(st.copy()).pin_memory()
        inputs.append(t.numpy())
    for _ in range(2):
        hst = ctx.evolve_jobs(inputs, None, dt, 2)
        for j in range(len(states)):
            assert np.array_equal(hst[j], expect_hst[j]), f"job {j}"
    ctx.close()
