"""The differentiated Z4c step on the device, through the C ABI:

* the tangent-linear step against central differences of the forward step;
* the adjoint step against the tangent-linear step (dot-product test
  <ubar_1, J udot_0> = <J^T ubar_1, udot_0> over every vertex);
* the objective (vol * sum of H^2 over the history cells) against the
  history norm, its tangent against differences, its adjoint against its
  tangent;
* revolve checkpointing: the gradient does not depend on the snapshot count;
* the gauge-wave adjoint benchmark at its stated size: 64^3 gauge wave (A = 0.05) with seeded 1e-6
  noise on the conformal metric, 100 rk4 steps, the gradient of the H-norm
  with respect to every initial Z4c value against central differences on 32
  seeded directions and against tangent-linear runs.

Tolerances: the adjoint and the tangent-linear model differentiate the same
discrete map, so they agree to rounding (1e-10 relative); central
differences carry a truncation error O(h^2) and a rounding error O(eps/h),
the bound on them is 1e-6 relative.

eps_floor = -1 in every run compared with differences.  AlgConstr rescales
g~ by regularize_nth_root(det g~, 1, eps_floor, -3) (z4c.cpp:677-799,
floating_point.hpp:120-131), which switches from det^(-1/3) to the constant
1 - eps_floor/3 where det g~ < 1 + eps_floor.  AlgConstr itself sets
det g~ = 1 every stage and the evolution keeps it there to rounding, so with
the default eps_floor = 1e-12 nearly every vertex sits on that switch: the
map is not differentiable along the determinant direction, the derivatives
take the branch of the linearisation point and a difference quotient of any
step averages the two.  A negative eps_floor selects det^(-1/3) everywhere
(the constraint the switch approximates) and the map is smooth."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PUNC = dict(diss=0.02, chi_div_floor=1e-5, damp_kappa1=0.02, damp_kappa2=0.0, shift_eta=2.0,
            r_max_con=1e300, eps_floor=-1.0)
GW = dict(lapse_harmonic=1.0, lapse_harmonicf=0.0, lapse_oplog=0.0, lapse_advect=0.0,
          shift_Gamma=0.0, shift_eta=0.0, shift_advect=0.0, diss=0.02, damp_kappa1=0.02,
          r_max_con=1e300, eps_floor=-1.0)


def make(nb, nx, params, lim=0.5, bc="periodic"):
    import z4c_b200 as Z
    mesh = Z.Mesh(nb, (nx,) * 3, (-lim,) * 3, (lim,) * 3, bc)
    ctx = Z.Z4c(mesh, Z.default_params(**params), "rk4")
    ctx.adj_setup()
    return Z, mesh, ctx


def rich_state(Z, mesh, ctx, amp=1e-3, seed=0):
    """A gauge wave (A = 0.05) with smooth periodic perturbations of size amp
    on every variable, and a shift of one sign per component (the upwind
    side never switches), so that every term of the right-hand side,
    advection included, is active and differentiable."""
    from z4c_b200 import initial_data as ID
    ID.load_adm(ctx, ID.gauge_wave1(mesh, amplitude=0.05))
    u = ctx.download(Z.REG_U)
    rng = np.random.default_rng(seed)
    for b in range(mesh.nblocks):
        xs, _ = mesh.block_coords(b)
        X, Y, Zc = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
        for n in range(22):
            k = rng.integers(1, 3, size=3)
            ph = rng.uniform(0, 2 * np.pi)
            wave = np.sin(2 * np.pi * (k[0] * Zc + k[1] * Y + k[2] * X) + ph)
            if n >= Z.BETAX:  # 0.5 amp .. 2.5 amp, signs +, -, +
                u[b, n] = (1 if n != Z.BETAY else -1) * amp * (1.5 + wave)
            else:
                u[b, n] += amp * wave
    ctx.upload(Z.REG_U, u)
    ctx.init_finalize()
    return ctx.download(Z.REG_U)


def dot(a, b):
    return float(np.sum(a * b))


def smooth_direction(Z, mesh, seed, amp=1e-3):
    """A smooth periodic direction on every variable and vertex (the outflow
    extrapolation multiplies rough data by up to ~10^3 per axis in the
    ghosts, which would leave the range where differences are linear)."""
    rng = np.random.default_rng(seed)
    out = np.zeros((mesh.nblocks, 22) + tuple(reversed(mesh.nn)))
    for b in range(mesh.nblocks):
        xs, _ = mesh.block_coords(b)
        X, Y, Zc = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
        for n in range(22):
            k = rng.integers(1, 3, size=3)
            ph = rng.uniform(0, 2 * np.pi)
            out[b, n] = amp * np.sin(2 * np.pi * (k[0] * Zc + k[1] * Y + k[2] * X) + ph)
    return out


CASES = [(PUNC, "periodic"), (GW, "periodic"), (PUNC, "outflow")]
CASE_IDS = ["puncture_gauge", "gauge_wave", "puncture_gauge_outflow"]


@pytest.mark.parametrize("params,bc", CASES, ids=CASE_IDS)
def test_tlm_step_matches_central_differences(params, bc):
    Z, mesh, ctx = make((2, 2, 1), 12, params, bc=bc)
    u0 = rich_state(Z, mesh, ctx)
    dt = 0.25 * float(ctx.dx().min())
    v = smooth_direction(Z, mesh, 1)
    ctx.upload(Z.REG_TAN, v)
    ctx.upload(Z.REG_U, u0)
    ctx.tlm_step(dt)
    tan = ctx.download(Z.REG_TAN)
    u1 = ctx.download(Z.REG_U)
    ctx.upload(Z.REG_U, u0)
    ctx.evolve(dt, 1)
    assert np.array_equal(ctx.download(Z.REG_U), u1), "tlm_step's values are the forward step's"
    h = 1e-4
    out = []
    for sgn in (1, -1):
        ctx.upload(Z.REG_U, u0 + sgn * h * v)
        ctx.evolve(dt, 1)
        out.append(ctx.download(Z.REG_U))
    fd = (out[0] - out[1]) / (2 * h)
    if bc == "periodic":
        err = np.abs(fd - tan).max() / np.abs(tan).max()
        tol = 1e-6
    else:
        # The reference's extrapolation (5, -10, 10, -5, 1, cascaded over four
        # ghost layers and three axes) multiplies the state's rounding by up
        # to ~1e9 in the corner ghosts, which makes a difference quotient
        # noise there; the interior is compared, and the exact transpose
        # test below covers the boundary conditions.
        I = (slice(None), slice(None), slice(4, -4), slice(4, -4), slice(4, -4))
        err = np.abs(fd - tan)[I].max() / np.abs(tan[I]).max()
        tol = 5e-5
    print(f"tlm vs central differences ({bc}): {err:.2e}")
    assert err <= tol
    ctx.close()


@pytest.mark.parametrize("params,bc", CASES, ids=CASE_IDS)
def test_adjoint_step_is_the_transpose_of_the_tlm_step(params, bc):
    Z, mesh, ctx = make((2, 2, 1), 12, params, bc=bc)
    u0 = rich_state(Z, mesh, ctx)
    dt = 0.25 * float(ctx.dx().min())
    rng = np.random.default_rng(2)
    for trial in range(3):
        ud = rng.standard_normal(u0.shape)
        ub = rng.standard_normal(u0.shape)
        ctx.upload(Z.REG_U, u0)
        ctx.upload(Z.REG_TAN, ud)
        ctx.tlm_step(dt)
        Jud = ctx.download(Z.REG_TAN)
        ctx.upload(Z.REG_U, u0)
        ctx.upload(Z.REG_ADJ, ub)
        ctx.adj_params(reset=True)
        ctx.adj_step(dt)
        assert np.array_equal(ctx.download(Z.REG_U), u0), "adj_step leaves u unchanged"
        JTub = ctx.download(Z.REG_ADJ)
        lhs, rhs = dot(ub, Jud), dot(JTub, ud)
        scale = np.abs(ub * Jud).sum()
        print(f"trial {trial}: <ub, J ud> = {lhs:.15e}, <J^T ub, ud> = {rhs:.15e}")
        assert abs(lhs - rhs) <= 1e-12 * scale
    ctx.close()


def test_parameter_adjoints_match_differences():
    """d<ub, u_1>/d eta and d/d kappa1 of one step: adjoint vs central
    differences of the forward step."""
    Z, mesh, ctx = make((2, 2, 1), 12, PUNC)
    u0 = rich_state(Z, mesh, ctx)
    dt = 0.25 * float(ctx.dx().min())
    ub = np.random.default_rng(4).standard_normal(u0.shape)
    ctx.upload(Z.REG_U, u0)
    ctx.upload(Z.REG_ADJ, ub)
    ctx.adj_params(reset=True)
    ctx.adj_step(dt)
    pb = ctx.adj_params()
    ctx.close()
    for k, name in enumerate(("shift_eta", "damp_kappa1")):
        states = []
        dp = 1e-3  # below ~1e-4 the rounding of the states dominates
        for sgn in (1, -1):
            p = dict(PUNC)
            p[name] = PUNC[name] + sgn * dp
            Z2, mesh2, c2 = make((2, 2, 1), 12, p)
            c2.upload(Z2.REG_U, u0)
            c2.evolve(dt, 1)
            states.append(c2.download(Z2.REG_U))
            c2.close()
        # difference the states first: <ub, u> itself is a sum of ~10^6 terms
        fd = dot(ub, states[0] - states[1]) / (2 * dp)
        print(f"{name}: adjoint {pb[k]:.12e}, differences {fd:.12e}")
        assert abs(fd - pb[k]) <= 1e-6 * abs(fd)


def test_objective_and_its_derivatives():
    Z, mesh, ctx = make((2, 2, 1), 12, PUNC)
    u0 = rich_state(Z, mesh, ctx)
    # J equals the history output's H-norm (volume-weighted sum of H^2)
    ctx.constraints()
    J, _ = ctx.objective(Z.REG_U)
    hst = ctx.hst_norms()[0]
    assert abs(J - hst) <= 1e-12 * hst, (J, hst)
    rng = np.random.default_rng(3)
    v = rng.standard_normal(u0.shape) * 1e-3
    ctx.upload(Z.REG_TAN, v)
    J0, Jd = ctx.objective(Z.REG_U, Z.REG_TAN)
    h = 1e-4
    Jp = Jm = None
    ctx.upload(Z.REG_W, u0 + h * v)
    Jp, _ = ctx.objective(Z.REG_W)
    ctx.upload(Z.REG_W, u0 - h * v)
    Jm, _ = ctx.objective(Z.REG_W)
    fd = (Jp - Jm) / (2 * h)
    print(f"J {J0:.6e}: tangent {Jd:.12e}, differences {fd:.12e}")
    assert abs(fd - Jd) <= 1e-7 * abs(Jd)
    ctx.upload(Z.REG_ADJ, np.zeros_like(u0))
    ctx.objective_adj(Z.REG_U, 1.0)
    g = ctx.download(Z.REG_ADJ)
    assert abs(dot(g, v) - Jd) <= 1e-12 * np.abs(g * v).sum()
    ctx.close()


def test_revolve_schedules_give_the_same_gradient():
    Z, mesh, ctx = make((2, 1, 1), 12, PUNC)
    u0 = rich_state(Z, mesh, ctx)
    dt = 0.25 * float(ctx.dx().min())
    nsteps = 7
    ref = None
    for nsnap, w_step in ((6, 0.0), (2, 0.0), (0, 0.0), (2, 0.5)):
        ctx.upload(Z.REG_U, u0)
        J, pb, st = ctx.gradient(dt, nsteps, nsnap, 1.0, w_step)
        g = ctx.download(Z.REG_ADJ)
        assert np.array_equal(ctx.download(Z.REG_U), u0)
        assert st["adjoint_steps"] == nsteps
        # forward sweep + schedule + (per-step source recomputation)
        extra = nsteps if w_step else 0
        assert st["forward_steps"] == nsteps + st["schedule_cost"] + extra, st
        if w_step == 0.0:
            if ref is None:
                ref = (J, g, pb)
            assert J == ref[0] and np.array_equal(g, ref[1]) and np.array_equal(pb, ref[2])
        else:
            # the time-integrated part through the step-by-step adjoint
            ctx.upload(Z.REG_U, u0)
            states = [u0]
            for _ in range(nsteps):
                ctx.evolve(dt, 1)
                states.append(ctx.download(Z.REG_U))
            ctx.upload(Z.REG_ADJ, np.zeros_like(u0))
            ctx.upload(Z.REG_U, states[-1])
            ctx.objective_adj(Z.REG_U, 1.0 + w_step)
            for k in range(nsteps - 1, -1, -1):
                ctx.upload(Z.REG_U, states[k])
                ctx.adj_step(dt)
                if k > 0:
                    ctx.objective_adj(Z.REG_U, w_step)
            g2 = ctx.download(Z.REG_ADJ)
            assert np.abs(g2 - g).max() <= 1e-12 * np.abs(g).max()
    ctx.close()


def gw64_adjoint_state(Z, mesh, ctx, seed=2024):
    from z4c_b200 import initial_data as ID
    ID.load_adm(ctx, ID.gauge_wave1(mesh, amplitude=0.05))
    u = ctx.download(Z.REG_U)
    rng = np.random.default_rng(seed)
    u[:, Z.GXX:Z.GZZ + 1] += rng.uniform(-1e-6, 1e-6, size=u[:, Z.GXX:Z.GZZ + 1].shape)
    ctx.upload(Z.REG_U, u)
    ctx.init_finalize()
    return ctx.download(Z.REG_U)


def test_gw64_gradient_against_differences_and_tangent_linear_runs():
    Z, mesh, ctx = make((1, 1, 1), 64, GW)
    u0 = gw64_adjoint_state(Z, mesh, ctx)
    dt = 0.25 / 64
    nsteps = 100
    ctx.upload(Z.REG_U, u0)
    J, pb, st = ctx.gradient(dt, nsteps, 9)
    g = ctx.download(Z.REG_ADJ)
    print(f"J = {J:.10e}, gradient in {st['seconds']:.2f} s, {st}")
    import time
    ctx.upload(Z.REG_U, u0)
    ctx.evolve(dt, 2)
    ctx.sync()
    t0 = time.perf_counter()
    ctx.evolve(dt, 20)
    ctx.sync()
    fwd = (time.perf_counter() - t0) / 20
    ctx.upload(Z.REG_U, u0)
    ctx.adj_step(dt)
    ctx.sync()
    t0 = time.perf_counter()
    for _ in range(5):
        ctx.adj_step(dt)
    ctx.sync()
    adj = (time.perf_counter() - t0) / 5
    print(f"forward step {fwd * 1e3:.3f} ms, adjoint step {adj * 1e3:.3f} ms, ratio {adj / fwd:.2f}")
    assert np.array_equal(ctx.download(Z.REG_U), u0)
    rng = np.random.default_rng(32)
    worst_tlm = 0.0
    errs, pairs = [], []
    # Fourth-order central differences, (-J(2h) + 8 J(h) - 8 J(-h) + J(-2h)) / 12h,
    # exact up to cubic terms: perturbations of the size of the initial noise
    # (1e-6) keep far above the rounding of 100 steps.  The directions leave
    # the shift alone: it is zero throughout the gauge wave (no shift
    # evolution), where the advection's upwind side switches with its sign,
    # so J is only one-sidedly differentiable along it (the adjoint takes the
    # side of beta >= 0); the tangent-linear runs below use full directions.
    import z4c_b200 as Zp
    h = 1.0  # perturbations of 1e-6 and 2e-6
    for d in range(32):
        v = rng.standard_normal(u0.shape) * 1e-6
        v_full = v.copy()
        v[:, Zp.BETAX:Zp.BETAZ + 1] = 0.0
        Js = {}
        for m in (2, 1, -1, -2):
            ctx.upload(Z.REG_U, u0 + m * h * v)
            ctx.evolve(dt, nsteps)
            Js[m] = ctx.objective(Z.REG_U)[0]
        fd = (-Js[2] + 8 * Js[1] - 8 * Js[-1] + Js[-2]) / (12 * h)
        ad = dot(g, v)
        errs.append(abs(fd - ad) / abs(ad))
        pairs.append((fd, ad))
        if d < 4:  # tangent-linear runs along the first directions, shift included
            ctx.upload(Z.REG_U, u0)
            ctx.upload(Z.REG_TAN, v_full)
            for _ in range(nsteps):
                ctx.tlm_step(dt)
            _, Jd = ctx.objective(Z.REG_U, Z.REG_TAN)
            ad_full = dot(g, v_full)
            worst_tlm = max(worst_tlm, abs(Jd - ad_full) / abs(ad_full))
    # A random direction's derivative can come out near zero, where a
    # relative difference means little: each difference is measured against
    # the root-mean-square derivative over the 32 directions.
    fds, ads = np.array(pairs).T
    rms = np.sqrt(np.mean(ads ** 2))
    worst_fd = float(np.max(np.abs(fds - ads)) / rms)
    print(f"64^3 gauge wave: relative difference to central differences: median {np.median(errs):.2e} "
          f"(own derivative), worst {worst_fd:.2e} (rms derivative); to tangent-linear runs "
          f"{worst_tlm:.2e}")
    assert worst_fd <= 1e-6
    assert worst_tlm <= 1e-9
    ctx.close()


# ---- the chain to the initial data (the binary adjoint benchmark's gradient, on a uniform mesh) ----

BL_Y, BL_Z = 0.13, 0.07  # the punctures sit off the x axis and off the vertices


def bl_adm(Z, mesh, params, m1, m2, d):
    """Brill-Lindquist data: masses m1, m2 at (+-d/2, +-0.13, +-0.07)."""
    from z4c_b200 import initial_data as ID
    return ID.punctures(mesh, params, masses=(m1, m2),
                        centres=((0.5 * d, BL_Y, BL_Z), (-0.5 * d, -BL_Y, -BL_Z)))


@pytest.mark.parametrize("bc", ["periodic", "outflow"])
def test_initial_data_adjoint_matches_differences(bc):
    """The adjoint of ADMToZ4c + the initial ghost finalisation against
    central differences of that map along a smooth direction in the ADM
    data.  On the outflow mesh the weights ub leave out the ghosts, where
    the extrapolation's amplification of rounding makes differences noise
    (the transposed extrapolation is covered by the step's transpose test)."""
    Z, mesh, ctx = make((2, 2, 1), 12, PUNC, lim=4.0, bc=bc)
    params = Z.default_params(**PUNC)
    adm = bl_adm(Z, mesh, params, 0.5, 0.5, 3.0)
    rng = np.random.default_rng(9)
    dirs = smooth_direction(Z, mesh, 11, amp=1e-2)[:, :17]
    dirs[:, Z.ADM_PSI4] = 0.0

    def u_of(a):
        ctx.upload(Z.REG_ADM, a)
        ctx.ADMToZ4c()
        ctx.init_finalize()
        return ctx.download(Z.REG_U)

    u0 = u_of(adm)
    ub = smooth_direction(Z, mesh, 12, amp=1.0) + 0.1 * rng.standard_normal(u0.shape)
    if bc == "outflow":
        interior = np.zeros_like(ub)
        interior[:, :, 4:-4, 4:-4, 4:-4] = 1.0
        ub *= interior
    ctx.upload(Z.REG_ADM, adm)
    ctx.upload(Z.REG_ADJ, ub)
    ctx.adj_adm_to_z4c()
    ab = ctx.download(Z.REG_ADM_ADJ)
    h = 1e-4
    fd = dot(ub, (u_of(adm + h * dirs) - u_of(adm - h * dirs))) / (2 * h)
    ad = dot(ab, dirs)
    print(f"initial data: adjoint {ad:.12e}, differences {fd:.12e}")
    assert abs(fd - ad) <= 1e-7 * abs(fd)
    ctx.close()


def test_binary_parameter_gradient_on_a_uniform_mesh():
    """The binary adjoint benchmark's gradient on a uniform mesh: the time-integrated H-norm
    of a binary Brill-Lindquist evolution (outflow faces, 1+log and
    Gamma-driver) with respect to the two masses, the separation and the
    Gamma-driver eta, through the revolve-checkpointed adjoint, the adjoint
    of ADMToZ4c and the derivative of the host-side initial data, against
    central differences of the full forward run."""
    Z, mesh, ctx = make((2, 2, 2), 12, PUNC, lim=4.0, bc="outflow")
    params = Z.default_params(**PUNC)
    theta = np.array([0.5, 0.45, 3.0])  # m1, m2, separation
    dt = 0.25 * float(ctx.dx().min())
    nsteps = 12

    def run(th, eta=PUNC["shift_eta"]):
        p = dict(PUNC, shift_eta=eta)
        Zr, meshr, c = make((2, 2, 2), 12, p, lim=4.0, bc="outflow")
        adm = bl_adm(Zr, meshr, Zr.default_params(**p), *th)
        c.upload(Zr.REG_ADM, adm)
        c.ADMToZ4c()
        c.init_finalize()
        J = 0.0
        for _ in range(nsteps):
            c.evolve(dt, 1)
            J += dt * c.objective(Zr.REG_U)[0]
        c.close()
        return J

    adm = bl_adm(Z, mesh, params, *theta)
    ctx.upload(Z.REG_ADM, adm)
    ctx.ADMToZ4c()
    ctx.init_finalize()
    J, pb, st = ctx.gradient(dt, nsteps, 3, w_final=0.0, w_step=dt)
    ctx.upload(Z.REG_ADM, adm)  # the steps rewrote it (Z4cToADM)
    ctx.adj_adm_to_z4c()
    ab = ctx.download(Z.REG_ADM_ADJ)
    ctx.close()
    assert abs(J - run(theta)) <= 1e-12 * abs(J)
    grads = []
    for j in range(3):
        e = np.zeros(3)
        e[j] = 1e-6
        dadm = (bl_adm(Z, mesh, params, *(theta + e)) - bl_adm(Z, mesh, params, *(theta - e))) / 2e-6
        grads.append(dot(ab, dadm))
    grads.append(pb[0])
    fds = []
    for j in range(3):
        e = np.zeros(3)
        e[j] = 1e-4
        fds.append((run(theta + e) - run(theta - e)) / 2e-4)
    fds.append((run(theta, PUNC["shift_eta"] + 1e-3) - run(theta, PUNC["shift_eta"] - 1e-3)) / 2e-3)
    names = ("m1", "m2", "separation", "eta")
    for n_, a, f in zip(names, grads, fds):
        print(f"dJ/d{n_}: adjoint {a:.12e}, differences {f:.12e}, rel {abs(a - f) / abs(f):.2e}")
    for a, f in zip(grads, fds):
        assert abs(a - f) <= 1e-6 * abs(f)


def test_torch_autograd_function_gives_the_adjoint_gradient():
    """The torch.autograd.Function harness: J.backward() returns the adjoint
    gradient, and a scaled upstream gradient scales it; torch's own
    central-difference check along a direction agrees."""
    import torch
    from z4c_b200.autograd import Z4cObjective
    Z, mesh, ctx = make((2, 1, 1), 12, GW)
    u0 = rich_state(Z, mesh, ctx)
    dt = 0.25 * float(ctx.dx().min())
    x = torch.tensor(u0, dtype=torch.float64, requires_grad=True)
    J = Z4cObjective.apply(x, ctx, dt, 5, 2)
    (3.0 * J).backward()
    ctx.upload(Z.REG_U, u0)
    J2, _, _ = ctx.gradient(dt, 5, 2)
    g = ctx.download(Z.REG_ADJ)
    assert J.item() == J2
    assert np.array_equal(x.grad.numpy(), 3.0 * g)
    v = torch.from_numpy(smooth_direction(Z, mesh, 21))
    h = 1e-3
    with torch.no_grad():
        Jp = Z4cObjective.apply(x + h * v, ctx, dt, 5, 2)
        Jm = Z4cObjective.apply(x - h * v, ctx, dt, 5, 2)
    fd = float(Jp - Jm) / (2 * h)
    ad = float(torch.sum(x.grad * v)) / 3.0
    print(f"autograd: {ad:.12e}, differences {fd:.12e}")
    assert abs(fd - ad) <= 1e-6 * abs(fd)
    ctx.close()
