"""The differentiated step on a statically refined mesh: the tangent-linear
and adjoint steps through the multilevel ghost fill (restriction, the
contribution-list gather, coarse-level BCs, prolongation, fine-level BCs)
and its transpose.

Mesh: 16^3 cells on [-4, 4]^3 as 2^3 root MeshBlocks of 8^3 with one root
block (x > 0, y < 0, z < 0) refined once, so its eight children sit between
coarse blocks in gid order and every kind of neighbour (finer, coarser,
same level across faces, edges and corners) occurs.

* the tangent-linear step against central differences of the forward step
  (interior vertices; tolerance as on uniform meshes);
* the adjoint step against the tangent-linear step, a dot-product test over
  every vertex of every block: the transpose of the whole step, the fill
  included, to rounding (the transpose scatters with atomic adds, so its
  sums are ordered differently from run to run);
* the gradient of the time-integrated H-norm through revolve checkpointing
  against central differences of the full forward run on smooth directions,
  and against tangent-linear runs;
* the initial-data adjoint (ADMToZ4c + the initial ghost finalisation) and
  the binary parameter gradient (masses, separation) on this mesh.

eps_floor = -1 throughout (see tests/test_gpu_adjoint.py)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PUNC = dict(diss=0.02, chi_div_floor=1e-5, damp_kappa1=0.02, damp_kappa2=0.0, shift_eta=2.0,
            r_max_con=1e300, eps_floor=-1.0)
REGION = dict(x1min=0.5, x1max=3.5, x2min=-3.5, x2max=-0.5, x3min=-3.5, x3max=-0.5, level=1)


def make(bc, params=PUNC):
    import z4c_b200 as Z
    mesh = Z.Mesh((2, 2, 2), (8, 8, 8), (-4.0,) * 3, (4.0,) * 3, bc, refinement=[REGION])
    ctx = Z.Z4c(mesh, Z.default_params(**params), "rk4")
    ctx.adj_setup()
    return Z, mesh, ctx


def smooth_field(Z, mesh, seed, amp):
    """Smooth periodic functions of position on every variable (the same
    function on every level, so the levels agree where they overlap)."""
    rng = np.random.default_rng(seed)
    ks = rng.integers(1, 3, size=(22, 3))
    ph = rng.uniform(0, 2 * np.pi, size=22)
    out = np.zeros((mesh.nblocks, 22) + tuple(reversed(mesh.nn)))
    for b in range(mesh.nblocks):
        xs, _ = mesh.block_coords(b)
        X, Y, Zc = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
        for n in range(22):
            k = ks[n]
            out[b, n] = amp * np.sin(2 * np.pi * (k[0] * Zc + k[1] * Y + k[2] * X) / 8.0 + ph[n])
    return out


def rich_state(Z, mesh, ctx, amp=1e-3):
    """Minkowski plus smooth perturbations on every variable and a shift of
    one sign per component (the upwind side never switches)."""
    u = smooth_field(Z, mesh, 0, amp)
    for c in (Z.CHI, Z.GXX, Z.GYY, Z.GZZ, Z.ALPHA):
        u[:, c] += 1.0
    for a, sgn in zip(range(3), (1, -1, 1)):
        u[:, Z.BETAX + a] = sgn * amp * (1.5 + u[:, Z.BETAX + a] / amp)
    ctx.upload(Z.REG_U, u)
    ctx.init_finalize()
    return ctx.download(Z.REG_U)


def dot(a, b):
    return float(np.sum(a * b))


def interior(u):
    return u[:, :, 4:-4, 4:-4, 4:-4]


@pytest.mark.parametrize("bc", ["periodic", "outflow"])
def test_tlm_step_matches_central_differences(bc):
    Z, mesh, ctx = make(bc)
    u0 = rich_state(Z, mesh, ctx)
    dt = 0.25 * min(min(mesh.block_coords(b)[1]) for b in range(mesh.nblocks))
    v = smooth_field(Z, mesh, 1, 1e-3)
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
    err = np.abs(interior(fd - tan)).max() / np.abs(interior(tan)).max()
    print(f"tlm vs central differences ({bc}, refined): {err:.2e}")
    assert err <= 5e-5
    ctx.close()


@pytest.mark.parametrize("bc", ["periodic", "outflow"])
def test_adjoint_step_is_the_transpose_of_the_tlm_step(bc):
    Z, mesh, ctx = make(bc)
    u0 = rich_state(Z, mesh, ctx)
    dt = 0.25 * min(min(mesh.block_coords(b)[1]) for b in range(mesh.nblocks))
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
        print(f"{bc} trial {trial}: <ub, J ud> = {lhs:.15e}, <J^T ub, ud> = {rhs:.15e}")
        assert abs(lhs - rhs) <= 1e-12 * scale
    ctx.close()


def test_gradient_against_differences_and_tangent_linear_runs():
    """dJ/du0 of the time-integrated H-norm over 6 steps, revolve with 2
    snapshots: against fourth-order central differences of the forward
    run along smooth directions and against tangent-linear runs."""
    Z, mesh, ctx = make("periodic")
    u0 = rich_state(Z, mesh, ctx)
    dt = 0.25 * min(min(mesh.block_coords(b)[1]) for b in range(mesh.nblocks))
    nsteps = 6

    def J(u):
        ctx.upload(Z.REG_U, u)
        tot = 0.0
        for _ in range(nsteps):
            ctx.evolve(dt, 1)
            tot += dt * ctx.objective()[0]
        return tot

    ctx.upload(Z.REG_U, u0)
    Jg, pb, st = ctx.gradient(dt, nsteps, 2, w_final=0.0, w_step=dt)
    grad = ctx.download(Z.REG_ADJ)
    assert np.isclose(Jg, J(u0), rtol=1e-12, atol=0)
    for seed in (5, 6):
        v = smooth_field(Z, mesh, seed, 1.0)
        v[:, Z.BETAX:Z.BETAZ + 1] = 0.0  # the upwind side stays put
        ctx.upload(Z.REG_U, u0)
        ctx.upload(Z.REG_TAN, v)
        jd = 0.0
        for _ in range(nsteps):
            ctx.tlm_step(dt)
            jd += dt * ctx.objective(reg_tan=Z.REG_TAN)[1]
        adj_dot = dot(grad, v)
        h = 1e-4
        f = [J(u0 + s * h * v) for s in (2, 1, -1, -2)]
        fd = (-f[0] + 8 * f[1] - 8 * f[2] + f[3]) / (12 * h)
        print(f"direction {seed}: adjoint {adj_dot:.12e} tlm {jd:.12e} fd {fd:.12e}")
        assert abs(adj_dot - jd) <= 1e-10 * abs(jd)
        assert abs(adj_dot - fd) <= 1e-6 * abs(fd)
    ctx.close()


BL_Y, BL_Z = 0.13, 0.07  # the punctures sit off the x axis and off the vertices


def bl_adm(Z, mesh, params, m1, m2, d):
    """Brill-Lindquist data: masses m1, m2 at (+-d/2, -+0.13, -+0.07), the
    first inside the refined root block near its coarse neighbours, with a
    constant shift of one sign per component: the advection stencils'
    upwind side, chosen by the sign of the shift, then never switches over
    the run (with zero initial shift it switches wherever the growing shift
    crosses zero, and the map is not differentiable there)."""
    from z4c_b200 import initial_data as ID
    return ID.punctures(mesh, params, masses=(m1, m2),
                        centres=((0.5 * d, -BL_Y, -BL_Z), (-0.5 * d, BL_Y, BL_Z)),
                        shift=(0.3, -0.3, 0.3))


def test_binary_parameter_gradient_on_the_refined_mesh():
    """The time-integrated H-norm of a binary Brill-Lindquist evolution on
    the two-level outflow mesh (1+log and Gamma-driver, 8 steps) with
    respect to the two masses, the separation and eta: revolve-checkpointed
    adjoint, the adjoint of ADMToZ4c and the initial multilevel ghost fill,
    and the derivative of the host-side initial data, against central
    differences of the full forward run."""
    Z, mesh, ctx = make("outflow")
    params = Z.default_params(**PUNC)
    theta = np.array([0.5, 0.45, 3.0])  # m1, m2, separation
    dt = 0.25 * min(min(mesh.block_coords(b)[1]) for b in range(mesh.nblocks))
    nsteps = 8

    def run(th, eta=PUNC["shift_eta"]):
        p = dict(PUNC, shift_eta=eta)
        Zr, meshr, c = make("outflow", p)
        c.upload(Zr.REG_ADM, bl_adm(Zr, meshr, Zr.default_params(**p), *th))
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
    J, pb, st = ctx.gradient(dt, nsteps, 2, w_final=0.0, w_step=dt)
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
    # fourth-order central differences: the data's third derivative with
    # respect to a puncture's position is large a fraction of a cell away
    fds = []
    for j in range(3):
        e = np.zeros(3)
        e[j] = 1e-4
        f = [run(theta + s_ * e) for s_ in (2, 1, -1, -2)]
        fds.append((-f[0] + 8 * f[1] - 8 * f[2] + f[3]) / (12 * 1e-4))
    eta = PUNC["shift_eta"]
    f = [run(theta, eta + s_ * 1e-3) for s_ in (2, 1, -1, -2)]
    fds.append((-f[0] + 8 * f[1] - 8 * f[2] + f[3]) / (12 * 1e-3))
    names = ("m1", "m2", "separation", "eta")
    for n_, a, f in zip(names, grads, fds):
        print(f"dJ/d{n_}: adjoint {a:.12e}, differences {f:.12e}, rel {abs(a - f) / abs(f):.2e}")
    for a, f in zip(grads, fds):
        assert abs(a - f) <= 1e-6 * abs(f)


# ---- the Weyl-scalar term of the objective ----

def weyl_setup(Z, ctx, radius=2.3, weight=1e3):
    w = Z.WaveExtract(ctx, radius=radius, nlev=6, lmax=2)
    ctx.adj_set_weyl(w, weight)
    return w


@pytest.mark.parametrize("bc", ["periodic", "outflow"])
def test_weyl_objective_gradient_against_differences(bc):
    """J = H-norm + weight * sum_p w_p |psi4(p)|^2 over a sphere of radius
    2.3 (crossing both levels) at one state: its adjoint (the interpolation
    and the Weyl ghost fill transposed, psi4's local inputs by forward mode,
    the transposed stencils and Z4cToADM) against fourth-order central
    differences along smooth directions, and the tangent the objective
    reports (the adjoint along the direction) against them too."""
    Z, mesh, ctx = make(bc)
    u0 = rich_state(Z, mesh, ctx, amp=3e-2)
    weyl_setup(Z, ctx)
    ctx.upload(Z.REG_U, u0)
    J0 = ctx.objective()[0]
    ctx.adj_set_weyl(None)
    JH = ctx.objective()[0]
    ctx.adj_set_weyl(0, 1e3)
    assert J0 > JH > 0
    ctx.upload(Z.REG_ADJ, np.zeros_like(u0))
    ctx.objective_adj(Z.REG_U, 1.0)
    grad = ctx.download(Z.REG_ADJ)
    for seed in (7, 8):
        v = smooth_field(Z, mesh, seed, 1.0)
        if bc == "outflow":  # directions the ghost fill reproduces: interior only
            v[:, :, :4] = v[:, :, -4:] = 0
            v[:, :, :, :4] = v[:, :, :, -4:] = 0
            v[:, :, :, :, :4] = v[:, :, :, :, -4:] = 0
        h = 1e-4

        def J(x):
            ctx.upload(Z.REG_U, x)
            return ctx.objective()[0]
        f = [J(u0 + s_ * h * v) for s_ in (2, 1, -1, -2)]
        fd = (-f[0] + 8 * f[1] - 8 * f[2] + f[3]) / (12 * h)
        ad = dot(grad, v)
        ctx.upload(Z.REG_U, u0)
        ctx.upload(Z.REG_TAN, v)
        jd = ctx.objective(reg_tan=Z.REG_TAN)[1]
        print(f"{bc} direction {seed}: adjoint {ad:.12e} tangent {jd:.12e} fd {fd:.12e}")
        assert abs(ad - fd) <= 1e-6 * abs(fd)
        assert abs(jd - ad) <= 1e-12 * abs(ad)
    ctx.close()


def test_binary_gradient_with_the_weyl_term():
    """The binary parameter gradient of the time-integrated H-norm plus the
    Weyl term on the sphere of radius 2.3 (two-level outflow mesh, 6 steps)
    against fourth-order differences of the full forward run."""
    Z, mesh, ctx = make("outflow")
    params = Z.default_params(**PUNC)
    theta = np.array([0.5, 0.45, 3.0])
    dt = 0.25 * min(min(mesh.block_coords(b)[1]) for b in range(mesh.nblocks))
    nsteps = 6

    def run(th):
        Zr, meshr, c = make("outflow")
        weyl_setup(Zr, c)
        c.upload(Zr.REG_ADM, bl_adm(Zr, meshr, params, *th))
        c.ADMToZ4c()
        c.init_finalize()
        J = 0.0
        for _ in range(nsteps):
            c.evolve(dt, 1)
            J += dt * c.objective(Zr.REG_U)[0]
        c.close()
        return J

    weyl_setup(Z, ctx)
    adm = bl_adm(Z, mesh, params, *theta)
    ctx.upload(Z.REG_ADM, adm)
    ctx.ADMToZ4c()
    ctx.init_finalize()
    J, pb, st = ctx.gradient(dt, nsteps, 2, w_final=0.0, w_step=dt)
    ctx.upload(Z.REG_ADM, adm)
    ctx.adj_adm_to_z4c()
    ab = ctx.download(Z.REG_ADM_ADJ)
    ctx.close()
    assert abs(J - run(theta)) <= 1e-12 * abs(J)
    for j, name in enumerate(("m1", "m2", "separation")):
        e = np.zeros(3)
        e[j] = 1e-6
        dadm = (bl_adm(Z, mesh, params, *(theta + e)) - bl_adm(Z, mesh, params, *(theta - e))) / 2e-6
        g = dot(ab, dadm)
        e[j] = 1e-4
        f = [run(theta + s_ * e) for s_ in (2, 1, -1, -2)]
        fd = (-f[0] + 8 * f[1] - 8 * f[2] + f[3]) / (12 * 1e-4)
        print(f"dJ/d{name}: adjoint {g:.12e}, differences {fd:.12e}, rel {abs(g - fd) / abs(fd):.2e}")
        assert abs(g - fd) <= 1e-6 * abs(fd)
