"""The compile-time 16^3 kernel instances against the oracle.

The golden fixtures use 8^3 MeshBlocks, which run the generic kernels; every
kernel of the step also exists in a form specialised for 16^3 MeshBlocks
(constant strides, whole-loop unrolling).  Here meshes of 2^3 and 3^3
MeshBlocks of 16^3 take one full step through the captured graph for each
integrator and boundary condition, including the Sommerfeld and Butcher
stage kernels, and are compared with the same step on the oracle."""
import numpy as np
import pytest

import z4c_oracle as O
from z4c_testlib import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-12
PARAMS = dict(diss=0.02, chi_div_floor=1e-5, damp_kappa1=0.02, damp_kappa2=0.0, shift_eta=2.0,
              r_max_con=1e300)


def oracle_step(mesh, p, u, dt, integ):
    """One GR_Z4c step on the oracle, blocks in grid order."""
    nb = mesh.nblocks
    nn = mesh.nn
    blocks = []
    for b in range(nb):
        xs, dxs = mesh.block_coords(b)
        blocks.append(O.Block(mesh.nx, dxs, xs))
    som = [O.sommerfeld_faces(mesh.nb, mesh.bc, b) for b in range(nb)]

    def rhs(v):
        r = np.stack([O.rhs(blocks[b], p, v[b]) for b in range(nb)])
        for b in range(nb):
            O.boundary_rhs(blocks[b], v[b], r[b], som[b])
        return r

    def exchange(v):
        v = O.mesh_exchange(mesh.nb, mesh.nx, mesh.bc, v)
        return np.stack([O.algconstr(blocks[b], p, v[b]) for b in range(nb)])

    u = u.copy()
    if integ == "rk4":
        u1 = np.zeros_like(u)
        for s in range(4):
            w = O.LS_RK4[s]
            r = rhs(u)
            for b in range(nb):
                O.weighted_ave(u1[b], u[b], None, [1.0, w["delta"], 0.0], nn)
                O.weighted_ave(u[b], u1[b], None, [w["gamma_1"], w["gamma_2"], w["gamma_3"]], nn)
                O.add_rhs(r[b], w["beta"] * dt, u[b], nn)
            u = exchange(u)
    else:
        un, ks = u.copy(), []
        for s in range(4):
            ks.append(rhs(u))
            u = un.copy()
            coefs = O.BT_RK4_A[s + 1][: s + 1] if s < 3 else O.BT_RK4_B
            for q, a in enumerate(coefs):
                if a != 0:
                    u += (a * dt) * ks[q]
            u = exchange(u)
    return u


@pytest.mark.parametrize("integ,bc,nb", [("rk4", "outflow", 2), ("rk4", "sommerfeld", 2),
                                         ("rk4", "periodic", 2), ("bt_rk4", "outflow", 2),
                                         ("bt_rk4", "sommerfeld", 2), ("rk4", "outflow", 3),
                                         ("bt_rk4", "sommerfeld", 3)])
def test_one_step_on_16cubed_blocks_matches_oracle(integ, bc, nb):
    """nb = 3 puts a MeshBlock in the middle that touches no physical face."""
    import z4c_b200 as Z
    from z4c_b200 import initial_data as ID
    lim = 2.0 * nb
    mesh = Z.Mesh((nb,) * 3, (16, 16, 16), (-lim,) * 3, (lim,) * 3, bc)
    params = Z.default_params(**PARAMS)
    ctx = Z.Z4c(mesh, params, integ)
    ID.load_adm(ctx, ID.punctures(mesh, params, masses=(0.5, 0.5),
                                  centres=((1.1, 0.2, 0.1), (-1.1, -0.3, 0.0))))
    u0 = ctx.download(Z.REG_U)
    dt = 0.25 * float(ctx.dx().min())
    ctx.evolve(dt, 1)
    got = ctx.download(Z.REG_U)
    ref = oracle_step(mesh, O.default_params(**PARAMS), u0, dt, integ)
    assert rel_err(got, ref) <= TOL
    ctx.close()
