"""The CPU oracle against the golden fixtures produced by the reference
build itself (tests/golden/make_golden.py).  The oracle restates the
reference's arithmetic in the same order, so agreement is bit for bit."""
import os

import numpy as np
import pytest

import z4c_oracle as O
from z4c_testlib import GOLDEN, Case, bitwise

OPS = ["ops_gw1", "ops_punc2", "ops_rs2", "ops_somm2"]


def _params(case):
    return O.default_params(**case.params)


def _som(case, g):
    """Sommerfeld faces of the block with reference gid g."""
    return O.sommerfeld_faces(case.nb, case.mesh["bc"], case.order[g])


@pytest.mark.parametrize("name", OPS)
def test_single_operators(name):
    c = Case(name)
    p = _params(c)
    blocks = c.blocks()
    u0, adm0 = c.rec["u0"], c.rec["adm0"]
    I = c.interior()
    rhs = np.stack([O.rhs(b, p, u0[g]) for g, b in enumerate(blocks)])
    assert bitwise(rhs[I], c.rec["rhs0"][I])
    if "brhs0" in c.rec:  # Z4cBoundaryRHS on the gr_sommerfeld faces
        for g, b in enumerate(blocks):
            O.boundary_rhs(b, u0[g], rhs[g], _som(c, g))
        assert bitwise(rhs[I], c.rec["brhs0"][I])
    alg = np.stack([O.algconstr(b, p, u0[g]) for g, b in enumerate(blocks)])
    assert bitwise(alg, c.rec["alg0"])
    adm = np.stack([O.z4c_to_adm(b, p, u0[g]) for g, b in enumerate(blocks)])
    assert bitwise(adm, adm0)
    con = np.stack([O.adm_constraints(b, p, adm0[g], u0[g]) for g, b in enumerate(blocks)])
    assert bitwise(con, c.rec["con0"])
    uadm = np.stack([O.adm_to_z4c(b, p, adm0[g]) for g, b in enumerate(blocks)])
    assert bitwise(uadm, c.rec["uadm0"])


@pytest.mark.parametrize("name", OPS)
def test_ghost_exchange(name):
    c = Case(name)
    bc = c.mesh["bc"]
    out = c.from_grid(O.mesh_exchange(c.nb, c.nx, bc, c.to_grid(c.rec["gx_pre"])))
    assert bitwise(out, c.rec["gx_post"])


def oracle_step(c, p, blocks, u, dt):
    """One full step of the GR_Z4c task list on the oracle (gid order)."""
    nb = len(blocks)
    u = u.copy()
    if c.integrator == "rk4":
        u1 = np.zeros_like(u)
        for s in range(4):
            w = O.LS_RK4[s]
            r = np.stack([O.rhs(blocks[b], p, u[b]) for b in range(nb)])
            for b in range(nb):
                O.boundary_rhs(blocks[b], u[b], r[b], _som(c, b))
            for b in range(nb):
                O.weighted_ave(u1[b], u[b], None, [1.0, w["delta"], 0.0], c.nn)
                O.weighted_ave(u[b], u1[b], None, [w["gamma_1"], w["gamma_2"], w["gamma_3"]], c.nn)
                O.add_rhs(r[b], w["beta"] * dt, u[b], c.nn)
            u = c.from_grid(O.mesh_exchange(c.nb, c.nx, c.mesh["bc"], c.to_grid(u)))
            u = np.stack([O.algconstr(blocks[b], p, u[b]) for b in range(nb)])
            yield u
    else:
        un, ks = u.copy(), []
        for s in range(4):
            ks.append(np.stack([O.rhs(blocks[b], p, u[b]) for b in range(nb)]))
            for b in range(nb):
                O.boundary_rhs(blocks[b], u[b], ks[-1][b], _som(c, b))
            u = un.copy()
            coefs = O.BT_RK4_A[s + 1][: s + 1] if s < 3 else O.BT_RK4_B
            for q, a in enumerate(coefs):
                if a != 0:
                    u += (a * dt) * ks[q]
            u = c.from_grid(O.mesh_exchange(c.nb, c.nx, c.mesh["bc"], c.to_grid(u)))
            u = np.stack([O.algconstr(blocks[b], p, u[b]) for b in range(nb)])
            yield u


@pytest.mark.parametrize("name", OPS)
def test_one_step_stage_by_stage(name):
    c = Case(name)
    p = _params(c)
    blocks = c.blocks()
    dt = c.rec["time_dt"][1]
    for s, u in enumerate(oracle_step(c, p, blocks, c.rec["u0"], dt)):
        assert bitwise(u, c.rec[f"s{s + 1}_alg"]), f"stage {s + 1}"
    adm = np.stack([O.z4c_to_adm(b, p, u[g]) for g, b in enumerate(blocks)])
    assert bitwise(adm, c.rec["s4_adm"])
    con = np.stack([O.adm_constraints(b, p, adm[g], u[g]) for g, b in enumerate(blocks)])
    assert bitwise(con, c.rec["s4_con"])


@pytest.mark.parametrize("name", ["evol_gw16", "evol_punc4", "evol_somm4"])
def test_evolution_and_history(name):
    """Multi-step run of the stock reference driver: final state and the
    history-output constraint norms (outputs/history.cpp:168-200)."""
    c = Case(name)
    p = _params(c)
    blocks = c.blocks()
    dt = c.rec["time_dt"][1]
    u = c.rec["u_init"]
    for _ in range(int(c.rec["nlim"])):
        for u in oracle_step(c, p, blocks, u, dt):
            pass
    assert bitwise(u, c.rec["u_final"])
    adm = np.stack([O.z4c_to_adm(b, p, u[g]) for g, b in enumerate(blocks)])
    con = np.stack([O.adm_constraints(b, p, adm[g], u[g]) for g, b in enumerate(blocks)])
    assert bitwise(con, c.rec["con_final"])
    hst = O.hst_norms(blocks, p, con, u)
    ref = c.rec["hst"][int(c.rec["nlim"]), 3:11]
    np.testing.assert_allclose(hst, ref, rtol=1e-13, atol=0)


@pytest.mark.parametrize("when", ["initial", "one_step"])
def test_weyl_psi4(when):
    """Z4cWeyl (Re, Im psi4) on the puncture of ops_punc2, bit for bit on the
    interior and NaN elsewhere, as the reference fills it: on the initial data
    (K_ab = 0) and after one RK4 step (K_ab nonzero, so the Codazzi and K K
    terms take part)."""
    c = Case("ops_punc2")
    z = np.load(os.path.join(GOLDEN, "weyl_punc2.npz"))
    ukey, akey, wkey = {"initial": ("u0", "adm0", "weyl0"),
                        "one_step": ("s4_alg", "s4_adm", "weyl1")}[when]
    u, adm = c.rec[ukey], c.rec[akey]
    assert bitwise(z[ukey], u[:, :1, :1, :1, :1])  # the same input state
    if when == "one_step":
        kdd = adm[:, 10:16][c.interior()]  # K_ab, the ADM variables 10..15
        assert np.abs(kdd).max() > 1e-3
    p = _params(c)
    blocks = c.blocks()
    w = np.stack([O.weyl(b, p, adm[g], u[g]) for g, b in enumerate(blocks)])
    ref = z[wkey]
    assert (np.isnan(w) == np.isnan(ref)).all()
    fin = ~np.isnan(ref)
    assert fin.sum() == 2 * 2 * 9 ** 3
    assert bitwise(w[fin], ref[fin])


def test_psi4_extraction():
    """psi4 extraction after the one RK4 step of ops_punc2, piece by piece
    against the reference: the SphericalGrid vertices and weights, the ghost
    exchange of the Weyl register, the SphericalPatch ownership, each block's
    (l, m) projections and their sum over blocks; two spheres, one of which
    leaves the domain."""
    import json
    c = Case("ops_punc2")
    z = np.load(os.path.join(GOLDEN, "weyl_punc2.npz"))
    W = json.loads(str(z["wave"]))
    wx = c.from_grid(O.mesh_exchange(c.nb, c.nx, c.mesh["bc"], c.to_grid(z["weyl1"])))
    assert bitwise(wx, z["wave_weylx"])
    blocks = c.blocks()
    for n in range(W["num_radii"]):
        rad = W[f"radius_{n}"]
        geo = O.sphere_grid(W["nlev"], rad)
        assert bitwise(geo, z[f"wave_geo{n}"])
        total = np.zeros_like(z[f"wave_psi{n}"])
        owned = []
        for g, b in enumerate(blocks):
            own, psi = O.wave_block(b, wx[g], geo, rad, W["lmax"])
            owned += [(g, i) for i in own]
            assert bitwise(psi, z[f"wave_loc{n}"][g]), (n, g)
            total = total + psi
        assert np.array_equal(np.array(owned), z[f"wave_patch{n}"].astype(np.int64))
        assert bitwise(total, z[f"wave_psi{n}"])
    assert len(z["wave_patch0"]) == 10 * W["nlev"] ** 2 + 2  # the inner sphere is whole
    assert 0 < len(z["wave_patch1"]) < 10 * W["nlev"] ** 2 + 2


def test_vc_refinement_operators():
    """Restriction (injection) and prolongation (injection + tensor-product
    Lagrange) of one MeshBlock of a statically refined mesh, bit for bit
    against MeshRefinement's own operators."""
    z = np.load(os.path.join(GOLDEN, "refine_vc.npz"))
    nx = [int(v) for v in z["nx"]]
    fine, coarse = z["rf_fine"], z["rf_coarse"]
    out = O.vc_restrict(nx, fine.copy(), np.zeros_like(coarse), z["rf_rbox"])
    assert bitwise(out, z["rf_restrict"])
    for q in range(4):
        out = O.vc_prolongate(nx, coarse.copy(), fine.copy(), z[f"rf_pbox{q}"])
        assert bitwise(out, z[f"rf_prolong{q}"]), q


def test_puncture_tracker():
    """PunctureTracker: the shift interpolated at the puncture at the start of
    every step, then pos -= dt * beta; matches the reference's tracker file
    (printed with 16 significant digits) on every step."""
    c = Case("evol_track4")
    p = _params(c)
    blocks = c.blocks()
    dt = c.rec["time_dt"][1]
    u = c.rec["u_init"]
    pos = c.rec["tracker_start"].astype(np.float64).copy()
    for row in c.rec["tracker"]:
        owner = [g for g, b in enumerate(blocks) if O.contains_exclusive(b, pos)]
        assert len(owner) == 1
        beta = O.tracker_interp(blocks[owner[0]], u[owner[0]], pos)
        for u in oracle_step(c, p, blocks, u, dt):
            pass
        pos = pos - dt * beta
        got = [float("%.15e" % v) for v in (*pos, *beta)]
        assert got == [float(v) for v in row[2:8]], row[0]
