"""Statically refined meshes: the multilevel vertex-centred ghost exchange
(restriction, additive unpack with node multiplicity, coarse-level BCs,
prolongation next to coarser blocks, fine-level BCs) and evolution on them.

CPU: the oracle's exchange bit for bit against the reference's on a two-level
mesh (tests/golden/ml_exchange_<bc>.npz: one root block of 2^3 refined once,
outflow and periodic faces), the host-side block tree (which blocks exist,
their gid order and coordinates) against the reference's, and the context's
neighbour search against the oracle's.  GPU: the same exchange through the C
ABI on all 22 variables, and full RK4 / Butcher steps against the oracle."""
import json
import os

import numpy as np
import pytest

import z4c_b200 as Z
import z4c_oracle as O
from z4c_testlib import GOLDEN, bitwise, rel_err

BCS = ("outflow", "periodic")


def _fixture(bc):
    z = np.load(os.path.join(GOLDEN, f"ml_exchange_{bc}.npz"))
    return {k: z[k] for k in z.files}


def hash_state(nblocks, nvar, nn):
    """The integer-hash state the reference driver exchanged (gx_hash)."""
    g, n, k, j, i = np.meshgrid(np.arange(nblocks), np.arange(nvar), np.arange(nn),
                                np.arange(nn), np.arange(nn), indexing="ij")
    return ((g * 131 + n * 31 + k * 7 + j * 3 + i) % 1009) / 1009.0 - 0.5


def _mesh(z, bc=None):
    region = json.loads(str(z["region"]))
    return Z.Mesh(z["nb"], z["nx"], z["xmin"], z["xmax"],
                  bc if bc is not None else [int(z["bc"])] * 6, refinement=[region])


@pytest.mark.parametrize("bc", BCS)
def test_oracle_exchange_matches_reference(bc):
    z = _fixture(bc)
    locs = z["meta"][:, 1:5]
    nb = len(locs)
    u = hash_state(nb, 22, 17)[:, z["vars"]]
    got = O.ml_exchange(z["nb"], 1, z["nx"], [int(z["bc"])] * 6, locs, u)
    assert bitwise(got, z["gx_post"])
    # ghosts next to the coarse blocks were prolonged, not left at zero
    assert np.count_nonzero(got[:, :, :4]) > 0.9 * got[:, :, :4].size


@pytest.mark.parametrize("bc", BCS)
def test_block_tree_matches_reference(bc):
    """Mesh(refinement=...) builds the reference's blocks, gid order and
    vertex coordinates."""
    z = _fixture(bc)
    mesh = _mesh(z)
    assert mesh.root_level == 1
    assert np.array_equal(mesh.locs, z["meta"][:, 1:5])
    nn = mesh.nn[0]
    for b in range(mesh.nblocks):
        (x, y, w), dxs = mesh.block_coords(b)
        assert bitwise(np.concatenate([x, y, w]), z["xf"][b]), b
        assert bitwise(np.array(dxs), z["dx"][b])
    assert mesh.nblocks == 15 and len(x) == nn


def test_deeper_tree_is_balanced():
    """A level-2 region inside a level-1 one: the tree refines the coarse
    neighbours so that adjacent levels differ by one (MeshBlockTree::Refine),
    and the context's neighbour lists equal the oracle's block by block."""
    mesh = Z.Mesh((2, 2, 2), (8, 8, 8), (-4.0,) * 3, (4.0,) * 3, "outflow",
                  refinement=[dict(x1min=0.5, x1max=3.5, x2min=-3.5, x2max=-0.5, x3min=-3.5,
                                   x3max=-0.5, level=1),
                              dict(x1min=0.2, x1max=0.8, x2min=-1.8, x2max=-1.2, x3min=-0.8,
                                   x3max=-0.2, level=2)])
    levels = mesh.locs[:, 0]
    assert set(levels.tolist()) == {2, 3}
    vol = sum(8 ** (3 - lv) for lv in levels)
    assert vol == 8 * 8 ** 2
    for b in range(mesh.nblocks):
        mine = mesh.neighbours(b)
        ref = O.ml_neighbours(mesh.nb, mesh.root_level, mesh.nx, mesh.bc, mesh.locs, b)
        assert np.array_equal(mine, ref), b
        lv = mesh.locs[b, 0]
        assert np.all(np.abs(mine[:, 1] - lv) <= 1)


@pytest.mark.parametrize("bc", BCS)
def test_neighbour_lists_match_oracle(bc):
    z = _fixture(bc)
    mesh = _mesh(z)
    for b in range(mesh.nblocks):
        mine = mesh.neighbours(b)
        ref = O.ml_neighbours(mesh.nb, 1, mesh.nx, mesh.bc, mesh.locs, b)
        assert np.array_equal(mine, ref), b
    # a fine block next to the coarse ones sees coarser faces, edges, corners
    fine = [b for b in range(mesh.nblocks) if mesh.locs[b, 0] == 2]
    assert any((mesh.neighbours(b)[:, 1] == 1).sum() >= 3 for b in fine)


@pytest.mark.parametrize("bc", BCS)
def test_exchange_plan_builds_inside_the_arrays(bc):
    """The whole plan is built and bounds-checked on the host: one
    prolongation box per coarser neighbour of a fine block, boundary faces
    only with outflow faces."""
    import ctypes as C
    z = _fixture(bc)
    mesh = _mesh(z)
    locs = np.ascontiguousarray(mesh.locs, dtype=np.int64)
    out = np.zeros(56 * 7, dtype=np.int32)
    n = Z.lib().z4c_refined_neighbours(C.byref(mesh.desc()), len(locs),
                                       locs.ctypes.data_as(C.POINTER(C.c_longlong)), -2,
                                       out.ctypes.data_as(C.POINTER(C.c_int)))
    assert n == 4
    nunpack, moved, npro, nbc = out[:4]
    ncoarser = sum((mesh.neighbours(b)[:, 1] < mesh.locs[b, 0]).sum()
                   for b in range(mesh.nblocks))
    assert npro == ncoarser > 0
    assert moved > nunpack > 26 * mesh.nblocks // 2
    assert (nbc > 0) == (bc == "outflow")


def test_bad_tilings_are_rejected():
    mesh = Z.Mesh((2, 2, 2), (8, 8, 8), (-4.0,) * 3, (4.0,) * 3, "outflow")
    root = np.array([(1, i, j, k) for k in range(2) for j in range(2) for i in range(2)])

    def check(locs):
        m = Z.Mesh(mesh.nb, mesh.nx, mesh.xmin, mesh.xmax, mesh.bc)
        m.locs = np.array(locs, dtype=np.int64)
        with pytest.raises(Z.Z4cError):
            m.neighbours(0)

    check(root[:7])                                    # a hole
    check(np.vstack([root, [[2, 0, 0, 0]]]))           # a block inside another
    check(np.vstack([root[:7], root[6:7]]))            # a duplicate
    # level 3 next to level 1 (2:1 balance broken)
    fine = [(2, 2 + (c & 1), (c >> 1) & 1, (c >> 2) & 1) for c in range(8)]
    finer = [(3, 4 + (c & 1), (c >> 1) & 1, (c >> 2) & 1) for c in range(8)]
    check([tuple(r) for r in root if tuple(r) != (1, 1, 0, 0)] + fine[1:] + finer)


@pytest.mark.gpu
@pytest.mark.parametrize("bc", BCS)
def test_exchange_matches_reference_and_oracle(bc):
    z = _fixture(bc)
    mesh = _mesh(z)
    ctx = Z.Z4c(mesh, Z.default_params(), "rk4")
    u = hash_state(mesh.nblocks, 22, 17)
    ctx.upload(Z.REG_U, u)
    ctx.ghost_fill(Z.REG_U)
    got = ctx.download(Z.REG_U)
    assert bitwise(got[:, z["vars"]], z["gx_post"])
    ref = O.ml_exchange(mesh.nb, mesh.root_level, mesh.nx, mesh.bc, mesh.locs, u)
    assert bitwise(got, ref)
    ctx.close()


def sommerfeld_faces(mesh, b):
    """gr_sommerfeld faces of block b of a refined mesh, from its logical
    location at its level."""
    lev, *loc = (int(v) for v in mesh.locs[b])
    n = [mesh.nb[a] << (lev - mesh.root_level) for a in range(3)]
    return [int(mesh.bc[2 * a + side] == 2 and loc[a] == (0 if side == 0 else n[a] - 1))
            for a in range(3) for side in range(2)]


def oracle_ml_step(mesh, p, u, dt, integ):
    """One GR_Z4c step on the oracle over a refined mesh."""
    nb = mesh.nblocks
    nn = mesh.nn
    blocks = []
    for b in range(nb):
        xs, dxs = mesh.block_coords(b)
        blocks.append(O.Block(mesh.nx, dxs, xs))
    som = [sommerfeld_faces(mesh, b) for b in range(nb)]

    def rhs(v):
        r = np.stack([O.rhs(blocks[b], p, v[b]) for b in range(nb)])
        for b in range(nb):
            O.boundary_rhs(blocks[b], v[b], r[b], som[b])
        return r

    def exchange(v):
        v = O.ml_exchange(mesh.nb, mesh.root_level, mesh.nx, mesh.bc, mesh.locs, v)
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


@pytest.mark.gpu
@pytest.mark.parametrize("integ,bc", [("rk4", "outflow"), ("bt_rk4", "outflow"),
                                      ("rk4", "periodic"), ("rk4", "sommerfeld"),
                                      ("bt_rk4", "sommerfeld")])
def test_step_on_refined_mesh_matches_oracle(integ, bc):
    """A binary puncture straddling the level boundary: one full step
    (gr_sommerfeld: the outflow fixture's mesh with Sommerfeld faces, whose
    right-hand side is overridden on the coarse and the fine blocks' faces)."""
    from z4c_b200 import initial_data as ID
    params = dict(diss=0.02, chi_div_floor=1e-5, damp_kappa1=0.02, damp_kappa2=0.0,
                  shift_eta=2.0, r_max_con=1e300)
    z = _fixture("outflow" if bc == "sommerfeld" else bc)
    mesh = _mesh(z, [2] * 6 if bc == "sommerfeld" else None)
    ctx = Z.Z4c(mesh, Z.default_params(**params), integ)
    ID.load_adm(ctx, ID.punctures(mesh, ctx.params, masses=(0.5, 0.5),
                                  centres=((0.9, -1.1, -0.7), (-1.2, 0.3, 0.2))))
    ctx.ghost_fill(Z.REG_U)
    u0 = ctx.download(Z.REG_U)
    dt = mesh.new_dt(0.25)
    assert dt == 0.25 * 0.25  # the fine blocks' spacing
    ctx.evolve(dt, 1)
    got = ctx.download(Z.REG_U)
    assert np.isfinite(got).all()
    ref = oracle_ml_step(mesh, O.default_params(**params), u0, dt, integ)
    assert rel_err(got, ref) <= 1e-12
    ctx.close()


def _refined_binary(bc="outflow", integ="rk4"):
    from z4c_b200 import initial_data as ID
    params = dict(diss=0.02, chi_div_floor=1e-5, damp_kappa1=0.02, damp_kappa2=0.0,
                  shift_eta=2.0, r_max_con=1e300)
    mesh = _mesh(_fixture(bc))
    ctx = Z.Z4c(mesh, Z.default_params(**params), integ)
    ID.load_adm(ctx, ID.punctures(mesh, ctx.params, masses=(0.5, 0.5),
                                  centres=((0.9, -1.1, -0.7), (-1.2, 0.3, 0.2))))
    return mesh, ctx, params


@pytest.mark.gpu
def test_tracker_on_refined_mesh_matches_oracle():
    """Two trackers, one in a fine block and one in a coarse block: the shift
    interpolated in the owning block at the start of the step, then
    pos -= dt beta (PunctureTracker::InterpolateShift / EvolveTracker)."""
    mesh, ctx, _ = _refined_binary()
    u0 = ctx.download(Z.REG_U)
    starts = [(1.37, -0.61, -1.23), (-1.45, 0.55, 0.35)]
    ids = [ctx.add_tracker(p) for p in starts]
    dt = mesh.new_dt(0.25)
    ctx.evolve(dt, 1)
    levels = []
    for tid, p in zip(ids, starts):
        owners = []
        for b in range(mesh.nblocks):
            xs, dxs = mesh.block_coords(b)
            blk = O.Block(mesh.nx, dxs, xs)
            if O.contains_exclusive(blk, p):
                owners.append(b)
        assert len(owners) == 1
        b = owners[0]
        levels.append(int(mesh.locs[b, 0]))
        xs, dxs = mesh.block_coords(b)
        beta = O.tracker_interp(O.Block(mesh.nx, dxs, xs), u0[b], p)
        pos, got_beta = ctx.tracker(tid)
        assert rel_err(np.asarray(got_beta), beta) <= 1e-13
        assert np.allclose(pos, np.asarray(p) - dt * beta, rtol=0, atol=1e-15)
    assert sorted(levels) == [1, 2]
    ctx.close()


@pytest.mark.gpu
def test_extraction_on_refined_mesh_matches_oracle():
    """psi4 multipoles on spheres that cross both levels: per-block
    projections summed over the blocks in gid order (the context's order on
    a refined mesh)."""
    mesh, ctx, _ = _refined_binary()
    ctx.evolve(mesh.new_dt(0.25), 1)
    spheres = [Z.WaveExtract(ctx, r, 10, 4) for r in (1.9, 3.1)]
    psis = ctx.psi4_multipoles(spheres)
    weyl = ctx.download(Z.REG_WEYL)
    assert np.isfinite(weyl).all()
    for w, psi in zip(spheres, psis):
        geo = O.sphere_grid(w.nlev, w.radius)
        total = np.zeros_like(psi)
        owned, lv = 0, set()
        for b in range(mesh.nblocks):
            xs, dxs = mesh.block_coords(b)
            own, loc = O.wave_block(O.Block(mesh.nx, dxs, xs), weyl[b], geo, w.radius, w.lmax)
            if len(own):
                lv.add(int(mesh.locs[b, 0]))
            owned += len(own)
            total = total + loc
        assert w.num_points() == owned == len(geo)
        assert lv == {1, 2}
        assert rel_err(psi, total) <= 1e-12
        assert np.abs(total).max() > 0
    ctx.close()


@pytest.mark.gpu
def test_constraints_and_history_on_refined_mesh_match_oracle():
    """ADMConstraints on every block (each with its own spacing) after a step
    with constraints, and the history norms summed over blocks of both
    levels, each weighted by its own cell volume."""
    mesh, ctx, params = _refined_binary()
    ctx.evolve(mesh.new_dt(0.25), 1, with_constraints=True)
    u = ctx.download(Z.REG_U)
    adm = ctx.download(Z.REG_ADM)
    con = ctx.download(Z.REG_CON)
    got = ctx.hst_norms()
    p = O.default_params(**params)
    blocks = []
    ref_con = np.empty_like(con)
    for b in range(mesh.nblocks):
        xs, dxs = mesh.block_coords(b)
        blk = O.Block(mesh.nx, dxs, xs)
        blocks.append(blk)
        ref_con[b] = O.adm_constraints(blk, p, adm[b], u[b])
    assert rel_err(con, ref_con) <= 1e-11
    ref = O.hst_norms(blocks, p, ref_con, u)
    np.testing.assert_allclose(got, ref, rtol=1e-9)
    assert got[0] > 0
    ctx.close()


@pytest.mark.gpu
def test_regrid_moves_the_refined_region_like_the_oracle():
    """A regrid that derefines the refined root block and refines another
    one: kept blocks copied, the new children prolonged from their parent
    (FillSameRankCoarseToFine), the new parent restricted from its eight
    children (FillSameRankFineToCoarse), then the ghost fill of the new
    mesh; against the oracle's transfers and exchange, and the tracker
    carried along."""
    mesh, ctx, params = _refined_binary()
    ctx.add_tracker((0.31, 0.27, -0.22))
    ctx.evolve(mesh.new_dt(0.25), 1)
    old = ctx.download(Z.REG_U)
    trk = ctx.tracker(0)
    moved = Z.Mesh(mesh.nb, mesh.nx, mesh.xmin, mesh.xmax, mesh.bc,
                   refinement=[dict(x1min=-3.5, x1max=-0.5, x2min=0.5, x2max=3.5, x3min=0.5,
                                    x3max=3.5, level=1)])
    new = Z.Z4c(moved, Z.default_params(**params), "rk4")
    new.regrid_from(ctx)
    got = new.download(Z.REG_U)
    # the oracle: transfers block by block, then exchange + AlgConstr on ghosts
    sidx = {tuple(l): b for b, l in enumerate(mesh.locs.tolist())}
    ref = np.zeros_like(got)
    kinds = set()
    for b, (lv, x, y, z) in enumerate(moved.locs.tolist()):
        if (lv, x, y, z) in sidx:
            ref[b] = old[sidx[(lv, x, y, z)]]
            kinds.add("kept")
        elif (lv - 1, x >> 1, y >> 1, z >> 1) in sidx:
            ref[b] = O.regrid_refine(mesh.nx, old[sidx[(lv - 1, x >> 1, y >> 1, z >> 1)]],
                                     ref[b], (x & 1, y & 1, z & 1))
            kinds.add("refined")
        else:
            for c in range(8):
                o = (c & 1, (c >> 1) & 1, (c >> 2) & 1)
                ch = sidx[(lv + 1, 2 * x + o[0], 2 * y + o[1], 2 * z + o[2])]
                ref[b] = O.regrid_derefine(mesh.nx, old[ch], ref[b], o)
            kinds.add("derefined")
    assert kinds == {"kept", "refined", "derefined"}
    ref = O.ml_exchange(moved.nb, moved.root_level, moved.nx, moved.bc, moved.locs, ref)
    p = O.default_params(**params)
    for b in range(moved.nblocks):
        xs, dxs = moved.block_coords(b)
        ref[b] = O.algconstr(O.Block(moved.nx, dxs, xs), p, ref[b], ghosts_only=True)
    assert rel_err(got, ref) <= 1e-14
    np.testing.assert_array_equal(np.concatenate(new.tracker(0)), np.concatenate(trk))
    new.evolve(moved.new_dt(0.25), 1)
    assert new.check_finite()
    ctx.close()
    new.close()
