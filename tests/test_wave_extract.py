"""psi4 extraction (WaveExtract, z4c/wave_extract.cpp) through the C ABI.

CPU: the library's own SphericalGrid (vertices, polar angles, weights) bit for
bit against the reference's.  GPU: the Weyl ghost exchange and the sphere
multipoles against the reference's records on the puncture of ops_punc2
(after its one RK4 step), and against the oracle on an evolved binary on 64
MeshBlocks, where the blocks' gid (Morton) order differs from the context's
grid order."""
import json
import os

import numpy as np
import pytest

import z4c_b200 as Z
from z4c_testlib import GOLDEN, NG, Case, bitwise, rel_err

TOL = 1e-12  # normwise relative, as every parity test of the RHS


def _fixture():
    z = np.load(os.path.join(GOLDEN, "weyl_punc2.npz"))
    return z, json.loads(str(z["wave"]))


def test_sphere_grid_matches_reference():
    z, W = _fixture()
    for n in range(W["num_radii"]):
        geo = Z.sphere_grid(W["nlev"], W[f"radius_{n}"])
        assert bitwise(geo, z[f"wave_geo{n}"]), n


def test_sphere_grid_properties():
    """Unit-sphere weights sum to 4 pi; bitant folds z to z >= 0."""
    for nlev in (1, 4, 11):
        geo = Z.sphere_grid(nlev, 2.0)
        assert geo.shape == (10 * nlev * nlev + 2, 6)
        assert abs(geo[:, 5].sum() / 4.0 - 4 * np.pi) < 1e-12
        np.testing.assert_allclose(np.linalg.norm(geo[:, 2:5], axis=1), 2.0, rtol=1e-14)
    assert (Z.sphere_grid(5, 1.0, bitant=True)[:, 4] >= 0).all()
    with pytest.raises(Z.Z4cError):
        Z.sphere_grid(0, 1.0)


@pytest.mark.gpu
def test_extraction_matches_reference():
    c = Case("ops_punc2")
    z, W = _fixture()
    m = c.mesh
    mesh = Z.Mesh(m["nb"], m["nx"], m["xmin"], m["xmax"], m["bc"])
    ctx = Z.Z4c(mesh, Z.default_params(**c.params), c.integrator)
    ctx.upload(Z.REG_U, c.to_grid(c.rec["s4_alg"]))
    ctx.upload(Z.REG_ADM, c.to_grid(c.rec["s4_adm"]))
    spheres = [Z.WaveExtract(ctx, W[f"radius_{n}"], W["nlev"], W["lmax"])
               for n in range(W["num_radii"])]
    ctx.Z4cWeyl()
    ctx.ghost_fill(Z.REG_WEYL)
    wx = c.from_grid(ctx.download(Z.REG_WEYL))
    assert np.isfinite(wx).all()
    assert rel_err(wx, z["wave_weylx"]) <= TOL
    for n, w in enumerate(spheres):
        assert w.num_points() == len(z[f"wave_patch{n}"])
        psi = w.ReduceMultipole()
        assert rel_err(psi, z[f"wave_psi{n}"]) <= TOL, n
    ctx.close()


@pytest.mark.gpu
def test_extraction_on_evolved_binary_matches_oracle(tmp_path):
    """64 blocks of 16^3 (gid order = Morton order of the 4^3 block grid), two
    spheres, one crossing many block faces; the oracle projects per block and
    sums over blocks in gid order."""
    import z4c_oracle as O
    from z4c_b200 import initial_data as ID
    params = dict(diss=0.02, chi_div_floor=1e-5, damp_kappa1=0.02, damp_kappa2=0.0,
                  shift_eta=2.0, r_max_con=1e300)
    mesh = Z.Mesh((4, 4, 4), (16, 16, 16), (-6.0,) * 3, (6.0,) * 3, "outflow")
    ctx = Z.Z4c(mesh, Z.default_params(**params), "rk4")
    ID.load_adm(ctx, ID.punctures(mesh, ctx.params, masses=(0.5, 0.5),
                                  centres=((1.3, 0.2, 0.1), (-1.3, -0.25, 0.0))))
    ctx.evolve(0.25 * float(ctx.dx().min()), 2)
    spheres = [Z.WaveExtract(ctx, r, 12, 4, filename=str(tmp_path / "wave")) for r in (2.7, 4.5)]
    psis = ctx.psi4_multipoles(spheres)
    weyl = ctx.download(Z.REG_WEYL)
    assert np.isfinite(weyl).all()

    def morton(b):  # interleaved bits of the logical location, x lowest
        loc = (b % 4, (b // 4) % 4, b // 16)
        return sum(((loc[a] >> i) & 1) << (3 * i + a) for i in range(2) for a in range(3))

    order = sorted(range(64), key=morton)
    assert order != list(range(64))
    for w, psi in zip(spheres, psis):
        geo = O.sphere_grid(w.nlev, w.radius)
        total = np.zeros_like(psi)
        owned = 0
        for b in order:
            xs, dxs = mesh.block_coords(b)
            own, loc = O.wave_block(O.Block(mesh.nx, dxs, xs), weyl[b], geo, w.radius, w.lmax)
            owned += len(own)
            total = total + loc
        assert w.num_points() == owned == len(geo)
        assert rel_err(psi, total) <= TOL
        assert np.abs(total).max() > 0
        w.Write(3, 0.5)
        w.Write(4, 0.75)
        lines = open(w.ofname).read().splitlines()
        assert lines[0].startswith("# 1:iter 2:time 3:l=2-m=-2-Re 4:l=2-m=-2-Im")
        assert len(lines) == 3 and len(lines[1].split()) == 2 + 2 * 21
    ctx.close()
