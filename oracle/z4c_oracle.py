"""ctypes binding of the CPU Z4c oracle (oracle/z4c_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by the CPU-baseline / reference arms of bench.py, as the checker or the timed
CPU baseline.  The product path (gr-athena_b200/) never imports it.

Arrays use the reference layout [var][k][j][i] per block (float64, C order).
"""
import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle_z4c.so")

NG = 4
NVAR, NADM, NCON = 22, 17, 7
BC_PERIODIC, BC_OUTFLOW = 0, 1


class Params(C.Structure):
    """Mirror of z4c_params_t (include/z4c_b200.h)."""

    _fields_ = [(n, C.c_double) for n in (
        "chi_psi_power", "chi_div_floor", "diss", "eps_floor", "damp_kappa1",
        "damp_kappa2", "lapse_oplog", "lapse_harmonicf", "lapse_harmonic",
        "lapse_advect", "lapse_K", "shift_Gamma", "shift_alpha2Gamma", "shift_H",
        "shift_advect", "shift_eta", "r_max_con")] + [
        ("tf_force_regularization", C.c_int), ("force_regularization", C.c_int)]


def default_params(**kw):
    """Reference defaults of z4c.cpp:318-410, overridden by keyword."""
    p = Params(chi_psi_power=-4.0, chi_div_floor=-1000.0, diss=0.0, eps_floor=1e-12,
               damp_kappa1=0.0, damp_kappa2=0.0, lapse_oplog=2.0, lapse_harmonicf=1.0,
               lapse_harmonic=0.0, lapse_advect=1.0, lapse_K=0.0, shift_Gamma=1.0,
               shift_alpha2Gamma=0.0, shift_H=0.0, shift_advect=1.0, shift_eta=2.0,
               r_max_con=math.inf, tf_force_regularization=1, force_regularization=0)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class _Block(C.Structure):
    _fields_ = [("nx", C.c_int * 3), ("dx", C.c_double * 3),
                ("x", C.POINTER(C.c_double) * 3), ("xc", C.POINTER(C.c_double) * 3)]


class _Derivs(C.Structure):
    _fields_ = [("dalpha", C.POINTER(C.c_double) * 3),
                ("dchi", C.POINTER(C.c_double) * 3),
                ("dbeta", (C.POINTER(C.c_double) * 3) * 3),
                ("dg", (C.POINTER(C.c_double) * 6) * 3),
                ("ddchi", C.POINTER(C.c_double) * 6)]


class _Mesh(C.Structure):
    _fields_ = [("nb", C.c_int * 3), ("nx", C.c_int * 3), ("bc", C.c_int * 6)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run make -C oracle)")
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        bp, pp, mp = C.POINTER(_Block), C.POINTER(Params), C.POINTER(_Mesh)
        Dp = C.POINTER(_Derivs)
        L.orc_derivs_alloc.argtypes = [bp, Dp]
        L.orc_derivs_free.argtypes = [Dp]
        L.orc_prepare_derivs.argtypes = [bp, dp, Dp]
        L.orc_rhs.argtypes = [bp, pp, dp, Dp, dp]
        L.orc_boundary_rhs.argtypes = [bp, dp, dp, C.POINTER(C.c_int)]
        L.orc_algconstr.argtypes = [bp, pp, dp]
        L.orc_tracker_interp.argtypes = [bp, dp, dp, dp]
        ip6 = C.POINTER(C.c_int)
        L.orc_vc_restrict.argtypes = [ip6, C.c_int, dp, dp, ip6]
        L.orc_vc_prolongate.argtypes = [ip6, C.c_int, dp, dp, ip6]
        L.orc_regrid_refine.argtypes = [ip6, C.c_int, dp, dp, ip6]
        L.orc_regrid_derefine.argtypes = [ip6, C.c_int, dp, dp, ip6]
        L.orc_algconstr_ghosts.argtypes = [bp, pp, dp]
        L.orc_z4c_to_adm.argtypes = [bp, pp, dp, dp]
        L.orc_z4c_to_adm_ghosts.argtypes = [bp, pp, dp, dp]
        L.orc_adm_to_z4c.argtypes = [bp, pp, dp, dp]
        L.orc_adm_constraints.argtypes = [bp, pp, dp, dp, Dp, dp]
        L.orc_weyl.argtypes = [bp, pp, dp, dp, Dp, dp]
        L.orc_sphere_grid.argtypes = [C.c_int, C.c_double, C.c_int, dp]
        L.orc_sylm.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, dp, dp]
        L.orc_wave_block.argtypes = [bp, dp, C.c_int, dp, C.c_double, C.c_int, C.c_int,
                                     C.POINTER(C.c_int), dp]
        L.orc_mesh_exchange.argtypes = [mp, C.c_int, dp]
        L.orc_ml_exchange.argtypes = [C.POINTER(_MlMesh), C.c_int, dp]
        L.orc_ml_neighbours.argtypes = [C.POINTER(_MlMesh), C.c_int, C.POINTER(C.c_int)]
        L.orc_hst_accumulate.argtypes = [bp, pp, dp, dp, dp]
        _lib = L
    return _lib


def _ptr(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Block:
    """Geometry of one vertex-centred MeshBlock: nx cells per axis, spacing dx,
    vertex coordinates xf[a] (nn entries) and cell centres xv[a] (nn-1)."""

    def __init__(self, nx, dx, xf, xv=None):
        self.nx = tuple(int(n) for n in nx)
        self.nn = tuple(n + 1 + 2 * NG for n in self.nx)
        self.dx = tuple(float(d) for d in dx)
        self.xf = [np.ascontiguousarray(x, dtype=np.float64) for x in xf]
        if xv is None:
            xv = [0.5 * (x[1:] + x[:-1]) for x in self.xf]
        self.xv = [np.ascontiguousarray(x, dtype=np.float64) for x in xv]
        s = _Block()
        for a in range(3):
            s.nx[a] = self.nx[a]
            s.dx[a] = self.dx[a]
            s.x[a] = _ptr(self.xf[a])
            s.xc[a] = _ptr(self.xv[a])
        self._s = s

    def shape(self, nvar):
        return (nvar, self.nn[2], self.nn[1], self.nn[0])


class _DerivsHolder:
    def __init__(self, blk, u):
        self.d = _Derivs()
        if lib().orc_derivs_alloc(C.byref(blk._s), C.byref(self.d)) != 0:
            raise MemoryError("oracle derivative arrays")
        lib().orc_prepare_derivs(C.byref(blk._s), _ptr(u), C.byref(self.d))

    def __del__(self):
        try:
            lib().orc_derivs_free(C.byref(self.d))
        except Exception:
            pass


def rhs(blk, p, u):
    """Z4c::Z4cRHS after PrepareZ4cDerivatives; interior written, rest zero."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    out = np.zeros(blk.shape(NVAR))
    d = _DerivsHolder(blk, u)
    lib().orc_rhs(C.byref(blk._s), C.byref(p), _ptr(u), C.byref(d.d), _ptr(out))
    return out


def sommerfeld_faces(nb, bc, block):
    """Faces (inner_x1, outer_x1, ...) of block `block` of an nb block grid
    that carry gr_sommerfeld (Z4C_BC_SOMMERFELD = 2)."""
    loc = (block % nb[0], (block // nb[0]) % nb[1], block // (nb[0] * nb[1]))
    return [int(bc[2 * a + side] == 2 and loc[a] == (0 if side == 0 else nb[a] - 1))
            for a in range(3) for side in range(2)]


def boundary_rhs(blk, u, rhs, som):
    """Z4c::Z4cBoundaryRHS on the faces flagged in som, in place on rhs."""
    if not any(som):
        return rhs
    u = np.ascontiguousarray(u, dtype=np.float64)
    assert rhs.flags.c_contiguous and rhs.dtype == np.float64
    lib().orc_boundary_rhs(C.byref(blk._s), _ptr(u), _ptr(rhs), (C.c_int * 6)(*som))
    return rhs


def algconstr(blk, p, u, ghosts_only=False):
    out = np.array(u, dtype=np.float64, copy=True, order="C")
    fn = lib().orc_algconstr_ghosts if ghosts_only else lib().orc_algconstr
    fn(C.byref(blk._s), C.byref(p), _ptr(out))
    return out


def z4c_to_adm(blk, p, u, adm=None, ghosts_only=False):
    u = np.ascontiguousarray(u, dtype=np.float64)
    out = np.zeros(blk.shape(NADM)) if adm is None else np.array(adm, copy=True, order="C")
    fn = lib().orc_z4c_to_adm_ghosts if ghosts_only else lib().orc_z4c_to_adm
    fn(C.byref(blk._s), C.byref(p), _ptr(u), _ptr(out))
    return out


def adm_to_z4c(blk, p, adm):
    adm = np.ascontiguousarray(adm, dtype=np.float64)
    out = np.zeros(blk.shape(NVAR))
    lib().orc_adm_to_z4c(C.byref(blk._s), C.byref(p), _ptr(adm), _ptr(out))
    return out


def adm_constraints(blk, p, adm, u):
    adm = np.ascontiguousarray(adm, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.float64)
    out = np.zeros(blk.shape(NCON))
    d = _DerivsHolder(blk, u)
    lib().orc_adm_constraints(C.byref(blk._s), C.byref(p), _ptr(adm), _ptr(u),
                              C.byref(d.d), _ptr(out))
    return out


def weyl(blk, p, adm, u):
    """Z4c::Z4cWeyl: Re and Im psi4 on the interior, NaN elsewhere."""
    adm = np.ascontiguousarray(adm, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.float64)
    out = np.zeros(blk.shape(2))
    d = _DerivsHolder(blk, u)
    lib().orc_weyl(C.byref(blk._s), C.byref(p), _ptr(adm), _ptr(u), C.byref(d.d), _ptr(out))
    return out


def regrid_refine(nx, parent, child, oct):
    """FillSameRankCoarseToFine: child's interior from the parent's octant."""
    parent = np.ascontiguousarray(parent, dtype=np.float64)
    out = np.array(child, dtype=np.float64, copy=True, order="C")
    lib().orc_regrid_refine((C.c_int * 3)(*nx), out.shape[0], _ptr(parent), _ptr(out),
                            (C.c_int * 3)(*[int(v) for v in oct]))
    return out


def regrid_derefine(nx, child, parent, oct):
    """FillSameRankFineToCoarse: the parent's octant from the child."""
    child = np.ascontiguousarray(child, dtype=np.float64)
    out = np.array(parent, dtype=np.float64, copy=True, order="C")
    lib().orc_regrid_derefine((C.c_int * 3)(*nx), out.shape[0], _ptr(child), _ptr(out),
                              (C.c_int * 3)(*[int(v) for v in oct]))
    return out


def sphere_grid(nlev, rad, bitant=False):
    """SphericalGrid(nlev, rad, bitant): rows (theta, phi, x, y, z, weight)."""
    np_ = 10 * nlev * nlev + 2
    out = np.zeros((np_, 6))
    assert lib().orc_sphere_grid(int(nlev), float(rad), int(bitant), _ptr(out)) == np_
    return out


def sylm(s, l, m, theta, phi):
    re, im = C.c_double(), C.c_double()
    lib().orc_sylm(s, l, m, float(theta), float(phi), C.byref(re), C.byref(im))
    return re.value, im.value


def wave_block(blk, weyl, geo, rad, lmax, bitant=False):
    """WaveExtractLocal::Decompose_multipole of one block: (the sphere
    vertices it owns, psi[l-2][m+l][re/im])."""
    weyl = np.ascontiguousarray(weyl, dtype=np.float64)
    geo = np.ascontiguousarray(geo, dtype=np.float64)
    owned = (C.c_int * len(geo))()
    psi = np.zeros((lmax - 1, 2 * lmax + 1, 2))
    n = lib().orc_wave_block(C.byref(blk._s), _ptr(weyl), len(geo), _ptr(geo), float(rad),
                             int(lmax), int(bitant), owned, _ptr(psi))
    return np.array(owned[:n], dtype=np.int64), psi


def mesh_exchange(nb, nx, bc, u_all):
    """Ghost exchange + physical BCs over a uniform block grid; u_all is
    [nblocks][nvar][k][j][i], updated copy returned."""
    out = np.array(u_all, dtype=np.float64, copy=True, order="C")
    m = _Mesh()
    for a in range(3):
        m.nb[a], m.nx[a] = int(nb[a]), int(nx[a])
    for f in range(6):
        m.bc[f] = int(bc[f])
    lib().orc_mesh_exchange(C.byref(m), int(out.shape[1]), _ptr(out))
    return out


class _MlMesh(C.Structure):
    _fields_ = [("nroot", C.c_int * 3), ("root_level", C.c_int), ("nx", C.c_int * 3),
                ("bc", C.c_int * 6), ("nblocks", C.c_int), ("loc", C.POINTER(C.c_int64))]


def _ml_mesh(nroot, root_level, nx, bc, locs):
    loc = np.ascontiguousarray(np.asarray(locs, dtype=np.int64).reshape(-1, 4))
    m = _MlMesh()
    for a in range(3):
        m.nroot[a], m.nx[a] = int(nroot[a]), int(nx[a])
    for f in range(6):
        m.bc[f] = int(bc[f])
    m.root_level, m.nblocks = int(root_level), len(loc)
    m.loc = loc.ctypes.data_as(C.POINTER(C.c_int64))
    return m, loc


def ml_neighbours(nroot, root_level, nx, bc, locs, b):
    """Neighbour list of block b on a multilevel mesh: rows (gid, level, ox1,
    ox2, ox3, fi1, fi2) in the reference's order."""
    m, keep = _ml_mesh(nroot, root_level, nx, bc, locs)
    out = np.zeros((56, 7), dtype=np.int32)
    n = lib().orc_ml_neighbours(C.byref(m), int(b), out.ctypes.data_as(C.POINTER(C.c_int)))
    return out[:n]


def ml_exchange(nroot, root_level, nx, bc, locs, u_all):
    """One ghost fill of a multilevel mesh (locs: per block, gid order,
    {level, lx1, lx2, lx3}); u_all is [nblocks][nvar][k][j][i], updated copy
    returned."""
    out = np.array(u_all, dtype=np.float64, copy=True, order="C")
    m, keep = _ml_mesh(nroot, root_level, nx, bc, locs)
    lib().orc_ml_exchange(C.byref(m), int(out.shape[1]), _ptr(out))
    return out


def hst_norms(blocks, p, con_all, u_all):
    out = np.zeros(8)
    for b, blk in enumerate(blocks):
        lib().orc_hst_accumulate(C.byref(blk._s), C.byref(p),
                                 _ptr(np.ascontiguousarray(con_all[b])),
                                 _ptr(np.ascontiguousarray(u_all[b])), _ptr(out))
    return out


# ---- RK register algebra (mesh/weighted_ave.cpp:20-150, add_z4c_rhs.cpp) ----

def _interior(nn):
    return (slice(None), slice(NG, nn[2] - NG), slice(NG, nn[1] - NG), slice(NG, nn[0] - NG))


def weighted_ave(u_out, u_in1, u_in2, w, nn):
    """WeightedAve_ with the VC interior range, in place on u_out (per block)."""
    s = _interior(nn)
    o, a = u_out[s], u_in1[s]
    if w[0] == 1.0:
        if w[2] != 0.0:
            o += w[1] * a + w[2] * u_in2[s]
        elif w[1] != 0.0:
            o += w[1] * a
    elif w[0] == 0.0:
        if w[2] != 0.0:
            o[...] = w[1] * a + w[2] * u_in2[s]
        elif w[1] == 1.0:
            o[...] = a
        else:
            o[...] = w[1] * a
    else:
        if w[2] != 0.0:
            o[...] = w[0] * o + w[1] * a + w[2] * u_in2[s]
        elif w[1] != 0.0:
            o[...] = w[0] * o + w[1] * a
        else:
            o *= w[0]
    u_out[s] = o


def add_rhs(rhs, wght, u_out, nn):
    s = _interior(nn)
    u_out[s] += wght * rhs[s]


# low-storage RK4()4[2S] weights, task_list_integrators_low_storage.cpp:112-142
LS_RK4 = [
    dict(delta=1.0, gamma_1=0.0, gamma_2=1.0, gamma_3=0.0, beta=1.193743905974738),
    dict(delta=0.217683334308543, gamma_1=0.121098479554482, gamma_2=0.721781678111411,
         gamma_3=0.0, beta=0.099279895495783),
    dict(delta=1.065841341361089, gamma_1=-3.843833699660025, gamma_2=2.121209265338722,
         gamma_3=0.0, beta=1.131678018054042),
    dict(delta=0.0, gamma_1=0.546370891121863, gamma_2=0.198653035682705, gamma_3=0.0,
         beta=0.310665766509336),
]
# classical Butcher RK4, task_list_integrators_butcher.cpp:37-48
BT_RK4_A = [[0, 0, 0, 0], [0.5, 0, 0, 0], [0, 0.5, 0, 0], [0, 0, 1, 0]]
BT_RK4_B = [1. / 6., 1. / 3., 1. / 3., 1. / 6.]


# ---- vertex-centred refinement operators (mesh/mesh_refinement_vc.cpp) ----

def vc_restrict(nx, fine, coarse, box):
    """MeshRefinement::RestrictVertexCenteredValues over the coarse box, in
    place on coarse ([nvar][cn3][cn2][cn1])."""
    assert fine.flags.c_contiguous and coarse.flags.c_contiguous
    lib().orc_vc_restrict((C.c_int * 3)(*nx), fine.shape[0], _ptr(fine), _ptr(coarse),
                          (C.c_int * 6)(*[int(b) for b in box]))
    return coarse


def vc_prolongate(nx, coarse, fine, box):
    """MeshRefinement::ProlongateVertexCenteredValues (3-D) over the coarse
    box, in place on fine ([nvar][nn3][nn2][nn1])."""
    assert fine.flags.c_contiguous and coarse.flags.c_contiguous
    lib().orc_vc_prolongate((C.c_int * 3)(*nx), coarse.shape[0], _ptr(coarse), _ptr(fine),
                            (C.c_int * 6)(*[int(b) for b in box]))
    return fine


# ---- puncture tracker (z4c/puncture_tracker.cpp) ----

def tracker_interp(blk, u, pos):
    """PunctureTracker::InterpolateShift in the block blk (pos inside it)."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    p = np.ascontiguousarray(pos, dtype=np.float64)
    out = np.zeros(3)
    lib().orc_tracker_interp(C.byref(blk._s), _ptr(u), _ptr(p), _ptr(out))
    return out


def contains_exclusive(blk, pos):
    """MeshBlock::PointContainedExclusive (mesh/meshblock.cpp:1186-1201)."""
    return all(blk.xf[a][NG] <= pos[a] < blk.xf[a][NG + blk.nx[a]] for a in range(3))
