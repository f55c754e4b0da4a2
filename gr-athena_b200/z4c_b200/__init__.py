"""Host-side mirror of the GR-Athena++ Z4c operator interface over the B200
C ABI (include/z4c_b200.h, library gr-athena_b200/_build/libz4c_b200.so).

The class :class:`Z4c` carries the reference member-function names
(src/z4c/z4c.hpp:448-539): ``Z4cRHS``, ``AddZ4cRHS``, ``WeightedAve``,
``ADMToZ4c``, ``Z4cToADM``, ``ADMConstraints``, ``AlgConstr``, plus the task
list pieces (ghost fill, stages, whole steps).  Registers stay on the device;
numpy arrays in the reference layout ``[block][var][k][j][i]`` move across
the boundary only through ``upload``/``download``.

There is no CPU fallback: constructing a context without the built library
or without a CUDA device raises.
"""
import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "_build", "libz4c_b200.so")

NG = 4
NVAR, NADM, NCON, NWEYL = 22, 17, 7, 2
(CHI, GXX, GXY, GXZ, GYY, GYZ, GZZ, KHAT, AXX, AXY, AXZ, AYY, AYZ, AZZ,
 GAMX, GAMY, GAMZ, THETA, ALPHA, BETAX, BETAY, BETAZ) = range(22)
(ADM_ALPHA, ADM_BETAX, ADM_BETAY, ADM_BETAZ, ADM_GXX, ADM_GXY, ADM_GXZ, ADM_GYY,
 ADM_GYZ, ADM_GZZ, ADM_KXX, ADM_KXY, ADM_KXZ, ADM_KYY, ADM_KYZ, ADM_KZZ,
 ADM_PSI4) = range(17)
CON_C, CON_H, CON_M, CON_Z, CON_MX, CON_MY, CON_MZ = range(7)
(REG_U, REG_U1, REG_RHS, REG_ADM, REG_CON, REG_W, REG_K1, REG_K2, REG_K3,
 REG_K4, REG_WEYL, REG_TAN, REG_ADJ, REG_ADM_ADJ) = range(14)
BC_PERIODIC, BC_OUTFLOW, BC_SOMMERFELD = 0, 1, 2
BC_NAMES = {"periodic": BC_PERIODIC, "outflow": BC_OUTFLOW, "extrapolate_outflow": BC_OUTFLOW,
            "sommerfeld": BC_SOMMERFELD, "gr_sommerfeld": BC_SOMMERFELD}
INTEG = {"rk4": 0, "bt_rk4": 1}
ERRORS = {-1: "EINVAL", -2: "ENOMEM", -3: "ECUDA", -4: "ENONFINITE", -5: "ETIMEOUT",
          -6: "ESTATE", -7: "ENODEV"}
HST_COLUMNS = ("H-norm2", "M-norm2", "Mx-norm2", "My-norm2", "Mz-norm2", "Z-norm2",
               "Theta-norm2", "C-norm2")

# symbols the library must export (one per declaration in include/z4c_b200.h)
EXPORTS = (
    "z4c_params_default", "z4c_last_error", "z4c_create", "z4c_destroy",
    "z4c_set_stream", "z4c_sync", "z4c_num_blocks", "z4c_block_nn", "z4c_reg_nvar",
    "z4c_dx", "z4c_block_coords", "z4c_mesh_block_coords", "z4c_mesh_new_dt",
    "z4c_mesh_loc_coords", "z4c_create_refined", "z4c_refined_neighbours", "z4c_restart_locs",
    "z4c_regrid", "z4c_upload", "z4c_download", "z4c_device_ptr",
    "z4c_rhs", "z4c_boundary_rhs", "z4c_add_rhs", "z4c_weighted_ave", "z4c_alg_constr", "z4c_adm_to_z4c",
    "z4c_z4c_to_adm", "z4c_adm_constraints", "z4c_weyl", "z4c_ghost_fill", "z4c_init_finalize",
    "z4c_hst_norms", "z4c_stage", "z4c_evolve", "z4c_evolve_jobs", "z4c_set_per_block", "z4c_set_tile",
    "z4c_get_tile", "z4c_autotune", "z4c_check_finite", "z4c_kernel_launches", "z4c_rhs_stage",
    "z4c_fp64_probe", "z4c_tracker_add", "z4c_tracker_get", "z4c_vc_restrict", "z4c_vc_prolongate",
    "z4c_regrid_refine", "z4c_regrid_derefine", "z4c_rhs_noalloc",
    "z4c_sphere_grid", "z4c_wave_add", "z4c_wave_points", "z4c_wave_decompose",
    "z4c_restart_info", "z4c_restart_text", "z4c_restart_read", "z4c_restart_write_host",
    "z4c_restart_load", "z4c_restart_save", "z4c_adj_setup", "z4c_tlm_step", "z4c_adj_step",
    "z4c_adj_objective", "z4c_adj_objective_adj", "z4c_adj_params", "z4c_adj_gradient",
    "z4c_adj_adm_to_z4c", "z4c_set_contract", "z4c_get_contract", "z4c_set_point_regs",
    "z4c_get_point_regs", "z4c_adj_snapshots", "z4c_adj_set_weyl", "z4c_set_merged",
    "z4c_get_merged")


class Z4cError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Params(C.Structure):
    """z4c_params_t; defaults of the reference (z4c.cpp:318-410)."""

    _fields_ = [(n, C.c_double) for n in (
        "chi_psi_power", "chi_div_floor", "diss", "eps_floor", "damp_kappa1",
        "damp_kappa2", "lapse_oplog", "lapse_harmonicf", "lapse_harmonic",
        "lapse_advect", "lapse_K", "shift_Gamma", "shift_alpha2Gamma", "shift_H",
        "shift_advect", "shift_eta", "r_max_con")] + [
        ("tf_force_regularization", C.c_int), ("force_regularization", C.c_int)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class RestartInfo(C.Structure):
    _fields_ = [("nbtotal", C.c_int), ("root_level", C.c_int), ("xmin", C.c_double * 3),
                ("xmax", C.c_double * 3), ("xrat", C.c_double * 3), ("mesh_nx", C.c_int * 3),
                ("time", C.c_double), ("dt", C.c_double), ("ncycle", C.c_int),
                ("datasize", C.c_ulonglong), ("nb", C.c_int * 3), ("block_nx", C.c_int * 3),
                ("ntrackers", C.c_int), ("trackers", (C.c_double * 6) * 8),
                ("text_bytes", C.c_longlong), ("nlevels", C.c_int)]


class MeshDesc(C.Structure):
    _fields_ = [("nb", C.c_int * 3), ("nx", C.c_int * 3), ("xmin", C.c_double * 3),
                ("xmax", C.c_double * 3), ("bc", C.c_int * 6)]


_lib = None


def lib():
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"z4c_b200 library not built: {LIB_PATH} "
                               "(run python gr-athena_b200/build.py)")
        L = C.CDLL(LIB_PATH)
        vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.c_int
        L.z4c_last_error.restype = C.c_char_p
        L.z4c_params_default.argtypes = [C.POINTER(Params)]
        L.z4c_params_default.restype = None
        L.z4c_create.argtypes = [C.POINTER(MeshDesc), C.POINTER(Params), ip, C.POINTER(vp)]
        L.z4c_destroy.argtypes = [vp]
        L.z4c_set_stream.argtypes = [vp, vp]
        L.z4c_sync.argtypes = [vp]
        L.z4c_num_blocks.argtypes = [vp]
        L.z4c_block_nn.argtypes = [vp, ip]
        L.z4c_reg_nvar.argtypes = [ip]
        L.z4c_dx.argtypes = [vp, dp]
        L.z4c_block_coords.argtypes = [vp, ip, ip, dp]
        L.z4c_mesh_block_coords.argtypes = [C.POINTER(MeshDesc), ip, ip, dp, dp]
        L.z4c_mesh_new_dt.argtypes = [C.POINTER(MeshDesc), C.c_double, dp]
        L.z4c_mesh_loc_coords.argtypes = [C.POINTER(MeshDesc), C.POINTER(C.c_longlong), ip, dp,
                                          dp]
        L.z4c_create_refined.argtypes = [C.POINTER(MeshDesc), ip, C.POINTER(C.c_longlong),
                                         C.POINTER(Params), ip, C.POINTER(vp)]
        L.z4c_restart_locs.argtypes = [C.c_char_p, C.POINTER(C.c_longlong), ip]
        L.z4c_regrid.argtypes = [vp, vp]
        L.z4c_refined_neighbours.argtypes = [C.POINTER(MeshDesc), ip, C.POINTER(C.c_longlong),
                                             ip, C.POINTER(C.c_int)]
        L.z4c_upload.argtypes = [vp, ip, ip, dp]
        L.z4c_download.argtypes = [vp, ip, ip, dp]
        L.z4c_device_ptr.argtypes = [vp, ip, C.POINTER(dp)]
        L.z4c_rhs.argtypes = [vp, ip, ip, ip]
        L.z4c_boundary_rhs.argtypes = [vp, ip, ip, ip]
        L.z4c_add_rhs.argtypes = [vp, ip, C.c_double, ip, ip]
        L.z4c_weighted_ave.argtypes = [vp, ip, ip, ip, dp, ip]
        L.z4c_alg_constr.argtypes = [vp, ip, ip]
        L.z4c_adm_to_z4c.argtypes = [vp, ip, ip, ip]
        L.z4c_z4c_to_adm.argtypes = [vp, ip, ip, ip]
        L.z4c_adm_constraints.argtypes = [vp, ip, ip, ip, ip]
        L.z4c_weyl.argtypes = [vp, ip, ip, ip, ip]
        L.z4c_ghost_fill.argtypes = [vp, ip]
        L.z4c_init_finalize.argtypes = [vp]
        L.z4c_hst_norms.argtypes = [vp, dp]
        L.z4c_stage.argtypes = [vp, ip, C.c_double]
        L.z4c_evolve.argtypes = [vp, C.c_double, ip, ip]
        L.z4c_evolve_jobs.argtypes = [vp, ip, C.POINTER(vp), C.POINTER(vp), dp, C.c_double, ip]
        L.z4c_set_per_block.argtypes = [vp, ip]
        L.z4c_set_tile.argtypes = [vp, ip, ip, ip]
        L.z4c_get_tile.argtypes = [vp, C.POINTER(C.c_int)]
        L.z4c_set_contract.argtypes = [vp, ip]
        L.z4c_set_merged.argtypes = [vp, ip]
        L.z4c_get_merged.argtypes = [vp, C.POINTER(C.c_int)]
        L.z4c_get_contract.argtypes = [vp, C.POINTER(C.c_int)]
        L.z4c_set_point_regs.argtypes = [vp, ip]
        L.z4c_adj_snapshots.argtypes = [vp, ip, C.POINTER(C.c_int)]
        L.z4c_adj_set_weyl.argtypes = [vp, ip, C.c_double]
        L.z4c_get_point_regs.argtypes = [vp, C.POINTER(C.c_int)]
        L.z4c_autotune.argtypes = [vp, ip, C.POINTER(C.c_float)]
        L.z4c_check_finite.argtypes = [vp, ip]
        L.z4c_rhs_stage.argtypes = [vp, ip, C.c_double]
        L.z4c_fp64_probe.argtypes = [vp, dp]
        ipp = C.POINTER(C.c_int)
        L.z4c_tracker_add.argtypes = [vp, dp, ipp]
        L.z4c_tracker_get.argtypes = [vp, ip, dp]
        L.z4c_vc_restrict.argtypes = [vp, vp, ip, ip, ipp, ipp, vp]
        L.z4c_vc_prolongate.argtypes = [vp, vp, ip, ip, ipp, ipp, vp]
        L.z4c_regrid_refine.argtypes = [vp, vp, vp, ip, ipp, ipp, vp]
        L.z4c_regrid_derefine.argtypes = [vp, vp, vp, ip, ipp, ipp, vp]
        L.z4c_rhs_noalloc.argtypes = [vp, vp, ip, C.POINTER(C.c_int), dp,
                                      C.POINTER(Params), vp]
        L.z4c_sphere_grid.argtypes = [ip, C.c_double, ip, dp]
        L.z4c_wave_add.argtypes = [vp, C.c_double, ip, ip, ip, ipp]
        L.z4c_wave_points.argtypes = [vp, ip]
        L.z4c_wave_decompose.argtypes = [vp, ip, ip, dp]
        cp = C.c_char_p
        L.z4c_restart_info.argtypes = [cp, C.POINTER(RestartInfo)]
        L.z4c_restart_text.argtypes = [cp, C.c_char_p, C.c_longlong]
        L.z4c_restart_text.restype = C.c_longlong
        L.z4c_restart_read.argtypes = [cp, dp]
        L.z4c_restart_write_host.argtypes = [cp, cp, C.POINTER(MeshDesc), dp, C.c_double,
                                             C.c_double, ip, ip, dp]
        L.z4c_restart_load.argtypes = [vp, cp, C.POINTER(RestartInfo)]
        L.z4c_restart_save.argtypes = [vp, cp, cp, C.c_double, C.c_double, ip]
        L.z4c_adj_setup.argtypes = [vp]
        L.z4c_tlm_step.argtypes = [vp, C.c_double]
        L.z4c_adj_step.argtypes = [vp, C.c_double]
        L.z4c_adj_objective.argtypes = [vp, ip, ip, dp, dp]
        L.z4c_adj_objective_adj.argtypes = [vp, ip, C.c_double]
        L.z4c_adj_params.argtypes = [vp, dp, ip]
        L.z4c_adj_adm_to_z4c.argtypes = [vp]
        L.z4c_adj_gradient.argtypes = [vp, C.c_double, ip, ip, C.c_double, C.c_double, dp, dp,
                                       dp]
        L.z4c_kernel_launches.argtypes = []
        L.z4c_kernel_launches.restype = C.c_longlong
        _lib = L
    return _lib


def _check(rc):
    if rc < 0:
        raise Z4cError(rc, lib().z4c_last_error().decode())
    return rc


def sphere_grid(nlev, rad, bitant=False):
    """SphericalGrid(nlev, rad, bitant) on the host: one row (theta, phi, x,
    y, z, weight) per geodesic vertex."""
    out = np.empty((10 * nlev * nlev + 2, 6))
    _check(lib().z4c_sphere_grid(int(nlev), float(rad), int(bool(bitant)),
                                 out.ctypes.data_as(C.POINTER(C.c_double))))
    return out


class WaveExtract:
    """WaveExtract (z4c/wave_extract.cpp): the (l, m) multipoles of psi4 on
    one coordinate sphere, 2 <= l <= lmax, as psi[l-2, m+l, re/im]; the
    <psi4_extraction> parameters nlev (default 3), radius_n (10.0), lmax (2),
    filename ("wave") and <mesh> bitant."""

    def __init__(self, ctx, radius=10.0, nlev=3, lmax=2, bitant=False, filename="wave"):
        self.ctx, self.radius, self.nlev, self.lmax = ctx, float(radius), int(nlev), int(lmax)
        i = C.c_int()
        _check(lib().z4c_wave_add(ctx._h, self.radius, self.nlev, self.lmax, int(bool(bitant)),
                                  C.byref(i)))
        self.id = i.value
        self.psi = np.zeros((self.lmax - 1, 2 * self.lmax + 1, 2))
        self.ofname = f"{filename}_r{self.radius:05.2f}.txt"

    def num_points(self):
        """Sphere vertices owned by some MeshBlock."""
        return _check(lib().z4c_wave_points(self.ctx._h, self.id))

    def ReduceMultipole(self, reg_weyl=REG_WEYL):
        """Decompose_multipole on every block plus the sum over blocks, from
        the Weyl register (ghosts filled)."""
        out = np.zeros_like(self.psi)
        _check(lib().z4c_wave_decompose(self.ctx._h, self.id, reg_weyl,
                                        out.ctypes.data_as(C.POINTER(C.c_double))))
        self.psi = out
        return out

    def Write(self, iteration, time):
        """Appends one line to the reference's wave_r<radius>.txt format,
        writing the column header first when the file is new."""
        new = not os.path.exists(self.ofname)
        with open(self.ofname, "a") as f:
            if new:
                cols, idx = ["# 1:iter 2:time"], 3
                for l in range(2, self.lmax + 1):
                    for m in range(-l, l + 1):
                        cols.append(f" {idx}:l={l}-m={m}-Re {idx + 1}:l={l}-m={m}-Im")
                        idx += 2
                f.write("".join(cols) + "\n")
            line = [f"{int(iteration)} {time:.17g} "]
            for l in range(2, self.lmax + 1):
                for m in range(-l, l + 1):
                    line.append(f"{self.psi[l - 2, m + l, 0]:.17g} {self.psi[l - 2, m + l, 1]:.17g} ")
            f.write("".join(line) + "\n")


def kernel_launches():
    """Kernels this library has launched in this process (graph replays
    count every kernel node)."""
    return int(lib().z4c_kernel_launches())


def default_params(**overrides):
    p = Params()
    lib().z4c_params_default(C.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


class Mesh:
    """Block grid of the reference's <mesh>/<meshblock> blocks: nb root
    blocks per axis of nx cells.  With `refinement` (the <refinementN>
    blocks: dicts of x1min, x1max, x2min, x2max, x3min, x3max and level) the
    mesh is statically refined as Mesh's constructor builds it
    (mesh/mesh.cpp:488-665, MeshBlockTree::AddMeshBlock / Refine,
    mesh/meshblock_tree.cpp:108-230): `locs` then lists every MeshBlock in gid
    order as (level, lx1, lx2, lx3)."""

    def __init__(self, nb, nx, xmin, xmax, bc="periodic", refinement=None):
        self.nb = tuple(int(v) for v in nb)
        self.nx = tuple(int(v) for v in nx)
        self.xmin = tuple(float(v) for v in xmin)
        self.xmax = tuple(float(v) for v in xmax)
        if isinstance(bc, str):
            bc = [BC_NAMES[bc]] * 6
        self.bc = tuple(int(v) for v in bc)
        self.root_level = max(0, (max(self.nb) - 1).bit_length())
        self.locs = None
        if refinement:
            self.locs = _smr_blocks(self, refinement)

    @property
    def nblocks(self):
        if self.locs is not None:
            return len(self.locs)
        return self.nb[0] * self.nb[1] * self.nb[2]

    @property
    def nn(self):
        return tuple(n + 1 + 2 * NG for n in self.nx)

    def desc(self):
        d = MeshDesc()
        for a in range(3):
            d.nb[a], d.nx[a] = self.nb[a], self.nx[a]
            d.xmin[a], d.xmax[a] = self.xmin[a], self.xmax[a]
        for f in range(6):
            d.bc[f] = self.bc[f]
        return d

    def block_coords(self, block):
        """Vertex coordinates (x, y, z) and spacing of one block, computed on
        the host exactly as the reference's Coordinates constructor does."""
        xs, dxs = [], []
        d = self.desc()
        loc = None
        if self.locs is not None:
            loc = (C.c_longlong * 4)(*[int(v) for v in self.locs[block]])
        for a in range(3):
            x = np.empty(self.nn[a])
            dx = C.c_double()
            xp = x.ctypes.data_as(C.POINTER(C.c_double))
            if loc is None:
                _check(lib().z4c_mesh_block_coords(C.byref(d), block, a, xp, C.byref(dx)))
            else:
                _check(lib().z4c_mesh_loc_coords(C.byref(d), loc, a, xp, C.byref(dx)))
            xs.append(x)
            dxs.append(dx.value)
        return xs, dxs

    def neighbours(self, block):
        """Neighbour list of one block of a refined mesh as the context builds
        it: rows (gid, level, ox1, ox2, ox3, fi1, fi2) in the reference's
        order."""
        locs = np.ascontiguousarray(self.locs, dtype=np.int64)
        out = np.zeros((56, 7), dtype=np.int32)
        n = lib().z4c_refined_neighbours(C.byref(self.desc()), len(locs),
                                         locs.ctypes.data_as(C.POINTER(C.c_longlong)), int(block),
                                         out.ctypes.data_as(C.POINTER(C.c_int)))
        _check(min(n, 0))
        return out[:n]

    def new_dt(self, cfl):
        """Time step of the mesh: NewBlockTimeStep on every block, minimum
        over blocks (cfl times the smallest cell width)."""
        if self.locs is not None:
            return min(min(self.block_coords(b)[1]) * float(cfl) for b in range(self.nblocks))
        dt = C.c_double()
        _check(lib().z4c_mesh_new_dt(C.byref(self.desc()), float(cfl), C.byref(dt)))
        return dt.value

    def zones(self):
        """Cells of the mesh (the reference's zone count, mesh.hpp:289-292)."""
        return self.nblocks * self.nx[0] * self.nx[1] * self.nx[2]

    @classmethod
    def from_restart(cls, path):
        """The mesh of a reference restart file: block grid and bounds from
        its header, boundary conditions from its <mesh> block."""
        info = restart_info(path)
        text = restart_text(path)
        bc = []
        for a in (1, 2, 3):
            for side in ("i", "o"):
                v = _param(text, "mesh", f"{side}x{a}_bc")
                bc.append(BC_NAMES[v or "periodic"])
        mesh = cls(info["nb"], info["block_nx"], info["xmin"], info["xmax"], bc)
        if info["nlevels"] > 1:  # a refined mesh: its blocks as the file lists them
            n = _check(lib().z4c_restart_locs(path.encode(), None, 0))
            locs = np.zeros((n, 4), dtype=np.int64)
            _check(lib().z4c_restart_locs(path.encode(),
                                          locs.ctypes.data_as(C.POINTER(C.c_longlong)), n))
            mesh.locs = locs
        return mesh


def _param(text, block, key):
    """Value of key in <block> of an input or restart parameter text."""
    inside = False
    for line in text.splitlines():
        s = line.split("#", 1)[0].strip()
        if s.startswith("<"):
            inside = s.startswith(f"<{block}>")
            continue
        if inside and "=" in s:
            k, v = s.split("=", 1)
            if k.strip() == key:
                return v.strip()
    return None


def _info_dict(I):
    return dict(nbtotal=I.nbtotal, root_level=I.root_level, xmin=tuple(I.xmin),
                xmax=tuple(I.xmax), xrat=tuple(I.xrat), mesh_nx=tuple(I.mesh_nx), time=I.time,
                dt=I.dt, ncycle=I.ncycle, datasize=I.datasize, nb=tuple(I.nb),
                block_nx=tuple(I.block_nx), nlevels=I.nlevels,
                trackers=[tuple(I.trackers[t]) for t in range(I.ntrackers)])


def restart_info(path):
    """Header of a reference restart file (outputs/restart.cpp layout)."""
    I = RestartInfo()
    _check(lib().z4c_restart_info(os.fsencode(path), C.byref(I)))
    return _info_dict(I)


def restart_text(path):
    """Parameter text of a restart file, through the byte after <par_end>."""
    n = _check(lib().z4c_restart_text(os.fsencode(path), None, 0))
    buf = C.create_string_buffer(n + 1)
    lib().z4c_restart_text(os.fsencode(path), buf, n + 1)
    return buf.raw[:n].decode()


def restart_read(path):
    """(header, state): the Z4c state of every MeshBlock of a restart file,
    [block][var][k][j][i] with blocks in grid order."""
    info = restart_info(path)
    nn = [n + 1 + 2 * NG for n in info["block_nx"]]
    u = np.empty((info["nbtotal"], NVAR, nn[2], nn[1], nn[0]))
    _check(lib().z4c_restart_read(os.fsencode(path), u.ctypes.data_as(C.POINTER(C.c_double))))
    return info, u


def restart_write(path, par_text, mesh, u, time, dt, ncycle, trackers=()):
    """RestartOutput::WriteOutputFile from host data: u in grid order,
    trackers as (x, y, z, betax, betay, betaz) rows."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    assert u.shape == (mesh.nblocks, NVAR) + tuple(reversed(mesh.nn))
    t = np.ascontiguousarray(np.asarray(trackers, dtype=np.float64).reshape(-1, 6))
    _check(lib().z4c_restart_write_host(
        os.fsencode(path), par_text.encode(), C.byref(mesh.desc()),
        u.ctypes.data_as(C.POINTER(C.c_double)), float(time), float(dt), int(ncycle), len(t),
        t.ctypes.data_as(C.POINTER(C.c_double)) if len(t) else None))


def _mesh_gen_x(index, nrange, x0, x1):
    """ComputeMeshGeneratorX (symmetric interval) and UniformMeshGeneratorX1,
    mesh/mesh.hpp:839-945."""
    rx = float(2 * index - nrange) / float(2 * nrange)
    return 0.5 * (x0 + x1) + (rx * x1 - rx * x0)


def _smr_blocks(mesh, regions):
    """Leaves of the statically refined block tree in gid order."""
    r0 = mesh.root_level
    leaves = {(r0, i, j, k) for k in range(mesh.nb[2]) for j in range(mesh.nb[1])
              for i in range(mesh.nb[0])}
    periodic = [mesh.bc[2 * a] == BC_NAMES["periodic"] for a in range(3)]

    def refine(node):  # MeshBlockTree::Refine: children, then the 26 neighbours' level
        lev, l = node[0], node[1:]
        leaves.discard(node)
        for c in range(8):
            leaves.add((lev + 1, 2 * l[0] + (c & 1), 2 * l[1] + ((c >> 1) & 1),
                        2 * l[2] + ((c >> 2) & 1)))
        n = [mesh.nb[a] << (lev - r0) for a in range(3)]
        for oz in (-1, 0, 1):
            for oy in (-1, 0, 1):
                for ox in (-1, 0, 1):
                    if ox == oy == oz == 0:
                        continue
                    nl = [l[0] + ox, l[1] + oy, l[2] + oz]
                    ok = True
                    for a in range(3):
                        if nl[a] < 0 or nl[a] >= n[a]:
                            if not periodic[a]:
                                ok = False
                            nl[a] %= n[a]
                    if ok:
                        add_block((lev, *nl))

    def add_block(loc):  # MeshBlockTree::AddMeshBlock from the root
        lev = loc[0]
        for lv in range(r0, lev):
            anc = (lv, *[x >> (lev - lv) for x in loc[1:]])
            if anc in leaves:
                refine(anc)

    for reg in regions:
        level = int(reg["level"])
        if level < 1:
            raise ValueError("refinement level must be larger than 0")
        lo, hi = [], []
        for a in range(3):
            lxmax = mesh.nb[a] << level
            rmin, rmax = float(reg[f"x{a + 1}min"]), float(reg[f"x{a + 1}max"])
            if rmin > rmax or rmin < mesh.xmin[a] or rmax > mesh.xmax[a]:
                raise ValueError("invalid refinement region")
            l0 = 0
            while l0 < lxmax and not _mesh_gen_x(l0 + 1, lxmax, mesh.xmin[a], mesh.xmax[a]) > rmin:
                l0 += 1
            l1 = l0
            while l1 < lxmax and not _mesh_gen_x(l1 + 1, lxmax, mesh.xmin[a], mesh.xmax[a]) >= rmax:
                l1 += 1
            if l0 % 2 == 1:
                l0 -= 1
            if l1 % 2 == 0:
                l1 += 1
            lo.append(l0)
            hi.append(l1)
        for k in range(lo[2], hi[2], 2):
            for j in range(lo[1], hi[1], 2):
                for i in range(lo[0], hi[0], 2):
                    add_block((r0 + level, i, j, k))
    maxlev = max(b[0] for b in leaves)

    def morton(b):
        sh = maxlev - b[0]
        x, y, z = (v << sh for v in b[1:])
        key = 0
        for bit in range(maxlev + 1):
            key |= (((x >> bit) & 1) << (3 * bit)) | (((y >> bit) & 1) << (3 * bit + 1)) \
                | (((z >> bit) & 1) << (3 * bit + 2))
        return key

    return np.array(sorted(leaves, key=morton), dtype=np.int64)


class Z4c:
    """A device context holding every MeshBlock of a mesh."""

    def __init__(self, mesh, params=None, integrator="rk4"):
        self.mesh = mesh
        self.params = params if params is not None else default_params()
        self.integrator = integrator
        h = C.c_void_p()
        if mesh.locs is None:
            _check(lib().z4c_create(C.byref(mesh.desc()), C.byref(self.params),
                                    INTEG[integrator], C.byref(h)))
        else:
            locs = np.ascontiguousarray(mesh.locs, dtype=np.int64)
            _check(lib().z4c_create_refined(
                C.byref(mesh.desc()), len(locs), locs.ctypes.data_as(C.POINTER(C.c_longlong)),
                C.byref(self.params), INTEG[integrator], C.byref(h)))
        self._h = h
        self.nblocks = mesh.nblocks
        self.nn = mesh.nn

    def close(self):
        if getattr(self, "_h", None):
            lib().z4c_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- data movement ----
    def shape(self, reg, block=-1):
        nv = lib().z4c_reg_nvar(reg)
        s = (nv, self.nn[2], self.nn[1], self.nn[0])
        return s if block >= 0 else (self.nblocks,) + s

    def upload(self, reg, arr, block=-1):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.shape != self.shape(reg, block):
            raise ValueError(f"shape {a.shape} != {self.shape(reg, block)}")
        _check(lib().z4c_upload(self._h, reg, block, a.ctypes.data_as(C.POINTER(C.c_double))))

    def download(self, reg, block=-1, out=None):
        a = np.empty(self.shape(reg, block)) if out is None else out
        if a.shape != self.shape(reg, block) or a.dtype != np.float64 or not a.flags.c_contiguous:
            raise ValueError("output array has the wrong shape, dtype or layout")
        _check(lib().z4c_download(self._h, reg, block, a.ctypes.data_as(C.POINTER(C.c_double))))
        return a

    def device_ptr(self, reg):
        p = C.POINTER(C.c_double)()
        _check(lib().z4c_device_ptr(self._h, reg, C.byref(p)))
        return C.cast(p, C.c_void_p).value

    def coords(self, block):
        """Vertex coordinates (x, y, z) of one block, the reference's x?f."""
        out = []
        for a in range(3):
            x = np.empty(self.nn[a])
            _check(lib().z4c_block_coords(self._h, block, a,
                                          x.ctypes.data_as(C.POINTER(C.c_double))))
            out.append(x)
        return out

    def dx(self):
        d = np.empty(3)
        _check(lib().z4c_dx(self._h, d.ctypes.data_as(C.POINTER(C.c_double))))
        return d

    def sync(self):
        _check(lib().z4c_sync(self._h))

    def set_stream(self, stream_handle):
        _check(lib().z4c_set_stream(self._h, C.c_void_p(stream_handle)))

    # ---- reference operator names ----
    def Z4cRHS(self, reg_u=REG_U, reg_rhs=REG_RHS, block=-1):
        _check(lib().z4c_rhs(self._h, reg_u, reg_rhs, block))

    def Z4cBoundaryRHS(self, reg_u=REG_U, reg_rhs=REG_RHS, block=-1):
        _check(lib().z4c_boundary_rhs(self._h, reg_u, reg_rhs, block))

    def AddZ4cRHS(self, reg_rhs, wght, reg_out, block=-1):
        _check(lib().z4c_add_rhs(self._h, reg_rhs, float(wght), reg_out, block))

    def WeightedAve(self, reg_out, reg_in1, reg_in2, wght, block=-1):
        w = (C.c_double * 3)(*[float(x) for x in wght])
        _check(lib().z4c_weighted_ave(self._h, reg_out, reg_in1, reg_in2, w, block))

    def AlgConstr(self, reg_u=REG_U, block=-1):
        _check(lib().z4c_alg_constr(self._h, reg_u, block))

    def ADMToZ4c(self, reg_adm=REG_ADM, reg_u=REG_U, block=-1):
        _check(lib().z4c_adm_to_z4c(self._h, reg_adm, reg_u, block))

    def Z4cToADM(self, reg_u=REG_U, reg_adm=REG_ADM, block=-1):
        _check(lib().z4c_z4c_to_adm(self._h, reg_u, reg_adm, block))

    def ADMConstraints(self, reg_con=REG_CON, reg_adm=REG_ADM, reg_u=REG_U, block=-1):
        _check(lib().z4c_adm_constraints(self._h, reg_con, reg_adm, reg_u, block))

    # ---- task-list pieces ----
    def Z4cWeyl(self, reg_adm=REG_ADM, reg_weyl=REG_WEYL, block=-1, reg_u=REG_U):
        """Z4c::Z4cWeyl: Re and Im psi4 on the interior, NaN elsewhere."""
        _check(lib().z4c_weyl(self._h, reg_adm, reg_u, reg_weyl, block))

    def ghost_fill(self, reg=REG_U):
        _check(lib().z4c_ghost_fill(self._h, reg))

    def init_finalize(self):
        _check(lib().z4c_init_finalize(self._h))

    def stage(self, stage, dt):
        _check(lib().z4c_stage(self._h, int(stage), float(dt)))

    def evolve(self, dt, nsteps, with_constraints=False):
        _check(lib().z4c_evolve(self._h, float(dt), int(nsteps), int(bool(with_constraints))))

    def rhs_stage(self, stage, dt):
        """Fused RHS + low-storage stage update, without the ghost exchange."""
        _check(lib().z4c_rhs_stage(self._h, int(stage), float(dt)))

    def fp64_probe(self):
        t = C.c_double()
        _check(lib().z4c_fp64_probe(self._h, C.byref(t)))
        return t.value

    def set_per_block(self, flag):
        _check(lib().z4c_set_per_block(self._h, int(bool(flag))))

    def set_tile(self, point_threads, column_threads, column_slabs):
        """Launch shape of the RHS passes (see z4c_set_tile)."""
        _check(lib().z4c_set_tile(self._h, int(point_threads), int(column_threads),
                                  int(column_slabs)))

    def set_contract(self, on=True):
        """Contracted right-hand side on or off (see z4c_set_contract)."""
        _check(lib().z4c_set_contract(self._h, int(bool(on))))

    def set_point_regs(self, regs):
        """Register budget of the heavy RHS passes (0 or 168, see
        z4c_set_point_regs)."""
        _check(lib().z4c_set_point_regs(self._h, int(regs)))

    def get_point_regs(self):
        v = C.c_int()
        _check(lib().z4c_get_point_regs(self._h, C.byref(v)))
        return v.value

    def get_contract(self):
        v = C.c_int()
        _check(lib().z4c_get_contract(self._h, C.byref(v)))
        return bool(v.value)

    def set_merged(self, on):
        """Allows (True, the default) or forbids the merged vertex grid of
        z4c_evolve on uniform meshes (see z4c_set_merged)."""
        _check(lib().z4c_set_merged(self._h, int(bool(on))))

    def get_merged(self):
        """Whether the next evolve runs on the merged vertex grid."""
        v = C.c_int()
        _check(lib().z4c_get_merged(self._h, C.byref(v)))
        return bool(v.value)

    def get_tile(self):
        t = (C.c_int * 3)()
        _check(lib().z4c_get_tile(self._h, t))
        return tuple(t)

    def autotune(self, reps=3):
        """Picks the fastest launch shape of the RHS passes on this mesh;
        returns (shape, stage milliseconds)."""
        ms = C.c_float()
        _check(lib().z4c_autotune(self._h, int(reps), C.byref(ms)))
        return self.get_tile(), ms.value

    def add_tracker(self, pos):
        """PunctureTracker at pos; returns its id."""
        p = (C.c_double * 3)(*[float(v) for v in pos])
        i = C.c_int()
        _check(lib().z4c_tracker_add(self._h, p, C.byref(i)))
        return i.value

    def tracker(self, tid):
        """(position, interpolated shift) of a tracker."""
        out = np.empty(6)
        _check(lib().z4c_tracker_get(self._h, int(tid), out.ctypes.data_as(C.POINTER(C.c_double))))
        return out[:3], out[3:]

    def restart_load(self, path):
        """Mesh restart constructor: state and puncture trackers of a reference
        restart file into this context; returns the header (time, dt,
        ncycle, ...)."""
        I = RestartInfo()
        _check(lib().z4c_restart_load(self._h, os.fsencode(path), C.byref(I)))
        return _info_dict(I)

    def restart_save(self, path, par_text, time, dt, ncycle):
        """RestartOutput::WriteOutputFile for this context's state and
        trackers; par_text is the parameter text the reference re-reads."""
        _check(lib().z4c_restart_save(self._h, os.fsencode(path), par_text.encode(),
                                      float(time), float(dt), int(ncycle)))

    def psi4_multipoles(self, spheres):
        """The extraction of the main loop after a step (main.hpp
        Z4c_DerivedQuantities): Z4cToADM, Z4cWeyl, the Weyl ghost exchange
        (Mesh::CommunicateAuxZ4c), then ReduceMultipole on every sphere."""
        self.Z4cToADM()
        self.Z4cWeyl()
        self.ghost_fill(REG_WEYL)
        for w in spheres:
            w.ReduceMultipole()
        return [w.psi for w in spheres]

    def regrid_from(self, old):
        """Carry the state and trackers of context `old` into this context
        (the regridded mesh), then fill the ghosts (z4c_regrid +
        z4c_init_finalize)."""
        _check(lib().z4c_regrid(self._h, old._h))
        self.init_finalize()

    def evolve_jobs(self, inputs, outputs, dt, nsteps, hst=None):
        """Evolves independent states from host memory (z4c_evolve_jobs):
        inputs[j] (u registers) -> outputs[j] after nsteps steps of dt, with
        the copies of one job overlapping the evolution of the next; returns
        the history norms, one row of eight per job.  outputs None: the norms
        only.  Page-locked arrays (e.g. torch's pin_memory) let the copies
        overlap."""
        n = len(inputs)
        if n < 1 or (outputs is not None and len(outputs) != n):
            raise ValueError("need as many outputs as inputs, at least one")
        shape = self.shape(REG_U)
        for a in list(inputs) + list(outputs or []):
            if a.shape != shape or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("job arrays must be contiguous float64 u registers")
        hin = (C.c_void_p * n)(*[a.ctypes.data for a in inputs])
        hout = None if outputs is None else (C.c_void_p * n)(*[a.ctypes.data for a in outputs])
        h = np.empty((n, 8)) if hst is None else hst
        _check(lib().z4c_evolve_jobs(self._h, n, hin, hout,
                                     h.ctypes.data_as(C.POINTER(C.c_double)), float(dt),
                                     int(nsteps)))
        return h

    def hst_norms(self):
        out = np.empty(8)
        _check(lib().z4c_hst_norms(self._h, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def check_finite(self, reg=REG_U):
        rc = lib().z4c_check_finite(self._h, reg)
        if rc == -4:
            return False
        _check(rc)
        return True

    # ---- differentiation (tangent-linear model and adjoint) ----------------
    def adj_setup(self):
        """Allocates the tangent / adjoint buffers (REG_TAN, REG_ADJ)."""
        _check(lib().z4c_adj_setup(self._h))

    def tlm_step(self, dt):
        """One step of u and of its tangent REG_TAN."""
        _check(lib().z4c_tlm_step(self._h, dt))

    def adj_step(self, dt):
        """REG_ADJ: adjoint of the state after one step from u -> adjoint of u."""
        _check(lib().z4c_adj_step(self._h, dt))

    def objective(self, reg=REG_U, reg_tan=-1):
        """J = vol * sum of H^2 over the history cells of register reg, and
        with reg_tan its derivative along that tangent: (J, Jdot)."""
        J, Jd = C.c_double(), C.c_double()
        _check(lib().z4c_adj_objective(self._h, reg, reg_tan, C.byref(J), C.byref(Jd)))
        return J.value, (Jd.value if reg_tan >= 0 else None)

    def objective_adj(self, reg=REG_U, scale=1.0):
        """REG_ADJ += scale * dJ/du at register reg."""
        _check(lib().z4c_adj_objective_adj(self._h, reg, scale))

    def adj_adm_to_z4c(self):
        """REG_ADJ (adjoint of u after ADMToZ4c + init_finalize) -> REG_ADM_ADJ,
        the adjoint of the ADM register's data."""
        _check(lib().z4c_adj_adm_to_z4c(self._h))

    def adj_params(self, reset=False):
        """Accumulated adjoints of (shift_eta, damp_kappa1)."""
        out = np.zeros(2)
        _check(lib().z4c_adj_params(self._h, out.ctypes.data_as(C.POINTER(C.c_double)),
                                    int(reset)))
        return out

    def adj_set_weyl(self, sphere, weight=1.0):
        """Adds weight * J_W (the weighted |psi4|^2 over the sphere's
        vertices; sphere: a WaveExtract or its id, None removes the term) to
        the objective of objective, objective_adj and gradient."""
        sid = -1 if sphere is None else int(getattr(sphere, "id", sphere))
        _check(lib().z4c_adj_set_weyl(self._h, sid, float(weight)))

    def snapshots(self, nsteps):
        """Revolve snapshots the free device memory holds for nsteps steps."""
        v = C.c_int()
        _check(lib().z4c_adj_snapshots(self._h, int(nsteps), C.byref(v)))
        return v.value

    def gradient(self, dt, nsteps, nsnap=-1, w_final=1.0, w_step=0.0):
        """dJ_total/du_0 into REG_ADJ with revolve checkpointing (nsnap
        snapshots; -1: as many as free device memory holds) for
        J_total = w_final J(u_n) + w_step sum_k J(u_k); returns
        (J_total, (d/d shift_eta, d/d damp_kappa1), stats)."""
        J = C.c_double()
        pb = np.zeros(2)
        st = np.zeros(4)
        dp = C.POINTER(C.c_double)
        _check(lib().z4c_adj_gradient(self._h, dt, nsteps, nsnap, w_final, w_step, C.byref(J),
                                      pb.ctypes.data_as(dp), st.ctypes.data_as(dp)))
        return J.value, pb, {"forward_steps": int(st[0]), "adjoint_steps": int(st[1]),
                             "seconds": float(st[2]), "schedule_cost": int(st[3])}

    def constraints(self):
        """Z4cToADM + ADMConstraints on the current state (last-stage tasks)."""
        self.Z4cToADM()
        self.ADMConstraints()
