"""Vertex-centred refinement operators through the C ABI: restriction
(injection) and prolongation (injection + tensor-product 6-point Lagrange
interpolation) against the reference's MeshRefinement operators on one
MeshBlock of a statically refined mesh (tests/golden/refine_vc.npz, made by
the reference build), and against the oracle on a second block in the same
batched launch."""
import ctypes as C
import os

import numpy as np
import pytest

import z4c_b200 as Z
import z4c_oracle as O
from z4c_testlib import GOLDEN, bitwise


def _fixture():
    z = np.load(os.path.join(GOLDEN, "refine_vc.npz"))
    return {k: z[k] for k in z.files}


def _call(fn, src_ptr, dst_ptr, nblocks, nvar, nx, box, stream=None):
    return fn(C.c_void_p(src_ptr), C.c_void_p(dst_ptr), int(nblocks), int(nvar),
              (C.c_int * 3)(*nx), (C.c_int * 6)(*[int(b) for b in box]), C.c_void_p(stream))


def test_boxes_outside_the_arrays_are_rejected():
    """Bad boxes and sizes fail before any launch (pointers never used)."""
    L = Z.lib()
    nx = (8, 8, 8)
    assert _call(L.z4c_vc_prolongate, 0x100, 0x200, 1, 3, nx, (0, 4, 4, 8, 4, 8)) == -1
    assert _call(L.z4c_vc_prolongate, 0x100, 0x200, 1, 3, nx, (4, 12, 4, 8, 4, 8)) == -1
    assert _call(L.z4c_vc_restrict, 0x100, 0x200, 1, 3, nx, (1, 10, 2, 10, 2, 10)) == -1
    assert _call(L.z4c_vc_restrict, 0x100, 0x200, 1, 3, (9, 8, 8), (2, 10, 2, 10, 2, 10)) == -1


@pytest.mark.gpu
def test_restrict_and_prolongate_match_reference():
    import torch
    z = _fixture()
    nx = [int(v) for v in z["nx"]]
    fine, coarse = z["rf_fine"], z["rf_coarse"]
    nvar = fine.shape[0]
    # two blocks per launch: the reference's block and a perturbed copy
    fine2 = np.stack([fine, fine * 1.5 - 0.25])
    coarse2 = np.stack([coarse, np.cos(coarse) + 0.5])
    dev = torch.device("cuda:0")
    L = Z.lib()
    s = torch.cuda.current_stream().cuda_stream

    f_d = torch.from_numpy(fine2).to(dev)
    c_out = torch.zeros(coarse2.shape, dtype=torch.float64, device=dev)
    assert _call(L.z4c_vc_restrict, f_d.data_ptr(), c_out.data_ptr(), 2, nvar, nx,
                 z["rf_rbox"], s) == 0, L.z4c_last_error()
    got = c_out.cpu().numpy()
    assert bitwise(got[0], z["rf_restrict"])
    assert bitwise(got[1], O.vc_restrict(nx, fine2[1].copy(), np.zeros_like(coarse),
                                         z["rf_rbox"]))

    c_d = torch.from_numpy(coarse2).to(dev)
    for q in range(4):
        f_out = torch.from_numpy(fine2.copy()).to(dev)
        box = z[f"rf_pbox{q}"]
        assert _call(L.z4c_vc_prolongate, c_d.data_ptr(), f_out.data_ptr(), 2, nvar, nx, box,
                     s) == 0, L.z4c_last_error()
        got = f_out.cpu().numpy()
        assert bitwise(got[0], z[f"rf_prolong{q}"]), q
        ref1 = O.vc_prolongate(nx, coarse2[1].copy(), fine2[1].copy(), box)
        assert bitwise(got[1], ref1), q


def test_regrid_oracle_matches_reference():
    """The oracle's regrid transfer (both directions, three octants) bit for
    bit against AMRRegistry::FillSameRank{CoarseToFine,FineToCoarse}."""
    z = _fixture()
    nx = [int(v) for v in z["nx"]]
    for q in range(3):
        oct_ = z[f"rg_oct{q}"]
        assert bitwise(O.regrid_refine(nx, z["rg_parent"], z["rg_child"], oct_), z[f"rg_c2f{q}"])
        assert bitwise(O.regrid_derefine(nx, z["rg_child"], z["rg_parent"], oct_),
                       z[f"rg_f2c{q}"])


def test_regrid_rejects_bad_octants():
    L = Z.lib()
    nx = (8, 8, 8)
    args = (C.c_void_p(0x100), C.c_void_p(0x200), C.c_void_p(0x300), 3, (C.c_int * 3)(*nx))
    assert L.z4c_regrid_refine(*args, (C.c_int * 3)(0, 2, 0), None) == -1
    assert L.z4c_regrid_derefine(*args, (C.c_int * 3)(0, 0, -1), None) == -1


@pytest.mark.gpu
def test_regrid_transfer_matches_reference():
    """Refinement of a parent into each recorded octant and derefinement of a
    child into it, on the device, against the reference; then all eight
    octants against the oracle."""
    import torch
    z = _fixture()
    nx = [int(v) for v in z["nx"]]
    dev = torch.device("cuda:0")
    L = Z.lib()
    s = torch.cuda.current_stream().cuda_stream
    parent, child = z["rg_parent"], z["rg_child"]
    nvar = parent.shape[0]
    cn = [n // 2 + 1 + 2 * Z4C_NCG for n in nx]
    scratch = torch.zeros((nvar, cn[2], cn[1], cn[0]), dtype=torch.float64, device=dev)
    p_d = torch.from_numpy(parent).to(dev)
    c_d = torch.from_numpy(child).to(dev)

    def run(fn, src, dst, oct_):
        out = dst.clone()
        rc = fn(C.c_void_p(src.data_ptr()), C.c_void_p(out.data_ptr()),
                C.c_void_p(scratch.data_ptr()), nvar, (C.c_int * 3)(*nx),
                (C.c_int * 3)(*[int(v) for v in oct_]), C.c_void_p(s))
        assert rc == 0, L.z4c_last_error()
        torch.cuda.synchronize()
        return out.cpu().numpy()

    for q in range(3):
        oct_ = z[f"rg_oct{q}"]
        assert bitwise(run(L.z4c_regrid_refine, p_d, c_d, oct_), z[f"rg_c2f{q}"])
        assert bitwise(run(L.z4c_regrid_derefine, c_d, p_d, oct_), z[f"rg_f2c{q}"])
    for o in range(8):
        oct_ = (o & 1, o >> 1 & 1, o >> 2 & 1)
        assert bitwise(run(L.z4c_regrid_refine, p_d, c_d, oct_),
                       O.regrid_refine(nx, parent, child, oct_))
        assert bitwise(run(L.z4c_regrid_derefine, c_d, p_d, oct_),
                       O.regrid_derefine(nx, child, parent, oct_))


Z4C_NCG = 4  # coarse ghost vertices, include/z4c_b200.h
