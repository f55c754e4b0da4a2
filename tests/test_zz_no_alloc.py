"""The allocation-free right-hand side, z4c_rhs_noalloc, called through the C
ABI.

It exists for callers that cannot call cudaMalloc: host programs whose own
allocator (a framework's caching allocator, or a pool reserved at start-up)
owns all device memory, and time-stepping loops that cannot take the
device-wide synchronisation an allocation implies.  It takes the state and the
output as caller-owned device pointers and keeps its scratch in a fixed
64 MiB array compiled into the library, processing MeshBlocks in chunks that
fit it.

The GPU test compares it with the context-based z4c_rhs on two calls in a row
(the second on a different state, so that the array's leftover contents from
the first call would show), on MeshBlocks of 40^3 cells, one per chunk, and on
64 MeshBlocks of 16^3 cells, whose kernels are the compile-time-geometry
instances, a dozen blocks per chunk.  Around the second call the device's free
memory is read: the call must not change it.  The file is named to be
collected last.
"""
import ctypes as C

import numpy as np
import pytest

import z4c_b200 as Z
from z4c_testlib import rel_err

TOL = 1e-12  # the normwise relative bound of every RHS parity test


def _call(u_ptr, rhs_ptr, nblocks, nx, dx, params, stream=None):
    nx_c = (C.c_int * 3)(*nx)
    dx_c = (C.c_double * 3)(*dx)
    return Z.lib().z4c_rhs_noalloc(C.c_void_p(u_ptr), C.c_void_p(rhs_ptr), int(nblocks), nx_c,
                                   dx_c, C.byref(params), C.c_void_p(stream))


def test_rejects_bad_sizes_before_any_work():
    """A MeshBlock whose scratch exceeds the fixed array, and malformed
    arguments, are rejected before anything is enqueued (the pointers here are
    never dereferenced)."""
    p = Z.default_params()
    rc = _call(0x1000, 0x2000, 1, (70, 70, 70), (0.1, 0.1, 0.1), p)
    assert rc == -1 and b"scratch" in Z.lib().z4c_last_error()
    assert _call(0x1000, 0x1000, 1, (16, 16, 16), (0.1, 0.1, 0.1), p) == -1
    assert _call(0x1000, 0x2000, 0, (16, 16, 16), (0.1, 0.1, 0.1), p) == -1
    assert _call(0x1000, 0x2000, 1, (4, 16, 16), (0.1, 0.1, 0.1), p) == -1


@pytest.mark.gpu
@pytest.mark.parametrize("nb,nx", [
    # 8 blocks of 40^3 cells: 46.5 MB of scratch per block (33 doubles per
    # vertex, 28 per interior vertex), so the 64 MiB array takes one block
    # per chunk
    ((2, 2, 2), 40),
    # 64 blocks of 16^3 cells (5.2 MB each, 12 per chunk): the fixed-geometry
    # kernel instances
    ((4, 4, 4), 16)])
def test_noalloc_rhs_matches_context_rhs_on_two_calls(nb, nx):
    from z4c_b200 import initial_data as ID
    import torch
    params = Z.default_params(diss=0.02, chi_div_floor=1e-5, damp_kappa1=0.02,
                              shift_eta=2.0, r_max_con=1e300)
    mesh = Z.Mesh(nb, (nx, nx, nx), (-8.0,) * 3, (8.0,) * 3, "outflow")
    ctx = Z.Z4c(mesh, params, "rk4")
    # one stream for the context and the allocation-free call, so that the
    # uploads, the call and the downloads are ordered
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    ID.load_adm(ctx, ID.punctures(mesh, params, masses=(0.5, 0.5),
                                  centres=((1.1, 0.2, 0.1), (-1.1, -0.3, 0.0))))
    dx = [float(v) for v in ctx.dx()]
    nn = mesh.nn
    I = (slice(None), slice(None), slice(4, nn[2] - 4), slice(4, nn[1] - 4), slice(4, nn[0] - 4))
    nan_fill = np.full(ctx.shape(Z.REG_W), np.nan)
    for call in range(2):
        if call == 1:
            ctx.evolve(0.25 * min(dx), 1)  # a different state for the second call
        ctx.Z4cRHS(Z.REG_U, Z.REG_RHS, -1)
        expect = ctx.download(Z.REG_RHS)
        ctx.upload(Z.REG_W, nan_fill)  # unwritten interior entries would stay NaN
        ctx.sync()
        free_before = torch.cuda.mem_get_info()[0]
        rc = _call(ctx.device_ptr(Z.REG_U), ctx.device_ptr(Z.REG_W), ctx.nblocks, mesh.nx, dx,
                   params, stream.cuda_stream)
        assert rc == 0, Z.lib().z4c_last_error()
        ctx.sync()
        if call == 1:  # the first call may load the module (documented); the second may not
            assert torch.cuda.mem_get_info()[0] == free_before, "the call allocated"
        got = ctx.download(Z.REG_W)
        assert np.isfinite(got[I]).all(), f"call {call}: interior left unwritten"
        assert rel_err(got[I], expect[I]) <= TOL, f"call {call}"
    ctx.close()
