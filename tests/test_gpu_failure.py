"""Failure detection without any GPU fault: non-finite state is reported as
an error status, bad arguments are rejected before any launch, and the
context stays usable afterwards."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_nonfinite_state_is_detected_and_context_survives():
    import z4c_b200 as Z
    from z4c_b200 import initial_data as ID
    mesh = Z.Mesh((2, 1, 1), (8, 8, 8), (-1, -0.5, -0.5), (1, 0.5, 0.5), "periodic")
    ctx = Z.Z4c(mesh, Z.default_params(r_max_con=1e300), "rk4")
    u = ID.noise_state(mesh)
    ctx.upload(Z.REG_U, u)
    assert ctx.check_finite()
    u[1, Z.ALPHA, 9, 9, 9] = np.nan
    ctx.upload(Z.REG_U, u)
    assert not ctx.check_finite()
    ctx.evolve(0.01, 1)
    assert not ctx.check_finite()  # NaN spreads through the stencils
    ctx.upload(Z.REG_U, ID.noise_state(mesh))
    ctx.evolve(0.01, 1)
    assert ctx.check_finite()
    ctx.close()


def test_bad_arguments_are_rejected():
    import z4c_b200 as Z
    mesh = Z.Mesh((1, 1, 1), (8, 8, 8), (0, 0, 0), (1, 1, 1), "periodic")
    ctx = Z.Z4c(mesh, Z.default_params(), "rk4")
    with pytest.raises(Z.Z4cError) as e:
        ctx.Z4cRHS(Z.REG_U, Z.REG_U)
    assert e.value.code == -1
    with pytest.raises(Z.Z4cError) as e:
        ctx.Z4cRHS(Z.REG_U, Z.REG_RHS, block=5)
    assert e.value.code == -1
    with pytest.raises(Z.Z4cError) as e:
        ctx.upload(Z.REG_K1, np.zeros(ctx.shape(Z.REG_K1)))
    assert e.value.code == -6  # Butcher registers are absent for rk4
    with pytest.raises(Z.Z4cError) as e:
        ctx.stage(5, 0.1)
    assert e.value.code == -1
    ctx.Z4cRHS()
    ctx.sync()
    ctx.close()
