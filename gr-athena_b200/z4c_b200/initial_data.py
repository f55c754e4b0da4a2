"""Initial data on the host, in the ADM register layout [block][17][k][j][i].

Each generator restates the reference problem generator it names; the
transcendental functions go through Python's ``math`` module (the C library
the reference links), so the data agree with the reference bit for bit.
The ADM data are then mapped to Z4c on the device (``Z4c.ADMToZ4c``) and the
ghosts finalised (``Z4c.init_finalize``), as Mesh::Initialize does.
"""
import math

import numpy as np

from . import (ADM_ALPHA, ADM_BETAX, ADM_GXX, ADM_GYY, ADM_GZZ, ADM_KXX, ADM_PSI4, NADM,
               NVAR, REG_ADM, REG_U)


def _minkowski(nn):
    """Z4c::ADMMinkowski (z4c/adm_z4c.cpp:936-951) plus unit lapse, zero shift."""
    adm = np.zeros((NADM, nn[2], nn[1], nn[0]))
    for c in (ADM_GXX, ADM_GYY, ADM_GZZ):
        adm[c] = 1.0
    adm[ADM_PSI4] = 1.0
    adm[ADM_ALPHA] = 1.0
    return adm


def gauge_wave1(mesh, amplitude=0.01, d_x=1.0, d_y=1.0):
    """Z4c::ADMGaugeWave1 + GaugeGaugeWave1 (z4c/awa_z4c.cpp:298-354):
    g_xx = 1 - A sin(2 pi x/d_x), K_xx = pi A cos(.)/sqrt(1 - A sin(.)) and
    alpha = sqrt(1 - A sin(.)), zero shift."""
    out = []
    for b in range(mesh.nblocks):
        (x, _, _), _ = mesh.block_coords(b)
        adm = _minkowski(mesh.nn)
        for i, xi in enumerate(x):
            arg = 2. * math.pi * (xi / d_x - 0. / d_y)
            s = amplitude * math.sin(arg)
            ds = -amplitude * 2. * math.pi * math.cos(arg)
            adm[ADM_GXX, :, :, i] -= s
            adm[ADM_KXX, :, :, i] = 0.5 * ds / math.sqrt(1.0 - s)
            adm[ADM_ALPHA, :, :, i] = math.sqrt(1.0 - s)
        out.append(adm)
    return np.stack(out)


def _psi4_regularized(psi4_bare, chi_div_floor, chi_psi_power):
    """Z4c::psi4Regularized (z4c/z4c.hpp:504-514)."""
    t = math.pow(chi_div_floor, 4. / chi_psi_power)
    return min(t, psi4_bare) if math.isfinite(psi4_bare) else t


def punctures(mesh, params, masses=(1.0,), centres=((0.0, 0.0, 0.0),), shift=(0.0, 0.0, 0.0)):
    """Conformally flat punctures with psi = 1 + sum_i m_i / (2 r_i), the
    precollapsed lapse alpha = psi^-2 and a constant shift (zero by
    default).  One puncture is Z4c::ADMOnePuncture + GaugePreCollapsedLapse
    (z4c/one_puncture_z4c.cpp:22-60, gauge.cpp:46-60); two or more give
    Brill-Lindquist data, the same construction summed over punctures (no
    reference counterpart: the reference ships no BL data)."""
    pw = params.chi_psi_power
    out = []
    for b in range(mesh.nblocks):
        (x, y, z), _ = mesh.block_coords(b)
        adm = _minkowski(mesh.nn)
        pow_ = np.frompyfunc(math.pow, 2, 1)
        X = x[None, None, :]
        Y = y[None, :, None]
        Zc = z[:, None, None]
        psi = np.ones((mesh.nn[2], mesh.nn[1], mesh.nn[0]))
        for m, (ox, oy, oz) in zip(masses, centres):
            r = np.sqrt((X - ox) * (X - ox) + (Y - oy) * (Y - oy) + (Zc - oz) * (Zc - oz))
            with np.errstate(divide="ignore", invalid="ignore"):
                term = 0.5 * m / r
            if len(masses) == 1:
                psi = 1.0 + term
            else:
                psi = psi + term
        psi4_bare = pow_(psi, 4.).astype(np.float64)
        # _psi4_regularized over the array: the threshold once, then
        # std::min(T, v) (v where v < T, else T) and T where v is not finite
        t = math.pow(params.chi_div_floor, 4. / pw)
        psi4 = np.where(np.isfinite(psi4_bare) & (psi4_bare < t), psi4_bare, t)
        adm[ADM_PSI4] = psi4
        for c in (ADM_GXX, ADM_GYY, ADM_GZZ):
            adm[c] = psi4
        adm[ADM_ALPHA] = pow_(psi4, -0.5).astype(np.float64)
        for a in range(3):
            adm[ADM_BETAX + a] = float(shift[a])
        out.append(adm)
    return np.stack(out)


def noise_state(mesh, amplitude=1e-10, seed=137):
    """Minkowski plus i.i.d. uniform noise in [-amplitude, amplitude) on all 22
    Z4c variables at every vertex (the robust-stability workload), seeded."""
    rng = np.random.default_rng(seed)
    nn = mesh.nn
    u = np.zeros((mesh.nblocks, NVAR, nn[2], nn[1], nn[0]))
    from . import ALPHA, CHI, GXX, GYY, GZZ
    for c in (CHI, GXX, GYY, GZZ, ALPHA):
        u[:, c] = 1.0
    u += rng.uniform(-amplitude, amplitude, size=u.shape)
    return u


def load_adm(ctx, adm):
    """Uploads ADM data, maps to Z4c on the device and finalises the ghosts."""
    ctx.upload(REG_ADM, adm)
    ctx.ADMToZ4c()
    ctx.init_finalize()


def load_z4c(ctx, u):
    """Uploads a Z4c state and finalises ghosts (exchange, boundary
    conditions, AlgConstr and Z4cToADM on the ghost vertices)."""
    ctx.upload(REG_U, u)
    ctx.Z4cToADM()
    ctx.init_finalize()
