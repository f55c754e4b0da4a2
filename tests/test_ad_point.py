"""The hand-written reverse sweeps of the pointwise Z4c algebra
(gr-athena_b200/csrc/z4c_ad.cuh) on the CPU: each against the forward-mode
derivative of the same forward function (dot-product test <ob, J v> =
<J^T ob, v> on random states and directions), the forward-mode derivative
against central differences of the forward function, and the parameter
adjoints (shift_eta, damp_kappa1) against central differences.

The header compiles for the host as well as the device; tests/ad/
ad_point_check.cpp wraps it in a small C library built here with g++."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import z4c_b200 as Z
from z4c_testlib import ROOT

SRC = os.path.join(ROOT, "tests", "ad", "ad_point_check.cpp")
DP = C.POINTER(C.c_double)

PARAM_SETS = {
    # the puncture benchmarks' gauge: 1+log, Gamma-driver, damping
    "puncture": dict(diss=0.02, chi_div_floor=1e-5, damp_kappa1=0.02, shift_eta=2.0),
    # the gauge-wave benchmarks' gauge: harmonic lapse, zero shift, kappa2 != 0
    "gauge_wave": dict(lapse_harmonic=1.0, lapse_harmonicf=0.0, lapse_oplog=0.0,
                       lapse_advect=0.0, shift_Gamma=0.0, shift_eta=0.0, shift_advect=0.0,
                       damp_kappa1=0.02, damp_kappa2=0.3),
    # every optional branch: shift_H, alpha^2 Gamma, lapse_K, chi^-2 conformal factor
    "branches": dict(shift_H=0.7, shift_alpha2Gamma=0.4, lapse_K=0.3, damp_kappa1=0.1,
                     chi_psi_power=-2.0, chi_div_floor=1e-5),
}


@pytest.fixture(scope="module")
def adp(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("adp") / "adp.so")
    subprocess.run(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-ffp-contract=off", "-o",
                    out, SRC], check=True)
    L = C.CDLL(out)
    L.adp_ham.restype = C.c_double
    return L


def ptr(a):
    return a.ctypes.data_as(DP)


def local_state(rng, n):
    """Random local inputs around a regular state: chi and alpha in (0.5, 1),
    g~ near the identity, everything else O(0.3)."""
    v = rng.uniform(-0.3, 0.3, n)
    v[Z.CHI] = rng.uniform(0.5, 1.0)
    for q, d in zip(range(Z.GXX, Z.GZZ + 1), (1, 0, 0, 1, 0, 1)):
        v[q] = d + 0.1 * rng.uniform(-1, 1)
    v[Z.ALPHA] = rng.uniform(0.5, 1.0)
    return v


@pytest.mark.parametrize("name", list(PARAM_SETS))
def test_rhs_reverse_sweep_is_the_transpose(adp, name):
    p = Z.default_params(**PARAM_SETS[name])
    N = adp.adp_rhs_size()
    rng = np.random.default_rng(11)
    for t in range(25):
        v, vd, ob = local_state(rng, N), rng.standard_normal(N), rng.standard_normal(22)
        res, vb = np.zeros(4), np.zeros(N)
        adp.adp_rhs_dot(ptr(v), ptr(vd), ptr(ob), C.byref(p), ptr(res), ptr(vb))
        scale = np.abs(vb * vd).sum()
        assert abs(res[0] - res[1]) <= 1e-13 * scale, (t, res[:2])


@pytest.mark.parametrize("name", list(PARAM_SETS))
def test_rhs_forward_mode_and_parameter_adjoints_match_differences(adp, name):
    kw = PARAM_SETS[name]
    p = Z.default_params(**kw)
    N = adp.adp_rhs_size()
    rng = np.random.default_rng(3)
    v, vd, ob = local_state(rng, N), rng.standard_normal(N), rng.standard_normal(22)
    res = np.zeros(4)
    adp.adp_rhs_dot(ptr(v), ptr(vd), ptr(ob), C.byref(p), ptr(res), None)

    def F(x, pp):
        out = np.zeros(22)
        adp.adp_rhs(ptr(x), C.byref(pp), ptr(out))
        return out @ ob

    h = 1e-6
    fd = (F(v + h * vd, p) - F(v - h * vd, p)) / (2 * h)
    assert abs(fd - res[0]) <= 1e-7 * max(1.0, abs(fd))
    for k, name_p in ((2, "shift_eta"), (3, "damp_kappa1")):
        hp = 1e-6
        p1, p2 = Z.default_params(**kw), Z.default_params(**kw)
        setattr(p1, name_p, getattr(p, name_p) + hp)
        setattr(p2, name_p, getattr(p, name_p) - hp)
        fd = (F(v, p1) - F(v, p2)) / (2 * hp)
        assert abs(fd - res[k]) <= 1e-7 * max(1.0, abs(fd)), name_p


@pytest.mark.parametrize("tf", [1, 0])
def test_alg_constr_reverse_sweep(adp, tf):
    p = Z.default_params(tf_force_regularization=tf, force_regularization=1)
    rng = np.random.default_rng(5)
    for t in range(40):
        u = local_state(rng, 22)
        if t % 2:
            u[Z.GXX:Z.GZZ + 1] *= 1.2  # det g~ > 1: the pow branch
        ud, ub, res = rng.standard_normal(22), rng.standard_normal(22), np.zeros(2)
        adp.adp_alg_dot(ptr(u), ptr(ud), ptr(ub), C.byref(p), ptr(res))
        assert abs(res[0] - res[1]) <= 1e-13 * max(1.0, abs(res[0])), (t, res)


def test_hamiltonian_reverse_sweep(adp):
    p = Z.default_params(chi_div_floor=1e-5)
    N = adp.adp_ham_size()
    rng = np.random.default_rng(7)
    for t in range(25):
        v = rng.uniform(-0.3, 0.3, N)
        v[0] = rng.uniform(0.5, 1.0)
        for q, d in zip(range(1, 7), (1, 0, 0, 1, 0, 1)):
            v[q] = d + 0.1 * rng.uniform(-1, 1)
        vd, res = rng.standard_normal(N), np.zeros(2)
        adp.adp_ham_dot(ptr(v), ptr(vd), C.byref(p), ptr(res))
        assert abs(res[0] - res[1]) <= 1e-12 * max(1.0, abs(res[0])), (t, res)
        if t == 0:
            h = 1e-6
            fd = (adp.adp_ham(ptr(v + h * vd), C.byref(p)) -
                  adp.adp_ham(ptr(v - h * vd), C.byref(p))) / (2 * h)
            assert abs(fd - res[0]) <= 1e-7 * max(1.0, abs(fd))
