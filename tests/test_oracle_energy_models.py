"""Invariants of the oracle's three energy models, called through the
per-material dispatch (orc_constitutive): von Mises with fracture (the
default), fixed-corotated (computeContributionFixedCorotated,
ExplicitTimeIntegrator.cu:22-47) and Neo-Hookean with phase-field fracture
driving (computeContributionNeoHookean, :372-446).  The GPU is compared with
these restatements in tests/test_gpu_energy_models.py; here the restatements
themselves are checked for the properties every such model has: no stress at
rest, objectivity, a symmetric V0 P F^T, and each model's own history rules."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

DX = 1.0 / 128
V0 = DX ** 3 / 8
MODELS = (0, 1, 2)  # von Mises + fracture, fixed-corotated, Neo-Hookean + fracture


def update(oracle, mat, F, g=1.0, alpha=0.0, c=1.0, psi=0.0):
    io = np.zeros(13)
    io[:9] = F.reshape(3, 3).T.ravel()  # column-major
    io[9:] = [g, alpha, c, psi]
    out = np.zeros(23)
    dp = C.POINTER(C.c_double)
    oracle.lib().orc_constitutive(C.byref(mat), V0, DX, io.ctypes.data_as(dp), out.ctypes.data_as(dp))
    return dict(F=out[:9].reshape(3, 3).T, g=out[9], alpha=out[10], psi=out[11], FP=out[12],
                sigma=out[13:22].reshape(3, 3).T, vol=out[22])


@pytest.fixture(scope="module")
def mats(pkg):
    out = {}
    for em in MODELS:
        d = pkg.gmpm.reference_defaults(DX, (64, 64, 64))
        pkg.scenes.config_material(d.materials[0], DX)
        d.materials[0].energy_model = em
        out[em] = d.materials[0]
    return out


def _rotation(rng):
    Q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    if np.linalg.det(Q) < 0:
        Q[:, 0] *= -1
    return Q


@pytest.mark.parametrize("em", MODELS, ids=["von_mises", "fixed_corotated", "neo_hookean"])
def test_rest_state_is_stress_free(oracle, mats, em):
    r = update(oracle, mats[em], np.eye(3), psi=0.25)
    if em == 2:
        # the reference's deviator subtracts (1.f/3.f) tr(b): the single-precision
        # third leaves mu * 3e-8 at rest (ExplicitTimeIntegrator.cu:411-425)
        assert np.abs(r["sigma"]).max() <= 1e-7 * V0 * mats[em].youngs_modulus
    else:
        assert np.array_equal(r["sigma"], np.zeros((3, 3)))
    assert np.array_equal(r["F"], np.eye(3))
    assert r["psi"] == 0.25 and r["alpha"] == 0.0
    assert r["vol"] == V0


@pytest.mark.parametrize("em", MODELS, ids=["von_mises", "fixed_corotated", "neo_hookean"])
def test_every_model_is_objective_and_symmetric(oracle, mats, em):
    rng = np.random.default_rng(11 + em)
    # Neo-Hookean takes J^(-2/3) in single precision, as the reference does
    rtol = 1e-6 if em == 2 else 1e-8
    for _ in range(40):
        F = np.eye(3) + 0.05 * rng.standard_normal((3, 3))
        Q = _rotation(rng)
        a = update(oracle, mats[em], F, g=0.8, alpha=0.01, c=0.9, psi=0.1)
        b = update(oracle, mats[em], Q @ F, g=0.8, alpha=0.01, c=0.9, psi=0.1)
        scale = np.abs(a["sigma"]).max()
        assert np.allclose(b["F"], Q @ a["F"], rtol=1e-9, atol=1e-12)
        assert np.allclose(b["sigma"], Q @ a["sigma"] @ Q.T, rtol=rtol, atol=rtol * scale)
        assert np.allclose(a["sigma"], a["sigma"].T, rtol=0, atol=1e-10 * scale)
        for k in ("g", "alpha", "psi", "FP", "vol"):
            assert np.isclose(a[k], b[k], rtol=rtol, atol=0), k


def test_fixed_corotated_is_elastic_without_fracture_driving(oracle, mats):
    rng = np.random.default_rng(5)
    m = mats[1]
    for _ in range(40):
        F = np.eye(3) + 0.2 * rng.standard_normal((3, 3))
        if np.linalg.det(F) <= 0.2:
            continue
        r = update(oracle, m, F, g=0.7, alpha=0.03, c=0.6, psi=0.4)
        assert np.array_equal(r["F"], F)  # no plastic projection
        assert (r["g"], r["alpha"], r["psi"], r["FP"]) == (0.7, 0.03, 0.4, 1.0)
    # uniaxial stretch s: P_11 = 2 mu (s - 1) + lambda (J - 1) J / s with J = s, and sigma_11 = V0 P_11 s
    lam, mu, kappa = C.c_double(), C.c_double(), C.c_double()
    oracle.lib().orc_lame(m.youngs_modulus, m.poisson_ratio, C.byref(lam), C.byref(mu), C.byref(kappa))
    s = 1.01
    r = update(oracle, m, np.diag([s, 1.0, 1.0]))
    P11 = 2 * mu.value * (s - 1) + lam.value * (s - 1)
    assert np.isclose(r["sigma"][0, 0], V0 * P11 * s, rtol=1e-12)


def test_neo_hookean_history_and_driving_force(oracle, mats):
    m = mats[2]
    L0 = DX / 2
    # The reference's volumetric energy kappa/2 ((J - 1)/2 - ln J) is negative for
    # 1 < J < 3.5, so a 2% uniaxial stretch carries no tension energy at all ...
    u = update(oracle, m, np.diag([1.02, 1.0, 1.0]), psi=0.0)
    assert u["psi"] == 0.0 and u["FP"] == 1.0
    # ... and the deviator drives the phase field: an isochoric stretch (J = 1)
    s = 1.05
    iso = np.diag([s, s ** -0.5, s ** -0.5])
    r = update(oracle, m, iso, c=0.8, psi=0.0)
    assert r["psi"] > 0
    assert np.isclose(r["FP"], 4 * L0 * float(np.float32(1) - np.float32(0.001)) * r["psi"] / 3 + 1, rtol=1e-14)
    assert np.isclose(r["g"], 0.8 ** 2 * float(np.float32(1) - np.float32(1e-4)) + float(np.float32(1e-4)),
                      rtol=1e-14)
    # a larger history value is kept
    big = update(oracle, m, iso, psi=10 * r["psi"])
    assert big["psi"] == 10 * r["psi"]
    # hydrostatic compression: J < 1 keeps only the deviatoric energy, which is
    # zero up to the rounding of the single-precision J^(-2/3)
    k = update(oracle, m, 0.98 * np.eye(3), psi=0.0)
    assert k["psi"] < 1e-5 * r["psi"] and k["FP"] - 1.0 < 1e-5 * (r["FP"] - 1.0)
    assert np.all(np.diag(k["sigma"]) < 0)  # it pushes back
