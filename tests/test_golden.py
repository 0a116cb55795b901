"""Golden fixtures generated from the reference (tests/golden/make_golden.py):
the CPU oracle and the CUDA path against the reference's own outputs and
known answers, without the reference present at run time."""
import json
import os

import numpy as np
import pytest

import oracle
from mbs_fast_b200 import abi, beams as B
from tests import common

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _case(key):
    batch = B.BeamBatch.load(os.path.join(GOLD, f"{key}_batch.npz"))
    z = np.load(os.path.join(GOLD, f"{key}_mueller.npz"))
    grid = B.grid(float(z["grid"][0]), float(z["grid"][1]), int(z["n_az"]), int(z["n_zen"]))
    return batch, grid, z["M"], z["Mns"], z["cext"]


def _extinction_cases():
    with open(os.path.join(GOLD, "extinction_reference.json")) as f:
        d = json.load(f)
    return d["run"], d["cases"]


def _extinction_batch(run, case):
    cfg = B.ParticleConfig(particle_type=case["type"], p=tuple(case["p"]), ri_re=run["ri"][0],
                           ri_im=run["ri"][1], wavelength=run["wavelength"],
                           max_reflections=run["max_reflections"])
    bs, gs, _ = B.symmetry(cfg)
    beta, gamma, w = B.euler_orientations(bs, gs, *run["euler_grid"])
    return cfg, B.trace(cfg, beta, gamma, w)


def test_jones_kat_fixture():
    z = np.load(os.path.join(GOLD, "jones_kat.npz"))
    mine = np.array([oracle.jones_to_mueller(j, w) for j, w in zip(z["jones"], z["weight"])])
    assert np.max(np.abs(mine - z["mueller"])) <= 2e-15   # test_mueller_direct.cpp:41


@pytest.mark.parametrize("key", ["hex10x20", "concave"])
def test_oracle_matches_golden(key):
    batch, grid, M, Mns, cext = _case(key)
    wave = B.wave(common.CASES[key])
    Mo, Mnso = oracle.po_diffract(batch, grid, wave, noshadow=True)
    assert common.weighted_l2(Mo, M, grid) < 5e-8
    assert common.weighted_l2(Mnso, Mns, grid) < 5e-8
    np.testing.assert_allclose(oracle.po_extinction(batch, wave), cext, rtol=1e-7)


def test_extinction_known_answer_bullet_host():
    """The reference's extinction known answer (bullet, 12 reflections,
    Euler 64 x 32, 0.3 %), from the reference tracer's optical-theorem
    extinction and from the oracle's restatement on the same beams."""
    run, cases = _extinction_cases()
    case = next(c for c in cases if c["case"] == "bullet")
    cfg, batch = _extinction_batch(run, case)
    cext = batch.extinction_ot.sum() / batch.orient_weight.sum()
    assert abs(cext / case["cext"] - 1) <= case["rel_tol"]
    mine = oracle.po_extinction(batch, B.wave(cfg)).sum() / batch.orient_weight.sum()
    assert abs(mine / case["cext"] - 1) <= case["rel_tol"]


@pytest.mark.gpu
@pytest.mark.parametrize("key", ["hex10x20", "concave"])
def test_gpu_matches_golden(key):
    from mbs_fast_b200.handler import GpuHandlerPO
    batch, grid, M, Mns, cext = _case(key)
    wave = B.wave(common.CASES[key])
    h = GpuHandlerPO(grid, wave)
    Mg, Mnsg = h.new_mueller(), h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, Mg, Mnsg, precision=abi.FP64)
    assert common.weighted_l2(Mg, M, grid) < 1e-7
    assert common.weighted_l2(Mnsg, Mns, grid) < 1e-7
    np.testing.assert_allclose(h.extinction(batch), cext, rtol=1e-7)
    M32 = h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, M32, precision=abi.FP32C)
    assert common.weighted_l2(M32, M, grid) < 2e-4
    h.close()


@pytest.mark.gpu
def test_extinction_known_answers_gpu():
    """Both of the reference's extinction known answers with the device
    extinction kernel on the reference tracer's beams."""
    from mbs_fast_b200.handler import GpuHandlerPO
    run, cases = _extinction_cases()
    for case in cases:
        cfg, batch = _extinction_batch(run, case)
        h = GpuHandlerPO(B.grid(0.0, 180.0, 1, 1), B.wave(cfg))
        cext = h.extinction(batch).sum() / batch.orient_weight.sum()
        h.close()
        assert abs(cext / case["cext"] - 1) <= case["rel_tol"], case["case"]


# The reference's basic functional test (tests/run_tests.sh:129-146): hexagonal
# column D = H = 10 um, m = 1.31, 6 reflections, 256 Sobol orientations, grid
# 48 x 90: Q_sca = 2.05 +/- 10 %.  For a non-absorbing particle the reference
# reports C_sca = C_ext from the optical theorem over the mean projected area
# (IntegralCharacteristics.cpp:128-137, 161-163); for a convex particle that mean
# is a quarter of the surface area (Cauchy), here with the circumscribed
# diameter of Hexagonal.cpp:54 (side = D / 2).
QSCA_CFG = B.ParticleConfig(particle_type=1, p=(10.0, 10.0), ri_re=1.31, ri_im=0.0,
                            wavelength=0.532, max_reflections=6)
QSCA_EXPECTED, QSCA_REL_TOL = 2.05, 0.10


def _qsca_batch():
    bs, gs, _ = B.symmetry(QSCA_CFG)
    beta, gamma, w = B.sobol_orientations(256, bs, gs, 42)
    return B.trace(QSCA_CFG, beta, gamma, w)


def _mean_projected_area():
    side, height = 10.0 / 2, 10.0
    surface = 2 * (3 * np.sqrt(3) / 2) * side ** 2 + 6 * side * height
    return surface / 4


def test_qsca_known_answer_host():
    """Q_sca of the reference's functional test from the reference tracer's
    optical-theorem extinction and from the oracle's restatement."""
    batch = _qsca_batch()
    area = _mean_projected_area()
    q_tracer = batch.extinction_ot.sum() / batch.orient_weight.sum() / area
    q_oracle = oracle.po_extinction(batch, B.wave(QSCA_CFG)).sum() / batch.orient_weight.sum() / area
    print("Q_sca tracer", q_tracer, "oracle", q_oracle)
    assert abs(q_tracer / QSCA_EXPECTED - 1) <= QSCA_REL_TOL
    assert abs(q_oracle / QSCA_EXPECTED - 1) <= QSCA_REL_TOL


@pytest.mark.gpu
def test_qsca_known_answer_gpu():
    """The same Q_sca from the device extinction kernel."""
    from mbs_fast_b200.handler import GpuHandlerPO
    batch = _qsca_batch()
    h = GpuHandlerPO(B.grid(0.0, 180.0, 48, 90), B.wave(QSCA_CFG))
    q = h.extinction(batch).sum() / batch.orient_weight.sum() / _mean_projected_area()
    h.close()
    assert abs(q / QSCA_EXPECTED - 1) <= QSCA_REL_TOL
