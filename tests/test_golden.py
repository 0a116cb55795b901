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
