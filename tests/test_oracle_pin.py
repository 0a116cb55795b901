"""Pins the CPU oracle (plain-C restatement) to the reference compiled from
its own sources, and the reference harness to the reference's own
known-answer tests.  CPU only."""
import numpy as np
import pytest

import oracle
from mbs_fast_b200 import beams as B
from tests import common

pytestmark = pytest.mark.skipif(not oracle.have_reference(),
                                reason="reference library not built")


def kat_samples():
    """The 64 analytic Jones samples of the reference's
    tests/test_mueller_direct.cpp:9-24 (inputs of that known-answer test)."""
    J, W = [], []
    for s in range(64):
        x = 0.125 * (s + 1)
        J.append([np.sin(x), np.cos(0.7 * x), np.cos(1.3 * x), -np.sin(0.4 * x),
                  -np.sin(0.9 * x), np.cos(1.1 * x), np.cos(0.6 * x), np.sin(1.7 * x)])
        W.append(0.03125 * (s + 1))
    return np.array(J), np.array(W)


def test_jones_to_mueller_kat():
    J, W = kat_samples()
    direct, legacy = oracle.ref_jones_kat(J, W)
    # the reference's own bound (test_mueller_direct.cpp:41)
    assert np.max(np.abs(direct - legacy)) <= 2e-15
    mine = np.array([oracle.jones_to_mueller(J[i], W[i]) for i in range(64)])
    assert np.max(np.abs(mine - direct)) <= 2e-15


@pytest.mark.parametrize("case,n,grid", [("hex40x100", 6, (0.0, 180.0, 16, 90)),
                                         ("concave", 8, (0.0, 180.0, 24, 60)),
                                         ("hex10x20", 4, (0.0, 180.0, 12, 180)),
                                         ("bullet30x10", 6, (0.0, 180.0, 16, 180)),
                                         ("droxtal20", 6, (0.0, 180.0, 16, 180)),
                                         ("hexagg20x10x3", 6, (0.0, 180.0, 16, 180))])
def test_oracle_matches_reference(case, n, grid):
    cfg = common.CASES[case]
    batch = common.sobol_batch(case, n)
    g = B.grid(*grid)
    wave = B.wave(cfg)
    M_ref, Mns_ref, cext_ref, _ = oracle.ref_batch(cfg, grid, batch)
    M, Mns = oracle.po_diffract(batch, g, wave, noshadow=True)
    # Rounding-level agreement: the oracle takes libm sincos where the
    # reference uses its own polynomial.  For scale, the reference reports
    # 9.6e-10 CPU vs CUDA FP64 (docs/releases/v1.0.0.md:29) and gates at 1e-5
    # (tests/run_cuda_release_gate.sh:8).
    assert common.weighted_l2(M, M_ref, g) < 5e-8
    assert common.weighted_l2(Mns, Mns_ref, g) < 5e-8
    assert common.grid_l2(M, M_ref) < 5e-8
    cext = oracle.po_extinction(batch, wave)
    np.testing.assert_allclose(cext, cext_ref, rtol=1e-7)
    # PrepareBeams' host extinction equals the unpacked batch's (lossless packing)
    np.testing.assert_array_equal(batch.extinction_ot, cext_ref)


def test_producer_batch_is_lossless():
    """The reference traced and diffracted by itself equals the reference
    diffracting the producer's flat batch (packing loses nothing)."""
    cfg = common.HEX_COLUMN_40x100
    bs, gs, _ = B.symmetry(cfg)
    beta, gamma, w = B.sobol_orientations(5, bs, gs)
    grid = (0.0, 180.0, 8, 45)
    batch = B.trace(cfg, beta, gamma, w)
    M_run, _, cext_run, _, _ = oracle.ref_run(cfg, grid, beta, gamma, w)
    M_bat, _, cext_bat, _ = oracle.ref_batch(cfg, grid, batch)
    assert common.grid_l2(M_run, M_bat) < 1e-14
    np.testing.assert_array_equal(cext_run, cext_bat)


def test_fixed_orientation_reference_paths_agree():
    """Fixed orientation (column 10x20 um at beta=30, gamma=15 deg): the
    reference's fixed path HandleBeams and the prepared
    path HandleBeamsToLocal give the same Mueller grid (both cutoffs are 0)."""
    cfg = common.HEX_COLUMN_10x20
    grid = (0.0, 180.0, 36, 120)
    beta, gamma = np.deg2rad(30.0), np.deg2rad(15.0)
    M_fixed, _ = oracle.ref_fixed(cfg, grid, beta, gamma)
    batch = B.trace(cfg, [beta], [gamma], [1.0])
    M_prep, _, _, _ = oracle.ref_batch(cfg, grid, batch)
    assert common.grid_l2(M_fixed, M_prep) < 1e-12


def test_phi_average_rows():
    """Azimuth average with the L(2 phi) rotation and pole projection: an
    azimuth-independent Mueller field returns its own rows; C_sca and g of a
    uniform M11 are 4*pi and 0."""
    g = B.grid(0.0, 180.0, 8, 36)
    M = np.zeros((8, 37, 16))
    M[..., 0] = 1.0
    rows, csca, asym = oracle.phi_average(M, g)
    np.testing.assert_allclose(rows[:, 0], 1.0)
    assert abs(csca - 4 * np.pi) < 1e-12
    assert abs(asym) < 1e-12


@pytest.mark.parametrize("scale", [0.6, 2.3])
def test_scale_batch_matches_direct_trace(scale):
    """The multi-size rescaling (ScalePreparedOrientation restated in
    oracle.scale_batch) equals tracing the particle at the scaled size with
    the reference tracer: geometry scales exactly, and the re-phased,
    re-absorbed Jones matrices agree up to the reference's fast_exp_im."""
    import dataclasses
    cfg = common.HEX_COLUMN_ABSORBING_10x20
    bs, gs, _ = B.symmetry(cfg)
    beta, gamma, w = B.sobol_orientations(4, bs, gs)
    base = B.trace(cfg, beta, gamma, w)
    big = dataclasses.replace(cfg, p=(cfg.p[0] * scale, cfg.p[1] * scale))
    direct = B.trace(big, beta, gamma, w)
    wave = B.wave(cfg)
    assert base.abs_paths is not None and len(base.abs_paths) > 0
    scaled = oracle.scale_batch(base, scale, wave.wave_index, wave.abs_coeff)
    assert scaled.n_beams == direct.n_beams
    np.testing.assert_allclose(scaled.vx, direct.vx, atol=1e-9 * scale * 20)
    g = B.grid(0.0, 180.0, 8, 90)
    M1 = oracle.po_diffract(scaled, g, wave)
    M2 = oracle.po_diffract(direct, g, B.wave(big))
    assert common.weighted_l2(M1, M2, g) < 1e-9


def test_thetas_oracle_matches_reference_single_beam():
    """DiffractThetasGpu's incoherent azimuth sum, pinned through orientations
    of one beam each (coherent = incoherent there): per zenith row,
    m11(t) = 4/(n_az+1) * sum_p M11_ref(p, t) with the reference's CPU
    HandleBeamsToLocal (CPU rotation carries the 0.5 the GPU one omits).
    The Mueller path takes the stable quotient of nearly singular edges, so
    the pin runs the restatement with it on; the reference's theta scan
    drops those edges (checked on the GPU against singular=False)."""
    cfg = common.HEX_COLUMN_10x20
    batch = common.single_beam_orientations(common.sobol_batch("hex10x20", 2))
    spec = (0.0, 180.0, 12, 60)
    g = B.grid(*spec)
    wave = B.wave(cfg)
    M_ref, _, _, _ = oracle.ref_batch(cfg, spec, batch)
    th = g.theta[1:-1]          # off the poles (the clamp moves them by 1e-6 rad)
    m11 = oracle.thetas_m11(batch, g.n_az, g.az_step, th, wave, singular=True)
    want = 4.0 / (g.n_az + 1) * M_ref[:, 1:-1, 0].sum(axis=0)
    # the reference evaluates sin/cos with its own polynomial (as above)
    np.testing.assert_allclose(m11, want, rtol=1e-6)
