"""Multi-size scan (HandleOrientationsToLocalGpuMultiK) and the zenith-list
M11 scan (DiffractThetasGpu) on the GPU, through the C ABI, against the CPU
oracle on the same inputs (run on the B200: pytest -m gpu)."""
import numpy as np
import pytest

import oracle
from mbs_fast_b200 import abi, beams as B
from mbs_fast_b200.handler import GpuHandlerPO
from tests import common

pytestmark = pytest.mark.gpu

SCALES = [0.5, 1.0, 1.7, 3.1]


@pytest.fixture(scope="module")
def absorbing():
    cfg = common.HEX_COLUMN_ABSORBING_10x20
    batch = common.sobol_batch("hexabs10x20", 6)
    grid = B.grid(0.0, 180.0, 16, 120)
    wave = B.wave(cfg)
    h = GpuHandlerPO(grid, wave)
    yield cfg, batch, grid, wave, h
    h.close()


def _multik(h, batch, scales, precision):
    ms = [h.new_mueller() for _ in scales]
    assert h.handle_orientations_to_local_gpu_multik(batch, 0, batch.n_orient, scales,
                                                     h.wave.wave_index, ms, precision=precision)
    return ms


def test_multisize_matches_oracle_fp64(absorbing):
    cfg, batch, grid, wave, h = absorbing
    ms = _multik(h, batch, SCALES, abi.FP64)
    # one diffraction launch for all sizes: polar rows + main kernel + reduce
    assert h.last_stats.launches <= 4
    assert h.last_stats.n_chunks % len(SCALES) == 0
    for s, M in zip(SCALES, ms):
        ref = oracle.po_diffract(oracle.scale_batch(batch, s, wave.wave_index, wave.abs_coeff),
                                 grid, wave)
        assert common.weighted_l2(M, ref, grid) < 1e-8, s
        assert common.grid_l2(M, ref) < 1e-8, s


def test_multisize_fp32c_against_fp64(absorbing):
    cfg, batch, grid, wave, h = absorbing
    m64 = _multik(h, batch, SCALES, abi.FP64)
    m32 = _multik(h, batch, SCALES, abi.FP32C)
    for s, a, b in zip(SCALES, m32, m64):
        wl2, err = common.weighted_l2(a, b, grid), common.element_errors(a, b, grid)
        print("scale", s, "FP32C vs FP64 weighted L2", wl2, err)
        # about ten times the measured 1.2e-6 and 1.4e-4
        assert wl2 < 1.5e-5
        assert err["M11_max_rel"] < 1.5e-3


def test_multisize_accumulates_and_scale_one_matches_direct(absorbing):
    cfg, batch, grid, wave, h = absorbing
    ms = [h.new_mueller()]
    assert h.handle_orientations_to_local_gpu_multik(batch, 0, batch.n_orient, [1.0],
                                                     wave.wave_index, ms)
    once = ms[0].copy()
    assert h.handle_orientations_to_local_gpu_multik(batch, 0, batch.n_orient, [1.0],
                                                     wave.wave_index, ms)
    np.testing.assert_array_equal(ms[0], 2 * once)
    direct = h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, direct)
    # J re-phased from the raw record (libm sincos) vs the tracer's J_phased
    # (the reference's fast_exp_im, ~3e-9 relative)
    assert common.weighted_l2(once, direct, grid) < 1e-7


def test_multisize_staged_equals_host(absorbing):
    import torch
    cfg, batch, grid, wave, h = absorbing
    host = _multik(h, batch, SCALES, abi.FP32C)
    st = h.stage_multisize(batch, SCALES, wave.wave_index)
    assert st.n_sets == len(SCALES)
    G = grid.n_az * (grid.n_zen + 1)
    dev = torch.zeros(len(SCALES) * G * 16, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    h.diffract_staged(st, dev.data_ptr(), precision=abi.FP32C)
    torch.cuda.synchronize()
    got = dev.cpu().numpy().reshape(len(SCALES), grid.n_az, grid.n_zen + 1, 16)
    for i in range(len(SCALES)):
        np.testing.assert_array_equal(got[i], host[i])
    st.free()


def test_multisize_rejects_missing_raw(absorbing):
    cfg, batch, grid, wave, h = absorbing
    bare = batch.select(0, 2)
    bare.beam_raw = None
    with pytest.raises(ValueError):
        h.handle_orientations_to_local_gpu_multik(bare, 0, 2, [1.0, 2.0], wave.wave_index,
                                                  [h.new_mueller(), h.new_mueller()])


def test_size_scan_plates_nonuniform_grid():
    """The size scan on its own grid: 16 plates (L = 0.2 D, D log-spaced
    10-200 um) from one trace at D = 10 um, 16 Sobol orientations, the
    non-uniform zenith grid (0.05 deg to 10 deg, 0.5 deg beyond: 541 rows) x
    48 azimuth bins, all sizes in one launch; every size against the oracle
    in FP64, and FP32C against FP64 size by size."""
    cfg = common.PLATE_D10
    batch = common.sobol_batch("plate10", 16)
    grid = B.grid(0.0, 180.0, 48, 0, theta_deg=common.size_scan_theta_deg())
    assert grid.n_zen + 1 == 541
    wave = B.wave(cfg)
    scales = common.size_scan_diameters() / 10.0
    h = GpuHandlerPO(grid, wave)
    ms = [h.new_mueller() for _ in scales]
    assert h.handle_orientations_to_local_gpu_multik(batch, 0, batch.n_orient, scales,
                                                     wave.wave_index, ms)
    for i in range(len(scales)):
        ref = oracle.po_diffract(oracle.scale_batch(batch, scales[i], wave.wave_index,
                                                    wave.abs_coeff), grid, wave)
        assert common.weighted_l2(ms[i], ref, grid) < 1e-8, i
    m32 = [h.new_mueller() for _ in scales]
    assert h.handle_orientations_to_local_gpu_multik(batch, 0, batch.n_orient, scales,
                                                     wave.wave_index, m32, precision=abi.FP32C)
    for i in range(len(scales)):
        wl2 = common.weighted_l2(m32[i], ms[i], grid)
        print("size", i, "FP32C vs FP64 weighted L2", wl2)
        assert wl2 < 1.5e-5, i      # about ten times the measured 1.6e-6
    # the forward peak grows about as D^4 (shadow area squared; beam
    # interference makes it non-monotonic over three orientations)
    f = np.array([m[0, 0, 0] for m in ms])
    assert f[-1] > 1e3 * f[0]
    h.close()


def test_thetas_matches_oracle(absorbing):
    cfg, batch, grid, wave, h = absorbing
    th = np.deg2rad(np.array([0.0, 0.3, 5.0, 22.0, 90.0, 150.5, 179.9, 180.0]))
    got = h.diffract_thetas_gpu(batch, th)
    want = oracle.thetas_m11(batch, grid.n_az, grid.az_step, th, wave, singular=False)
    np.testing.assert_allclose(got, want, rtol=1e-9)
    # empty list and empty batch
    assert len(h.diffract_thetas_gpu(batch, [])) == 0
    bad = batch.select(0, 1)
    bad.vert_offsets = bad.vert_offsets.copy()
    bad.vert_offsets[1] = bad.vert_offsets[0] + 2
    bad.vert_offsets[2:] = np.maximum(bad.vert_offsets[2:], bad.vert_offsets[1])
    assert h.diffract_thetas_gpu(bad, th) is None
