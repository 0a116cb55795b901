"""FFT-phi azimuth interpolation (reference GpuDiffraction.cu:3206-3320 and
:3504-3760): the oracle's numpy restatement of the zero-padded FFT
upsampling, the device interpolation against it, the low-resolution direct
evaluation plus interpolation against the oracle applied to the direct
result, and the interpolation error against the direct evaluation on the
full azimuth grid."""
import numpy as np
import pytest

import oracle
from mbs_fast_b200 import abi, beams as B
from tests import common


@pytest.mark.parametrize("n_low,n_full", [(24, 48), (17, 50), (16, 96), (25, 25)])
def test_oracle_upsampling_is_exact_for_band_limited_series(n_low, n_full):
    """A trigonometric series with frequencies below n_low/2 is reproduced
    exactly at every output azimuth; the zero-padded FFT rule is pinned by it."""
    rng = np.random.default_rng(n_low)
    kmax = (n_low - 1) // 2
    a, b = rng.normal(size=kmax + 1), rng.normal(size=kmax + 1)

    def f(phi):
        k = np.arange(kmax + 1)[:, None]
        return (a[:, None] * np.cos(k * phi) + b[:, None] * np.sin(k * phi)).sum(axis=0)

    low = np.zeros((n_low, 2, 16))
    low[:, 1, 3] = f(2 * np.pi * np.arange(n_low) / n_low)
    up = oracle.phi_upsample_fft(low, n_full)
    np.testing.assert_allclose(up[:, 1, 3], f(2 * np.pi * np.arange(n_full) / n_full), atol=1e-12)
    assert np.all(up[:, 0, :] == 0.0)


def test_oracle_upsampling_keeps_samples_when_factor_is_integral():
    rng = np.random.default_rng(3)
    low = rng.normal(size=(24, 5, 16))
    up = oracle.phi_upsample_fft(low, 72)
    np.testing.assert_allclose(up[::3], low, atol=1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("n_low,n_full", [(24, 48), (17, 50), (16, 96)])
def test_device_interpolation_matches_oracle(n_low, n_full):
    import torch
    from mbs_fast_b200.handler import GpuHandlerPO
    cfg = common.HEX_COLUMN_10x20
    grid = B.grid(0.0, 180.0, 16, 30)
    h = GpuHandlerPO(grid, B.wave(cfg))
    rng = np.random.default_rng(n_full)
    rows = 37
    low = rng.normal(size=(n_low, rows, 16))
    base = rng.normal(size=(n_full, rows, 16))
    low_d = torch.tensor(low, device="cuda:0")
    out_d = torch.tensor(base, device="cuda:0")
    h.phi_interpolate(low_d.data_ptr(), n_low, rows, out_d.data_ptr(), n_full)
    torch.cuda.synchronize()
    want = base + oracle.phi_upsample_fft(low, n_full)     # accumulated +=
    got = out_d.cpu().numpy()
    assert np.max(np.abs(got - want)) < 1e-12 * np.max(np.abs(want))
    h.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [abi.FP64, abi.FP32C])
def test_fft_phi_path_is_direct_low_grid_plus_interpolation(precision):
    from mbs_fast_b200.handler import GpuHandlerPO
    cfg = common.HEX_COLUMN_40x100
    batch = common.sobol_batch("hex40x100", 16)
    full = B.grid(0.0, 180.0, 48, 360)
    low = full.with_azimuths(24)
    h = GpuHandlerPO(full, B.wave(cfg))
    M, Mns = h.diffract_fft_phi(batch, low, 48, precision, noshadow=True)
    hl = GpuHandlerPO(low, B.wave(cfg))
    Ml, Mlns = hl.new_mueller(), hl.new_mueller()
    assert hl.handle_orientations_to_local_gpu(batch, Ml, Mlns, precision=precision)
    for got, lowm in ((M, Ml), (Mns, Mlns)):
        want = oracle.phi_upsample_fft(lowm, 48)
        assert np.sqrt(np.sum((got - want) ** 2) / np.sum(want ** 2)) < 1e-13
    # the mirror of HandleOrientationsToLocalGpuFftPhi picks factor 2 for 48
    # bins; without no-shadow sums the kernel runs another launch shape, so
    # the agreement is to the rounding of the precision (FP32 sums in FP32C)
    acc = h.new_mueller()
    assert h.handle_orientations_to_local_gpu_fft_phi(batch, acc, precision=precision)
    tol = 1e-13 if precision == abi.FP64 else 1e-6
    assert np.sqrt(np.sum((acc - M) ** 2) / np.sum(M ** 2)) < tol
    h.close()
    hl.close()


@pytest.mark.gpu
def test_fft_phi_error_against_direct_full_grid():
    """The interpolated grid approximates the direct one (64 orientations,
    48 azimuth bins from 24: about 0.5 % weighted L2 on the azimuth-averaged
    rows and on the grid)."""
    from mbs_fast_b200.handler import GpuHandlerPO
    cfg = common.HEX_COLUMN_40x100
    batch = common.sobol_batch("hex40x100", 64)
    full = B.grid(0.0, 180.0, 48, 360)
    h = GpuHandlerPO(full, B.wave(cfg))
    direct = h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, direct, precision=abi.FP64)
    fft = h.new_mueller()
    assert h.handle_orientations_to_local_gpu_fft_phi(batch, fft, precision=abi.FP64)
    rows_err = common.weighted_l2(fft, direct, full)
    grid_err = common.grid_l2(fft, direct)
    print("fft-phi error: rows", rows_err, "grid", grid_err)
    assert 0.0 < rows_err < 2e-2
    assert 0.0 < grid_err < 2e-2
    h.close()
