"""Parity on the reference's other particle shapes: bullet (--particle 2 L D),
droxtal (--particle 4 size) and hexagonal aggregate (--particle 12 L D n),
whose beams carry 7-12 vertices, so the FP32C kernel's general vertex loop
(apertures above six vertices) runs beside the fixed-count forms.  The CUDA
path against the oracle and the reference's own CPU result of the same beams,
FP64 and FP32C, with and without the no-shadow sums (run on the B200 box:
pytest -m gpu)."""
import numpy as np
import pytest

import oracle
from mbs_fast_b200 import abi, beams as B
from mbs_fast_b200.handler import GpuHandlerPO
from tests import common

pytestmark = pytest.mark.gpu

GRID = (0.0, 180.0, 16, 180)


@pytest.fixture(scope="module", params=common.SHAPE_CASES)
def shape_case(request):
    cfg = common.CASES[request.param]
    batch = common.sobol_batch(request.param, 6)
    grid = B.grid(*GRID)
    wave = B.wave(cfg)
    h = GpuHandlerPO(grid, wave, device=0)
    M_ref, Mns_ref = oracle.po_diffract(batch, grid, wave, noshadow=True)
    yield request.param, cfg, batch, grid, h, M_ref, Mns_ref
    h.close()


def test_shape_has_long_apertures(shape_case):
    name, _, batch, _, _, _, _ = shape_case
    assert np.diff(batch.vert_offsets).max() > 6, name


def test_shape_fp64_matches_oracle(shape_case):
    name, _, batch, grid, h, M_ref, Mns_ref = shape_case
    M, Mns = h.new_mueller(), h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, M, Mns, precision=abi.FP64)
    assert common.weighted_l2(M, M_ref, grid) < 1e-8, name
    assert common.weighted_l2(Mns, Mns_ref, grid) < 1e-8, name
    assert np.max(np.abs(M - M_ref)) < 1e-9 * np.max(np.abs(M_ref[..., 0])), name


def test_shape_fp64_matches_reference(shape_case):
    name, cfg, batch, grid, h, _, _ = shape_case
    if not oracle.have_reference():
        pytest.skip("reference library not built")
    M_ref, Mns_ref, _, _ = oracle.ref_batch(cfg, GRID, batch)
    M, Mns = h.new_mueller(), h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, M, Mns, precision=abi.FP64)
    assert common.weighted_l2(M, M_ref, grid) < 1e-7, name
    assert common.weighted_l2(Mns, Mns_ref, grid) < 1e-7, name


def test_shape_fp32c_against_fp64(shape_case):
    name, _, batch, grid, h, _, _ = shape_case
    M64, M32 = h.new_mueller(), h.new_mueller()
    N64, N32 = h.new_mueller(), h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, M64, N64, precision=abi.FP64)
    assert h.handle_orientations_to_local_gpu(batch, M32, N32, precision=abi.FP32C)
    wl2 = common.weighted_l2(M32, M64, grid)
    err = common.element_errors(M32, M64, grid)
    print(name, "FP32C vs FP64 weighted L2", wl2, common.weighted_l2(N32, N64, grid), err)
    # measured: weighted L2 0.1-2.1e-6, M11 max rel 0.4-2.3e-4; the no-shadow
    # sums (internal beams only, without the large external ones they are
    # normalised by) 0.7-2.7e-5
    assert wl2 < 2e-5, name
    assert common.weighted_l2(N32, N64, grid) < 1e-4, name
    assert err["M11_max_rel"] < 2e-3, name
