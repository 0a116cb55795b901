"""Host tracing overlapped with device diffraction (mbs_fast_b200.pipeline)
gives the same orientation average as tracing everything first."""
import numpy as np
import pytest

from mbs_fast_b200 import abi, beams as B
from tests import common

pytestmark = pytest.mark.gpu


def test_pipelined_average_equals_sequential():
    from mbs_fast_b200.handler import GpuHandlerPO
    from mbs_fast_b200.pipeline import orientation_average
    cfg = common.HEX_COLUMN_40x100
    bs, gs, _ = B.symmetry(cfg)
    beta, gamma, w = B.sobol_orientations(96, bs, gs, 42)
    grid = B.grid(0.0, 180.0, 16, 90)
    h = GpuHandlerPO(grid, B.wave(cfg))
    M, Mns, t = orientation_average(h, cfg, beta, gamma, w, precision=abi.FP64, batch=20,
                                    noshadow=True)
    batch = B.trace(cfg, beta, gamma, w)
    R, Rns = h.new_mueller(), h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, R, Rns, precision=abi.FP64)
    assert t["beams"] == batch.n_beams
    assert common.grid_l2(M, R) < 1e-13
    assert common.grid_l2(Mns, Rns) < 1e-13
    h.close()
