"""The non-convex aggregate (8 touching hexagonal columns, thousands of beams
per orientation, so every orientation spans several shared-memory stages)
on the GPU against the oracle, both precisions, and the diffraction step
captured into a CUDA graph and replayed."""
import numpy as np
import pytest

import oracle
from mbs_fast_b200 import abi, beams as B
from tests import common

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def agg(tmp_path_factory):
    from mbs_fast_b200.handler import GpuHandlerPO
    cfg = common.aggregate_config(str(tmp_path_factory.mktemp("agg") / "agg8.particle"))
    bs, gs, _ = B.symmetry(cfg)
    beta, gamma, w = B.sobol_orientations(3, bs, gs, 42)
    batch = B.trace(cfg, beta, gamma, w)
    grid = B.grid(0.0, 180.0, 16, 60)
    wave = B.wave(cfg)
    h = GpuHandlerPO(grid, wave)
    yield cfg, batch, grid, wave, h
    h.close()


def test_aggregate_fp64_and_fp32c(agg):
    cfg, batch, grid, wave, h = agg
    assert np.diff(batch.beam_offsets).min() > 1000          # many stages per orientation
    M_ref, Mns_ref = oracle.po_diffract(batch, grid, wave, noshadow=True)
    M, Mns = h.new_mueller(), h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, M, Mns, precision=abi.FP64)
    assert common.weighted_l2(M, M_ref, grid) < 1e-8
    assert common.weighted_l2(Mns, Mns_ref, grid) < 1e-8
    M32 = h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, M32, precision=abi.FP32C)
    assert common.weighted_l2(M32, M, grid) < 2e-4


def test_graph_captured_step_replays_the_same(agg):
    import torch
    cfg, batch, grid, wave, h = agg
    st = h.stage(batch)
    n = grid.n_az * (grid.n_zen + 1) * 16
    ref = torch.zeros(n, dtype=torch.float64, device="cuda:0")
    acc = torch.zeros_like(ref)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        h.diffract_staged(st, ref.data_ptr(), precision=abi.FP32C, stream=s.cuda_stream, stats=False)
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        acc.zero_()
        h.diffract_staged(st, acc.data_ptr(), precision=abi.FP32C, stream=s.cuda_stream,
                          stats=False)
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    assert torch.equal(acc, ref)
    del g
    st.free()


def test_aggregate_bench_configuration_and_repeated_table(tmp_path):
    """The aggregate as the bench runs it (6 reflections, importance cutoffs
    1e-4 / 1e-3, about a thousand beams per orientation): 12 orientations
    against the oracle in FP64 and FP32C, and the bench's step -- an
    orientation table cycling over the staged orientations, captured into a
    CUDA graph -- against the direct sums with the table's weights."""
    import dataclasses
    import torch
    from mbs_fast_b200 import workloads as W
    from mbs_fast_b200.handler import GpuHandlerPO
    cfg = dataclasses.replace(W.aggregate_config(str(tmp_path / "agg.particle")),
                              trace_cutoff_importance=1e-4, beam_cutoff_importance=1e-3)
    bs, gs, _ = B.symmetry(cfg)
    beta, gamma, w = B.sobol_orientations(12, bs, gs, 42)
    batch = B.trace(cfg, beta, gamma, w)
    bpo = np.diff(batch.beam_offsets)
    assert 30 <= bpo.min() and bpo.max() <= 3000
    grid = B.grid(0.0, 180.0, 16, 60)
    wave = B.wave(cfg)
    h = GpuHandlerPO(grid, wave)
    M_ref = oracle.po_diffract(batch, grid, wave)
    M = h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, M, precision=abi.FP64)
    assert common.weighted_l2(M, M_ref, grid) < 1e-8
    M32 = h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, M32, precision=abi.FP32C)
    assert common.weighted_l2(M32, M, grid) < 2e-5
    # 36 evaluations cycling over the 12 orientations, weight 1/36 each:
    # the same as the 12-orientation average with weights 3/36 = 1/12 each
    src = h.stage(batch)
    rep = h.stage_repeat(src, np.arange(36) % 12, np.full(36, 1.0 / 36))
    n = grid.n_az * (grid.n_zen + 1) * 16
    acc = torch.zeros(n, dtype=torch.float64, device="cuda:0")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        h.diffract_staged(rep, acc.data_ptr(), precision=abi.FP64, stream=s.cuda_stream, stats=False)
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        acc.zero_()
        h.diffract_staged(rep, acc.data_ptr(), precision=abi.FP64, stream=s.cuda_stream, stats=False)
    g.replay()
    torch.cuda.synchronize()
    got = acc.cpu().numpy().reshape(M.shape)
    assert np.allclose(w, 1.0 / 12)               # the batch's own weights
    assert np.sqrt(np.sum((got - M) ** 2) / np.sum(M ** 2)) < 1e-13
    del g
    rep.free()
    src.free()
    h.close()
