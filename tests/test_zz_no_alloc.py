"""The allocation-free entry point mbs_po_diffract_staged_noalloc.

It serves callers that cannot allocate device memory when they diffract:
callers whose device memory belongs to an external pool or a fixed budget,
and real-time loops that must not stall on cudaMalloc/cudaFree, which can
synchronise the device.  Its chunk partials live
in the library's fixed device array instead of context memory, so it must
give the same Mueller sums as mbs_po_diffract_staged, call after call, with
the array reused.  This file is collected last (after every other test).
"""
import numpy as np
import pytest

from mbs_fast_b200 import abi, beams as B
from mbs_fast_b200.handler import GpuHandlerPO
from tests import common

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 32 << 20          # MBS_PO_NOALLOC_SCRATCH_BYTES in include/mbs_po_b200.h


@pytest.mark.parametrize("precision", [abi.FP64, abi.FP32C])
def test_noalloc_matches_allocating_path_twice(precision):
    import torch
    cfg = common.HEX_COLUMN_40x100
    batch = common.sobol_batch("hex40x100", 24)
    grid = B.grid(0.0, 180.0, 32, 360)
    h = GpuHandlerPO(grid, B.wave(cfg))
    staged = h.stage(batch)
    n = grid.n_dirs * 16
    ref = torch.zeros(n, dtype=torch.float64, device="cuda:0")
    ref_ns = torch.zeros_like(ref)
    h.diffract_staged(staged, ref.data_ptr(), ref_ns.data_ptr(), precision=precision)
    torch.cuda.synchronize()
    ref_np, ref_ns_np = ref.cpu().numpy(), ref_ns.cpu().numpy()
    for call in range(2):   # the second call reuses the array the first one filled
        out = torch.zeros_like(ref)
        out_ns = torch.zeros_like(ref)
        h.diffract_staged_noalloc(staged, out.data_ptr(), out_ns.data_ptr(), precision=precision)
        torch.cuda.synchronize()
        # same per-orientation values, chunk sums in a different grouping:
        # agreement to FP64 rounding
        for got, want in ((out.cpu().numpy(), ref_np), (out_ns.cpu().numpy(), ref_ns_np)):
            rel = np.sqrt(np.sum((got - want) ** 2) / np.sum(want ** 2))
            assert rel < 1e-12, (call, rel)
    staged.free()
    h.close()


def test_noalloc_accumulates_and_rejects_oversized_grids():
    import torch
    cfg = common.HEX_COLUMN_10x20
    batch = common.sobol_batch("hex10x20", 3)
    grid = B.grid(0.0, 180.0, 8, 90)
    h = GpuHandlerPO(grid, B.wave(cfg))
    staged = h.stage(batch)
    acc = torch.zeros(grid.n_dirs * 16, dtype=torch.float64, device="cuda:0")
    h.diffract_staged_noalloc(staged, acc.data_ptr(), precision=abi.FP64)
    h.diffract_staged_noalloc(staged, acc.data_ptr(), precision=abi.FP64)
    once = torch.zeros_like(acc)
    h.diffract_staged(staged, once.data_ptr(), precision=abi.FP64)
    torch.cuda.synchronize()
    np.testing.assert_allclose(acc.cpu().numpy(), 2 * once.cpu().numpy(), rtol=1e-12, atol=0)
    staged.free()
    h.close()
    # a grid whose single partial plane exceeds the fixed array is refused
    n_az = 64
    n_zen = SCRATCH_BYTES // (16 * 8 * n_az) + 10
    big = B.grid(0.0, 180.0, n_az, n_zen)
    hb = GpuHandlerPO(big, B.wave(cfg))
    sb = hb.stage(batch)
    out = torch.zeros(big.n_dirs * 16, dtype=torch.float64, device="cuda:0")
    with pytest.raises(RuntimeError, match="ERANGE.*no-allocation scratch"):
        hb.diffract_staged_noalloc(sb, out.data_ptr(), precision=abi.FP32C)
    sb.free()
    hb.close()


def test_noalloc_allocates_nothing_on_a_fresh_handler():
    """On a handler whose first diffraction is the allocation-free call (no
    allocating call before it, so the context holds no partial planes), the
    call leaves the device's free memory unchanged; its result equals the
    allocating path's afterwards."""
    import torch
    cfg = common.HEX_COLUMN_40x100
    batch = common.sobol_batch("hex40x100", 8)
    grid = B.grid(0.0, 180.0, 16, 180)
    # load the library's module (and its fixed array) on this device first
    warm = GpuHandlerPO(grid, B.wave(cfg))
    ws = warm.stage(batch.select(0, 1))
    wacc = torch.zeros(grid.n_dirs * 16, dtype=torch.float64, device="cuda:0")
    warm.diffract_staged_noalloc(ws, wacc.data_ptr(), precision=abi.FP64)
    torch.cuda.synchronize()
    ws.free()
    warm.close()
    h = GpuHandlerPO(grid, B.wave(cfg))
    staged = h.stage(batch)
    out = torch.zeros(grid.n_dirs * 16, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for precision in (abi.FP64, abi.FP32C):
        out.zero_()
        h.diffract_staged_noalloc(staged, out.data_ptr(), precision=precision)
        torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    ref = torch.zeros_like(out)
    h.diffract_staged(staged, ref.data_ptr(), precision=abi.FP32C)
    torch.cuda.synchronize()
    got, want = out.cpu().numpy(), ref.cpu().numpy()
    assert np.sqrt(np.sum((got - want) ** 2) / np.sum(want ** 2)) < 1e-12
    staged.free()
    h.close()
