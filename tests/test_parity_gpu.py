"""Parity of the CUDA path with the CPU oracle and the reference, through the
C ABI (run on the B200 box: pytest -m gpu)."""
import numpy as np
import pytest

import oracle
from mbs_fast_b200 import abi, beams as B
from mbs_fast_b200.handler import GpuHandlerPO
from tests import common

pytestmark = pytest.mark.gpu

# Tolerances.  FP64: rounding-level agreement with the oracle (the
# reference reports 9.6e-10 CPU vs CUDA FP64 and gates at 1e-5,
# tests/run_cuda_release_gate.sh:8).  FP32C: the FP32 path against the FP64
# path on the same inputs.
FP64_WL2 = 1e-8          # against the oracle (both evaluate sin/cos to < 1 ulp)
FP64_REF_WL2 = 1e-7      # against the reference (its own AVX sin/cos polynomial)
FP32C_WL2 = 2e-5         # about 10x what FP32C reaches on these cases
FP32C_M11_MAX_REL = 2e-3


@pytest.fixture(scope="module")
def hex_case():
    cfg = common.HEX_COLUMN_40x100
    batch = common.sobol_batch("hex40x100", 8)
    grid = B.grid(0.0, 180.0, 16, 180)
    wave = B.wave(cfg)
    h = GpuHandlerPO(grid, wave, device=0)
    M_ref, Mns_ref = oracle.po_diffract(batch, grid, wave, noshadow=True)
    yield cfg, batch, grid, wave, h, M_ref, Mns_ref
    h.close()


def test_fp64_matches_oracle(hex_case):
    cfg, batch, grid, wave, h, M_ref, Mns_ref = hex_case
    M, Mns = h.new_mueller(), h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, M, Mns, precision=abi.FP64)
    assert common.weighted_l2(M, M_ref, grid) < FP64_WL2
    assert common.weighted_l2(Mns, Mns_ref, grid) < FP64_WL2
    assert common.grid_l2(M, M_ref) < FP64_WL2
    # pointwise, relative to the forward peak
    assert np.max(np.abs(M - M_ref)) < 1e-9 * np.max(np.abs(M_ref[..., 0]))


def test_fp64_matches_reference(hex_case):
    cfg, batch, grid, wave, h, _, _ = hex_case
    if not oracle.have_reference():
        pytest.skip("reference library not built")
    M_ref, Mns_ref, _, _ = oracle.ref_batch(cfg, (0.0, 180.0, 16, 180), batch)
    M, Mns = h.new_mueller(), h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, M, Mns, precision=abi.FP64)
    assert common.weighted_l2(M, M_ref, grid) < FP64_REF_WL2
    assert common.weighted_l2(Mns, Mns_ref, grid) < FP64_REF_WL2


def test_fp32c_against_fp64(hex_case):
    cfg, batch, grid, wave, h, M_ref, _ = hex_case
    M64, M32 = h.new_mueller(), h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, M64, precision=abi.FP64)
    assert h.handle_orientations_to_local_gpu(batch, M32, precision=abi.FP32C)
    wl2 = common.weighted_l2(M32, M64, grid)
    err = common.element_errors(M32, M64, grid)
    print("FP32C vs FP64 weighted L2", wl2, err)
    assert wl2 < FP32C_WL2
    assert err["M11_max_rel"] < FP32C_M11_MAX_REL


def _n_variants(h, precision):
    """Launch shapes the library offers for a precision (set_variant refuses
    the first index past them)."""
    n = 0
    while True:
        try:
            h.set_variant(precision, n)
        except RuntimeError:
            return n
        n += 1


def test_every_launch_shape_matches_oracle(hex_case):
    """The autotuner may pick any launch shape (threads per CTA, directions
    per thread, CTAs per SM; each also sets the orientation chunking): every
    one of them against the oracle."""
    cfg, batch, grid, wave, h, M_ref, _ = hex_case
    try:
        for prec, gate in ((abi.FP64, FP64_WL2), (abi.FP32C, FP32C_WL2)):
            nv = _n_variants(h, prec)
            assert nv >= 5
            for v in range(nv):
                h.set_variant(prec, v)
                M = h.new_mueller()
                assert h.handle_orientations_to_local_gpu(batch, M, precision=prec)
                wl2 = common.weighted_l2(M, M_ref, grid)
                assert wl2 < gate, (prec, v, wl2)
    finally:
        h.set_variant(abi.FP64, 0)
        h.set_variant(abi.FP32C, 0)


@pytest.fixture(scope="module")
def headline_case():
    """The headline configuration's particle and grid at full size: column
    D = 40 um, L = 100 um, m = 1.3116 + 1e-9 i, 4 reflections, 64 Sobol
    orientations, zenith 0-180 deg in 0.1 deg steps x 48 azimuth bins
    (86,448 directions), with the reference's own CPU result of the same
    beams."""
    if not oracle.have_reference():
        pytest.skip("reference library not built")
    cfg = common.HEX_COLUMN_40x100
    batch = common.sobol_batch("hex40x100", 64)
    spec = (0.0, 180.0, 48, 1800)
    grid = B.grid(*spec)
    M_ref, Mns_ref, cext_ref, _ = oracle.ref_batch(cfg, spec, batch)
    h = GpuHandlerPO(grid, B.wave(cfg), device=0)
    yield batch, grid, h, M_ref, Mns_ref, cext_ref
    h.close()


def test_headline_grid_fp64_against_reference(headline_case):
    """FP64 on the headline grid against the reference's CPU double path:
    the reference's release-gate metric (weighted L2 of the azimuth-averaged
    rows) at rounding level, pointwise agreement relative to the forward
    peak, C_ext from the device extinction kernel."""
    batch, grid, h, M_ref, Mns_ref, cext_ref = headline_case
    M, Mns = h.new_mueller(), h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, M, Mns, precision=abi.FP64)
    wl2 = common.weighted_l2(M, M_ref, grid)
    err = common.element_errors(M, M_ref, grid)
    print("FP64 vs reference, headline grid: weighted L2", wl2, err)
    assert wl2 < FP64_REF_WL2
    assert common.weighted_l2(Mns, Mns_ref, grid) < FP64_REF_WL2
    assert np.max(np.abs(M - M_ref)) < 1e-8 * np.max(np.abs(M_ref[..., 0]))
    # relative to rows whose M11 is orders of magnitude below the forward
    # peak (the reference evaluates sin/cos with its own polynomial)
    assert err["M11_max_rel"] < 1e-5
    cext = h.extinction(batch)
    np.testing.assert_allclose(cext, cext_ref, rtol=1e-9)


def test_headline_grid_fp32c_against_reference(headline_case):
    """FP32C on the headline grid against the reference's CPU double path
    (the reference's own FP32 CUDA build reports 3.5e-6 weighted L2,
    docs/releases/v1.0.0.md:30)."""
    batch, grid, h, M_ref, _, _ = headline_case
    M = h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, M, precision=abi.FP32C)
    wl2 = common.weighted_l2(M, M_ref, grid)
    err = common.element_errors(M, M_ref, grid)
    print("FP32C vs reference, headline grid: weighted L2", wl2, err)
    assert wl2 < FP32C_WL2
    assert err["M11_max_rel"] < FP32C_M11_MAX_REL
    for k in ("M12/M11_max_abs", "M22/M11_max_abs", "M33/M11_max_abs", "M34/M11_max_abs",
              "M44/M11_max_abs"):
        assert err[k] < 1e-3, k


def test_accumulates_not_overwrites(hex_case):
    cfg, batch, grid, wave, h, M_ref, _ = hex_case
    M = h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, M, precision=abi.FP64)
    once = M.copy()
    assert h.handle_orientations_to_local_gpu(batch, M, precision=abi.FP64)
    np.testing.assert_array_equal(M, 2 * once)


def test_deterministic_and_range_split(hex_case):
    """Bitwise repeatable; orientation ranges add up to the whole batch."""
    cfg, batch, grid, wave, h, M_ref, _ = hex_case
    a, b = h.new_mueller(), h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, a, precision=abi.FP64)
    assert h.handle_orientations_to_local_gpu(batch, b, precision=abi.FP64)
    np.testing.assert_array_equal(a, b)
    c = h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, c, start=0, count=3, precision=abi.FP64)
    assert h.handle_orientations_to_local_gpu(batch, c, start=3, count=100, precision=abi.FP64)
    assert common.grid_l2(c, a) < 1e-14


def test_staged_path_equals_host_path(hex_case):
    import torch
    cfg, batch, grid, wave, h, M_ref, _ = hex_case
    M = h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, M, precision=abi.FP32C)
    st = h.stage(batch)
    dev = torch.zeros(grid.n_az * (grid.n_zen + 1) * 16, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    h.diffract_staged(st, dev.data_ptr(), precision=abi.FP32C)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dev.cpu().numpy().reshape(M.shape), M)
    st.free()


def test_restage_equals_fresh_stage(hex_case):
    """mbs_po_restage re-fills a staged batch (smaller, larger, then smaller
    batches than it held) with results bitwise equal to a freshly staged
    batch; a malformed batch is rejected and leaves nothing to diffract."""
    import torch
    cfg, batch, grid, wave, h, _, _ = hex_case
    n = grid.n_az * (grid.n_zen + 1) * 16

    def run(st):
        dev = torch.zeros(n, dtype=torch.float64, device="cuda:0")
        torch.cuda.synchronize()
        h.diffract_staged(st, dev.data_ptr(), precision=abi.FP32C)
        torch.cuda.synchronize()
        return dev.cpu().numpy()

    ring = h.stage(batch.select(2, 3))
    bigger = common.sobol_batch("hex40x100", 24)
    for b in (batch.select(0, 2), bigger, batch, batch.select(5, 1)):
        fresh = h.stage(b)
        np.testing.assert_array_equal(run(h.restage(ring, b)), run(fresh))
        assert ring.n_orient == b.n_orient and ring.n_beams == b.n_beams
        fresh.free()
    bad = batch.select(0, 1)
    bad.vert_offsets = bad.vert_offsets.copy()
    bad.vert_offsets[1] = bad.vert_offsets[0] + 2
    bad.vert_offsets[2:] = np.maximum(bad.vert_offsets[2:], bad.vert_offsets[1])
    with pytest.raises(Exception):
        h.restage(ring, bad)
    assert not run(ring).any()
    np.testing.assert_array_equal(run(h.restage(ring, batch)), run(h.stage(batch)))
    ring.free()


def test_growing_batches_on_one_context(hex_case):
    """Host calls whose batches grow and shrink on one context (the upload
    area, the staged batch and the chunk partials grow in stream order
    between them) give bitwise the results of a fresh context per batch."""
    cfg, batch, grid, wave, h, _, _ = hex_case
    big = common.sobol_batch("hex40x100", 40)
    for prec in (abi.FP64, abi.FP32C):
        for b in (big.select(0, 2), big.select(2, 8), big, big.select(7, 3)):
            M = h.new_mueller()
            assert h.handle_orientations_to_local_gpu(b, M, precision=prec)
            fresh = GpuHandlerPO(grid, wave)
            R = fresh.new_mueller()
            assert fresh.handle_orientations_to_local_gpu(b, R, precision=prec)
            fresh.close()
            np.testing.assert_array_equal(M, R)


def test_extinction_on_device(hex_case):
    cfg, batch, grid, wave, h, _, _ = hex_case
    cext = h.extinction(batch)
    np.testing.assert_allclose(cext, batch.extinction_ot, rtol=1e-9)


def test_release_gate_particle():
    """The reference's CUDA release-gate particle (concave hexagon, absorbing,
    cutoffs off): FP64 against the reference's CPU path."""
    cfg = common.CONCAVE_ABSORBING
    batch = common.sobol_batch("concave", 16)
    spec = (0.0, 180.0, 24, 90)
    grid = B.grid(*spec)
    wave = B.wave(cfg)
    h = GpuHandlerPO(grid, wave)
    M, Mns = h.new_mueller(), h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, M, Mns, precision=abi.FP64)
    M_ref, Mns_ref = oracle.po_diffract(batch, grid, wave, noshadow=True)
    assert common.weighted_l2(M, M_ref, grid) < FP64_WL2
    assert common.weighted_l2(Mns, Mns_ref, grid) < FP64_WL2
    if oracle.have_reference():
        R, Rns, _, _ = oracle.ref_batch(cfg, spec, batch)
        assert common.weighted_l2(M, R, grid) < 1e-5   # the reference's own gate
    h.close()


def test_fixed_orientation_config0():
    """Fixed orientation: hexagonal column 10x20 um at beta=30, gamma=15 deg, grid
    theta 0..180 in 0.25 deg x phi 0..360 in 2 deg, against the reference's
    fixed-orientation path HandleBeams."""
    cfg = common.HEX_COLUMN_10x20
    spec = (0.0, 180.0, 180, 720)
    grid = B.grid(*spec)
    wave = B.wave(cfg)
    beta, gamma = np.deg2rad(30.0), np.deg2rad(15.0)
    batch = B.trace(cfg, [beta], [gamma], [1.0])
    h = GpuHandlerPO(grid, wave)
    M = h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, M, precision=abi.FP64)
    if oracle.have_reference():
        R, _ = oracle.ref_fixed(cfg, spec, beta, gamma)
    else:
        R = oracle.po_diffract(batch, grid, wave)
    assert common.weighted_l2(M, R, grid) < FP64_WL2
    assert common.grid_l2(M, R) < FP64_WL2
    h.close()


def test_pinned_result_equals_host_accumulation(hex_case):
    """mbs_po_diffract_pinned hands back exactly what mbs_po_diffract adds
    (both precisions, with and without the no-shadow sums); an empty batch
    gives no planes."""
    cfg, batch, grid, wave, h, _, _ = hex_case
    for prec in (abi.FP64, abi.FP32C):
        M, Mns = h.new_mueller(), h.new_mueller()
        assert h.handle_orientations_to_local_gpu(batch, M, Mns, precision=prec)
        a, an = h.diffract_pinned(batch, noshadow=True, precision=prec)
        np.testing.assert_array_equal(a, M)
        np.testing.assert_array_equal(an, Mns)
        # without no-shadow sums the launch shape differs: compare with the
        # plain host call
        M1 = h.new_mueller()
        assert h.handle_orientations_to_local_gpu(batch, M1, precision=prec)
        b, bn = h.diffract_pinned(batch, precision=prec)
        np.testing.assert_array_equal(b, M1)
        assert bn is None
    assert h.diffract_pinned(batch.select(0, 0)) == (None, None)


def test_staged_pinned_equals_pinned(hex_case):
    """mbs_po_diffract_staged_pinned on a staged batch (the drop-in's
    packed-beam cache) gives bitwise what mbs_po_diffract_pinned gives for the
    same batch from host arrays, call after call."""
    cfg, batch, grid, wave, h, _, _ = hex_case
    st = h.stage(batch)
    for prec in (abi.FP64, abi.FP32C):
        a, an = h.diffract_pinned(batch, noshadow=True, precision=prec)
        for _ in range(2):
            b, bn = h.diffract_staged_pinned(st, noshadow=True, precision=prec)
            np.testing.assert_array_equal(a, b)
            np.testing.assert_array_equal(an, bn)
    st.free()


def test_repeated_orientation_table(hex_case):
    """mbs_po_stage_repeat: an orientation table over a staged batch's
    records (repeats, a backward and a forward jump) gives the sums of the
    batch's orientations with the table's weights."""
    import torch
    cfg, batch, grid, wave, h, _, _ = hex_case
    n = grid.n_az * (grid.n_zen + 1) * 16
    st = h.stage(batch)

    def run(s):
        dev = torch.zeros(n, dtype=torch.float64, device="cuda:0")
        torch.cuda.synchronize()
        h.diffract_staged(s, dev.data_ptr(), precision=abi.FP64)
        torch.cuda.synchronize()
        return dev.cpu().numpy()

    per = []
    for o in range(batch.n_orient):
        one = batch.select(o, 1)
        one.orient_weight = np.ones(1)
        s1 = h.stage(one)
        per.append(run(s1))
        s1.free()
    idx = [0, 1, 2, 0, 1, 2, 5, 3, 7]
    w = np.arange(1, len(idx) + 1) * 0.125
    rep = h.stage_repeat(st, idx, w)
    got = run(rep)
    want = sum(wi * per[i] for wi, i in zip(w, idx))
    assert np.sqrt(np.sum((got - want) ** 2) / np.sum(want ** 2)) < 1e-13
    rep.free()
    st.free()


def test_edge_cases(hex_case):
    cfg, batch, grid, wave, h, _, _ = hex_case
    # empty batch: nothing added
    M = h.new_mueller()
    assert h.handle_orientations_to_local_gpu(batch, M, start=0, count=0)
    assert not M.any()
    # an orientation without beams contributes nothing
    empty = B.BeamBatch(beam_offsets=np.zeros(2, np.int64), orient_weight=np.ones(1),
                        vert_offsets=np.zeros(1, np.int64), vx=np.zeros(0), vy=np.zeros(0),
                        slope_yx=np.zeros(0), slope_xy=np.zeros(0),
                        edge_flags=np.zeros(0, np.uint8),
                        beam_geom=np.zeros((0, abi.GEOM_STRIDE)), beam_flags=np.zeros(0, np.uint8))
    mixed = B.BeamBatch.concat([empty, batch.select(0, 2), empty])
    a, b = h.new_mueller(), h.new_mueller()
    assert h.handle_orientations_to_local_gpu(mixed, a)
    assert h.handle_orientations_to_local_gpu(batch.select(0, 2), b)
    np.testing.assert_array_equal(a, b)
    # a beam with too few vertices is rejected like the reference's
    # "bad-edge-data" (returns False, nothing added)
    bad = batch.select(0, 1)
    bad.vert_offsets = bad.vert_offsets.copy()
    bad.vert_offsets[1] = bad.vert_offsets[0] + 2
    bad.vert_offsets[2:] = np.maximum(bad.vert_offsets[2:], bad.vert_offsets[1])
    M = h.new_mueller()
    assert not h.handle_orientations_to_local_gpu(bad, M)
    assert not M.any()


def test_phi_average_on_device(hex_case):
    """Azimuth-averaged rows, C_sca and g computed on the device from the
    device accumulator equal the oracle's writer restatement on the copied grid."""
    import torch
    cfg, batch, grid, wave, h, M_ref, _ = hex_case
    st = h.stage(batch)
    dev = torch.zeros(grid.n_az * (grid.n_zen + 1) * 16, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    h.diffract_staged(st, dev.data_ptr(), precision=abi.FP64)
    torch.cuda.synchronize()
    rows, csca, g = h.phi_average_gpu(dev.data_ptr())
    M = dev.cpu().numpy().reshape(grid.n_az, grid.n_zen + 1, 16)
    want, csca_w, g_w = oracle.phi_average(M, grid)
    scale = np.max(np.abs(want[:, 0]))
    assert np.max(np.abs(rows - want)) <= 1e-13 * scale
    assert abs(csca - csca_w) <= 1e-12 * abs(csca_w)
    assert abs(g - g_w) <= 1e-12
    # and against the oracle's own Mueller grid (parity of C_sca and g)
    _, csca_o, g_o = oracle.phi_average(M_ref, grid)
    assert abs(csca - csca_o) <= 1e-8 * abs(csca_o)
    assert abs(g - g_o) <= 1e-8
    st.free()
