"""The producer's restatement of HandlerPO::PrepareBeams (host/prepare.cpp)
against the reference's own PrepareBeams on the same traced beams: every
array of the flat batch, the extinction per orientation included, equal bit
for bit.  The cases cover absorbing and non-absorbing particles (facet tracks
and absorption paths), the relative beam cutoffs of the cutoff profiles, a
concave particle and the non-convex particle-file aggregate."""
import dataclasses

import numpy as np
import pytest

from mbs_fast_b200 import beams as B
from tests import common

ARRAYS = ("beam_offsets", "orient_weight", "vert_offsets", "vx", "vy", "slope_yx", "slope_xy",
          "edge_flags", "beam_geom", "beam_flags", "beam_raw", "abs_offsets", "abs_paths",
          "extinction_ot")


def _both(cfg, n, seed=7):
    bs, gs, _ = B.symmetry(cfg)
    beta, gamma, w = B.sobol_orientations(n, bs, gs, seed)
    ref = B.trace(dataclasses.replace(cfg, reference_prepare=True), beta, gamma, w)
    new = B.trace(dataclasses.replace(cfg, reference_prepare=False), beta, gamma, w)
    return ref, new


def _assert_identical(ref, new):
    assert ref.n_beams == new.n_beams and ref.n_verts == new.n_verts
    for name in ARRAYS:
        a, b = getattr(ref, name), getattr(new, name)
        assert a.shape == b.shape, name
        assert a.dtype == b.dtype, name
        # bitwise, NaN payloads and signed zeros included
        assert a.tobytes() == b.tobytes(), name


@pytest.mark.parametrize("key", ["hex40x100", "hex10x20", "concave", "hexabs10x20", "plate10"])
def test_prepare_matches_reference(key):
    ref, new = _both(common.CASES[key], 48)
    assert ref.n_beams > 0
    _assert_identical(ref, new)


@pytest.mark.parametrize("profile", ["safe", "fast"])
def test_prepare_matches_reference_with_beam_cutoffs(profile):
    cfg = dataclasses.replace(common.HEX_COLUMN_ABSORBING_10x20, cutoff_profile=profile)
    ref, new = _both(cfg, 48)
    _assert_identical(ref, new)


def test_prepare_matches_reference_on_aggregate(tmp_path):
    cfg = common.aggregate_config(str(tmp_path / "agg.dat"), max_reflections=3)
    ref, new = _both(cfg, 2)
    assert ref.n_beams > 100
    _assert_identical(ref, new)


def test_prepare_is_faster_on_absorbing_column():
    """The restatement's reason to exist: the same result for less host time
    in PrepareBeams (thread-summed seconds reported by the producer)."""
    ref, new = _both(common.HEX_COLUMN_40x100, 256)
    assert new.phase_seconds[1] < 0.5 * ref.phase_seconds[1], (ref.phase_seconds, new.phase_seconds)
