"""Shared cases and error measures for the tests.

Particle cases follow the reference's configurations and tests:
  HEX_COLUMN_40x100   orientation-averaged column (--particle 1 100 40, m=1.3116+1e-9i)
  HEX_COLUMN_10x20    fixed-orientation column (--particle 1 20 10, m=1.3116)
  CONCAVE_ABSORBING   the CUDA release-gate particle of the reference
                      (tests/run_cuda_release_gate.sh:31-44: --particle 10 1.0
                      0.7 43.4114540493, m=1.3116+0.01i, --absorption,
                      --cutoff-profile off)
"""
from __future__ import annotations

import functools

import numpy as np

from mbs_fast_b200 import beams as B
from mbs_fast_b200 import workloads as W

from mbs_fast_b200.workloads import PLATE_D10, aggregate_config, size_scan_diameters, \
    size_scan_theta_deg  # noqa: F401  (shared with bench.py)

HEX_COLUMN_40x100 = W.COLUMN_40x100
HEX_COLUMN_10x20 = W.COLUMN_10x20
CONCAVE_ABSORBING = B.ParticleConfig(particle_type=10, p=(1.0, 0.7, 43.4114540493), ri_re=1.3116,
                                     ri_im=0.01, absorption=True, wavelength=0.532,
                                     max_reflections=4, cutoff_off=True)


@functools.lru_cache(maxsize=None)
def sobol_batch(cfg_key: str, n: int, seed: int = 42) -> B.BeamBatch:
    cfg = CASES[cfg_key]
    bs, gs, _ = B.symmetry(cfg)
    beta, gamma, w = B.sobol_orientations(n, bs, gs, seed)
    return B.trace(cfg, beta, gamma, w)


# Absorbing column for the multi-size re-phasing (absorption paths present).
HEX_COLUMN_ABSORBING_10x20 = B.ParticleConfig(particle_type=1, p=(20.0, 10.0), ri_re=1.3116,
                                              ri_im=0.002, absorption=True, wavelength=0.532,
                                              max_reflections=4)
# The reference's other particle shapes (its main.cpp --particle 2, 4, 12):
# apertures of 7-12 vertices.
BULLET_30x10 = B.ParticleConfig(particle_type=2, p=(30.0, 10.0), ri_re=1.3116, ri_im=0.0,
                                wavelength=0.532, max_reflections=4)
DROXTAL_20 = B.ParticleConfig(particle_type=4, p=(20.0,), ri_re=1.3116, ri_im=0.0,
                              wavelength=0.532, max_reflections=4)
HEXAGG_20x10x3 = B.ParticleConfig(particle_type=12, p=(20.0, 10.0, 3), ri_re=1.3116, ri_im=0.0,
                                  wavelength=0.532, max_reflections=4)
CASES = {"hex40x100": HEX_COLUMN_40x100, "hex10x20": HEX_COLUMN_10x20,
         "concave": CONCAVE_ABSORBING, "hexabs10x20": HEX_COLUMN_ABSORBING_10x20,
         "plate10": PLATE_D10, "bullet30x10": BULLET_30x10, "droxtal20": DROXTAL_20,
         "hexagg20x10x3": HEXAGG_20x10x3}
SHAPE_CASES = ("bullet30x10", "droxtal20", "hexagg20x10x3")


def single_beam_orientations(batch: B.BeamBatch) -> B.BeamBatch:
    """Every beam of `batch` as an orientation of its own, with its original
    orientation's weight: coherent and incoherent sums coincide there."""
    out = batch.select(0, batch.n_orient)
    w = np.repeat(batch.orient_weight, np.diff(batch.beam_offsets))
    out.beam_offsets = np.arange(batch.n_beams + 1, dtype=np.int64)
    out.orient_weight = np.ascontiguousarray(w, dtype=np.float64)
    if getattr(out, "extinction_ot", None) is not None:
        out.extinction_ot = None
    return out


def weighted_l2(Ma: np.ndarray, Mb: np.ndarray, grid: B.GridTables) -> float:
    """Solid-angle weighted relative L2 over all 16 elements of the azimuth-
    averaged rows: the metric of the reference's CUDA release gate
    (tests/run_cuda_release_gate.sh:70-86), computed on rows like the .dat
    writer produces them."""
    import oracle
    ra, _, _ = oracle.phi_average(Ma, grid)
    rb, _, _ = oracle.phi_average(Mb, grid)
    w = grid.dcos2pi[:, None]
    return float(np.sqrt(np.sum(w * (ra - rb) ** 2) / max(np.sum(w * rb ** 2), 1e-300)))


def grid_l2(Ma: np.ndarray, Mb: np.ndarray) -> float:
    """Relative L2 over the full direction grid (no azimuth averaging)."""
    return float(np.sqrt(np.sum((Ma - Mb) ** 2) / max(np.sum(Mb ** 2), 1e-300)))


def element_errors(M: np.ndarray, Mref: np.ndarray, grid: B.GridTables) -> dict:
    """Errors of azimuth-averaged rows: relative for M11, absolute for the
    normalised elements M12/M11, M22/M11, M33/M11, M34/M11, M44/M11."""
    import oracle
    r, _, _ = oracle.phi_average(M, grid)
    q, _, _ = oracle.phi_average(Mref, grid)
    out = {"M11_max_rel": float(np.max(np.abs(r[:, 0] - q[:, 0]) / np.abs(q[:, 0])))}
    for name, idx in (("M12", 1), ("M22", 5), ("M33", 10), ("M34", 11), ("M44", 15)):
        out[name + "/M11_max_abs"] = float(np.max(np.abs(r[:, idx] / r[:, 0] - q[:, idx] / q[:, 0])))
    return out

