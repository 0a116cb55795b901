"""Particle and grid definitions of the benchmark workloads.

  COLUMN_40x100   orientation-averaged hexagonal column, --particle 1 100 40,
                  m = 1.3116 + 1e-9 i, 4 reflections (headline workload)
  COLUMN_10x20    fixed-orientation column, --particle 1 20 10, m = 1.3116
  PLATE_D10       size-scan plate family (L = 0.2 D) traced at D = 10 um
  aggregate_config  8 touching hexagonal columns D = 20 um, L = 60 um from a
                  particle file, 6 reflections, cutoff profile fast
"""
from __future__ import annotations

import numpy as np

from . import beams as B

COLUMN_40x100 = B.ParticleConfig(particle_type=1, p=(100.0, 40.0), ri_re=1.3116, ri_im=1e-9,
                                 wavelength=0.532, max_reflections=4)
COLUMN_10x20 = B.ParticleConfig(particle_type=1, p=(20.0, 10.0), ri_re=1.3116, ri_im=0.0,
                                wavelength=0.532, max_reflections=4)
PLATE_D10 = B.ParticleConfig(particle_type=1, p=(2.0, 10.0), ri_re=1.3116, ri_im=0.0,
                             wavelength=0.532, max_reflections=4)


def size_scan_diameters(n: int = 16, d_min: float = 10.0, d_max: float = 200.0) -> np.ndarray:
    """Size scan: plate diameters log-spaced from d_min to d_max (um)."""
    return np.geomspace(d_min, d_max, n)


def size_scan_theta_deg() -> np.ndarray:
    """Size-scan zenith grid: 0.05 deg steps over 0-10 deg (201 rows), then
    0.5 deg steps over 10.5-180 deg (340 rows)."""
    return np.concatenate([np.arange(201) * 0.05, 10.5 + np.arange(340) * 0.5])


def aggregate_config(path: str, max_reflections: int = 6, profile: str = "fast"):
    """Non-convex aggregate of 8 hexagonal columns (D=20 um, L=60 um,
    seed-drawn orientations, touching, written as a reference particle file
    at `path`), m=1.3116, `max_reflections` reflections, cutoff profile
    `profile`."""
    from . import particles as PT
    PT.write_particle_file(path, PT.column_aggregate())
    return B.ParticleConfig(particle_type=0, particle_file=path, ri_re=1.3116, ri_im=0.0,
                            wavelength=0.532, max_reflections=max_reflections,
                            cutoff_profile=profile)
