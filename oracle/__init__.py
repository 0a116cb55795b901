"""TEST INFRASTRUCTURE (the checker), not product code.

Python access to the two CPU oracles built by oracle/Makefile into
oracle/_ref/:

* ``libpo_oracle.so`` — plain-C restatement of the reference's CPU PO path
  (po_oracle.c), run on the same flat beam batch the CUDA path receives.
* ``libmbs_ref.so``   — the reference's own CPU double path compiled from its
  sources (ref_harness.cpp), used to pin the restatement and as the CPU
  baseline of bench.py.

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline import this.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from mbs_fast_b200 import abi
from mbs_fast_b200.beams import BeamBatch, GridTables, ParticleConfig

REF_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref")


def _load(name: str) -> C.CDLL:
    path = os.path.join(REF_DIR, name)
    if not os.path.exists(path):
        raise RuntimeError(f"oracle library {path} not built (make -C oracle)")
    return C.CDLL(path)


def have_reference() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libmbs_ref.so"))


_po = None
_ref = None


def _po_lib():
    global _po
    if _po is None:
        _po = _load("libpo_oracle.so")
        _po.po_oracle_diffract.argtypes = [C.POINTER(abi.Beams), C.POINTER(abi.Grid),
                                           C.POINTER(abi.Wave), C.c_int, abi._dp, abi._dp]
        _po.po_oracle_jones.argtypes = [C.POINTER(abi.Beams), C.POINTER(abi.Grid),
                                        C.POINTER(abi.Wave), C.c_int, abi._dp, abi._dp]
        _po.po_oracle_jones_to_mueller.argtypes = [abi._dp, C.c_double, abi._dp]
        _po.po_oracle_extinction.argtypes = [C.POINTER(abi.Beams), C.POINTER(abi.Wave), C.c_int]
        _po.po_oracle_extinction.restype = C.c_double
        _po.po_oracle_phi_average.argtypes = [abi._dp, C.c_int, C.c_int, abi._dp, abi._dp,
                                              abi._dp, abi._dp, abi._dp]
        _po.po_oracle_thetas_m11.argtypes = [C.POINTER(abi.Beams), C.POINTER(abi.Wave), C.c_int,
                                             C.c_double, abi._dp, C.c_int, C.c_int, abi._dp]
    return _po


class GridSpec(C.Structure):
    _fields_ = [("zen_start_deg", C.c_double), ("zen_end_deg", C.c_double),
                ("n_az", C.c_int32), ("n_zen", C.c_int32), ("theta_deg", abi._dp)]


def _ref_lib():
    global _ref
    if _ref is None:
        _ref = _load("libmbs_ref.so")
        cfgp = C.POINTER(abi.HostConfig)   # same layout as mbs_ref_config
        _ref.mbs_ref_run.argtypes = [cfgp, C.POINTER(GridSpec), C.c_int, abi._dp, abi._dp,
                                     abi._dp, abi._dp, abi._dp, abi._dp, abi._dp,
                                     abi._dp, abi._dp]
        _ref.mbs_ref_batch.argtypes = [cfgp, C.POINTER(GridSpec), C.POINTER(abi.Beams), C.c_int,
                                       abi._dp, abi._dp, abi._dp, abi._dp]
        _ref.mbs_ref_fixed.argtypes = [cfgp, C.POINTER(GridSpec), C.c_double, C.c_double,
                                       C.c_double, abi._dp, abi._dp]
        _ref.mbs_ref_jones_kat.argtypes = [C.c_int, abi._dp, abi._dp, abi._dp, abi._dp]
        _ref.mbs_ref_orientations.argtypes = [cfgp, C.c_int, C.c_uint, abi._dp, abi._dp, abi._dp]
    return _ref


# ------------------------------------------------------------ restatement ---

def po_diffract(batch: BeamBatch, grid: GridTables, wave: abi.Wave, n_threads: int = 0,
                noshadow: bool = False):
    """Mueller sums [n_az, n_zen+1, 16] (and no-shadow sums) from the C oracle."""
    lib = _po_lib()
    M = np.zeros((grid.n_az, grid.n_zen + 1, 16))
    Mns = np.zeros_like(M) if noshadow else None
    b, g = batch.as_c(), grid.as_c()
    abi.check(lib.po_oracle_diffract(C.byref(b), C.byref(g), C.byref(wave), n_threads,
                                     abi.ptr(M, C.c_double), abi.ptr(Mns, C.c_double)),
              "po_oracle_diffract")
    return (M, Mns) if noshadow else M


def po_jones(batch: BeamBatch, grid: GridTables, wave: abi.Wave, orient: int):
    lib = _po_lib()
    J = np.zeros((grid.n_az, grid.n_zen + 1, 8))
    Jns = np.zeros_like(J)
    b, g = batch.as_c(), grid.as_c()
    abi.check(lib.po_oracle_jones(C.byref(b), C.byref(g), C.byref(wave), orient,
                                  abi.ptr(J, C.c_double), abi.ptr(Jns, C.c_double)),
              "po_oracle_jones")
    return J, Jns


def jones_to_mueller(j: np.ndarray, weight: float) -> np.ndarray:
    lib = _po_lib()
    j = np.ascontiguousarray(j, np.float64)
    out = np.zeros(16)
    lib.po_oracle_jones_to_mueller(abi.ptr(j, C.c_double), weight, abi.ptr(out, C.c_double))
    return out


def po_extinction(batch: BeamBatch, wave: abi.Wave) -> np.ndarray:
    lib = _po_lib()
    b = batch.as_c()
    return np.array([lib.po_oracle_extinction(C.byref(b), C.byref(wave), o)
                     for o in range(batch.n_orient)])


def phi_average(M: np.ndarray, grid: GridTables):
    """(rows [n_zen+1,16], C_sca, g) of the orientation-average writer."""
    lib = _po_lib()
    M = np.ascontiguousarray(M, np.float64)
    rows = np.zeros((grid.n_zen + 1, 16))
    cs, g = C.c_double(), C.c_double()
    lib.po_oracle_phi_average(abi.ptr(M, C.c_double), grid.n_az, grid.n_zen,
                              abi.ptr(grid.theta, C.c_double), abi.ptr(grid.dcos2pi, C.c_double),
                              abi.ptr(rows, C.c_double), C.byref(cs), C.byref(g))
    return rows, cs.value, g.value


# ------------------------------------------------------------- reference ---

def _gridspec(zen_start, zen_end, n_az, n_zen, theta_deg=None):
    td = None if theta_deg is None else np.ascontiguousarray(theta_deg, np.float64)
    gs = GridSpec(zen_start, zen_end, n_az, (len(td) - 1) if td is not None else n_zen,
                  abi.ptr(td, C.c_double))
    return gs, td


def ref_run(cfg: ParticleConfig, gridspec: tuple, beta, gamma, weight, alpha=None,
            n_threads: int = 0):
    """Reference phase 1 + phase 2 on the CPU: (M, Mns, cext, t_trace, t_diffract)."""
    lib = _ref_lib()
    gs, keep = _gridspec(*gridspec)
    n_az, n_zen = gs.n_az, gs.n_zen
    beta = np.ascontiguousarray(beta, np.float64)
    gamma = np.ascontiguousarray(gamma, np.float64)
    weight = np.ascontiguousarray(weight, np.float64)
    alpha = None if alpha is None else np.ascontiguousarray(alpha, np.float64)
    M = np.zeros((n_az, n_zen + 1, 16))
    Mns = np.zeros_like(M)
    cext = np.zeros(len(beta))
    tt, td = C.c_double(), C.c_double()
    c = cfg.as_c()
    c.n_threads = n_threads
    rc = lib.mbs_ref_run(C.byref(c), C.byref(gs), len(beta), abi.ptr(beta, C.c_double),
                         abi.ptr(gamma, C.c_double), abi.ptr(alpha, C.c_double),
                         abi.ptr(weight, C.c_double), abi.ptr(M, C.c_double),
                         abi.ptr(Mns, C.c_double), abi.ptr(cext, C.c_double),
                         C.byref(tt), C.byref(td))
    if rc != 0:
        raise RuntimeError("mbs_ref_run failed")
    return M, Mns, cext, tt.value, td.value


def ref_orientations(cfg: ParticleConfig, n: int, seed: int = 42):
    """Sobol orientations (beta, gamma, weight) over the particle's symmetry
    domain from the reference's own code (TraceFromSobolSeed)."""
    lib = _ref_lib()
    beta, gamma, w = np.empty(n), np.empty(n), np.empty(n)
    c = cfg.as_c()
    if lib.mbs_ref_orientations(C.byref(c), n, seed, abi.ptr(beta, C.c_double),
                                abi.ptr(gamma, C.c_double), abi.ptr(w, C.c_double)) != 0:
        raise RuntimeError("mbs_ref_orientations failed")
    return beta, gamma, w


def ref_batch(cfg: ParticleConfig, gridspec: tuple, batch: BeamBatch, n_threads: int = 0):
    """Reference HandleBeamsToLocal on exactly this batch: (M, Mns, cext, seconds)."""
    lib = _ref_lib()
    gs, keep = _gridspec(*gridspec)
    M = np.zeros((gs.n_az, gs.n_zen + 1, 16))
    Mns = np.zeros_like(M)
    cext = np.zeros(batch.n_orient)
    sec = C.c_double()
    b = batch.as_c()
    c = cfg.as_c()
    rc = lib.mbs_ref_batch(C.byref(c), C.byref(gs), C.byref(b), n_threads,
                           abi.ptr(M, C.c_double), abi.ptr(Mns, C.c_double),
                           abi.ptr(cext, C.c_double), C.byref(sec))
    if rc != 0:
        raise RuntimeError("mbs_ref_batch failed")
    return M, Mns, cext, sec.value


def ref_fixed(cfg: ParticleConfig, gridspec: tuple, beta, gamma, alpha=0.0):
    """Reference fixed-orientation HandlerPO::HandleBeams: (M, seconds)."""
    lib = _ref_lib()
    gs, keep = _gridspec(*gridspec)
    M = np.zeros((gs.n_az, gs.n_zen + 1, 16))
    sec = C.c_double()
    c = cfg.as_c()
    rc = lib.mbs_ref_fixed(C.byref(c), C.byref(gs), beta, gamma, alpha,
                           abi.ptr(M, C.c_double), C.byref(sec))
    if rc != 0:
        raise RuntimeError("mbs_ref_fixed failed")
    return M, sec.value


def ref_jones_kat(jones: np.ndarray, weights: np.ndarray):
    lib = _ref_lib()
    jones = np.ascontiguousarray(jones, np.float64)
    weights = np.ascontiguousarray(weights, np.float64)
    n = len(weights)
    direct = np.zeros((n, 16))
    legacy = np.zeros((n, 16))
    lib.mbs_ref_jones_kat(n, abi.ptr(jones, C.c_double), abi.ptr(weights, C.c_double),
                          abi.ptr(direct, C.c_double), abi.ptr(legacy, C.c_double))
    return direct, legacy


def scale_batch(batch: BeamBatch, scale: float, wave_index: float, abs_coeff: float) -> BeamBatch:
    """The batch of a particle `scale` times larger, restating the
    reference's ScalePreparedOrientation (src/scattering/TracerPOTotal.cpp:
    2682-2747): vertex coordinates, beam centre and optical path times s, area
    times s^2, and J_phased rebuilt from the unphased Jones matrix,
        J_phased = sign * absorption(s) * J * exp(i k s path),
        absorption(s) = mean over paths L of (L > DBL_EPSILON ? exp(cAbs L s) : 1).
    Needs the batch's raw records (beam_raw, abs_offsets, abs_paths)."""
    if batch.beam_raw is None:
        raise ValueError("scale_batch needs beam_raw")
    s = float(scale)
    out = batch.select(0, batch.n_orient)
    out.vx = batch.vx * s
    out.vy = batch.vy * s
    g = batch.beam_geom.copy()
    g[:, abi.G_CEN:abi.G_CEN + 3] *= s
    g[:, abi.G_AREA] *= s * s
    g[:, abi.G_OPATH] *= s
    raw = batch.beam_raw
    arg = wave_index * raw[:, abi.R_PATH] * s
    cs, sn = np.cos(arg), np.sin(arg)
    absorption = np.ones(batch.n_beams)
    ao, ap = batch.abs_offsets, batch.abs_paths
    if ao is not None and ap is not None and len(ap):
        for b in range(batch.n_beams):
            a0, a1 = int(ao[b]), int(ao[b + 1])
            if a1 > a0:
                L = ap[a0:a1]
                absorption[b] = np.mean(np.where(L > np.finfo(float).eps, np.exp(abs_coeff * L * s), 1.0))
    f = raw[:, abi.R_SIGN] * absorption
    for i in range(4):
        jr, ji = raw[:, abi.R_J + 2 * i], raw[:, abi.R_J + 2 * i + 1]
        g[:, abi.G_JP + 2 * i] = f * (jr * cs - ji * sn)
        g[:, abi.G_JP + 2 * i + 1] = f * (jr * sn + ji * cs)
    out.beam_geom = np.ascontiguousarray(g)
    return out


def thetas_m11(batch: BeamBatch, grid_n_az: int, az_step: float, theta_rad, wave: abi.Wave,
               singular: bool = False):
    """Incoherent azimuth-summed M11 on a zenith list, restating
    HandlerPO::DiffractThetasGpu and theta_m11_kernel (reference
    src/cuda/GpuDiffraction.cu:1909-1956, 4780-4970) on the oracle's
    per-beam Jones: sum_o w_o sum_beams sum_{p<n_az} 0.5 |d|^2 / (n_az + 1),
    d with the GPU rotation convention (no 0.5 factor), zenith angles clamped
    1e-6 off the poles, nearly singular edges dropped (singular=False, as the
    reference does there) or given their stable quotient (singular=True)."""
    th = np.asarray(theta_rad, dtype=np.float64).copy()
    th = np.where(th <= 1e-14, 1e-6, np.where(th >= np.pi - 1e-14, np.pi - 1e-6, th))
    L = _po_lib()
    n = len(th)
    out = np.zeros(n)
    b = batch.as_c(with_raw=False)
    w = wave
    L.po_oracle_thetas_m11(C.byref(b), C.byref(w), grid_n_az, az_step,
                           abi.ptr(np.ascontiguousarray(th), C.c_double), n,
                           1 if singular else 0, abi.ptr(out, C.c_double))
    return out


def phi_upsample_fft(low: np.ndarray, n_full: int) -> np.ndarray:
    """Azimuth upsampling of the reference's FFT-phi path, restated with numpy
    FFTs: fft_upsample_phi_arr2d_impl and fft_phi_pad_kernel
    (src/cuda/GpuDiffraction.cu:3206-3320, :794-814).  Every (zenith row,
    element) series over the n_low azimuth bins of low [n_low, rows, 16] is
    transformed, bin k goes to frequency k (k <= n_low/2) or k - n_low, scaled
    by 1/n_low and placed in an n_full-bin spectrum (negative frequencies at
    n_full + f), transformed back unnormalised (cuFFT's inverse), and the
    real part is returned as [n_full, rows, 16]."""
    low = np.asarray(low, dtype=np.float64)
    n_low = low.shape[0]
    X = np.fft.fft(low, axis=0)
    Y = np.zeros((n_full,) + low.shape[1:], dtype=np.complex128)
    for k in range(n_low):
        f = k if k <= n_low // 2 else k - n_low
        d = f if f >= 0 else n_full + f
        if 0 <= d < n_full:
            Y[d] = X[k] / n_low
    return np.real(np.fft.ifft(Y, axis=0) * n_full)
