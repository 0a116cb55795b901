"""Beam batches (the mbs_po_beams payload) and the reference host producer.

``BeamBatch`` owns numpy copies of the flat arrays that cross the C ABI.
``trace()`` runs MBS-fast's own tracer + HandlerPO::PrepareBeams (compiled from
the reference sources into ``libmbs_host.so``) for a list of orientations, the
way phase 1 of TracerPOTotal::TraceWeightedOrientations does
(reference src/scattering/TracerPOTotal.cpp:5815-5898).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi


@dataclass
class BeamBatch:
    beam_offsets: np.ndarray          # int64 [n_orient+1]
    orient_weight: np.ndarray         # f64   [n_orient]
    vert_offsets: np.ndarray          # int64 [n_beams+1]
    vx: np.ndarray
    vy: np.ndarray
    slope_yx: np.ndarray
    slope_xy: np.ndarray
    edge_flags: np.ndarray            # uint8 [n_verts]
    beam_geom: np.ndarray             # f64   [n_beams, GEOM_STRIDE]
    beam_flags: np.ndarray            # uint8 [n_beams]
    beam_raw: np.ndarray | None = None
    abs_offsets: np.ndarray | None = None
    abs_paths: np.ndarray | None = None
    extinction_ot: np.ndarray | None = None   # host CPU PreparedOrientation::extinctionOt
    trace_seconds: float = 0.0
    # thread-summed tracer and PrepareBeams seconds, wall seconds of packing
    phase_seconds: tuple = (0.0, 0.0, 0.0)
    _keep: list = field(default_factory=list, repr=False)

    @property
    def n_orient(self) -> int:
        return len(self.orient_weight)

    @property
    def n_beams(self) -> int:
        return len(self.beam_flags)

    @property
    def n_verts(self) -> int:
        return len(self.vx)

    def nv(self) -> np.ndarray:
        return np.diff(self.vert_offsets)

    def beams_per_orient(self) -> np.ndarray:
        return np.diff(self.beam_offsets)

    def as_c(self, with_raw: bool = True) -> abi.Beams:
        raw = self.beam_raw if with_raw else None
        b = abi.Beams(
            n_orient=self.n_orient, n_beams=self.n_beams, n_verts=self.n_verts,
            beam_offsets=abi.ptr(self.beam_offsets, C.c_int64),
            orient_weight=abi.ptr(self.orient_weight, C.c_double),
            vert_offsets=abi.ptr(self.vert_offsets, C.c_int64),
            vx=abi.ptr(self.vx, C.c_double), vy=abi.ptr(self.vy, C.c_double),
            slope_yx=abi.ptr(self.slope_yx, C.c_double),
            slope_xy=abi.ptr(self.slope_xy, C.c_double),
            edge_flags=abi.ptr(self.edge_flags, C.c_uint8),
            beam_geom=abi.ptr(self.beam_geom, C.c_double),
            beam_flags=abi.ptr(self.beam_flags, C.c_uint8),
            beam_raw=abi.ptr(raw, C.c_double),
            abs_offsets=abi.ptr(self.abs_offsets if raw is not None else None, C.c_int64),
            abs_paths=abi.ptr(self.abs_paths if raw is not None and self.abs_paths is not None
                              and len(self.abs_paths) else None, C.c_double),
        )
        return b

    def select(self, start: int, count: int) -> "BeamBatch":
        """Orientations [start, start+count) as a new, rebased batch."""
        count = min(count, self.n_orient - start)
        b0, b1 = int(self.beam_offsets[start]), int(self.beam_offsets[start + count])
        v0, v1 = int(self.vert_offsets[b0]), int(self.vert_offsets[b1])
        out = BeamBatch(
            beam_offsets=np.ascontiguousarray(self.beam_offsets[start:start + count + 1] - b0),
            orient_weight=np.ascontiguousarray(self.orient_weight[start:start + count]),
            vert_offsets=np.ascontiguousarray(self.vert_offsets[b0:b1 + 1] - v0),
            vx=np.ascontiguousarray(self.vx[v0:v1]), vy=np.ascontiguousarray(self.vy[v0:v1]),
            slope_yx=np.ascontiguousarray(self.slope_yx[v0:v1]),
            slope_xy=np.ascontiguousarray(self.slope_xy[v0:v1]),
            edge_flags=np.ascontiguousarray(self.edge_flags[v0:v1]),
            beam_geom=np.ascontiguousarray(self.beam_geom[b0:b1]),
            beam_flags=np.ascontiguousarray(self.beam_flags[b0:b1]),
        )
        if self.beam_raw is not None:
            out.beam_raw = np.ascontiguousarray(self.beam_raw[b0:b1])
            a0, a1 = int(self.abs_offsets[b0]), int(self.abs_offsets[b1])
            out.abs_offsets = np.ascontiguousarray(self.abs_offsets[b0:b1 + 1] - a0)
            out.abs_paths = np.ascontiguousarray(self.abs_paths[a0:a1])
        if self.extinction_ot is not None:
            out.extinction_ot = np.ascontiguousarray(self.extinction_ot[start:start + count])
        return out

    @staticmethod
    def concat(parts: list["BeamBatch"]) -> "BeamBatch":
        bo = [np.zeros(1, np.int64)]
        vo = [np.zeros(1, np.int64)]
        ao = [np.zeros(1, np.int64)]
        nb = nv = na = 0
        for p in parts:
            bo.append(p.beam_offsets[1:] + nb)
            vo.append(p.vert_offsets[1:] + nv)
            if p.abs_offsets is not None:
                ao.append(p.abs_offsets[1:] + na)
                na += int(p.abs_offsets[-1])
            nb += p.n_beams
            nv += p.n_verts
        cat = np.concatenate
        out = BeamBatch(
            beam_offsets=cat(bo), orient_weight=cat([p.orient_weight for p in parts]),
            vert_offsets=cat(vo), vx=cat([p.vx for p in parts]), vy=cat([p.vy for p in parts]),
            slope_yx=cat([p.slope_yx for p in parts]), slope_xy=cat([p.slope_xy for p in parts]),
            edge_flags=cat([p.edge_flags for p in parts]),
            beam_geom=cat([p.beam_geom for p in parts]),
            beam_flags=cat([p.beam_flags for p in parts]),
        )
        if all(p.beam_raw is not None for p in parts):
            out.beam_raw = cat([p.beam_raw for p in parts])
            out.abs_offsets = cat(ao)
            out.abs_paths = cat([p.abs_paths for p in parts])
        if all(p.extinction_ot is not None for p in parts):
            out.extinction_ot = cat([p.extinction_ot for p in parts])
        return out

    def save(self, path: str) -> None:
        arrays = {k: v for k, v in self.__dict__.items()
                  if isinstance(v, np.ndarray)}
        np.savez_compressed(path, **arrays)

    @staticmethod
    def load(path: str) -> "BeamBatch":
        with np.load(path) as z:
            kw = {k: z[k] for k in z.files}
        return BeamBatch(**kw)


# ---------------------------------------------------------------- producer ---

@dataclass
class ParticleConfig:
    """Reference CLI particle/run options (see include/mbs_host.h)."""
    particle_type: int = 1
    p: tuple = (100.0, 40.0, 0.0, 0.0)
    particle_file: str | None = None
    resize: float = 0.0
    ri_re: float = 1.3116
    ri_im: float = 0.0
    absorption: bool = False
    wavelength: float = 0.532
    max_reflections: int = 4
    cutoff_off: bool = False
    # --cutoff-profile by name ("legacy-default", "off", "safe", "balanced",
    # "fast"); None: "off" when cutoff_off is set, else "legacy-default"
    cutoff_profile: str | None = None
    shadow_off: bool = False
    legacy_sign: bool = False
    n_threads: int = 0
    # True: the reference's PrepareBeams; False: the producer's bit-identical
    # restatement of it (host/prepare.cpp), several times faster
    reference_prepare: bool = False
    # individual importance thresholds (> 0) over the profile's:
    # --trace-cutoff-importance and --beam-cutoff-importance
    trace_cutoff_importance: float = 0.0
    beam_cutoff_importance: float = 0.0

    PROFILES = ("legacy-default", "off", "safe", "balanced", "fast")

    def _profile(self) -> int:
        if self.cutoff_profile is None:
            return 1 if self.cutoff_off else 0
        return self.PROFILES.index(self.cutoff_profile)

    def as_c(self) -> abi.HostConfig:
        p = (C.c_double * 4)(*([float(x) for x in self.p] + [0.0] * (4 - len(self.p)))[:4])
        return abi.HostConfig(
            particle_type=self.particle_type, p=p,
            particle_file=(self.particle_file.encode() if self.particle_file else None),
            resize=self.resize, ri_re=self.ri_re, ri_im=self.ri_im,
            absorption=int(self.absorption), wavelength=self.wavelength,
            max_reflections=self.max_reflections, cutoff_profile=self._profile(),
            shadow_off=int(self.shadow_off), legacy_sign=int(self.legacy_sign),
            n_threads=self.n_threads, reference_prepare=int(self.reference_prepare),
            trace_cutoff_importance=self.trace_cutoff_importance,
            beam_cutoff_importance=self.beam_cutoff_importance)


def _host():
    lib = abi.load("libmbs_host.so")
    if not getattr(lib, "_mbs_typed", False):
        lib.mbs_host_trace.argtypes = [C.POINTER(abi.HostConfig), C.c_int,
                                       abi._dp, abi._dp, abi._dp, abi._dp,
                                       C.POINTER(C.c_void_p), C.c_char_p, C.c_int]
        lib.mbs_host_batch_view.restype = C.POINTER(abi.Beams)
        lib.mbs_host_batch_view.argtypes = [C.c_void_p]
        lib.mbs_host_batch_extinction.restype = C.c_double
        lib.mbs_host_batch_extinction.argtypes = [C.c_void_p, C.c_int]
        lib.mbs_host_batch_trace_seconds.restype = C.c_double
        lib.mbs_host_batch_trace_seconds.argtypes = [C.c_void_p]
        lib.mbs_host_batch_phase_seconds.restype = C.c_int
        lib.mbs_host_batch_phase_seconds.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        lib.mbs_host_batch_free.argtypes = [C.c_void_p]
        lib.mbs_host_symmetry.argtypes = [C.POINTER(abi.HostConfig), abi._dp, abi._dp, abi._dp]
        lib.mbs_host_sobol_orientations.argtypes = [C.c_int, C.c_uint, C.c_double, C.c_double,
                                                    abi._dp, abi._dp, abi._dp]
        lib.mbs_host_wave.argtypes = [C.POINTER(abi.HostConfig), C.POINTER(abi.Wave)]
        lib.mbs_host_grid.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int, abi._dp,
                                      abi._dp, abi._dp, abi._dp, abi._dp]
        lib._mbs_typed = True
    return lib


def _copy(ptr, n, dtype):
    if n == 0 or not ptr:
        return np.zeros(n, dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


def trace(cfg: ParticleConfig, beta, gamma, weight, alpha=None) -> BeamBatch:
    """Trace + prepare orientations with the reference host code."""
    lib = _host()
    beta = np.ascontiguousarray(beta, np.float64)
    gamma = np.ascontiguousarray(gamma, np.float64)
    weight = np.ascontiguousarray(weight, np.float64)
    alpha = None if alpha is None else np.ascontiguousarray(alpha, np.float64)
    n = len(beta)
    handle = C.c_void_p()
    err = C.create_string_buffer(512)
    c = cfg.as_c()
    rc = lib.mbs_host_trace(C.byref(c), n, abi.ptr(beta, C.c_double),
                            abi.ptr(gamma, C.c_double), abi.ptr(alpha, C.c_double),
                            abi.ptr(weight, C.c_double), C.byref(handle), err, 512)
    abi.check(rc, "mbs_host_trace", err.value.decode(errors="replace"))
    try:
        v = lib.mbs_host_batch_view(handle).contents
        nb, nv = v.n_beams, v.n_verts
        out = BeamBatch(
            beam_offsets=_copy(v.beam_offsets, n + 1, np.int64),
            orient_weight=_copy(v.orient_weight, n, np.float64),
            vert_offsets=_copy(v.vert_offsets, nb + 1, np.int64),
            vx=_copy(v.vx, nv, np.float64), vy=_copy(v.vy, nv, np.float64),
            slope_yx=_copy(v.slope_yx, nv, np.float64),
            slope_xy=_copy(v.slope_xy, nv, np.float64),
            edge_flags=_copy(v.edge_flags, nv, np.uint8),
            beam_geom=_copy(v.beam_geom, nb * abi.GEOM_STRIDE, np.float64).reshape(nb, abi.GEOM_STRIDE),
            beam_flags=_copy(v.beam_flags, nb, np.uint8),
            beam_raw=_copy(v.beam_raw, nb * abi.RAW_STRIDE, np.float64).reshape(nb, abi.RAW_STRIDE),
            abs_offsets=_copy(v.abs_offsets, nb + 1, np.int64),
        )
        out.abs_paths = _copy(v.abs_paths, int(out.abs_offsets[-1]), np.float64)
        out.extinction_ot = np.array([lib.mbs_host_batch_extinction(handle, o) for o in range(n)])
        out.trace_seconds = lib.mbs_host_batch_trace_seconds(handle)
        ph = (C.c_double * 3)()
        if lib.mbs_host_batch_phase_seconds(handle, ph) == 0:
            out.phase_seconds = (ph[0], ph[1], ph[2])
    finally:
        lib.mbs_host_batch_free(handle)
    return out


def symmetry(cfg: ParticleConfig) -> tuple[float, float, float]:
    lib = _host()
    b, g, d = C.c_double(), C.c_double(), C.c_double()
    c = cfg.as_c()
    abi.check(lib.mbs_host_symmetry(C.byref(c), C.byref(b), C.byref(g), C.byref(d)),
              "mbs_host_symmetry")
    return b.value, g.value, d.value


def sobol_orientations(n: int, beta_sym: float, gamma_sym: float, seed: int = 42):
    lib = _host()
    beta, gamma, w = np.empty(n), np.empty(n), np.empty(n)
    abi.check(lib.mbs_host_sobol_orientations(n, seed, beta_sym, gamma_sym,
                                              abi.ptr(beta, C.c_double), abi.ptr(gamma, C.c_double),
                                              abi.ptr(w, C.c_double)), "mbs_host_sobol_orientations")
    return beta, gamma, w


def euler_orientations(beta_sym: float, gamma_sym: float, n_beta: int, n_gamma: int):
    """Gauss-Legendre nodes in cos(beta) x midpoint gamma over the symmetry
    domain, weights summing to 1 (the orientation set of
    TracerPOTotal::BuildEulerOrientations, reference
    src/scattering/TracerPOTotal.cpp:5225-5264)."""
    mu_min, mu_max = sorted((np.cos(beta_sym), 1.0))
    x, wx = np.polynomial.legendre.leggauss(n_beta)
    mu = 0.5 * (mu_max - mu_min) * x + 0.5 * (mu_max + mu_min)
    wmu = 0.5 * (mu_max - mu_min) * wx
    beta = np.arccos(np.clip(mu, -1.0, 1.0))
    bw = wmu / (mu_max - mu_min) if mu_max > mu_min else np.full(n_beta, 1.0 / n_beta)
    gam = gamma_sym * (np.arange(n_gamma) + 0.5) / n_gamma
    B = np.repeat(beta, n_gamma)
    Gm = np.tile(gam, n_beta)
    W = np.repeat(bw / n_gamma, n_gamma)
    return B, Gm, W / W.sum()


def wave(cfg: ParticleConfig) -> abi.Wave:
    lib = _host()
    w = abi.Wave()
    c = cfg.as_c()
    abi.check(lib.mbs_host_wave(C.byref(c), C.byref(w)), "mbs_host_wave")
    return w


@dataclass
class GridTables:
    n_az: int
    n_zen: int
    az_step: float
    theta: np.ndarray      # [n_zen+1]
    vf: np.ndarray         # [n_az, n_zen+1, 3]
    dcos2pi: np.ndarray    # [n_zen+1] Compute2PiDcos
    # how the zenith rows were made: (zen_start_deg, zen_end_deg, n_zen,
    # theta_deg or None), so that the same rows can be paired with another
    # azimuth count (with_azimuths)
    zenith: tuple | None = None

    def with_azimuths(self, n_az: int) -> "GridTables":
        """The same zenith rows on n_az equally spaced azimuth bins (the
        reference's ScatteringRange with nAzimuth and azinuthStep changed)."""
        if self.zenith is None:
            raise ValueError("grid without its zenith construction")
        z0, z1, n_zen, theta_deg = self.zenith
        return grid(z0, z1, n_az, n_zen, theta_deg)

    def as_c(self) -> abi.Grid:
        return abi.Grid(n_az=self.n_az, n_zen=self.n_zen, az_step=self.az_step,
                        theta=abi.ptr(self.theta, C.c_double),
                        vf=abi.ptr(self.vf, C.c_double))

    @property
    def n_dirs(self) -> int:
        return self.n_az * (self.n_zen + 1)


def grid(zen_start_deg: float, zen_end_deg: float, n_az: int, n_zen: int,
         theta_deg=None) -> GridTables:
    """ScatteringRange tables; theta_deg gives a non-uniform zenith grid."""
    lib = _host()
    if theta_deg is not None:
        theta_deg = np.ascontiguousarray(theta_deg, np.float64)
        n_zen = len(theta_deg) - 1
    theta = np.empty(n_zen + 1)
    vf = np.empty((n_az, n_zen + 1, 3))
    dc = np.empty(n_zen + 1)
    step = C.c_double()
    abi.check(lib.mbs_host_grid(zen_start_deg, zen_end_deg, n_az, n_zen,
                                abi.ptr(theta_deg, C.c_double), abi.ptr(theta, C.c_double),
                                abi.ptr(vf, C.c_double), abi.ptr(dc, C.c_double),
                                C.byref(step)), "mbs_host_grid")
    return GridTables(n_az, n_zen, step.value, theta, vf, dc,
                      zenith=(zen_start_deg, zen_end_deg, n_zen, theta_deg))
