"""Python mirror of HandlerPO's GPU entry points over the C ABI.

Names, argument meaning and error behaviour follow the reference's
HandlerPO GPU interface (reference src/handler/HandlerPO.h:102-162,
src/cuda/GpuDiffraction.cu:4159-4778):

* ``handle_orientations_to_local_gpu`` adds (never overwrites) the
  weighted Mueller sums of orientations [start, start+count) into
  ``local_m`` (and the no-shadow sums into ``local_m_noshadow``) and returns
  True; it returns False for a batch the GPU path rejects (a beam without
  valid edge data), like the reference, and raises on CUDA errors.
* ``select_gpu_orientation_batch_size`` bounds a batch by device memory.

Mueller arrays are numpy [n_az, n_zen+1, 16] in the reference's
direction order (row p, column t, 16 row-major elements).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi
from .beams import BeamBatch, GridTables

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        L = abi.load("libmbs_po_b200.so")
        vp = C.c_void_p
        L.mbs_po_create.argtypes = [C.POINTER(vp), C.c_int]
        L.mbs_po_destroy.argtypes = [vp]
        L.mbs_po_last_error.argtypes = [vp]
        L.mbs_po_last_error.restype = C.c_char_p
        L.mbs_po_version.restype = C.c_char_p
        L.mbs_po_set_grid.argtypes = [vp, C.POINTER(abi.Grid)]
        L.mbs_po_set_wave.argtypes = [vp, C.POINTER(abi.Wave)]
        L.mbs_po_diffract.argtypes = [vp, C.POINTER(abi.Beams), C.c_int, abi._dp, abi._dp,
                                      C.POINTER(abi.Stats)]
        L.mbs_po_diffract_pinned.argtypes = [vp, C.POINTER(abi.Beams), C.c_int,
                                             C.POINTER(abi._dp), C.POINTER(abi._dp), C.POINTER(abi.Stats)]
        L.mbs_po_diffract_staged_pinned.argtypes = [vp, vp, C.c_int, C.POINTER(abi._dp),
                                                    C.POINTER(abi._dp), C.POINTER(abi.Stats)]
        L.mbs_po_stage.argtypes = [vp, C.POINTER(abi.Beams), C.POINTER(vp)]
        L.mbs_po_staged_free.argtypes = [vp, vp]
        L.mbs_po_restage.argtypes = [vp, C.POINTER(abi.Beams), vp]
        L.mbs_po_stage_repeat.argtypes = [vp, vp, C.c_int, C.POINTER(C.c_int32), abi._dp,
                                          C.POINTER(vp)]
        L.mbs_po_diffract_staged.argtypes = [vp, vp, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.POINTER(abi.Stats)]
        L.mbs_po_extinction.argtypes = [vp, C.POINTER(abi.Beams), abi._dp]
        L.mbs_po_select_batch.argtypes = [vp, C.POINTER(abi.Beams), C.c_int, C.c_int, C.c_double,
                                          C.POINTER(C.c_int)]
        L.mbs_po_probe_fp32_peak.argtypes = [vp, abi._dp]
        L.mbs_po_probe_fp64_peak.argtypes = [vp, abi._dp]
        L.mbs_po_autotune.argtypes = [vp, vp, C.c_int, C.c_int, C.POINTER(C.c_int), abi._dp, C.c_int]
        L.mbs_po_set_variant.argtypes = [vp, C.c_int, C.c_int]
        L.mbs_po_diffract_staged_noalloc.argtypes = [vp, vp, C.c_int, C.c_void_p, C.c_void_p,
                                                     C.c_void_p]
        L.mbs_po_diffract_multisize.argtypes = [vp, C.POINTER(abi.Beams), abi._dp, C.c_int,
                                                C.c_double, C.c_int, abi._dp, abi._dp,
                                                C.POINTER(abi.Stats)]
        L.mbs_po_stage_multisize.argtypes = [vp, C.POINTER(abi.Beams), abi._dp, C.c_int,
                                             C.c_double, C.POINTER(vp)]
        L.mbs_po_staged_sets.argtypes = [vp]
        L.mbs_po_diffract_thetas.argtypes = [vp, C.POINTER(abi.Beams), abi._dp, C.c_int, abi._dp]
        L.mbs_po_phi_average.argtypes = [vp, C.c_void_p, abi._dp, abi._dp, abi._dp, abi._dp,
                                         C.c_void_p]
        L.mbs_po_orientation_rows.argtypes = [vp, C.POINTER(abi.Beams), C.c_int, abi._dp]
        L.mbs_po_phi_interpolate.argtypes = [vp, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                             C.c_void_p]
        L.mbs_po_diffract_fft_phi.argtypes = [vp, C.POINTER(abi.Beams), C.c_int, C.c_int, abi._dp,
                                              abi._dp, C.POINTER(abi.Stats)]
        _lib = L
    return _lib


class Staged:
    """A batch resident in device memory (mbs_po_stage)."""

    def __init__(self, handler: "GpuHandlerPO", handle: C.c_void_p, batch: BeamBatch | None,
                 counts: tuple | None = None, source: "Staged | None" = None):
        self._h = handler
        self.handle = handle
        self._source = source          # a repeated view keeps its source alive
        if batch is not None:
            self._count(batch)
        else:
            self.n_sets = 1
            self.n_orient, self.n_beams, self.n_verts = counts

    def _count(self, batch: BeamBatch) -> None:
        self.n_sets = int(lib().mbs_po_staged_sets(self.handle))
        self.n_orient = batch.n_orient * self.n_sets
        self.n_beams = batch.n_beams * self.n_sets
        self.n_verts = batch.n_verts * self.n_sets

    def free(self) -> None:
        if self.handle:
            lib().mbs_po_staged_free(self._h.ctx, self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class GpuHandlerPO:
    """One device context (the reference's thread_local GpuWorkspace)."""

    def __init__(self, grid: GridTables, wave: abi.Wave, device: int = 0):
        L = lib()
        self.ctx = C.c_void_p()
        abi.check(L.mbs_po_create(C.byref(self.ctx), device), "mbs_po_create")
        self.grid = grid
        self.wave = wave
        self._call(L.mbs_po_set_grid(self.ctx, C.byref(grid.as_c())), "mbs_po_set_grid")
        self._call(L.mbs_po_set_wave(self.ctx, C.byref(wave)), "mbs_po_set_wave")
        self.last_stats = abi.Stats()

    def _call(self, rc: int, what: str) -> None:
        if rc != abi.MBS_PO_OK:
            msg = lib().mbs_po_last_error(self.ctx)
            abi.check(rc, what, msg.decode(errors="replace") if msg else None)

    def close(self) -> None:
        if self.ctx:
            lib().mbs_po_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def new_mueller(self) -> np.ndarray:
        return np.zeros((self.grid.n_az, self.grid.n_zen + 1, 16))

    # -- HandlerPO::HandleOrientationsToLocalGpu ----------------------------
    def handle_orientations_to_local_gpu(self, prepared: BeamBatch, local_m: np.ndarray,
                                         local_m_noshadow: np.ndarray | None = None,
                                         start: int = 0, count: int | None = None,
                                         precision: int = abi.FP64) -> bool:
        if start < 0 or (count is not None and count < 0) or start > prepared.n_orient:
            return False
        if count is None:
            count = prepared.n_orient - start
        batch = prepared if (start == 0 and count >= prepared.n_orient) else prepared.select(start, count)
        assert local_m.shape == (self.grid.n_az, self.grid.n_zen + 1, 16) and local_m.flags.c_contiguous
        b = batch.as_c(with_raw=False)
        rc = lib().mbs_po_diffract(self.ctx, C.byref(b), precision, abi.ptr(local_m, C.c_double),
                                   abi.ptr(local_m_noshadow, C.c_double), C.byref(self.last_stats))
        if rc == -2:   # MBS_PO_EBEAM: the reference returns false ("bad-edge-data")
            return False
        self._call(rc, "mbs_po_diffract")
        return True

    def diffract_pinned(self, batch: BeamBatch, noshadow: bool = False,
                        precision: int = abi.FP64):
        """mbs_po_diffract_pinned: this call's Mueller sums as copies of the
        library's page-locked planes, (M, M_noshadow or None); (None, None)
        when the batch holds no beams."""
        b = batch.as_c(with_raw=False)
        m, mn = abi._dp(), abi._dp()
        rc = lib().mbs_po_diffract_pinned(self.ctx, C.byref(b), precision, C.byref(m),
                                          C.byref(mn) if noshadow else None, C.byref(self.last_stats))
        self._call(rc, "mbs_po_diffract_pinned")
        shape = (self.grid.n_az, self.grid.n_zen + 1, 16)
        n = shape[0] * shape[1] * shape[2]

        def grab(ptr):
            return np.ctypeslib.as_array(ptr, (n,)).reshape(shape).copy() if ptr else None
        return grab(m), grab(mn)

    def diffract_staged_pinned(self, staged: "Staged", noshadow: bool = False,
                               precision: int = abi.FP64):
        """mbs_po_diffract_staged_pinned: diffract_pinned of a batch staged
        earlier (no upload)."""
        m, mn = abi._dp(), abi._dp()
        rc = lib().mbs_po_diffract_staged_pinned(self.ctx, staged.handle, precision, C.byref(m),
                                                 C.byref(mn) if noshadow else None,
                                                 C.byref(self.last_stats))
        self._call(rc, "mbs_po_diffract_staged_pinned")
        shape = (self.grid.n_az, self.grid.n_zen + 1, 16)
        n = shape[0] * shape[1] * shape[2]

        def grab(ptr):
            return np.ctypeslib.as_array(ptr, (n,)).reshape(shape).copy() if ptr else None
        return grab(m), grab(mn)

    # -- HandlerPO::HandleOrientationsToLocalGpuFftPhi ----------------------
    @staticmethod
    def fft_phi_factor(n_full: int, configured: int = 0) -> int:
        """Azimuth factor of the FFT-phi path (reference
        GpuDiffraction.cu:712-726): the configured one, else
        MBS_FFT_PHI_FACTOR (1-64), else 8 / 6 / 3 / 2 for at least 2400 /
        600 / 240 / fewer output azimuths."""
        if configured > 0:
            return configured
        v = os.environ.get("MBS_FFT_PHI_FACTOR", "")
        if v.isdigit() and 1 <= int(v) <= 64:
            return int(v)
        return 8 if n_full >= 2400 else 6 if n_full >= 600 else 3 if n_full >= 240 else 2

    def diffract_fft_phi(self, batch: BeamBatch, low: GridTables, n_full: int,
                         precision: int = abi.FP64, noshadow: bool = False):
        """Direct evaluation on `low` (same zenith rows, fewer azimuth bins),
        interpolated on the device to n_full bins (mbs_po_diffract_fft_phi).
        Returns (M, Mns or None), each [n_full, n_zen+1, 16]."""
        shape = (n_full, low.n_zen + 1, 16)
        M = np.zeros(shape)
        Mns = np.zeros(shape) if noshadow else None
        b = batch.as_c(with_raw=False)
        self._call(lib().mbs_po_set_grid(self.ctx, C.byref(low.as_c())), "mbs_po_set_grid")
        try:
            rc = lib().mbs_po_diffract_fft_phi(self.ctx, C.byref(b), precision, n_full,
                                               abi.ptr(M, C.c_double), abi.ptr(Mns, C.c_double),
                                               C.byref(self.last_stats))
            self._call(rc, "mbs_po_diffract_fft_phi")
        finally:
            self._call(lib().mbs_po_set_grid(self.ctx, C.byref(self.grid.as_c())), "mbs_po_set_grid")
        return M, Mns

    def handle_orientations_to_local_gpu_fft_phi(self, prepared: BeamBatch, local_m: np.ndarray,
                                                 local_m_noshadow: np.ndarray | None = None,
                                                 factor: int = 0,
                                                 precision: int = abi.FP64) -> bool:
        """The FFT-phi path on this handler's grid (reference
        GpuDiffraction.cu:3504-3760): direct evaluation on n_az / factor
        azimuth bins (at least 16), interpolated to n_az; the plain direct
        evaluation when the factor is 1, the grid has fewer than 32 azimuth
        bins or the reduced count would not be smaller."""
        n_full = self.grid.n_az
        f = self.fft_phi_factor(n_full, factor)
        n_low = n_full // f if f > 1 else n_full
        if n_low < 16:
            n_low = min(n_full, 16)
        if f <= 1 or n_full < 32 or n_low >= n_full:
            return self.handle_orientations_to_local_gpu(prepared, local_m, local_m_noshadow,
                                                         precision=precision)
        M, Mns = self.diffract_fft_phi(prepared, self.grid.with_azimuths(n_low), n_full,
                                       precision, noshadow=local_m_noshadow is not None)
        local_m += M
        if local_m_noshadow is not None:
            local_m_noshadow += Mns
        return True

    def phi_interpolate(self, low_dev_ptr: int, n_low: int, n_rows: int, full_dev_ptr: int,
                        n_full: int, stream: int = 0) -> None:
        """mbs_po_phi_interpolate on device arrays (+= into the full grid)."""
        self._call(lib().mbs_po_phi_interpolate(self.ctx, C.c_void_p(low_dev_ptr), n_low, n_rows,
                                                C.c_void_p(full_dev_ptr), n_full, C.c_void_p(stream)),
                   "mbs_po_phi_interpolate")

    # -- HandlerPO::HandleOrientationsToLocalGpuMultiK ----------------------
    def handle_orientations_to_local_gpu_multik(self, prepared: BeamBatch, start: int, count: int,
                                                scales, wave_index: float,
                                                local_ms: list[np.ndarray] | np.ndarray,
                                                precision: int = abi.FP64) -> bool:
        """Adds the Mueller sums of orientations [start, start+count) at every
        size factor in ``scales`` into ``local_ms[i]`` (reference
        GpuDiffraction.cu:3956-4158).  The batch must carry the unphased
        Jones records (traced with raw output).  Returns False where the
        reference does (invalid beams)."""
        if start < 0 or count < 0 or start > prepared.n_orient:
            return False
        sc = np.ascontiguousarray(np.asarray(scales, dtype=np.float64))
        if count == 0 or len(sc) == 0:
            return True
        if len(local_ms) < len(sc):
            return False
        batch = prepared if (start == 0 and count >= prepared.n_orient) else prepared.select(start, count)
        if batch.beam_raw is None:
            raise ValueError("multi-size diffraction needs the unphased Jones records (beam_raw)")
        shape = (self.grid.n_az, self.grid.n_zen + 1, 16)
        out = np.zeros((len(sc),) + shape)
        b = batch.as_c(with_raw=True)
        rc = lib().mbs_po_diffract_multisize(self.ctx, C.byref(b), abi.ptr(sc, C.c_double), len(sc),
                                             float(wave_index), precision,
                                             abi.ptr(out, C.c_double), None,
                                             C.byref(self.last_stats))
        if rc == -2:
            return False
        self._call(rc, "mbs_po_diffract_multisize")
        for i in range(len(sc)):
            local_ms[i] += out[i]
        return True

    def stage_multisize(self, batch: BeamBatch, scales, wave_index: float = 0.0) -> "Staged":
        sc = np.ascontiguousarray(np.asarray(scales, dtype=np.float64))
        h = C.c_void_p()
        b = batch.as_c(with_raw=True)
        self._call(lib().mbs_po_stage_multisize(self.ctx, C.byref(b), abi.ptr(sc, C.c_double),
                                                len(sc), float(wave_index), C.byref(h)),
                   "mbs_po_stage_multisize")
        return Staged(self, h, batch)

    # -- HandlerPO::DiffractThetasGpu ----------------------------------------
    def diffract_thetas_gpu(self, prepared: BeamBatch, theta_rads) -> np.ndarray | None:
        """Incoherent azimuth-summed M11 at the given zenith angles (reference
        GpuDiffraction.cu:4780-4970); None where the reference returns false."""
        th = np.ascontiguousarray(np.asarray(theta_rads, dtype=np.float64))
        out = np.zeros(len(th))
        b = prepared.as_c(with_raw=False)
        rc = lib().mbs_po_diffract_thetas(self.ctx, C.byref(b), abi.ptr(th, C.c_double), len(th),
                                          abi.ptr(out, C.c_double))
        if rc == -2:
            return None
        self._call(rc, "mbs_po_diffract_thetas")
        return out

    # -- HandlerPOTotal::WriteMatricesToFile rows, on the device ----------------
    def phi_average_gpu(self, m_dev_ptr: int, stream: int = 0):
        """Azimuth-averaged rows [(n_zen+1), 16], C_sca and the asymmetry
        parameter g of a device-resident Mueller grid."""
        rows = np.zeros((self.grid.n_zen + 1, 16))
        csca, g = C.c_double(), C.c_double()
        dc = np.ascontiguousarray(self.grid.dcos2pi, dtype=np.float64)
        self._call(lib().mbs_po_phi_average(self.ctx, C.c_void_p(m_dev_ptr), abi.ptr(dc, C.c_double),
                                            abi.ptr(rows, C.c_double), C.byref(csca), C.byref(g),
                                            C.c_void_p(stream)), "mbs_po_phi_average")
        return rows, csca.value, g.value

    def orientation_rows(self, batch: BeamBatch, precision: int = abi.FP64) -> np.ndarray:
        """Azimuth-averaged rows of every orientation alone (times its
        weight): [n_orient, n_zen+1, 16]."""
        out = np.zeros((batch.n_orient, self.grid.n_zen + 1, 16))
        b = batch.as_c(with_raw=False)
        self._call(lib().mbs_po_orientation_rows(self.ctx, C.byref(b), precision,
                                                 abi.ptr(out, C.c_double)),
                   "mbs_po_orientation_rows")
        return out

    # -- HandlerPO::SelectGpuOrientationBatchSize ---------------------------
    def select_gpu_orientation_batch_size(self, prepared: BeamBatch, start: int, max_count: int,
                                          mem_fraction: float = 0.88) -> int:
        b = prepared.as_c(with_raw=False)
        out = C.c_int()
        self._call(lib().mbs_po_select_batch(self.ctx, C.byref(b), start, max_count, mem_fraction,
                                             C.byref(out)), "mbs_po_select_batch")
        return out.value

    # -- HandlerPO::ComputeForwardExtinctionOt on the device ----------------
    def extinction(self, prepared: BeamBatch) -> np.ndarray:
        out = np.zeros(prepared.n_orient)
        b = prepared.as_c(with_raw=False)
        self._call(lib().mbs_po_extinction(self.ctx, C.byref(b), abi.ptr(out, C.c_double)),
                   "mbs_po_extinction")
        return out

    def probe_fp32_peak(self) -> float:
        """Measured FP32 FMA throughput of this device, TFLOP/s."""
        v = C.c_double()
        self._call(lib().mbs_po_probe_fp32_peak(self.ctx, C.byref(v)), "mbs_po_probe_fp32_peak")
        return v.value

    def probe_fp64_peak(self) -> float:
        """Measured FP64 FMA throughput of this device, TFLOP/s."""
        v = C.c_double()
        self._call(lib().mbs_po_probe_fp64_peak(self.ctx, C.byref(v)), "mbs_po_probe_fp64_peak")
        return v.value

    def diffract_staged_noalloc(self, staged: Staged, m_dev_ptr: int,
                                mns_dev_ptr: int | None = None, precision: int = abi.FP64,
                                stream: int = 0) -> None:
        """mbs_po_diffract_staged_noalloc: the same accumulation with the
        chunk partials in the library's fixed device array (no allocation).
        Calls sharing the array must not overlap on the GPU."""
        self._call(lib().mbs_po_diffract_staged_noalloc(
            self.ctx, staged.handle, precision, C.c_void_p(m_dev_ptr),
            C.c_void_p(mns_dev_ptr) if mns_dev_ptr else None, C.c_void_p(stream)),
            "mbs_po_diffract_staged_noalloc")

    def autotune(self, staged: "Staged", precision: int, max_orient: int = 256):
        """Time every compiled launch shape on the staged batch; keep the
        fastest.  Returns (best index, per-shape kernel ms)."""
        best = C.c_int()
        ms = np.zeros(16)
        self._call(lib().mbs_po_autotune(self.ctx, staged.handle, precision, max_orient,
                                         C.byref(best), abi.ptr(ms, C.c_double), len(ms)),
                   "mbs_po_autotune")
        return best.value, [m for m in ms if m > 0]

    def set_variant(self, precision: int, variant: int) -> None:
        self._call(lib().mbs_po_set_variant(self.ctx, precision, variant), "mbs_po_set_variant")

    # -- device-resident path -------------------------------------------------
    def stage(self, batch: BeamBatch) -> Staged:
        h = C.c_void_p()
        b = batch.as_c(with_raw=False)
        self._call(lib().mbs_po_stage(self.ctx, C.byref(b), C.byref(h)), "mbs_po_stage")
        return Staged(self, h, batch)

    def stage_repeat(self, src: Staged, orient_index, weight) -> Staged:
        """mbs_po_stage_repeat: orientations orient_index of `src` (which
        must outlive the result) with the given weights, sharing src's
        device records."""
        idx = np.ascontiguousarray(orient_index, dtype=np.int32)
        w = np.ascontiguousarray(weight, dtype=np.float64)
        h = C.c_void_p()
        self._call(lib().mbs_po_stage_repeat(self.ctx, src.handle, len(idx), abi.ptr(idx, C.c_int32),
                                             abi.ptr(w, C.c_double), C.byref(h)), "mbs_po_stage_repeat")
        return Staged(self, h, None, counts=(int(len(idx)), src.n_beams, src.n_verts), source=src)

    def restage(self, staged: Staged, batch: BeamBatch) -> Staged:
        """mbs_po_restage: re-fill `staged` with `batch` in the device memory
        it holds (every diffraction reading it must have completed)."""
        b = batch.as_c(with_raw=False)
        rc = lib().mbs_po_restage(self.ctx, C.byref(b), staged.handle)
        staged._count(batch if rc == 0 else batch.select(0, 0))
        self._call(rc, "mbs_po_restage")
        return staged

    def diffract_staged(self, staged: Staged, m_dev_ptr: int, mns_dev_ptr: int | None = None,
                        precision: int = abi.FP64, stream: int = 0,
                        stats: abi.Stats | None | bool = None) -> None:
        """Accumulate the staged batch into device arrays on `stream`.  With
        stats=False no statistics are taken, so the call neither waits for
        the device nor does anything a CUDA graph capture forbids (after one
        earlier call has sized the context's scratch)."""
        if stats is False:
            sp = None
        else:
            sp = C.byref(stats if stats is not None else self.last_stats)
        self._call(lib().mbs_po_diffract_staged(self.ctx, staged.handle, precision,
                                                C.c_void_p(m_dev_ptr),
                                                C.c_void_p(mns_dev_ptr) if mns_dev_ptr else None,
                                                C.c_void_p(stream), sp),
                   "mbs_po_diffract_staged")
