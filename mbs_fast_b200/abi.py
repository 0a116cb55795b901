"""ctypes mirror of the C ABI in include/mbs_po_b200.h and include/mbs_host.h.

The structures below must match the C declarations field for field.  Libraries
are loaded from the package's ``_lib`` directory (built in-tree by
``__graft_entry__.build()``); a missing library raises immediately, there is
no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib")

MBS_PO_OK = 0
ERRORS = {
    -1: "EINVAL", -2: "EBEAM", -3: "ECUDA", -4: "ENOMEM",
    -5: "ESTATE", -6: "ETIMEOUT", -7: "ERANGE",
}
FP64 = 0
FP32C = 1

G_BD, G_HOR, G_VER, G_CEN, G_AREA = 0, 3, 6, 9, 12
G_NT, G_NP, G_NXDT, G_NXDP, G_JP, G_OPATH = 13, 16, 19, 22, 25, 33
GEOM_STRIDE = 34
R_J, R_PATH, R_SIGN = 0, 8, 9
RAW_STRIDE = 10
EDGE_VALID_X, EDGE_VALID_Y = 1, 2
BEAM_EXTERNAL = 1

_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_u8p = C.POINTER(C.c_uint8)


class Beams(C.Structure):
    """struct mbs_po_beams"""
    _fields_ = [
        ("n_orient", C.c_int32), ("n_beams", C.c_int64), ("n_verts", C.c_int64),
        ("beam_offsets", _i64p), ("orient_weight", _dp), ("vert_offsets", _i64p),
        ("vx", _dp), ("vy", _dp), ("slope_yx", _dp), ("slope_xy", _dp),
        ("edge_flags", _u8p), ("beam_geom", _dp), ("beam_flags", _u8p),
        ("beam_raw", _dp), ("abs_offsets", _i64p), ("abs_paths", _dp),
    ]


class Grid(C.Structure):
    """struct mbs_po_grid"""
    _fields_ = [("n_az", C.c_int32), ("n_zen", C.c_int32), ("az_step", C.c_double),
                ("theta", _dp), ("vf", _dp)]


class Wave(C.Structure):
    """struct mbs_po_wave"""
    _fields_ = [
        ("wave_index", C.c_double), ("wavelength", C.c_double),
        ("compl_wave_re", C.c_double), ("compl_wave_im", C.c_double),
        ("inv_compl_wave_re", C.c_double), ("inv_compl_wave_im", C.c_double),
        ("eps1", C.c_double), ("abs_coeff", C.c_double),
        ("ot_far_reference_path", C.c_double), ("ot_ping_distance", C.c_double),
        ("legacy_sign", C.c_int32), ("ot_phase_average", C.c_int32),
    ]


class Stats(C.Structure):
    """struct mbs_po_stats"""
    _fields_ = [
        ("kernel_ms", C.c_double), ("reduce_ms", C.c_double),
        ("h2d_ms", C.c_double), ("d2h_ms", C.c_double),
        ("beam_dir_evals", C.c_int64), ("vert_dir_evals", C.c_int64),
        ("launches", C.c_int32), ("n_chunks", C.c_int32),
    ]


class HostConfig(C.Structure):
    """struct mbs_host_config"""
    _fields_ = [
        ("particle_type", C.c_int32), ("p", C.c_double * 4),
        ("particle_file", C.c_char_p), ("resize", C.c_double),
        ("ri_re", C.c_double), ("ri_im", C.c_double), ("absorption", C.c_int32),
        ("wavelength", C.c_double), ("max_reflections", C.c_int32),
        ("cutoff_profile", C.c_int32), ("shadow_off", C.c_int32),
        ("legacy_sign", C.c_int32), ("n_threads", C.c_int32),
        ("reference_prepare", C.c_int32),
        ("trace_cutoff_importance", C.c_double), ("beam_cutoff_importance", C.c_double),
    ]


def ptr(a: np.ndarray | None, ctype):
    """Pointer to a contiguous numpy array (None -> NULL)."""
    if a is None:
        return C.cast(None, C.POINTER(ctype))
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(C.POINTER(ctype))


_LIBS: dict[str, C.CDLL] = {}


def load(name: str) -> C.CDLL:
    """Load an in-tree shared library; raise if it was not built."""
    if name in _LIBS:
        return _LIBS[name]
    path = os.path.join(LIB_DIR, name)
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build the native libraries first "
            "(python -c 'import __graft_entry__ as g; g.build()')")
    lib = C.CDLL(path, mode=C.RTLD_GLOBAL)
    _LIBS[name] = lib
    return lib


def check(rc: int, what: str, msg: str | None = None) -> None:
    if rc != MBS_PO_OK:
        raise RuntimeError(f"{what} failed: {ERRORS.get(rc, rc)}"
                           + (f": {msg}" if msg else ""))
