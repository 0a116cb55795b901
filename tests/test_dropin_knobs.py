"""The drop-in's environment knobs, through the library's pure helpers (CPU):
the multi-device split of MBS_GPU_MULTI / MBS_GPU_MULTI_MAX
(gpu_multi_device_count, reference src/cuda/GpuDiffraction.cu:595-626, and
the contiguous ranges of :4224-4226), the MBS_GPU_EPS1 override
(gpu_effective_eps1, :498-512) and the MBS_GPU_BEAM_STATS line (:4354-4443)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from mbs_fast_b200 import abi, beams as B

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _lib():
    L = abi.load("libmbs_po_b200.so")
    L.mbs_po_multi_devices.argtypes = [C.c_int, C.c_int, C.c_char_p, C.c_char_p, C.c_int]
    L.mbs_po_device_range.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int),
                                      C.POINTER(C.c_int)]
    L.mbs_po_eps1_override.argtypes = [C.c_double, C.c_char_p]
    L.mbs_po_eps1_override.restype = C.c_double
    L.mbs_po_beam_stats.argtypes = [C.POINTER(abi.Beams), C.c_char_p, C.c_int]
    return L


def _enc(v):
    return None if v is None else v.encode()


@pytest.mark.parametrize("work,devices,multi,cap,mpi,want", [
    (100, 8, None, None, 0, 8),      # default: every visible device
    (100, 8, "0", None, 0, 1),       # MBS_GPU_MULTI=0 disables
    (100, 8, "3", None, 0, 3),       # a limit
    (100, 8, "12", None, 0, 8),      # limit above the device count
    (100, 8, None, "2", 0, 2),       # MBS_GPU_MULTI_MAX caps
    (100, 8, "6", "4", 0, 4),
    (100, 8, None, None, 1, 1),      # off under MPI unless asked for
    (100, 8, "4", None, 1, 4),
    (3, 8, None, None, 0, 3),        # never more devices than orientations
    (1, 8, None, None, 0, 1),
    (100, 1, None, None, 0, 1),
    (100, 8, "x", None, 0, 8),       # unparsable values are ignored
    (100, 8, "-2", "0", 0, 8),
    (100, 8, "", None, 1, 1),
])
def test_multi_device_count(work, devices, multi, cap, mpi, want):
    assert _lib().mbs_po_multi_devices(work, devices, _enc(multi), _enc(cap), mpi) == want


@pytest.mark.parametrize("start,count,n", [(0, 100, 8), (17, 5, 3), (3, 1, 1), (0, 1023, 7)])
def test_device_ranges_partition_the_batch(start, count, n):
    L = _lib()
    b, c = C.c_int(), C.c_int()
    edges = []
    for d in range(n):
        L.mbs_po_device_range(start, count, n, d, C.byref(b), C.byref(c))
        assert b.value == start + count * d // n and c.value >= 0
        edges.append((b.value, b.value + c.value))
    assert edges[0][0] == start and edges[-1][1] == start + count
    assert all(edges[i][1] == edges[i + 1][0] for i in range(n - 1))


@pytest.mark.parametrize("value,want", [(None, 2.2e-7), ("1e-3", 1e-3), ("0", 2.2e-7),
                                        ("-1e-3", 2.2e-7), ("1e-3x", 2.2e-7), ("", 2.2e-7),
                                        ("5e-6", 5e-6)])
def test_eps1_override(value, want):
    assert _lib().mbs_po_eps1_override(2.2e-7, _enc(value)) == want


def test_beam_stats_line():
    batch = B.BeamBatch.load(os.path.join(GOLD, "hex10x20_batch.npz"))
    buf = C.create_string_buffer(1024)
    b = batch.as_c(with_raw=False)
    assert _lib().mbs_po_beam_stats(C.byref(b), buf, 1024) == 0
    line = buf.value.decode()
    per = np.diff(batch.beam_offsets)
    nv = np.diff(batch.vert_offsets)
    ext = int(np.count_nonzero(batch.beam_flags & 1))
    ex = np.count_nonzero(batch.edge_flags & 1) / batch.n_beams
    ey = np.count_nonzero(batch.edge_flags & 2) / batch.n_beams
    want = (f"GPU beam stats orient={batch.n_orient} beams={batch.n_beams} beams/orient "
            f"min={per.min()} mean={batch.n_beams / batch.n_orient:.3f} max={per.max()} "
            f"external={ext} internal={batch.n_beams - ext} valid_edges_x/beams={ex:.3f} "
            f"valid_edges_y/beams={ey:.3f} vertices:")
    assert line.startswith(want), (line, want)
    hist = dict((int(k), int(v)) for k, v in re.findall(r" (\d+):(\d+)", line[len(want):]))
    vals, cnts = np.unique(nv, return_counts=True)
    assert hist == {int(k): int(c) for k, c in zip(vals, cnts)}
