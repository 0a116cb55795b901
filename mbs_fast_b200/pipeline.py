"""Host tracing overlapped with device diffraction.

Once the diffraction runs on the B200, the orientation average is bound by
the host's beam-splitting tracer (the reference runs it as phase 1,
TracerPOTotal.cpp:5815-5898, before diffracting).  This pipeline traces
batch k+1 on the host cores (the reference tracer behind include/mbs_host.h,
OpenMP) while the device diffracts batch k into one device accumulator, so
the wall time approaches max(trace, diffract) instead of their sum.  The
accumulator receives the batches in order, so the result is the same as one
call over all orientations split the same way.
"""
from __future__ import annotations

import dataclasses
import os
import queue
import threading
import time

import numpy as np

from . import abi, beams as B


def batch_edges(n: int, batch: int) -> list[int]:
    """Boundaries of the pipeline's batches over n orientations: a quarter
    batch first, full batches, and the remainder split so that the last
    batch is at most half a batch."""
    if n <= batch:
        return [0, n] if n > 0 else [0]
    edges = [0, min(n, max(1, batch // 4))]
    while n - edges[-1] > batch + batch // 2:
        edges.append(edges[-1] + batch)
    rest = n - edges[-1]
    if rest > batch // 2:
        edges.append(edges[-1] + rest - batch // 2)
    edges.append(n)
    return edges


def orientation_average(handler, cfg, beta, gamma, weight, precision: int = abi.FP32C,
                        batch: int = 2048, depth: int = 2, noshadow: bool = False):
    """Weighted Mueller sums [n_az, n_zen+1, 16] (and no-shadow sums) of the
    orientations (beta, gamma, weight), traced in batches on the host while
    the previous batch diffracts.  Returns (M, Mns or None, timings)."""
    import torch
    g = handler.grid
    n = len(beta)
    dev = torch.device(f"cuda:{torch.cuda.current_device()}")
    acc = torch.zeros(g.n_az * (g.n_zen + 1) * 16, dtype=torch.float64, device=dev)
    acc_ns = torch.zeros_like(acc) if noshadow else None
    q: queue.Queue = queue.Queue(maxsize=max(1, depth))
    err: list = []
    t_trace = [0.0]

    # the tracer's OpenMP threads leave one core to this thread, which stages
    # each batch (page copies, record building) while they trace the next:
    # on all cores the staging waited for a core and some passes took twice
    # as long (16-core host: 0.83-1.83 s against 0.82-0.89 s per 16,384
    # orientations)
    if cfg.n_threads <= 0:
        cfg = dataclasses.replace(cfg, n_threads=max(1, (os.cpu_count() or 2) - 1))

    # batch boundaries: a short first batch (the device starts sooner) and a
    # short last one (less device work left once tracing ends), `batch`
    # orientations in between
    edges = batch_edges(n, batch)

    def producer():
        try:
            for s, e in zip(edges[:-1], edges[1:]):
                t0 = time.perf_counter()
                b = B.trace(cfg, beta[s:e], gamma[s:e], weight[s:e])
                t_trace[0] += time.perf_counter() - t0
                q.put(b)
        except Exception as ex:      # surfaced to the caller after the join
            err.append(ex)
        finally:
            q.put(None)

    t0 = time.perf_counter()
    th = threading.Thread(target=producer, daemon=True)
    th.start()
    cur = torch.cuda.current_stream(dev)
    stream = cur.cuda_stream
    # a ring of depth + 1 staged batches, each re-filled (mbs_po_restage) once
    # the stream has passed the diffraction that read it: the next batch is
    # staged while the previous ones diffract, and nothing is freed (cudaFree
    # would wait for the whole device) or allocated once the slots have grown
    ring = []
    n_beams = 0
    while True:
        b = q.get()
        if b is None:
            break
        n_beams += b.n_beams
        if len(ring) > depth:
            st, ev = ring.pop(0)
            ev.synchronize()
            handler.restage(st, b)
        else:
            st = handler.stage(b)
        # stats=False: the call neither times nor waits for its kernels
        handler.diffract_staged(st, acc.data_ptr(), acc_ns.data_ptr() if noshadow else None,
                                precision=precision, stream=stream, stats=False)
        ev = torch.cuda.Event()
        ev.record(cur)
        ring.append((st, ev))
    th.join()
    cur.synchronize()
    for st, _ in ring:
        st.free()
    if err:
        raise err[0]
    wall = time.perf_counter() - t0
    M = acc.cpu().numpy().reshape(g.n_az, g.n_zen + 1, 16)
    Mns = acc_ns.cpu().numpy().reshape(g.n_az, g.n_zen + 1, 16) if noshadow else None
    return M, Mns, {"wall_s": wall, "trace_s": t_trace[0], "beams": n_beams}
