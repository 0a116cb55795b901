"""Error measures of a Mueller grid against a reference grid.

The measures follow the reference's release gate and the error statement
of the PO path:

* weighted L2: solid-angle weighted relative L2 over the 16 elements of
  the azimuth-averaged rows (reference tests/run_cuda_release_gate.sh:70-86,
  rows as HandlerPOTotal::WriteMatricesToFile writes them,
  src/handler/HandlerPOTotal.cpp:23-122);
* M11: maximum and weighted relative error of the azimuth-averaged rows;
* M12/M11, M22/M11, M33/M11, M34/M11, M44/M11: maximum absolute error of
  the normalised elements;
* C_sca and the asymmetry parameter g of the rows, C_ext of the batch.

Rows come from the library's own device azimuth average
(mbs_po_phi_average), so the measures need no CPU restatement.
"""
from __future__ import annotations

import numpy as np

NORMALISED = (("M12", 1), ("M22", 5), ("M33", 10), ("M34", 11), ("M44", 15))


def device_rows(handler, M: np.ndarray):
    """Azimuth-averaged rows [(n_zen+1), 16], C_sca and g of a host Mueller
    grid [n_az, n_zen+1, 16], averaged on the handler's device."""
    import torch
    dev = torch.from_numpy(np.ascontiguousarray(M, dtype=np.float64).reshape(-1)).to(
        f"cuda:{torch.cuda.current_device()}")
    torch.cuda.synchronize()
    rows, csca, g = handler.phi_average_gpu(dev.data_ptr())
    torch.cuda.synchronize()
    return rows, csca, g


def row_errors(rows: np.ndarray, ref: np.ndarray, dcos2pi: np.ndarray) -> dict:
    """Errors of azimuth-averaged rows against reference rows (rows with a
    zero reference M11 are left out of the relative measures)."""
    w = np.asarray(dcos2pi, dtype=np.float64)
    ok = np.abs(ref[:, 0]) > 0
    rel = np.abs(rows[ok, 0] - ref[ok, 0]) / np.abs(ref[ok, 0])
    out = {"M11_max_rel": float(rel.max()) if rel.size else 0.0,
           "M11_weighted_rel": float(np.sqrt(np.sum(w[ok] * (rows[ok, 0] - ref[ok, 0]) ** 2)
                                             / max(np.sum(w[ok] * ref[ok, 0] ** 2), 1e-300)))}
    for name, idx in NORMALISED:
        d = rows[ok, idx] / rows[ok, 0] - ref[ok, idx] / ref[ok, 0]
        out[name + "/M11_max_abs"] = float(np.max(np.abs(d))) if d.size else 0.0
    out["weighted_L2_all16"] = float(np.sqrt(np.sum(w[:, None] * (rows - ref) ** 2)
                                             / max(np.sum(w[:, None] * ref ** 2), 1e-300)))
    return out


def compare(handler, M: np.ndarray, M_ref: np.ndarray, cext=None, cext_ref=None) -> dict:
    """All error measures of grid M against M_ref (both host arrays on the
    handler's grid); C_ext errors when per-orientation values are given."""
    r, csca, g = device_rows(handler, M)
    q, csca_r, g_r = device_rows(handler, M_ref)
    out = row_errors(r, q, handler.grid.dcos2pi)
    out["Csca_rel"] = float(abs(csca / csca_r - 1.0)) if csca_r else None
    out["g_abs"] = float(abs(g - g_r))
    if cext is not None and cext_ref is not None:
        a, b = float(np.sum(cext)), float(np.sum(cext_ref))
        out["Cext_rel"] = float(abs(a / b - 1.0)) if b else None
    return out
