"""Learned orientation proposal for the adaptive orientation average.

The orientation average of MBS-fast integrates per-orientation Mueller rows
f(q) over the symmetry-reduced orientation domain, parameterised by the unit
square (u, v) of its Sobol sampler:
    beta = acos(1 - (1 - cos beta_sym) u),   gamma = gamma_sym v
(the azimuth alpha is integrated by the scattering grid's phi bins).  Plain
quasi-random averaging takes Sobol points with equal weights 1/N.  Here a
network trained on a pilot run predicts, from the unit quaternion of an
orientation, the log of that orientation's contribution to the variance of the
averaged rows; the proposal density is a defensive mixture of the network's
density and the uniform one, tabulated on a C x C cell grid of the unit
square, and sampled by a 2-D inverse transform of scrambled Sobol points.
Every sample carries the importance weight p0 / g / N, so the weighted sum
(which the diffraction kernels compute with these weights as orientation
weights) is an unbiased estimate of the same average.  The plain Sobol
average remains the fallback (used when the fit is poor, or when the held-out
pilot orientations predict no clear variance reduction) and the measure of the
error.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def to_angles(u, v, beta_sym: float, gamma_sym: float):
    """Unit-square coordinates -> (beta, gamma), the Sobol sampler's map."""
    u, v = np.asarray(u, dtype=np.float64), np.asarray(v, dtype=np.float64)
    beta = np.arccos(np.clip(1.0 - (1.0 - np.cos(beta_sym)) * u, -1.0, 1.0))
    return beta, gamma_sym * v


def quaternion(beta, gamma, alpha=0.0) -> np.ndarray:
    """Unit quaternion (w, x, y, z) of the ZYZ Euler rotation
    Rz(alpha) Ry(beta) Rz(gamma)."""
    beta, gamma = np.asarray(beta, dtype=np.float64), np.asarray(gamma, dtype=np.float64)
    a = np.broadcast_to(np.asarray(alpha, dtype=np.float64), beta.shape)
    cb, sb = np.cos(beta / 2), np.sin(beta / 2)
    cs, ss = np.cos((a + gamma) / 2), np.sin((a + gamma) / 2)
    cd, sd = np.cos((a - gamma) / 2), np.sin((a - gamma) / 2)
    return np.stack([cb * cs, -sb * sd, sb * cd, cb * ss], axis=-1)


def variance_targets(rows: np.ndarray, rows_mask=None, eps: float = 1e-12) -> np.ndarray:
    """Per-orientation importance from pilot rows [n, n_t, 16] (each
    orientation alone, equal weights): the RMS over the zenith rows selected
    by rows_mask (all rows when None) of its influence on the relative error
    of the averaged M11 and on the error of the ratio M12/M11,
        a_i(t) = f11_i(t) / mean f11(t),
        b_i(t) = (f12_i(t) - R(t) f11_i(t)) / mean f11(t),  R = mean f12 / mean f11,
    h_i = sqrt(mean_t (a_i^2 + b_i^2)); returns log h_i."""
    if rows_mask is not None:
        rows = rows[:, np.asarray(rows_mask, dtype=bool), :]
    f11, f12 = rows[:, :, 0], rows[:, :, 1]
    m11 = f11.mean(axis=0)
    ok = np.abs(m11) > eps * np.max(np.abs(m11))
    m11 = np.where(ok, m11, 1.0)
    R = np.where(ok, f12.mean(axis=0) / m11, 0.0)
    a = f11 / m11
    b = (f12 - R * f11) / m11
    h = np.sqrt(np.mean((a * a + b * b)[:, ok], axis=1))
    return np.log(h + eps)


@dataclass
class Proposal:
    """Piecewise-constant density on a C x C grid of the unit square."""
    prob: np.ndarray          # [C, C] cell probabilities (rows: u, columns: v), sum 1
    learned: bool             # False: the uniform (plain Sobol) fallback

    @property
    def cells(self) -> int:
        return self.prob.shape[0]

    def sample(self, n: int, seed: int = 0):
        """n points (u, v) and their importance weights p0 / g / n by the
        inverse transform of scrambled Sobol points (row by the u-marginal,
        column by the conditional in that row, the remainders place the point
        inside its cell)."""
        from scipy.stats import qmc
        C = self.cells
        s = qmc.Sobol(d=2, scramble=True, seed=seed).random(n)
        row_p = self.prob.sum(axis=1)
        row_cdf = np.concatenate([[0.0], np.cumsum(row_p)])
        row_cdf[-1] = 1.0
        r = np.clip(np.searchsorted(row_cdf, s[:, 0], side="right") - 1, 0, C - 1)
        fu = np.clip((s[:, 0] - row_cdf[r]) / np.maximum(row_p[r], 1e-300), 0.0, 1.0 - 1e-12)
        cond = self.prob[r] / np.maximum(row_p[r], 1e-300)[:, None]
        col_cdf = np.concatenate([np.zeros((n, 1)), np.cumsum(cond, axis=1)], axis=1)
        col_cdf[:, -1] = 1.0
        c = np.clip((col_cdf <= s[:, 1:2]).sum(axis=1) - 1, 0, C - 1)
        lo = col_cdf[np.arange(n), c]
        fv = np.clip((s[:, 1] - lo) / np.maximum(cond[np.arange(n), c], 1e-300), 0.0, 1.0 - 1e-12)
        u = (r + fu) / C
        v = (c + fv) / C
        w = 1.0 / (C * C * self.prob[r, c]) / n
        return u, v, w


def proposal_density(prop: "Proposal", u, v) -> np.ndarray:
    """Density g(u, v) of a proposal on the unit square (C^2 times the
    probability of the point's cell; the uniform density is 1)."""
    C = prop.cells
    r = np.clip((np.asarray(u) * C).astype(np.int64), 0, C - 1)
    c = np.clip((np.asarray(v) * C).astype(np.int64), 0, C - 1)
    return C * C * prop.prob[r, c]


def balance_weights(prop: "Proposal", n_pilot: int, pilot_uv, main_uv):
    """Weights that combine a plain pilot (n_pilot points from the uniform
    density) and N points from the proposal into one unbiased estimate of the
    average (the balance heuristic of multiple importance sampling): every
    point x, whichever sampler drew it, gets 1 / (n_pilot + N g(x)), so
    E[sum] = n_pilot int f/(n_pilot+Ng) + N int f g/(n_pilot+Ng) = int f.
    Returns (pilot weights, main weights)."""
    n_main = len(main_uv[0])
    wp = 1.0 / (n_pilot + n_main * proposal_density(prop, *pilot_uv))
    wm = 1.0 / (n_pilot + n_main * proposal_density(prop, *main_uv))
    return wp, wm


def uniform_proposal(cells: int = 128) -> Proposal:
    return Proposal(np.full((cells, cells), 1.0 / (cells * cells)), learned=False)


def plain_sobol(n: int, seed: int = 0):
    """Plain quasi-random points with equal weights (the fallback and the error reference)."""
    from scipy.stats import qmc
    s = qmc.Sobol(d=2, scramble=True, seed=seed).random(n)
    return s[:, 0], s[:, 1], np.full(n, 1.0 / n)


class LearnedProposal:
    """Trains the network on pilot (orientation, log importance) pairs and
    tabulates the proposal."""

    def __init__(self, beta_sym: float, gamma_sym: float, device: int = 0, seed: int = 1):
        from .mlp import ProposalNet
        self.beta_sym, self.gamma_sym = beta_sym, gamma_sym
        self.net = ProposalNet(device=device, seed=seed)
        self.mean = 0.0
        self.std = 1.0
        self.fit_r2 = None

    def quats(self, u, v) -> np.ndarray:
        b, g = to_angles(u, v, self.beta_sym, self.gamma_sym)
        return quaternion(b, g).astype(np.float32)

    def fit(self, u, v, log_h, epochs: int = 300, batch: int = 256, lr: float = 2e-3,
            holdout: float = 0.2, seed: int = 7) -> float:
        """Train on the pilot points; returns the held-out R^2 of the fit."""
        q = self.quats(u, v)
        y = np.asarray(log_h, dtype=np.float64)
        self.mean, self.std = float(y.mean()), float(y.std() + 1e-12)
        t = ((y - self.mean) / self.std).astype(np.float32)
        n = len(t)
        rng = np.random.default_rng(seed)
        perm = rng.permutation(n)
        nh = max(1, int(holdout * n))
        te, tr = perm[:nh], perm[nh:]
        self.holdout = te
        self.net.train(q[tr], t[tr], epochs=epochs, batch=batch, lr=lr, seed=seed)
        pred = self.net.forward(q[te])
        ss_res = float(np.sum((pred - t[te]) ** 2))
        ss_tot = float(np.sum((t[te] - t[te].mean()) ** 2)) + 1e-30
        self.fit_r2 = 1.0 - ss_res / ss_tot
        return self.fit_r2

    def proposal(self, cells: int = 128, mix: float = 0.7, min_r2: float = 0.2) -> Proposal:
        """Cell probabilities mix * h / sum h + (1 - mix) / C^2, h the network's
        importance at the cell centres; the uniform proposal when the fit's
        held-out R^2 is below min_r2."""
        if self.fit_r2 is None or self.fit_r2 < min_r2:
            return uniform_proposal(cells)
        c = (np.arange(cells) + 0.5) / cells
        U, V = np.meshgrid(c, c, indexing="ij")
        y = self.net.forward(self.quats(U.ravel(), V.ravel())).astype(np.float64)
        h = np.exp(y * self.std + self.mean).reshape(cells, cells)
        p = mix * h / h.sum() + (1.0 - mix) / (cells * cells)
        return Proposal(p / p.sum(), learned=True)

    def close(self) -> None:
        self.net.close()


def predicted_variance_ratio(rows: np.ndarray, g: np.ndarray, rows_mask=None,
                             eps: float = 1e-12) -> float:
    """Variance of the importance-sampled estimate against plain sampling,
    predicted from uniformly drawn pilot orientations (rows [n, n_t, 16],
    orientation weight 1) and the proposal density g at them: summed over
    the rows of rows_mask, for the relative M11 error and the -M12/M11 error
    (the quantities variance_targets weighs),
        plain:      mean_i x_i^2 - (mean_i x_i)^2
        importance: mean_i x_i^2 / g_i - (mean_i x_i)^2
    for x = a_i(t) and b_i(t).  Below 1 the proposal should help."""
    if rows_mask is not None:
        rows = rows[:, np.asarray(rows_mask, dtype=bool), :]
    f11, f12 = rows[:, :, 0], rows[:, :, 1]
    m11 = f11.mean(axis=0)
    ok = np.abs(m11) > eps * np.max(np.abs(m11))
    m11 = np.where(ok, m11, 1.0)
    R = np.where(ok, f12.mean(axis=0) / m11, 0.0)
    a = (f11 / m11)[:, ok]
    b = ((f12 - R * f11) / m11)[:, ok]
    g = np.asarray(g, dtype=np.float64)[:, None]
    plain = sum(float(np.sum(np.mean(x * x, axis=0) - np.mean(x, axis=0) ** 2)) for x in (a, b))
    imp = sum(float(np.sum(np.mean(x * x / g, axis=0) - np.mean(x, axis=0) ** 2)) for x in (a, b))
    return imp / plain if plain > 0 else 1.0


def row_errors(rows: np.ndarray, ref: np.ndarray, rows_mask=None, eps: float = 1e-12) -> dict:
    """Errors of averaged rows [n_t, 16] against a reference over the zenith
    rows selected by rows_mask (all when None): RMS and max of the relative
    M11 error and of the absolute error of -M12/M11."""
    if rows_mask is not None:
        k = np.asarray(rows_mask, dtype=bool)
        rows, ref = rows[k], ref[k]
    m, r = rows[:, 0], ref[:, 0]
    ok = np.abs(r) > eps * np.max(np.abs(r))
    rel = (m[ok] - r[ok]) / r[ok]
    p, pr = -rows[ok, 1] / m[ok], -ref[ok, 1] / r[ok]
    return {"M11_rms_rel": float(np.sqrt(np.mean(rel ** 2))),
            "M11_max_rel": float(np.max(np.abs(rel))),
            "P_rms_abs": float(np.sqrt(np.mean((p - pr) ** 2))),
            "P_max_abs": float(np.max(np.abs(p - pr)))}


def averaged_rows(handler, batch, precision: int, stream: int = 0):
    """Orientation-averaged, azimuth-averaged rows [n_t, 16] of a batch
    (weights as given) on the device: staged diffraction into a device
    accumulator, then the device azimuth average; also C_sca and g."""
    import torch
    g = handler.grid
    dev = torch.zeros(g.n_az * (g.n_zen + 1) * 16, dtype=torch.float64,
                      device=f"cuda:{torch.cuda.current_device()}")
    st = handler.stage(batch)
    try:
        torch.cuda.synchronize()
        handler.diffract_staged(st, dev.data_ptr(), precision=precision, stream=stream)
        rows, csca, asym = handler.phi_average_gpu(dev.data_ptr(), stream=stream)
    finally:
        st.free()
    return rows, csca, asym


def orientation_sample_batch(cfg, u, v, w, beta_sym: float, gamma_sym: float):
    """Traced beams of the orientations (u, v) with weights w (the host
    tracer of the reference, include/mbs_host.h)."""
    from . import beams as B
    beta, gamma = to_angles(u, v, beta_sym, gamma_sym)
    return B.trace(cfg, beta, gamma, w)


# A learned proposal is kept only when the held-out pilot orientations predict
# at most this fraction of plain sampling's variance (else plain Sobol).
MAX_VARIANCE_RATIO = 0.8


@dataclass
class TrainedProposal:
    """A proposal with its pilot run: the pilot's points (u, v) and
    per-orientation rows [n_pilot, n_t, 16] (orientation weight 1), which
    balance_weights lets the final estimate reuse when the pilot ran on the
    handler's grid (pilot_rows is None when it ran on a row subset), and the
    seconds spent in the pilot (tracing and device rows) and in the network
    fit."""
    proposal: Proposal
    fit_r2: float
    pilot_u: np.ndarray
    pilot_v: np.ndarray
    pilot_rows: np.ndarray | None
    pilot_s: float
    fit_s: float
    parts: dict | None = None    # seconds per part of the pilot and the fit
    variance_ratio: float | None = None   # predicted on the held-out pilot points


def pilot_theta_rows(theta_deg: np.ndarray, rows_mask=None, every: int = 1) -> np.ndarray:
    """Zenith angles (degrees) of a pilot grid: the rows of rows_mask (all
    rows when None), every `every`-th of them.  The importance target is an
    RMS over rows, so a pilot on these rows alone gives the same targets (all
    the chosen rows) or nearly (a thinned set) at a fraction of the cost."""
    th = np.asarray(theta_deg, dtype=np.float64)
    if rows_mask is not None:
        th = th[np.asarray(rows_mask, dtype=bool)]
    return np.ascontiguousarray(th[::max(1, int(every))])


def train_proposal_with_pilot(handler, cfg, n_pilot: int, rows_mask=None, pilot_seed: int = 777,
                              cells: int = 128, mix: float = 0.8, epochs: int = 400,
                              batch: int = 256, min_r2: float = 0.2, device: int = 0,
                              precision: int = 1, pilot_theta_deg=None,
                              lr: float = 2e-3,
                              max_variance_ratio: float = MAX_VARIANCE_RATIO) -> TrainedProposal:
    """Pilot run (plain Sobol, per-orientation rows), network training on the
    log importance, proposal table.  The pilot's rows are the handler's grid
    (and rows_mask selects the target rows among them), or, with
    pilot_theta_deg, only those zenith rows (same azimuth bins): then every
    pilot row is a target row."""
    import time
    from . import beams as B
    t0 = time.perf_counter()
    parts = {}
    bs, gs, _ = B.symmetry(cfg)
    u, v, _ = plain_sobol(n_pilot, seed=pilot_seed)
    pb = orientation_sample_batch(cfg, u, v, np.ones(n_pilot), bs, gs)
    parts["trace_s"] = time.perf_counter() - t0
    if pilot_theta_deg is None:
        rows = handler.orientation_rows(pb, precision=precision)
        keep = rows
    else:
        from .handler import GpuHandlerPO
        th = np.asarray(pilot_theta_deg, dtype=np.float64)
        ph = GpuHandlerPO(B.grid(float(th[0]), float(th[-1]), handler.grid.n_az, len(th) - 1,
                                 theta_deg=th), handler.wave, device=device)
        try:
            rows = ph.orientation_rows(pb, precision=precision)
        finally:
            ph.close()
        rows_mask, keep = None, None
    t1 = time.perf_counter()
    parts["rows_s"] = t1 - t0 - parts["trace_s"]
    logh = variance_targets(rows, rows_mask)
    lp = LearnedProposal(bs, gs, device=device)
    t2 = time.perf_counter()
    parts["targets_and_net_s"] = t2 - t1
    try:
        r2 = lp.fit(u, v, logh, epochs=epochs, batch=batch, lr=lr)
        t3 = time.perf_counter()
        parts["train_s"] = t3 - t2
        prop = lp.proposal(cells=cells, mix=mix, min_r2=min_r2)
        # the fit may rank orientations well and still not pay: keep the
        # learned density only where the held-out pilot points predict a
        # clear variance reduction
        te = lp.holdout
        ratio = predicted_variance_ratio(rows[te], proposal_density(prop, u[te], v[te]), rows_mask)
        if prop.learned and ratio > max_variance_ratio:
            prop = uniform_proposal(cells)
        parts["table_s"] = time.perf_counter() - t3
    finally:
        lp.close()
    return TrainedProposal(prop, r2, u, v, keep, t1 - t0, time.perf_counter() - t1, parts, ratio)


def train_proposal(handler, cfg, n_pilot: int, rows_mask=None, pilot_seed: int = 777,
                   cells: int = 128, mix: float = 0.8, epochs: int = 400, min_r2: float = 0.2,
                   device: int = 0, precision: int = 1):
    """train_proposal_with_pilot without the pilot data.  Returns
    (proposal, fit R^2, seconds spent)."""
    t = train_proposal_with_pilot(handler, cfg, n_pilot, rows_mask, pilot_seed, cells, mix, epochs,
                                  min_r2=min_r2, device=device, precision=precision)
    return t.proposal, t.fit_r2, t.pilot_s + t.fit_s
