"""Differentiable detector response: a torch.autograd.Function over the C ABI.

Forward: the wavefront engine tallies N photons at theta = (abs_length,
scat_length, reflectivity, tau) and returns the arrival-time histogram h
(time_bins + 1 counts, last = overflow) and the detected fraction D.

Backward: ``optx_engine_run_adjoint`` replays the same photons from their
Philox counters (no stored paths) and accumulates, in FP64, the score-function
(likelihood-ratio) estimator of d E[h_b] / d theta weighted by the incoming
gradients. For a photon history with path length s, n_s scatterings, k
reflections at painted faces and emission time t_e, the score of its
probability density is

    S_La  = s / La^2 - [absorbed in bulk] / La
    S_Ls  = s / Ls^2 - n_s / Ls
    S_R   = k / R - [absorbed at a painted face] / (1 - R)
    S_tau = t_e / tau^2 - 1 / tau

(exponential free paths of mean La, Ls; Bernoulli reflection with probability
R; exponential emission time). Only detected photons enter the histogram, so
the absorbed-photon terms drop out. d E[h_b] / d theta = E[1_b S] and the
estimate sum_photons 1_b S is unbiased; it is checked against common-random-
number central finite differences and the oracle's FP64 CPU gradient.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from .params import LAMBERTIAN, SPECULAR, SimParams, TallyConfig
from .wavefront import WaveConfig, WavefrontEngine

THETA_NAMES = ("abs_length", "scat_length", "reflectivity", "tau")


def with_theta(p: SimParams, theta) -> SimParams:
    """p at theta = (abs_length, scat_length, R, tau). R is the reflectivity of
    the painted (specular and Lambertian) faces: with per-face surfaces it is
    written to each painted face, and faces of other models keep their values."""
    t = [float(np.float32(v)) for v in theta]
    kw = dict(abs_length=t[0], scat_length=t[1], reflectivity=t[2], tau=t[3])
    if p.face_reflectivity is not None:
        surf = p.face_surface or [p.surface] * 6
        kw["face_reflectivity"] = [t[2] if i < 5 and int(surf[i]) in (SPECULAR, LAMBERTIAN) else float(r)
                                   for i, r in enumerate(p.face_reflectivity)]
    return p.replace(**kw)


class ResponseModel:
    """Owns a single-configuration wavefront engine for forward and replay runs."""

    def __init__(self, base: SimParams, n: int, tally: TallyConfig | None = None, first_id: int = 0,
                 config: WaveConfig | None = None):
        self.base = base
        self.n = n
        self.first_id = first_id
        self.tally = tally or TallyConfig(500, 50.0, 1)
        self.engine = WavefrontEngine(self.tally, 1, n, config or WaveConfig())
        self._theta = None

    def _upload(self, theta):
        key = tuple(float(np.float32(v)) for v in theta)
        if key != self._theta:
            self.engine.set_events([with_theta(self.base, key)], [self.n], self.first_id)
            self._theta = key

    def forward(self, theta) -> tuple[np.ndarray, int]:
        """(arrival-time histogram incl. overflow, detected count) at theta."""
        self._upload(theta)
        self.engine.run_tally()
        flat = self.engine.tallies()[0]
        tb = self.tally.time_bins
        return flat[5:5 + tb + 1].astype(np.float64), int(flat[0])

    def replay(self, theta, w_bin: torch.Tensor, w_det: float) -> np.ndarray:
        """FP64 sum over detected photons of (w_bin[bin] + w_det) * score."""
        self._upload(theta)
        w = w_bin.detach().to(device="cuda", dtype=torch.float64).contiguous()
        if w.numel() != self.tally.time_bins + 1:  # the kernel reads time_bins + 1 weights
            raise ValueError(f"w_bin must hold time_bins + 1 = {self.tally.time_bins + 1} weights, "
                             f"got {w.numel()}")
        grad = torch.zeros(4, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        _lib.call("optx_engine_run_adjoint", self.engine._h, ctypes.c_void_p(w.data_ptr()),
                  float(w_det), ctypes.c_void_p(grad.data_ptr()), ctypes.c_void_p(stream))
        self.engine.stats(stream)  # raises if the run ended on the watchdog or a full queue
        return grad.cpu().numpy()

    def score_moments(self, theta) -> tuple[np.ndarray, np.ndarray]:
        """(histogram h incl. overflow, Jacobian J) at theta from one replay.

        J[b, j] = sum over photons detected in bin b of S_j, an unbiased estimate
        of dE[h_b]/dtheta_j; h comes from the same photons (exact integer counts)."""
        self._upload(theta)
        tb = self.tally.time_bins
        m = torch.empty((tb + 1) * 5, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        _lib.call("optx_engine_run_score_moments", self.engine._h, ctypes.c_void_p(m.data_ptr()),
                  ctypes.c_void_p(stream))
        self.engine.stats(stream)  # raises if the run ended on the watchdog or a full queue
        M = m.view(tb + 1, 5).cpu().numpy()
        return M[:, 0].copy(), M[:, 1:].copy()

    def close(self):
        self.engine.close()


class _Response(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta: torch.Tensor, model: ResponseModel):
        th = theta.detach().cpu().numpy().astype(np.float64)
        hist, det = model.forward(th)
        ctx.model = model
        ctx.theta = th
        return (torch.as_tensor(hist, dtype=torch.float64, device=theta.device),
                torch.tensor(det / model.n, dtype=torch.float64, device=theta.device))

    @staticmethod
    def backward(ctx, grad_hist, grad_det):
        model = ctx.model
        w_bin = grad_hist if grad_hist is not None else torch.zeros(model.tally.time_bins + 1)
        w_det = float(grad_det) / model.n if grad_det is not None else 0.0
        g = model.replay(ctx.theta, w_bin, w_det)
        return torch.as_tensor(g, dtype=torch.float64), None


def response(theta: torch.Tensor, model: ResponseModel):
    """(histogram h, detected fraction D) as differentiable functions of theta (4,)."""
    return _Response.apply(theta, model)


def poisson_nll(hist: torch.Tensor, target: torch.Tensor, n: int, bins: int) -> torch.Tensor:
    """Poisson negative log-likelihood of the first `bins` bins, per photon.

    lambda_b = h_b + 1 (one pseudo-count keeps log finite in empty bins)."""
    lam = hist[:bins] + 1.0
    k = target[:bins]
    return (lam - k * torch.log(lam)).sum() / n


def loss_fn(theta: torch.Tensor, model: ResponseModel, target: torch.Tensor) -> torch.Tensor:
    """The calibration loss: Poisson NLL of the arrival-time histogram plus D."""
    h, d = response(theta, model)
    return poisson_nll(h, target, model.n, model.tally.time_bins) + d


def loss_value(theta, model: ResponseModel, target: np.ndarray) -> float:
    hist, det = model.forward(theta)
    lam = hist[:model.tally.time_bins] + 1.0
    k = target[:model.tally.time_bins]
    return float((lam - k * np.log(lam)).sum() / model.n + det / model.n)


def crn_central_fd(theta, model: ResponseModel, target: np.ndarray, rel_step: float = 1e-3):
    """Central finite differences with common random numbers (same photons / seed).

    The step is rel_step * theta_j rounded to the float32 grid; the divisor is the
    actual difference of the float32 parameters."""
    theta = np.asarray(theta, np.float64)
    g = np.zeros(4)
    for j in range(4):
        up, dn = theta.copy(), theta.copy()
        up[j] = float(np.float32(theta[j] * (1 + rel_step)))
        dn[j] = float(np.float32(theta[j] * (1 - rel_step)))
        g[j] = (loss_value(up, model, target) - loss_value(dn, model, target)) / (up[j] - dn[j])
    return g


def target_histogram(base: SimParams, theta_target, n: int, seed: int = 777,
                     tally: TallyConfig | None = None) -> np.ndarray:
    """Arrival-time histogram of a run at theta_target with its own seed."""
    m = ResponseModel(base.replace(seed=seed), n, tally)
    try:
        hist, _ = m.forward(theta_target)
    finally:
        m.close()
    return hist


def nll_loss(theta: torch.Tensor, model: ResponseModel, target: torch.Tensor) -> torch.Tensor:
    """Poisson NLL of the arrival-time histogram alone (the calibration objective)."""
    h, _ = response(theta, model)
    return poisson_nll(h, target, model.n, model.tally.time_bins)


def _phi_of(theta) -> np.ndarray:
    t = np.asarray(theta, np.float64)
    return np.array([math.log(t[0]), math.log(t[1]), math.log(1.0 - t[2]), math.log(t[3])])


def _theta_of(phi) -> np.ndarray:
    e = np.exp(np.asarray(phi, np.float64))
    return np.array([e[0], e[1], 1.0 - e[2], e[3]])


def _dtheta_dphi(theta) -> np.ndarray:
    t = np.asarray(theta, np.float64)
    return np.array([t[0], t[1], -(1.0 - t[2]), t[3]])


def fisher_information(hist: np.ndarray, jac: np.ndarray, theta, bins: int) -> np.ndarray:
    """Poisson Fisher information of the first `bins` histogram bins with respect
    to phi = (log La, log Ls, log(1-R), log tau):
        F = sum_b (d lambda_b/d phi)(d lambda_b/d phi)^T / lambda_b,
    lambda_b = h_b + 1, d lambda/d phi from the score Jacobian."""
    Jp = jac[:bins] * _dtheta_dphi(theta)
    lam = hist[:bins] + 1.0
    return (Jp.T / lam) @ Jp


def parameter_errors(model: "ResponseModel", theta) -> np.ndarray:
    """One-sigma statistical errors of theta fitted (as `calibrate` does) to a
    target histogram of as many photons as the model runs: covariance 2 F^-1 in
    phi — the target's Poisson counts and the model's own sampling noise
    contribute equally — mapped from phi to theta. Parameters whose process is
    off (zero Fisher information) get 0."""
    hist, jac = model.score_moments(theta)
    bins = model.tally.time_bins
    F = fisher_information(hist, jac, theta, bins)
    on = np.diag(F) > 0
    cov = np.zeros((4, 4))
    cov[np.ix_(on, on)] = 2.0 * np.linalg.inv(F[np.ix_(on, on)])
    return np.sqrt(np.diag(cov)) * np.abs(_dtheta_dphi(theta))


def _to_theta(phi: torch.Tensor) -> torch.Tensor:
    # phi = (log La, log Ls, log(1 - R), log tau): unconstrained and well scaled
    e = torch.exp(phi)
    return torch.stack([e[0], e[1], 1.0 - e[2], e[3]])


def calibrate(base: SimParams, theta0, target: np.ndarray, n: int, steps: int = 20,
              lr: float | None = None, model: ResponseModel | None = None, method: str = "fisher"):
    """Fits theta to a target arrival-time histogram by minimising its Poisson NLL.

    method "fisher": Fisher scoring (natural-gradient descent) on
    phi = (log La, log Ls, log(1-R), log tau): each step runs one score-moment
    replay, which gives the histogram, the gradient g = sum_b (1 - k_b/lambda_b)
    d lambda_b/d phi and the Fisher information F, and moves phi by
    -lr (F + 1e-6 diag F)^-1 g (lr 1; each component limited to 0.25 per step).
    The Monte Carlo noise of the model makes the iterates wander inside the
    target's error ellipse once they reach it, so the estimate is the average of
    phi over the second half of the steps (Polyak-Ruppert averaging).
    Trajectory: [(theta_i, loss_i)] for i = 0..steps, then (estimate, its loss).
    method "adam": Adam (lr 0.04) on phi with gradients from the adjoint replay
    through the autograd Function; trajectory [(theta_i, loss_i)] for
    i = 0..steps, the last being the estimate. loss = the NLL per photon."""
    own = model is None
    model = model or ResponseModel(base, n)
    if method == "fisher":
        try:
            return _calibrate_fisher(model, theta0, target, steps, 1.0 if lr is None else lr)
        finally:
            if own:
                model.close()
    if method != "adam":
        raise ValueError(f"unknown method {method!r}")
    lr = 0.04 if lr is None else lr
    tgt = torch.as_tensor(target, dtype=torch.float64)
    t0 = np.asarray(theta0, np.float64)
    phi = torch.tensor([math.log(t0[0]), math.log(t0[1]), math.log(1.0 - t0[2]), math.log(t0[3])],
                       dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([phi], lr=lr)
    traj = []
    try:
        for _ in range(steps):
            opt.zero_grad()
            theta = _to_theta(phi)
            loss = nll_loss(theta, model, tgt)
            loss.backward()  # adjoint replay, then the chain rule through _to_theta
            traj.append((theta.detach().numpy().copy(), float(loss.detach())))
            opt.step()
        theta = _to_theta(phi).detach().numpy()
        with torch.no_grad():
            traj.append((theta.copy(), float(nll_loss(torch.as_tensor(theta), model, tgt))))
    finally:
        if own:
            model.close()
    return traj


def _calibrate_fisher(model: ResponseModel, theta0, target: np.ndarray, steps: int, lr: float,
                      max_step: float = 0.25):
    bins = model.tally.time_bins
    k = np.asarray(target, np.float64)[:bins]
    phi = _phi_of(theta0)
    traj, phis = [], []
    for it in range(steps + 2):
        if it == steps + 1:  # the estimate: iterates steps/2 .. steps averaged
            phi = np.mean(phis[steps // 2:], axis=0)
        theta = _theta_of(phi)
        hist, jac = model.score_moments(theta)
        lam = hist[:bins] + 1.0
        traj.append((theta.copy(), float((lam - k * np.log(lam)).sum() / model.n)))
        phis.append(phi.copy())
        if it >= steps:
            continue
        Jp = jac[:bins] * _dtheta_dphi(theta)
        g = ((1.0 - k / lam)[:, None] * Jp).sum(0)
        F = (Jp.T / lam) @ Jp
        on = np.diag(F) > 0
        d = np.zeros(4)
        Fa = F[np.ix_(on, on)]
        d[on] = np.linalg.solve(Fa + 1e-6 * np.diag(np.diag(Fa)), g[on])
        phi = phi - np.clip(lr * d, -max_step, max_step)
    return traj


def main(argv=None):
    """Calibration from the command line: fits theta to a target histogram made
    at --target with its own seed, and prints one JSON line (trajectory, estimate,
    one-sigma errors).

        python -m gpu_optical_photons_b200.adjoint --n 1e7 --steps 20
    """
    import argparse
    import json
    from .params import config2
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--n", type=float, default=1e7, help="photons per evaluation")
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--method", default="fisher", choices=["fisher", "adam"])
    ap.add_argument("--theta0", type=float, nargs=4, default=[1000.0, 700.0, 0.95, 4.0],
                    metavar=("LA", "LS", "R", "TAU"))
    ap.add_argument("--target", type=float, nargs=4, default=[800.0, 600.0, 0.93, 3.5],
                    metavar=("LA", "LS", "R", "TAU"))
    ap.add_argument("--target-seed", type=int, default=777)
    ap.add_argument("--time_bins", type=int, default=500)
    ap.add_argument("--time_max", type=float, default=50.0)
    a = ap.parse_args(argv)
    base = config2()[0]
    n = int(a.n)
    tally = TallyConfig(a.time_bins, a.time_max, 1)
    target = target_histogram(base, a.target, n, seed=a.target_seed, tally=tally)
    model = ResponseModel(base, n, tally)
    try:
        traj = calibrate(base, a.theta0, target, n, steps=a.steps, model=model, method=a.method)
        est = traj[-1][0]
        sig = parameter_errors(model, est)
    finally:
        model.close()
    print(json.dumps({"method": a.method, "photons": n, "theta_names": THETA_NAMES,
                      "target": a.target, "estimate": est.tolist(), "sigma": sig.tolist(),
                      "trajectory": [[t.tolist(), l] for t, l in traj]}))


if __name__ == "__main__":
    main()
