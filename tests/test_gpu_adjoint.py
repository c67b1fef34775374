"""Path-replay adjoint (optx_engine_run_adjoint behind a torch.autograd.Function):
against the oracle's FP64 CPU gradient (same estimator, same photons), against
common-random-number central finite differences (independent estimator of the
same gradient), its cost relative to one forward run, and a calibration."""
import math

import numpy as np
import pytest
import torch

from gpu_optical_photons_b200 import params as P
from gpu_optical_photons_b200.adjoint import (ResponseModel, calibrate, crn_central_fd, loss_fn,
                                             parameter_errors, response, target_histogram,
                                             with_theta)
from gpu_optical_photons_b200.wavefront import WaveConfig

pytestmark = pytest.mark.gpu

BASE = P.config2()[0]                       # wrapped Lambertian, Rayleigh, volume source
THETA0 = np.array([1000.0, 700.0, 0.95, 4.0])
THETA_T = np.array([800.0, 600.0, 0.93, 3.5])
TC = P.TallyConfig(500, 50.0, 1)


@pytest.mark.parametrize("math_mode,tol", [("exact", 1e-10), ("fast", 2e-3)])
def test_adjoint_equals_fp64_oracle_gradient(engine, oracle, math_mode, tol):
    n = 200_000
    m = ResponseModel(BASE, n, TC, first_id=5, config=WaveConfig(math=math_mode))
    try:
        w = np.random.default_rng(1).normal(size=TC.time_bins + 1)
        g = m.replay(THETA0, torch.as_tensor(w), 0.7)
        hist, det = m.forward(THETA0)
    finally:
        m.close()
    mode = oracle.PORTABLE if math_mode == "exact" else oracle.PLATFORM
    go, ho, do = oracle.adjoint(with_theta(BASE, THETA0), TC, n, w_bin=w, w_det=0.7, first_id=5, mode=mode)
    assert np.all(np.abs(g - go) <= tol * np.abs(go)), (g, go)
    if math_mode == "exact":
        assert np.array_equal(hist, ho.astype(np.float64)) and det == do


@pytest.mark.parametrize("math_mode,bins", [("exact", 500), ("fast", 500), ("exact", 1000)])
def test_score_moments_equal_fp64_oracle(engine, oracle, math_mode, bins):
    """Per-bin (count, score sums) against the oracle; the counts are the forward
    histogram and J^T w reproduces the replay gradient. 500 bins accumulate in a
    shared-memory table per block, 1000 bins (past its 818-bin limit) directly
    with global atomics."""
    n = 200_000
    tc = P.TallyConfig(bins, 50.0, 1)
    m = ResponseModel(BASE, n, tc, first_id=5, config=WaveConfig(math=math_mode))
    try:
        hist, jac = m.score_moments(THETA0)
        h_fwd, det = m.forward(THETA0)
        w = np.random.default_rng(2).normal(size=tc.time_bins + 1)
        g = m.replay(THETA0, torch.as_tensor(w), 0.7)
    finally:
        m.close()
    assert np.array_equal(hist, h_fwd) and hist.sum() == det
    assert np.allclose(jac.T @ w + 0.7 * jac.sum(0), g, rtol=1e-9, atol=0.0)
    mode = oracle.PORTABLE if math_mode == "exact" else oracle.PLATFORM
    mo = oracle.score_moments(with_theta(BASE, THETA0), tc, n, first_id=5, mode=mode)
    if math_mode == "exact":
        assert np.array_equal(hist, mo[:, 0])
        scale = np.abs(mo[:, 1:]).max(axis=0)
        assert np.all(np.abs(jac - mo[:, 1:]) <= 1e-10 * np.abs(mo[:, 1:]) + 1e-12 * scale)
    else:  # FMA-contracted libm: a handful of photons may change bin
        assert abs(hist.sum() - mo[:, 0].sum()) <= 1e-3 * mo[:, 0].sum()
        assert np.all(np.abs(jac.sum(0) - mo[:, 1:].sum(0)) <= 2e-3 * np.abs(mo[:, 1:]).sum(0))


def _batch_gradients(n_batch, k_batches, fn_adj, fn_fd):
    G, F = [], []
    for k in range(k_batches):
        m = ResponseModel(BASE, n_batch, TC, first_id=k * n_batch)
        try:
            G.append(fn_adj(m))
            F.append(fn_fd(m))
        finally:
            m.close()
    G, F = np.array(G), np.array(F)
    D = G - F
    z = D.mean(0) / (D.std(0, ddof=1) / math.sqrt(k_batches))
    return G.mean(0), F.mean(0), z


def test_loss_gradient_within_2_sigma_of_crn_fd(engine):
    """Loss = Poisson NLL of the 500-bin histogram (target: theta_T, seed 777) + D."""
    nb, kb = 1_000_000, 16
    target = target_histogram(BASE, THETA_T, nb, seed=777, tally=TC)
    tgt = torch.as_tensor(target)

    def adj(m):
        th = torch.tensor(THETA0, requires_grad=True)
        loss_fn(th, m, tgt).backward()
        return th.grad.numpy().copy()

    g, f, z = _batch_gradients(nb, kb, adj, lambda m: crn_central_fd(THETA0, m, target, 1e-3))
    print("adjoint", g, "crn fd", f, "z", z)
    assert np.all(np.abs(z) < 2.0), z
    assert np.all(np.sign(g) == np.sign(f))


def test_detected_fraction_gradient_within_2_sigma_of_crn_fd(engine):
    nb, kb = 1_000_000, 16

    def adj(m):
        th = torch.tensor(THETA0, requires_grad=True)
        _, d = response(th, m)
        d.backward()
        return th.grad.numpy().copy()

    def fd(m):
        out = np.zeros(4)
        for j in range(4):
            up, dn = THETA0.copy(), THETA0.copy()
            up[j] = float(np.float32(THETA0[j] * 1.001))
            dn[j] = float(np.float32(THETA0[j] * 0.999))
            out[j] = (m.forward(up)[1] - m.forward(dn)[1]) / m.n / (up[j] - dn[j])
        return out

    g, f, z = _batch_gradients(nb, kb, adj, fd)
    print("dD/dtheta adjoint", g, "crn fd", f, "z", z)
    # tau does not change detection: both estimates are noise around 0
    assert np.all(np.abs(z) < 2.0), z


def test_adjoint_cost_at_most_1p5_forward(engine):
    n = 10_000_000
    m = ResponseModel(BASE, n, TC)
    try:
        import ctypes
        from gpu_optical_photons_b200 import _lib
        w = torch.ones(TC.time_bins + 1, dtype=torch.float64)
        th = THETA0
        m.forward(th)
        m.replay(th, w, 0.5)
        wd, gd = w.cuda(), torch.zeros(4, dtype=torch.float64, device="cuda")
        st = torch.cuda.current_stream().cuda_stream
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fwd, adj = [], []
        for _ in range(3):  # the bare runs: no host read-back inside the events
            s.record(); m.engine.run_tally(); e.record(); torch.cuda.synchronize()
            fwd.append(s.elapsed_time(e))
            s.record()
            _lib.call("optx_engine_run_adjoint", m.engine._h, ctypes.c_void_p(wd.data_ptr()), 0.5,
                      ctypes.c_void_p(gd.data_ptr()), ctypes.c_void_p(st))
            e.record(); torch.cuda.synchronize()
            adj.append(s.elapsed_time(e))
    finally:
        m.close()
    ratio = min(adj) / min(fwd)
    print(f"forward {min(fwd):.3f} ms, adjoint replay {min(adj):.3f} ms, ratio {ratio:.3f}")
    assert ratio <= 1.5


def test_fisher_calibration_recovers_target_theta(engine):
    """20 Fisher-scoring steps from theta0 on 1e7 photons per evaluation recover
    the target theta within 3 sigma of the fit's statistical error, every
    parameter ends closer than it started, and the estimate fits the target
    histogram as well as the true theta does."""
    n = 10_000_000
    target = target_histogram(BASE, THETA_T, n, seed=777, tally=TC)
    m = ResponseModel(BASE, n, TC)
    try:
        traj = calibrate(BASE, THETA0, target, n, steps=20, model=m)
        th, loss = traj[-1]
        sig = parameter_errors(m, th)
        h_t, _ = m.score_moments(THETA_T)
    finally:
        m.close()
    lam = h_t[:TC.time_bins] + 1.0
    loss_t = float((lam - target[:TC.time_bins] * np.log(lam)).sum() / n)
    print("calibration", [(np.round(t, 4).tolist(), round(l, 7)) for t, l in traj])
    print("estimate", th, "sigma", sig, "pull", (th - THETA_T) / sig, "n*(loss - loss(theta_T))",
          n * (loss - loss_t))
    assert loss < traj[0][1]
    assert np.all(np.abs(th - THETA_T) < 3.0 * sig)
    assert np.all(np.abs(th - THETA_T) < np.abs(THETA0 - THETA_T))
    # the arrival-time histogram pins tau and R to under 1 %
    assert sig[3] < 0.01 * THETA_T[3] and sig[2] < 0.01 * THETA_T[2]
    # the estimate is at the noise floor: no worse a fit than the true theta by
    # more than a few units of log-likelihood
    assert n * (loss - loss_t) < 5.0


def test_adam_calibration_reduces_loss(engine):
    """Plain first-order descent (Adam on the adjoint gradient) for comparison:
    it lowers the loss and moves tau, the best-identified parameter, at least
    halfway to its target in 20 steps."""
    n = 4_000_000
    target = target_histogram(BASE, THETA_T, n, seed=777, tally=TC)
    traj = calibrate(BASE, THETA0, target, n, steps=20, method="adam")
    l0, l1 = traj[0][1], traj[-1][1]
    th = traj[-1][0]
    print("adam calibration", [(np.round(t, 4).tolist(), round(l, 6)) for t, l in traj])
    assert l1 < l0
    assert abs(th[3] - THETA_T[3]) < abs(THETA0[3] - THETA_T[3]) / 2


def test_score_moments_rejects_bad_arguments(engine):
    import ctypes
    from gpu_optical_photons_b200 import _lib
    from gpu_optical_photons_b200.wavefront import WavefrontEngine
    m = ResponseModel(BASE, 1000, TC)
    try:
        with pytest.raises(_lib.OptxError) as e:
            _lib.call("optx_engine_run_score_moments", m.engine._h, None, None)
        assert e.value.code == 1
        buf = torch.zeros((TC.time_bins + 1) * 5 + 1, dtype=torch.float64, device="cuda")
        with pytest.raises(_lib.OptxError):  # not 8-byte aligned
            _lib.call("optx_engine_run_score_moments", m.engine._h,
                      ctypes.c_void_p(buf.data_ptr() + 4), None)
        grad = torch.zeros(4, dtype=torch.float64, device="cuda")
        with pytest.raises(_lib.OptxError, match="8-byte aligned"):  # bin weights not 8-byte aligned
            _lib.call("optx_engine_run_adjoint", m.engine._h, ctypes.c_void_p(buf.data_ptr() + 4), 0.0,
                      ctypes.c_void_p(grad.data_ptr()), None)
    finally:
        m.close()
    eng = WavefrontEngine(TC, 2, 2000)
    try:
        eng.set_events([BASE, BASE], [1000, 1000])
        buf = torch.zeros((TC.time_bins + 1) * 5, dtype=torch.float64, device="cuda")
        with pytest.raises(_lib.OptxError):  # the adjoint runs on one configuration only
            _lib.call("optx_engine_run_score_moments", eng._h, ctypes.c_void_p(buf.data_ptr()), None)
    finally:
        eng.close()


def test_replay_rejects_weights_of_another_length(engine):
    """The replay kernel reads time_bins + 1 bin weights: a shorter or longer
    vector is refused before the launch, and the model stays usable."""
    m = ResponseModel(BASE, 1000, TC)
    try:
        for k in (TC.time_bins, TC.time_bins + 2):
            with pytest.raises(ValueError, match="time_bins \\+ 1"):
                m.replay(THETA0, torch.ones(k, dtype=torch.float64), 0.0)
        g = m.replay(THETA0, torch.ones(TC.time_bins + 1, dtype=torch.float64), 0.0)
        assert g.shape == (4,) and np.all(np.isfinite(g))
    finally:
        m.close()


def test_reflectivity_parameter_with_per_face_surfaces(engine):
    """R is the reflectivity of the painted faces. (1) The same Lambertian box
    given as per-face lists replays the plain configuration's gradient exactly;
    (2) a black face's own reflectivity (which no photon uses) does not change
    the gradient; (3) painted faces with different reflectivities have no single
    R: the replay and the score moments are refused. A reflectivity taken from
    the wrong face would scale the R score by 0.95 / 0.2 or 0.95 / 0.5."""
    import ctypes
    from gpu_optical_photons_b200 import _lib
    from gpu_optical_photons_b200.wavefront import WavefrontEngine
    n = 100_000
    lam = P.SimParams(surface=P.LAMBERTIAN, reflectivity=0.95, n_det=1.5, source=P.VOLUME,
                      abs_length=2000.0, scat_length=500.0, tau=4.0)
    w = torch.as_tensor(np.random.default_rng(3).normal(size=TC.time_bins + 1))

    def grad(base):
        m = ResponseModel(base, n, TC, first_id=9, config=WaveConfig(math="exact"))
        try:
            return m.replay(THETA0, w, 0.3)
        finally:
            m.close()

    # The same photons and scores; the FP64 sums are atomics, so equal up to the
    # order of their additions.
    same = dict(rtol=1e-12, atol=0.0)
    plain = grad(lam)
    listed = grad(lam.replace(face_surface=[P.LAMBERTIAN] * 5 + [0], face_reflectivity=[0.5] * 6))
    assert np.allclose(listed, plain, **same), (listed, plain)  # theta's R on every painted face
    black = [P.BLACK] + [P.LAMBERTIAN] * 4 + [0]
    g1 = grad(lam.replace(face_surface=black, face_reflectivity=[0.2] + [0.95] * 5))
    g2 = grad(lam.replace(face_surface=black, face_reflectivity=[0.9] + [0.95] * 5))
    assert np.allclose(g1, g2, **same) and g1[2] != 0.0, (g1, g2)
    mixed = lam.replace(face_surface=[P.LAMBERTIAN] * 5 + [0], face_reflectivity=[0.9] + [0.95] * 5)
    eng = WavefrontEngine(TC, 1, 1000)
    try:
        eng.set_events([mixed], [1000])
        buf = torch.zeros(4, dtype=torch.float64, device="cuda")
        wb = torch.zeros(TC.time_bins + 1, dtype=torch.float64, device="cuda")
        with pytest.raises(_lib.InvalidArgument, match="painted faces must share one reflectivity"):
            _lib.call("optx_engine_run_adjoint", eng._h, ctypes.c_void_p(wb.data_ptr()), 0.0,
                      ctypes.c_void_p(buf.data_ptr()), None)
        mom = torch.zeros((TC.time_bins + 1) * 5, dtype=torch.float64, device="cuda")
        with pytest.raises(_lib.InvalidArgument, match="painted faces must share one reflectivity"):
            _lib.call("optx_engine_run_score_moments", eng._h, ctypes.c_void_p(mom.data_ptr()), None)
    finally:
        eng.close()


def test_calibration_command_line(engine, capsys):
    import json
    from gpu_optical_photons_b200.adjoint import main
    main(["--n", "1e6", "--steps", "4"])
    out = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert len(out["trajectory"]) == 4 + 2 and len(out["estimate"]) == 4 and len(out["sigma"]) == 4
    assert out["trajectory"][-1][1] < out["trajectory"][0][1]
