"""Test helpers: golden-case parameters, record comparison, statistics and
the analytic references of the reference project (include/optphot/analytic.hpp,
restated in double precision)."""
import math

import numpy as np
from scipy import stats as ss

from gpu_optical_photons_b200 import params as P


def params_from_meta(d: dict) -> P.SimParams:
    return P.SimParams(**{k: (float(v) if isinstance(v, float) else v) for k, v in d.items()})


def golden_records(arrays, name, tag):
    return {k: arrays[f"{name}/{tag}/{k}"] for k in
            ("fate", "n_boundary", "n_scatter", "t", "x", "y", "z", "path")}


def compare_histories(a, b) -> dict:
    """Photon-by-photon agreement (src/core/compare.cpp:103-127 of the reference)."""
    discrete = ((np.asarray(a["fate"]) == np.asarray(b["fate"]))
                & (np.asarray(a["n_boundary"]) == np.asarray(b["n_boundary"]))
                & (np.asarray(a["n_scatter"]) == np.asarray(b["n_scatter"])))
    same = discrete.copy()
    for k in ("t", "x", "y", "z", "path"):
        same &= np.asarray(a[k]).view(np.uint32) == np.asarray(b[k]).view(np.uint32)
    n = len(a["fate"])
    bad = np.nonzero(~discrete)[0]
    return {"n": n, "bitwise_identical": int(same.sum()), "same_discrete": int(discrete.sum()),
            "fate_differs": int((np.asarray(a["fate"]) != np.asarray(b["fate"])).sum()),
            "first_divergent": int(bad[0]) if len(bad) else -1}


def steps_of(r) -> np.ndarray:
    return (np.asarray(r["n_boundary"]).astype(np.int64) + np.asarray(r["n_scatter"])
            + (np.asarray(r["fate"]) == P.ABSORBED_BULK))


def binomial_pull(k, n, p):
    return (k - n * p) / math.sqrt(n * p * (1 - p))


def chi2_two_sample(a, b):
    """NR 14.3 two-sample chi-square (include/optphot/stats.hpp:262-280 of the reference)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    A, B = a.sum(), b.sum()
    m = (a + b) > 0
    d = math.sqrt(B / A) * a[m] - math.sqrt(A / B) * b[m]
    chi2 = float((d * d / (a[m] + b[m])).sum())
    ndf = int(m.sum()) - 1
    return chi2, ndf, float(ss.chi2.sf(chi2, ndf))


def ks_two_sample(x, y):
    r = ss.ks_2samp(x, y)
    return float(r.statistic), float(r.pvalue)


# ---- analytic references (analytic.hpp of the reference, restated) -----------

def rect_solid_angle(x1, x2, y1, y2, h):
    F = lambda x, y: math.atan(x * y / (h * math.sqrt(x * x + y * y + h * h)))
    return F(x2, y2) - F(x1, y2) - F(x2, y1) + F(x1, y1)


def face_frame(p: P.SimParams, face: int):
    half = [p.hx, p.hy, p.hz]
    src = [p.src_x, p.src_y, p.src_z]
    a = face >> 1
    s = 1.0 if face & 1 else -1.0
    ua, va = (a + 1) % 3, (a + 2) % 3
    return (half[a] - s * src[a], -half[ua] - src[ua], half[ua] - src[ua], -half[va] - src[va],
            half[va] - src[va])


def face_solid_angle_fraction(p, face):
    h, u1, u2, v1, v2 = face_frame(p, face)
    return rect_solid_angle(u1, u2, v1, v2, h) / (4 * math.pi)


def face_survival_fraction(p, face, L, panels=24, order=16):
    """(1/4pi) Int_face exp(-r/L) dOmega by composite Gauss-Legendre."""
    h, u1, u2, v1, v2 = face_frame(p, face)
    gx, gw = np.polynomial.legendre.leggauss(order)

    def edges(a, b):
        cuts = [a, 0.0, b] if a < 0.0 < b else [a, b]
        e = []
        for k in range(len(cuts) - 1):
            e.extend(cuts[k] + (cuts[k + 1] - cuts[k]) * np.arange(panels) / panels)
        e.append(b)
        return np.array(e)

    eu, ev = edges(u1, u2), edges(v1, v2)
    cu, hu = 0.5 * (eu[1:] + eu[:-1]), 0.5 * (eu[1:] - eu[:-1])
    cv, hv = 0.5 * (ev[1:] + ev[:-1]), 0.5 * (ev[1:] - ev[:-1])
    U = (cu[:, None] + hu[:, None] * gx[None, :]).ravel()
    WU = (hu[:, None] * gw[None, :]).ravel()
    V = (cv[:, None] + hv[:, None] * gx[None, :]).ravel()
    WV = (hv[:, None] * gw[None, :]).ravel()
    r = np.sqrt(U[:, None] ** 2 + V[None, :] ** 2 + h * h)
    att = 1.0 if math.isinf(L) else np.exp(-r / L)
    return float((WU[:, None] * WV[None, :] * h / r ** 3 * att).sum() / (4 * math.pi))


def mirror_box_escape_fraction(n_scint, n_det):
    if n_det >= n_scint:
        return 1.0
    s = n_det / n_scint
    return 1.0 - math.sqrt(1.0 - s * s)


def check_tally_consistency(flat, c) -> None:
    """Internal consistency of a flat tally: the arrival-time histogram (with its
    overflow bin) and the hit map each count every detected photon once."""
    flat = np.asarray(flat, dtype=np.uint64)
    det = int(flat[0])
    t0, x0 = 5, 5 + c.time_bins + 1
    assert int(flat[t0:x0].sum()) == det, "time histogram != detected"
    assert int(flat[x0:x0 + c.xy_bins * c.xy_bins].sum()) == det, "hit map != detected"
