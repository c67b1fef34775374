"""Comparison of two sets of photon records (the reference's src/core/compare.cpp).

* `compare_histories(a, b)`: same-seed, photon-by-photon agreement — bitwise
  identical records, same discrete history (fate, boundary and scatter counts),
  different fates, the largest time and position differences over the histories
  with the same discrete path, the first divergent photon (compare.cpp:39-65).
* `compare_distributions(a, b, p)`: independent-seed agreement — detection
  efficiency z-test, two-sample chi-square of the arrival-time and hit-map
  histograms, two-sample Kolmogorov-Smirnov test of the arrival times
  (compare.cpp:67-99; statistics of stats.hpp: Numerical Recipes 3rd ed.
  sections 6.2 and 14.3).
* `history_json` / `distribution_json`: the reference's JSON text of both
  results (compare.cpp:101-120), key for key, numbers with 10 significant digits.

Histograms are binned in float32 with the reference's operations; chi-square
sums run bin by bin in order, and the incomplete gamma function calls the C
library's `lgamma`, so statistics and p-values equal the reference's to the
last bit on the same records.
"""
from __future__ import annotations

import ctypes
import ctypes.util
import math
from dataclasses import dataclass, field

import numpy as np

from .params import DETECTED, SimParams

_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_libm.lgamma.restype = ctypes.c_double
_libm.lgamma.argtypes = [ctypes.c_double]


def _lgamma(a: float) -> float:
    return _libm.lgamma(a)


# ---- statistics (stats.hpp) ------------------------------------------------

def gamma_q(a: float, x: float) -> float:
    """Regularised upper incomplete gamma Q(a, x): series for x < a + 1, Lentz
    continued fraction otherwise (Numerical Recipes 3rd ed. 6.2)."""
    if x <= 0.0:
        return 1.0
    gln = _lgamma(a)
    if x < a + 1.0:
        ap, s = a, 1.0 / a
        d = s
        for _ in range(10000):
            ap += 1.0
            d *= x / ap
            s += d
            if abs(d) < abs(s) * 1e-15:
                break
        return 1.0 - s * math.exp(-x + a * math.log(x) - gln)
    tiny = 1e-300
    b = x + 1.0 - a
    c = 1.0 / tiny
    d = 1.0 / b
    h = d
    for i in range(1, 10000):
        an = -i * (i - a)
        b += 2.0
        d = an * d + b
        if abs(d) < tiny:
            d = tiny
        c = b + an / c
        if abs(c) < tiny:
            c = tiny
        d = 1.0 / d
        de = d * c
        h *= de
        if abs(de - 1.0) < 1e-15:
            break
    return math.exp(-x + a * math.log(x) - gln) * h


def chi2_pvalue(chi2: float, ndf: float) -> float:
    return gamma_q(0.5 * ndf, 0.5 * chi2)


@dataclass
class Chi2Result:
    chi2: float = 0.0
    ndf: int = 0
    pvalue: float = 1.0


def chi2_two_sample(a, b) -> Chi2Result:
    """chi2 = sum (sqrt(B/A) a_i - sqrt(A/B) b_i)^2 / (a_i + b_i) over bins not
    empty in both; ndf = such bins - 1 (Numerical Recipes 3rd ed. 14.3)."""
    a = [float(v) for v in a]
    b = [float(v) for v in b]
    A = B = 0.0
    for x, y in zip(a, b):
        A += x
        B += y
    with np.errstate(divide="ignore", invalid="ignore"):  # IEEE results for empty totals, as in C++
        ra = float(np.sqrt(np.float64(B) / np.float64(A)))
        rb = float(np.sqrt(np.float64(A) / np.float64(B)))
    r = Chi2Result()
    nbins = 0
    for x, y in zip(a, b):
        if x + y <= 0.0:
            continue
        d = ra * x - rb * y
        r.chi2 += d * d / (x + y)
        nbins += 1
    r.ndf = nbins - 1
    r.pvalue = chi2_pvalue(r.chi2, r.ndf)
    return r


def kolmogorov_q(lam: float) -> float:
    """Q_KS(lambda) = 2 sum_j (-1)^(j-1) exp(-2 j^2 lambda^2)."""
    if lam < 0.2:
        return 1.0
    s, sign = 0.0, 1.0
    for j in range(1, 101):
        term = sign * math.exp(-2.0 * j * j * lam * lam)
        s += term
        if abs(term) < 1e-16:
            break
        sign = -sign
    return min(max(2.0 * s, 0.0), 1.0)


@dataclass
class KsResult:
    d: float = 0.0
    pvalue: float = 1.0


def ks_two_sample(a, b) -> KsResult:
    """Two-sample KS statistic over the union of the samples' values, with the
    Stephens-corrected Kolmogorov p-value."""
    a = np.sort(np.asarray(a, dtype=np.float64))
    b = np.sort(np.asarray(b, dtype=np.float64))
    na, nb = float(a.size), float(b.size)
    r = KsResult()
    if a.size and b.size:
        v = np.unique(np.concatenate([a, b]))
        # The walk stops when either sample is exhausted: values past min(max a, max b)
        # cannot raise the maximum difference.
        v = v[v <= min(a[-1], b[-1])]
        fa = np.searchsorted(a, v, side="right") / na
        fb = np.searchsorted(b, v, side="right") / nb
        r.d = float(np.max(np.abs(fa - fb))) if v.size else 0.0
    with np.errstate(divide="ignore", invalid="ignore"):  # an empty sample gives NaN, as in C++
        ne = np.sqrt(np.float64(na) * nb / (np.float64(na) + nb))
        lam = float((ne + 0.12 + 0.11 / ne) * r.d)
    r.pvalue = kolmogorov_q(lam)
    return r


# ---- history agreement -------------------------------------------------------

@dataclass
class HistoryAgreement:
    n: int = 0
    bitwise_identical: int = 0
    same_discrete: int = 0
    fate_differs: int = 0
    max_abs_dt: float = 0.0
    max_abs_dpos: float = 0.0
    first_divergent: int = -1


def _bits(x) -> np.ndarray:
    return np.asarray(x, dtype=np.float32).view(np.uint32)


def compare_histories(a, b) -> HistoryAgreement:
    n = len(a["fate"])
    if len(b["fate"]) != n:
        raise ValueError("compare_histories: different sizes")
    fa, fb = np.asarray(a["fate"]), np.asarray(b["fate"])
    discrete = ((fa == fb) & (np.asarray(a["n_boundary"]) == np.asarray(b["n_boundary"]))
                & (np.asarray(a["n_scatter"]) == np.asarray(b["n_scatter"])))
    h = HistoryAgreement(n=n)
    h.fate_differs = int(np.count_nonzero(fa != fb))
    h.same_discrete = int(np.count_nonzero(discrete))
    bad = np.flatnonzero(~discrete)
    h.first_divergent = int(bad[0]) if bad.size else -1
    same = discrete.copy()
    for k in ("t", "x", "y", "z", "path"):
        same &= _bits(a[k]) == _bits(b[k])
    h.bitwise_identical = int(np.count_nonzero(same))
    if h.same_discrete:
        d = discrete
        dt = np.abs(np.asarray(a["t"], np.float64)[d] - np.asarray(b["t"], np.float32)[d].astype(np.float64))
        h.max_abs_dt = float(dt.max())
        dx = np.asarray(a["x"], np.float32)[d].astype(np.float64) - np.asarray(b["x"], np.float32)[d]
        dy = np.asarray(a["y"], np.float32)[d].astype(np.float64) - np.asarray(b["y"], np.float32)[d]
        dz = np.asarray(a["z"], np.float32)[d].astype(np.float64) - np.asarray(b["z"], np.float32)[d]
        h.max_abs_dpos = float(np.sqrt(dx * dx + dy * dy + dz * dz).max())
    return h


# ---- distribution agreement ----------------------------------------------------

@dataclass
class DistributionComparison:
    n_a: int = 0
    n_b: int = 0
    det_a: int = 0
    det_b: int = 0
    eff_a: float = 0.0
    eff_b: float = 0.0
    err_a: float = 0.0
    err_b: float = 0.0
    eff_z: float = 0.0
    time_chi2: Chi2Result = field(default_factory=Chi2Result)
    xy_chi2: Chi2Result = field(default_factory=Chi2Result)
    time_ks: KsResult = field(default_factory=KsResult)


def _histograms(r, p: SimParams, time_bins: int, t_max: np.float32, xy_bins: int):
    det = np.asarray(r["fate"]) == DETECTED
    t = np.asarray(r["t"], np.float32)[det]
    x = np.asarray(r["x"], np.float32)[det]
    y = np.asarray(r["y"], np.float32)[det]
    f32 = np.float32
    with np.errstate(over="ignore", invalid="ignore"):
        tb = np.minimum(time_bins, (t / t_max * f32(time_bins)).astype(np.int64))
        hx, hy = f32(p.hx), f32(p.hy)
        ix = np.minimum(xy_bins - 1, ((x + hx) / (f32(2) * hx) * f32(xy_bins)).astype(np.int64))
        iy = np.minimum(xy_bins - 1, ((y + hy) / (f32(2) * hy) * f32(xy_bins)).astype(np.int64))
    ht = np.bincount(tb, minlength=time_bins + 1).astype(np.float64)
    hxy = np.bincount(iy * xy_bins + ix, minlength=xy_bins * xy_bins).astype(np.float64)
    return ht, hxy, t.astype(np.float64), int(det.sum())


def compare_distributions(a, b, p: SimParams, time_bins: int = 100, t_max: float = 0.0,
                          xy_bins: int = 20) -> DistributionComparison:
    """t_max <= 0: the latest detected arrival in either sample, moved up by one
    float ulp so that it falls inside the range (compare.cpp:70-77)."""
    tm = np.float32(t_max)
    if tm <= 0:
        for r in (a, b):
            det = np.asarray(r["fate"]) == DETECTED
            if det.any():
                tm = max(tm, np.asarray(r["t"], np.float32)[det].max())
        tm = np.nextafter(np.float32(tm), np.float32(np.inf))
    ta, xya, ts_a, da = _histograms(a, p, time_bins, tm, xy_bins)
    tb, xyb, ts_b, db = _histograms(b, p, time_bins, tm, xy_bins)
    d = DistributionComparison(n_a=len(a["fate"]), n_b=len(b["fate"]), det_a=da, det_b=db)
    d.eff_a = da / d.n_a
    d.eff_b = db / d.n_b
    d.err_a = math.sqrt(d.eff_a * (1 - d.eff_a) / d.n_a)
    d.err_b = math.sqrt(d.eff_b * (1 - d.eff_b) / d.n_b)
    err = math.sqrt(d.err_a * d.err_a + d.err_b * d.err_b)
    d.eff_z = (d.eff_a - d.eff_b) / err if err > 0 else 0.0
    d.time_chi2 = chi2_two_sample(ta, tb)
    d.xy_chi2 = chi2_two_sample(xya, xyb)
    d.time_ks = ks_two_sample(ts_a, ts_b)
    return d


# ---- JSON (compare.cpp:101-120) ----------------------------------------------

def _g(v: float) -> str:
    if math.isnan(v):
        return "nan"
    if math.isinf(v):
        return "inf" if v > 0 else "-inf"
    return format(v, ".10g")


def history_json(h: HistoryAgreement) -> str:
    return (f"{{\"n\": {h.n}, \"bitwise_identical\": {h.bitwise_identical}, "
            f"\"same_discrete\": {h.same_discrete}, \"fate_differs\": {h.fate_differs}, "
            f"\"frac_bitwise\": {_g(h.bitwise_identical / h.n if h.n else math.nan)}, "
            f"\"frac_same_discrete\": {_g(h.same_discrete / h.n if h.n else math.nan)}, "
            f"\"max_abs_dt_ns\": {_g(h.max_abs_dt)}, \"max_abs_dpos_mm\": {_g(h.max_abs_dpos)}, "
            f"\"first_divergent\": {h.first_divergent}}}")


def distribution_json(d: DistributionComparison) -> str:
    return (f"{{\"n_a\": {d.n_a}, \"n_b\": {d.n_b}, \"det_a\": {d.det_a}, \"det_b\": {d.det_b}, "
            f"\"eff_a\": {_g(d.eff_a)}, \"eff_b\": {_g(d.eff_b)}, \"err_a\": {_g(d.err_a)}, "
            f"\"err_b\": {_g(d.err_b)}, \"eff_z\": {_g(d.eff_z)}, "
            f"\"time_chi2\": {_g(d.time_chi2.chi2)}, \"time_ndf\": {d.time_chi2.ndf}, "
            f"\"time_chi2_p\": {_g(d.time_chi2.pvalue)}, \"xy_chi2\": {_g(d.xy_chi2.chi2)}, "
            f"\"xy_ndf\": {d.xy_chi2.ndf}, \"xy_chi2_p\": {_g(d.xy_chi2.pvalue)}, "
            f"\"time_ks_d\": {_g(d.time_ks.d)}, \"time_ks_p\": {_g(d.time_ks.pvalue)}}}")


# ---- command line --------------------------------------------------------------

def params_from_meta(meta: dict) -> SimParams:
    """SimParams of a run from its meta.json (the fields the comparison needs and
    the rest of the physics keys)."""
    from .params import SURFACE_NAMES, POINT, VOLUME

    def num(key, default):
        v = meta.get(key, default)
        return math.inf if v == "inf" else float(v)

    return SimParams(hx=num("size_x", 50.0) / 2, hy=num("size_y", 50.0) / 2, hz=num("size_z", 50.0) / 2,
                     n_scint=num("n_scint", 1.63), n_det=num("n_det", 1.63), n_out=num("n_out", 1.0),
                     abs_length=num("abs_length", 1000.0), scat_length=num("scat_length", math.inf),
                     surface=SURFACE_NAMES.get(meta.get("surface", "polished"), 0),
                     reflectivity=num("reflectivity", 0.95),
                     source=VOLUME if meta.get("source") == "volume" else POINT,
                     src_x=num("src_x", 0.0), src_y=num("src_y", 0.0), src_z=num("src_z", 0.0),
                     tau=num("tau", 4.0), max_steps=int(meta.get("max_steps", 10000)),
                     seed=int(meta.get("seed", 12345)))


def main(argv=None) -> int:
    """Compares two record directories (the reference's optphot --out layout, or
    this package's io.write_records) and prints {"history": ..., "distribution": ...}:

        python -m gpu_optical_photons_b200.compare DIR_A DIR_B [--time_bins 100]
            [--t_max 0] [--xy_bins 20]

    The histories are compared photon by photon when both hold the same number of
    photons ("history": null otherwise). Hit-map bins use DIR_A's box size.
    """
    import argparse
    import json

    from . import io

    ap = argparse.ArgumentParser(description=main.__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("dir_a")
    ap.add_argument("dir_b")
    ap.add_argument("--time_bins", type=int, default=100)
    ap.add_argument("--t_max", type=float, default=0.0)
    ap.add_argument("--xy_bins", type=int, default=20)
    a = ap.parse_args(argv)
    ra, rb = io.read_records(a.dir_a), io.read_records(a.dir_b)
    p = params_from_meta(io.read_meta(a.dir_a))
    h = compare_histories(ra, rb) if len(ra["fate"]) == len(rb["fate"]) else None
    d = compare_distributions(ra, rb, p, a.time_bins, a.t_max, a.xy_bins)
    text = ("{\"history\": " + (history_json(h) if h else "null") + ",\n\"distribution\": "
            + distribution_json(d) + "}")
    json.loads(text)  # well-formed
    print(text)
    return 0


if __name__ == "__main__":
    import sys

    sys.exit(main())
