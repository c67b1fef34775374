"""The algorithmic work per photon-step used as the roofline numerator in
bench.py is the oracle's op count (op-counting scalar type) of the benchmark
workload; this pins the constant so it cannot drift from the physics."""
import importlib.util
import os

import numpy as np

from gpu_optical_photons_b200.wavefront import batched_events

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def bench_module():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_ops_per_step_constant_matches_oracle(oracle):
    events, _ = batched_events()
    agg = None
    for i in range(0, 4096, 64):
        c = oracle.opcount(events[i], 500, 0)
        agg = c if agg is None else {k: tuple(a + b for a, b in zip(agg[k], c[k])) for k in c}
    steps = sum(v[0] for k, v in agg.items() if k != "start")
    ops = sum(v[1] + v[2] + v[3] for v in agg.values())
    assert abs(ops / steps - bench_module().OPS_PER_STEP) < 0.05


def test_philox_block_is_98_integer_ops(oracle):
    # 10 rounds x (2 mul-lo + 2 mul-hi + 4 xor) + 9 x 2 key additions
    c = oracle.opcount(oracle_params(), 1, 0)
    per_block = 98
    # emission of a point-source photon draws 3 words: exactly one Philox block
    assert c["start"][3] == per_block + 3 * 4


def oracle_params():
    from gpu_optical_photons_b200 import params as P
    return P.SimParams()
