"""Seeded synthetic workloads for the batched and served forms.

* batched uneven filters: F unicycle filters whose particle counts are
  log-uniform over [lo, hi], rounded to multiples of `granule` (numpy PCG64
  generator seeded with `seed`); filter i uses landmarks, ground truth and
  measurements generated from seed `seed + i` by pf_make_trace.
"""
import numpy as np

from . import MODEL_UNICYCLE, make_trace, unicycle_params


def log_uniform_counts(n, lo, hi, granule, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    x = np.exp(rng.uniform(np.log(lo), np.log(hi), size=n))
    c = np.clip(np.rint(x / granule).astype(np.int64) * granule, lo, hi)
    return c.astype(np.int32)


def batched_unicycle(num_filters=4096, steps=200, lo=256, hi=65536, granule=256, seed=4):
    """(counts [F], params [F], inputs [F, steps] STEP_INPUT_DTYPE, truth [F, steps, 3])."""
    counts = log_uniform_counts(num_filters, lo, hi, granule, seed)
    params, inputs, truth = [], [], []
    for i in range(num_filters):
        p = unicycle_params(seed + i)
        inp, tr = make_trace(MODEL_UNICYCLE, p, seed + i, steps)
        params.append(p)
        inputs.append(inp)
        truth.append(tr)
    return counts, params, np.stack(inputs), np.stack(truth)
