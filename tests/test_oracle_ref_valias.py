"""The oracle's Vose alias build against the reference's own OpenCL resampler
(resampling-valias.cl), from golden vectors that tests/golden/
make_ref_valias_golden.py recorded by running it on a GPU (built as CUDA by
oracle/build_ref_valias.sh).  The reference fills its work lists with atomics,
so its tables' order is the hardware's: compared are the normalised, scaled
starting probabilities (bit for bit), each slot's selection probability
implied by the finished tables (within FP32 rounding) and the draw rule on the
reference's own tables (bit for bit)."""
from pathlib import Path

import numpy as np
import pytest

G = np.load(Path(__file__).resolve().parent / "golden" / "ref_valias.npz")


@pytest.mark.parametrize("m", [32, 64, 256, 512, 1024])
def test_oracle_vose_against_reference_golden(O, m):
    w, u2 = G["w_%d" % m], G["u2_%d" % m]
    scaled, rprob, ralias, rsel = G["scaled_%d" % m], G["prob_%d" % m], G["alias_%d" % m], G["sel_%d" % m]
    assert np.array_equal(O.vose_scaled(w, m).view(np.uint32), scaled.view(np.uint32))
    oprob, oalias = O.vose_build(w, m)
    small = scaled <= 1.0
    assert np.array_equal(oprob[small], scaled[small])  # slots that start small are never changed
    ri, oi = O.implied_selection(rprob, ralias, m), O.implied_selection(oprob, oalias, m)
    assert np.all(np.abs(ri - oi) <= 1e-6 + 1e-4 * ri), np.max(np.abs(ri - oi))
    assert np.array_equal(O.vose_draws(rprob, ralias, u2, m), rsel)
