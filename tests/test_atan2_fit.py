"""The atan polynomial compiled into pf_atan2: the committed coefficients are
the project's own least-squares + Lawson fit (esthera_b200/csrc/fit_atan2.py
regenerates them) and meet the stated error bounds against FP64 atan2."""
import importlib.util
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def _fit():
    spec = importlib.util.spec_from_file_location("fit_atan2", ROOT / "esthera_b200" / "csrc" / "fit_atan2.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_refit_reproduces_committed_coefficients():
    m = _fit()
    c, e = m.fit(4000, 60)
    cur = m.committed().astype(np.float64)
    assert len(cur) == 8
    assert e < 5e-8
    # the refit lands within a few FP32 ulps of every committed coefficient
    assert np.all(np.abs(c[::-1] - cur) <= 4 * np.spacing(np.abs(cur).astype(np.float32)).astype(np.float64) + 2e-8)


def test_committed_coefficients_meet_the_bounds():
    assert _fit().main([]) == 0
