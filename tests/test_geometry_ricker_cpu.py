"""The Ricker source time function (prepare_stf) against the reference's own
Python restatement of the wavelet OWL injects (test/lamb_reference.py
`ricker_owl`: peak at 1/f0, normalised to unit maximum), from the golden
fixture tests/golden/lamb_flat.npz (20 Hz at a 0.2 ms step): the same 501
samples (2 / f0 / dt formed in single precision rounds up past 500, as the
helper's round(2 / f0 / dt) + 1), equal to single precision."""
import os

import numpy as np

from owl_b200.geometry import Source, prepare_stf


def test_ricker_matches_reference_helper():
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "lamb_flat.npz"))
    stf, hnt = prepare_stf(Source(x=0.0, z=0.0, f0=float(g["f0"])), float(g["dt"]))
    ref = g["stf"]
    n = len(stf)
    assert n == np.count_nonzero(ref) == 501
    assert np.max(np.abs(stf.astype(np.float64) - ref[:n])) < 2e-6
    assert hnt == int(np.floor(n / 2.0 + 0.5))
