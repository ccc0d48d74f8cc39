"""CPU check of the envelope-feature oracle (oracle/features.py) against the
fixtures made from the reference tutorial's own ``envelope`` function
(tests/golden/make_feature_golden.py): bit for bit."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

from oracle import features as ofeat


def load_features():
    with np.load(os.path.join(GOLDEN, "features.npz")) as z:
        g = {k: z[k] for k in z.files}
    names = sorted(k[2:] for k in g if k.startswith("x_"))
    return g, names


G, NAMES = load_features()


def test_fixture_cases():
    assert {"even_1000", "odd_1001", "prime_997", "spike_clipped", "zeros"} <= set(NAMES)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_tutorial_envelope(name):
    got = ofeat.envelope(G[f"x_{name}"])
    assert np.array_equal(got.view(np.uint32), G[f"feature_{name}"].view(np.uint32))


def test_oracle_rows():
    x = np.stack([G["x_even_1000"], G["x_even_1000"][::-1]])
    f = ofeat.waveform_features(x[None])
    assert f.shape == (1, 2, 1000)
    assert np.array_equal(f[0, 0], G["feature_even_1000"])
