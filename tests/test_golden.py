"""The oracle against its committed golden fixtures (CPU).  A failure means
the restatement changed; regenerate only for a deliberate change."""
import os

import numpy as np
import pytest

from tests.golden import make_golden as G

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", sorted(G.FIXTURES))
def test_oracle_matches_golden(name):
    ref = np.load(os.path.join(HERE, name + ".npz"))
    got = G.run(name)
    for key in ref.files:
        r, g = ref[key], got[key]
        assert r.shape == g.shape, key
        scale = np.max(np.abs(r)) if r.size else 0.0
        assert np.max(np.abs(g - r)) <= 1e-12 * max(scale, 1e-300), key
