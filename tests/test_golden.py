"""The oracle reproduces the committed golden fixtures bit for bit (pins the
oracle against regressions; fixtures: tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from golden_cases import GOLDEN, load_golden

pytestmark = []


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_oracle_reproduces_golden(name, workdir):
    import make_golden
    img, recs = make_golden.render_case(name, workdir)
    gimg, grecs = load_golden(name)
    assert np.array_equal(img.view(np.uint32), gimg.view(np.uint32))
    for f in ("hash", "bounces", "nee_tests", "nee_occluded", "primary_mesh", "primary_tri"):
        assert np.array_equal(recs[f], grecs[f]), f
    assert np.array_equal(recs["rgb"].view(np.uint32), grecs["rgb"].view(np.uint32))
