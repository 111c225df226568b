"""Direction sets: level-symmetric construction, published weights, the INPUT_QUAD ordering contract."""
import math
import os
import re

import numpy as np
import pytest

from common import pkg

Q = pkg.quadrature
# The reference's INPUTS.f08, when a copy of the reference tree is at hand (TRT_REFERENCE_ROOT names its
# root directory); the comparison is skipped otherwise.
REF_INPUTS = os.path.join(os.environ.get("TRT_REFERENCE_ROOT", ""), "MainSrc", "INPUTS.f08")


@pytest.mark.parametrize("n,nm", [(8, 40), (12, 84), (16, 144)])
def test_level_symmetric_counts_and_contract(n, nm):
    ox, oy, w = Q.level_symmetric(n)
    assert len(ox) == nm
    q = nm // 4
    assert np.all(ox[:q] > 0) and np.all(oy[:q] > 0)
    assert np.array_equal(ox[q:2 * q], -ox[:q]) and np.array_equal(oy[q:2 * q], oy[:q])
    assert np.array_equal(ox[2 * q:3 * q], -ox[:q]) and np.array_equal(oy[2 * q:3 * q], -oy[:q])
    assert np.array_equal(ox[3 * q:], ox[:q]) and np.array_equal(oy[3 * q:], -oy[:q])
    assert abs(np.sum(w) - 4 * math.pi) < 1e-12
    assert np.all(ox ** 2 + oy ** 2 < 1.0)


@pytest.mark.parametrize("n", [4, 6, 8, 12, 16])
def test_level_symmetric_weights_match_published_table(n):
    P, W, classes, wc = Q._lqn_octant(n)
    assert np.max(np.abs(wc - np.array(Q.LQN_WEIGHTS[n]))) < 2e-6
    # directions lie on the unit sphere and the even moments are integrated exactly
    assert np.max(np.abs(np.sum(P * P, axis=1) - 1.0)) < 1e-6
    for a in range(0, n // 2 + 1):
        assert abs(np.sum(W * P[:, 0] ** (2 * a)) - 1.0 / (2 * a + 1)) < 1e-7   # mu_1 has 7 digits


def test_second_moments_of_2d_sets():
    for name in ("S8", "S12", "S16"):
        ox, oy, w = Q.by_name(name)
        assert abs(np.sum(w * ox * ox) / np.sum(w) - 1.0 / 3.0) < 1e-10
        assert abs(np.sum(w * ox * oy)) < 1e-12


@pytest.mark.skipif(not os.path.exists(REF_INPUTS), reason="reference tree not present")
def test_reference_sets_match_inputs_f08():
    """The abu36/abu20/1d_test tables equal the first-quadrant lists of INPUT_QUAD."""
    src = open(REF_INPUTS).read()
    block = src[src.index("SUBROUTINE INPUT_QUAD"):src.index("END SUBROUTINE INPUT_QUAD")]
    num = r"[-+]?\d*\.\d+d[-+]?\d+|[-+]?\d*\.?\d+d0"
    for name in ("abu36", "abu20"):
        # the table follows the last test of the name (the first one only sets N_m)
        at = max(m.start() for m in re.finditer(r"IF\s*\(quadrature \.EQ\. '" + name + r"'\)", block))
        seg = block[at:]
        lists = re.findall(r"\(/(.*?)/\)", seg, flags=re.S)[:3]
        vals = [np.array([float(x.replace("d", "e")) for x in re.findall(num, L)]) for L in lists]
        ox, oy, w = Q.reference_set(name)
        q = len(ox) // 4
        assert np.array_equal(ox[:q], vals[0]) and np.array_equal(oy[:q], vals[1])
        w1 = vals[2]
        w_exp = np.concatenate([w1] * 4)
        w_exp = 4.0 * math.pi * w_exp / np.sum(w_exp)
        assert np.max(np.abs(w - w_exp)) < 1e-15
