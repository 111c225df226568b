"""Discrete-ordinates direction sets in the reference's ordering contract.

INPUT_QUAD (MainSrc/INPUTS.f08:1579-1671) defines the contract the sweep relies on:
  * N_m = 4 * N_q directions; the first quadrant (Omega_x > 0, Omega_y > 0) is listed first and the
    other three are sign flips of it, in the order (-,+), (-,-), (+,-) (:1658-1664);
  * weights repeat per quadrant and are normalised to sum to 4*pi (:1666-1669).
Reflective boundaries (UPDATES.f08:34-102) pair direction m with m +/- N_m/4 etc., which holds only
under this ordering.

Level-symmetric LQ_n sets (S8, S12, S16) are built here: direction cosines
mu_i^2 = mu_1^2 + (i-1) * 2 (1 - 3 mu_1^2) / (n - 2), points (mu_i, mu_j, mu_k) with i+j+k = n/2+2 in
one octant, point weights shared by permutation class.  The class weights solve the even-moment
conditions sum_p w_p mu_p^(2a) = 1/(2a+1), a = 0..n/2; where that system leaves a free direction
(S16) it is fixed by the nearest point to the published weights.  mu_1 and the published weights are
those of the standard LQ_n table (Lewis & Miller, Computational Methods of Neutron Transport, 1984,
Table 4-1); the tests check the solved weights against that table.
"""
import itertools
import math

import numpy as np

# mu_1 of the standard LQ_n sets and their published point weights (octant sum 1), by class in the
# order of sorted index triples.
LQN_MU1 = {2: 0.5773503, 4: 0.3500212, 6: 0.2666355, 8: 0.2182179, 12: 0.1672126, 16: 0.1389568}
LQN_WEIGHTS = {
    2: [1.0],
    4: [0.3333333],
    6: [0.1761263, 0.1572071],
    8: [0.1209877, 0.0907407, 0.0925926],
    12: [0.0707626, 0.0558811, 0.0373377, 0.0502819, 0.0258513],
    16: [0.0489872, 0.0413296, 0.0212326, 0.0256207, 0.0360486, 0.0144589, 0.0344958, 0.0085179],
}


def _lqn_octant(n):
    """Points (mu, eta, xi) and weights (sum 1) of one octant of LQ_n."""
    if n not in LQN_MU1:
        raise ValueError(f"level-symmetric order {n} not supported (have {sorted(LQN_MU1)})")
    h = n // 2
    if n == 2:
        mu = np.array([LQN_MU1[2]])
    else:
        m1 = LQN_MU1[n] ** 2
        delta = 2.0 * (1.0 - 3.0 * m1) / (n - 2)
        mu = np.sqrt(m1 + np.arange(h) * delta)
    pts = [p for p in itertools.product(range(1, h + 1), repeat=3) if sum(p) == h + 2]
    classes = sorted(set(tuple(sorted(p)) for p in pts))
    cls = np.array([classes.index(tuple(sorted(p))) for p in pts])
    # even-moment conditions on the class weights
    rows, rhs = [], []
    for a in range(0, h + 1):
        rows.append([sum(mu[p[0] - 1] ** (2 * a) for p, c in zip(pts, cls) if c == k) for k in range(len(classes))])
        rhs.append(1.0 / (2 * a + 1))
    A = np.array(rows)
    b = np.array(rhs)
    w0, *_ = np.linalg.lstsq(A, b, rcond=None)
    # free directions of the moment system: move to the published weights along them
    _, s, vt = np.linalg.svd(A)
    rank = int(np.sum(s > 1e-12 * s[0]))
    null = vt[rank:]
    wc = w0
    if null.shape[0]:
        pub = np.array(LQN_WEIGHTS[n])
        wc = w0 + null.T @ (null @ (pub - w0))
    P = np.array([[mu[p[0] - 1], mu[p[1] - 1], mu[p[2] - 1]] for p in pts])
    W = wc[cls]
    return P, W, np.array(classes), wc


def level_symmetric(n):
    """LQ_n set for 2D x-y geometry in the reference ordering: returns (Omega_x, Omega_y, w) with
    N_m = n(n+2)/2 directions, weights summing to 4*pi."""
    P, W, _, _ = _lqn_octant(n)
    # first quadrant, ordered by increasing Omega_y, then decreasing Omega_x
    order = np.lexsort((-P[:, 0], P[:, 1]))
    ox1, oy1, w1 = P[order, 0], P[order, 1], W[order]
    return expand_quadrants(ox1, oy1, w1)


def expand_quadrants(ox1, oy1, w1):
    """Quadrant expansion and 4*pi normalisation of INPUT_QUAD (INPUTS.f08:1658-1669)."""
    ox1 = np.asarray(ox1, dtype=np.float64)
    oy1 = np.asarray(oy1, dtype=np.float64)
    w1 = np.asarray(w1, dtype=np.float64)
    ox = np.concatenate([ox1, -ox1, -ox1, ox1])
    oy = np.concatenate([oy1, oy1, -oy1, -oy1])
    w = np.concatenate([w1, w1, w1, w1])
    w = 4.0 * math.pi * w / np.sum(w)
    return ox, oy, w


def by_name(name):
    """'S8', 'S12', 'S16' (level-symmetric) or a reference set name (see reference_set)."""
    if name.upper().startswith("S") and name[1:].isdigit():
        return level_symmetric(int(name[1:]))
    return reference_set(name)


def reference_set(name):
    """The fixed sets of INPUT_QUAD (INPUTS.f08:1587-1656): 'abu36' (144 directions), 'abu20' (80),
    '1d_test' (8).  First-quadrant values as listed there, expanded by expand_quadrants."""
    if name == "1d_test":
        return expand_quadrants([0.92388, 0.382683], [0.382683, 0.92388], [0.5, 0.5])
    if name == "abu20":
        ox = [9.713274064903e-1, 7.645615896150e-1, 4.424202396002e-1, 9.586898685237e-1, 7.375714298063e-1,
              1.409476441875e-1, 9.028558915298e-1, 3.858240341629e-1, 6.313311043797e-1, 7.770210099715e-1,
              5.837054752370e-1, 4.332989313333e-1, 2.221674140412e-1, 3.596178122512e-1, 4.908227124734e-2,
              2.057068622698e-1, 1.593344524838e-1, 4.982847370367e-2, 4.210110375297e-2, 3.157215799340e-2]
        w = [2.419260514149e-2, 2.998205782366e-2, 2.932993043666e-2, 5.213067212540e-2, 6.147460425028e-2,
             1.802505216045e-2, 7.185542471164e-2, 5.322055875020e-2, 7.796304620960e-2, 8.182604839076e-2]
        w = w + w[::-1]
        return expand_quadrants(ox, ox[::-1], w)
    if name == "abu36":
        ox = [9.717784813336e-1, 7.656319455497e-1, 4.445439440056e-1, 9.701698603928e-1, 7.633693960835e-1,
              1.483114568272e-1, 9.622473153642e-1, 7.524467626583e-1, 9.410672772109e-1, 4.288508824476e-1,
              7.241384940891e-1, 8.997294996538e-1, 6.711819639118e-1, 1.293388490485e-1, 8.335743322378e-1,
              3.670788892962e-1, 5.909368760506e-1, 7.417637460141e-1, 6.279014865859e-1, 4.869502395267e-1,
              2.519357740235e-1, 4.996274255819e-1, 7.447663982495e-2, 3.685670882907e-1, 3.673697853806e-1,
              2.488983098158e-1, 1.196054590036e-1, 2.426233944222e-1, 1.419535016004e-1, 1.362124657777e-1,
              1.670387759191e-2, 5.995074957044e-2, 5.695764868253e-2, 2.447911451942e-2, 1.160393058611e-2,
              1.096881837272e-2]
        w = [8.454511187252e-3, 8.352354145856e-3, 1.460888798152e-2, 1.913728513580e-2, 1.873220073879e-2,
             6.404244616724e-3, 2.863542971348e-2, 2.759429759588e-2, 3.648716160597e-2, 2.995376809966e-2,
             3.442681426024e-2, 4.244873302980e-2, 3.901232700510e-2, 1.162080754372e-2, 4.642823955812e-2,
             3.798783310581e-2, 4.130171453748e-2, 4.841339013884e-2]
        w = w + w[::-1]
        return expand_quadrants(ox, ox[::-1], w)
    raise ValueError(f"unknown quadrature {name!r}")
