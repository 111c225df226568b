"""Reduced-order model path: the POD of snapshots (the decomposer's POD_Calc with SVD_Calc_Cntr,
Decomposer/DecompSrc/POD_ROUTINES.c:75-120, LA_ROUTINES.c:50-170) and POD_RECONSTRUCT
(MainSrc/POD_ROUTINES.f08:372-432), on the device (trt_pod_calc, trt_pod_reconstruct) against the oracle
(oracle.pod_calc: centring in the decomposer's order + LAPACK SVD; oracle.pod_reconstruct: the Fortran loop).

Singular values agree to 1e-12 of the largest; singular vectors are unique only up to sign (and only where
the singular values are separated), so they are compared after aligning signs, on well-separated spectra.
The centring vector and the reconstruction follow the reference's operation order and agree bit for bit.
"""
import ctypes

import numpy as np
import pytest

from common import pkg


def snapshots(clen, n_g, n_t, seed, decay=0.5):
    """data(clen, n_g, n_t): per block a mean field plus modes with geometrically decaying singular values
    (ratio `decay`, so each is separated from the next); the time coefficients have zero mean, so the
    centred matrix has exactly these singular values."""
    rng = np.random.default_rng(seed)
    out = np.empty((clen, max(n_g, 1), n_t), order="F")
    for g in range(max(n_g, 1)):
        k = min(clen, n_t - 1)
        Q1, _ = np.linalg.qr(rng.standard_normal((clen, k)))
        Q2, _ = np.linalg.qr(np.hstack([np.ones((n_t, 1)), rng.standard_normal((n_t, k))]))
        s = 3.0 * decay ** np.arange(k) * (1 + 0.1 * g)
        out[:, g, :] = 0.3 + rng.standard_normal((clen, 1)) * 0.01 + (Q1 * s) @ Q2[:, 1:k + 1].T
    return out


def align(A, B):
    """Flip the columns of A to the signs of B."""
    sgn = np.sign(np.sum(A * B, axis=0))
    sgn[sgn == 0] = 1.0
    return A * sgn


# ------------------------------------------------------------------------------------------------ CPU

def test_oracle_pod_reproduces_the_snapshots(oracle):
    data = snapshots(40, 3, 12, 1)
    for g in range(3):
        c, u, s, vt = oracle.pod_calc(data, 12, 3, 40, g)
        assert np.all(np.diff(s) <= 0)
        np.testing.assert_allclose(c[:, None] + (u * s) @ vt, data[:, g, :], rtol=0, atol=1e-13)
        for t in range(1, 13):   # full-rank reconstruction of block g at every time level
            r = oracle.pod_reconstruct(c, s, u, vt, [len(s)], 40, 1, 12, t, 1)
            np.testing.assert_allclose(r, data[:, g, t - 1], rtol=0, atol=1e-13)


def test_oracle_groupwise_reconstruction_layout(oracle):
    clen, ng, nt, rank = 30, 3, 8, [2, 4, 3]
    data = snapshots(clen, ng, nt, 2)
    C, S, U, V = [], [], [], []
    for g in range(ng):
        c, u, s, vt = oracle.pod_calc(data, nt, ng, clen, g)
        C.append(c)
        S.append(s[:rank[g]])
        U.append(u[:, :rank[g]].ravel(order="F"))
        V.append(vt[:rank[g]].ravel(order="F"))
    for t in (1, 5, 8):
        r = oracle.pod_reconstruct(np.concatenate(C), np.concatenate(S), np.concatenate(U), np.concatenate(V), rank,
                                   clen * ng, ng, nt, t, 0)
        for g in range(ng):
            c, u, s, vt = oracle.pod_calc(data, nt, ng, clen, g)
            k = rank[g]
            np.testing.assert_allclose(r[g * clen:(g + 1) * clen], c + (u[:, :k] * s[:k]) @ vt[:k, t - 1],
                                       rtol=0, atol=1e-13)


# ------------------------------------------------------------------------------------------------ GPU

@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(500, 0, 20, 0), (300, 4, 16, 2), (12, 2, 30, 1), (1, 0, 5, 0)])
def test_device_pod_matches_oracle(oracle, shape):
    clen, ng, nt, g = shape
    data = snapshots(clen, ng, nt, 3 + clen)
    c, u, s, vt = pkg.POD_Calc(data, nt, ng, clen, g)
    rc, ru, rs, rvt = oracle.pod_calc(data, nt, ng, clen, g)
    assert np.array_equal(c, rc)
    np.testing.assert_allclose(s, rs, rtol=0, atol=1e-12 * rs[0])
    k = int(np.sum(rs > 1e-10 * rs[0]))   # the modes the data carries (the rest are round-off)
    np.testing.assert_allclose(align(u[:, :k], ru[:, :k]), ru[:, :k], rtol=0, atol=1e-9)
    np.testing.assert_allclose(align(vt[:k].T, rvt[:k].T), rvt[:k].T, rtol=0, atol=1e-9)
    # the decomposition reproduces the data
    blk = data[:, g, :] if ng else data[:, 0, :]
    np.testing.assert_allclose(c[:, None] + (u * s) @ vt, blk, rtol=0, atol=1e-12 * np.abs(blk).max())


@pytest.mark.gpu
@pytest.mark.parametrize("gsum", [0, 1])
def test_device_pod_reconstruct_bit_identical(oracle, gsum):
    clen, ng, nt = 64, 3, 10
    data = snapshots(clen, ng, nt, 9)
    if gsum == 0:
        rank = [3, 5, 2]
        parts = [oracle.pod_calc(data, nt, ng, clen, g) for g in range(ng)]
        C = np.concatenate([p[0] for p in parts])
        S = np.concatenate([p[2][:r] for p, r in zip(parts, rank)])
        U = np.concatenate([p[1][:, :r].ravel(order="F") for p, r in zip(parts, rank)])
        V = np.concatenate([p[3][:r].ravel(order="F") for p, r in zip(parts, rank)])
        length = clen * ng
    else:
        whole = data.reshape(clen * ng, 1, nt, order="F")
        c, u, s, vt = oracle.pod_calc(whole, nt, 0, clen * ng, 0)
        rank = [7]
        C, S, U, V = c, s[:7], u[:, :7].ravel(order="F"), vt[:7].ravel(order="F")
        length = clen * ng
    for t in (1, 4, nt):
        out = np.zeros(length)
        pkg.POD_RECONSTRUCT(out, C, S, U, V, rank, length, ng, nt, t, gsum)
        assert np.array_equal(out, oracle.pod_reconstruct(C, S, U, V, rank, length, ng, nt, t, gsum))


@pytest.mark.gpu
def test_rom_of_qd_factor_snapshots_from_the_device_time_loop(oracle):
    """Snapshots of fg_avg_xx from device time steps (the transport-only loop on a small problem), stored in
    HBM by trt_snapshot_output (with FP32 I_avg snapshots from trt_snapshot_angular), decomposed by
    trt_pod_calc_device; a truncated POD reproduces the snapshots to its tail energy."""
    import ctypes
    import torch
    P = pkg.problems
    prob = P.random_small(51, 12, 10, 3, "S8")
    ts = P.fc_timestep_setup(prob)
    ox, oy, w = prob.directions()
    nt = 8
    clen = prob.nx * prob.ny
    snaps = torch.empty((nt, prob.ng, clen), dtype=torch.float64, device="cuda")
    with pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, prob.delx, prob.dely, prob.ng) as s:
        s.init_state(ts.Tini_eV, list(ts.bcT_eV), P.COMP_UNIT, ts.nu_eV)
        s.tstep_setup(ts.nu_eV, ts.kappa_mult, ts.cv, np.full((prob.nx, prob.ny), ts.Tini_eV), ts.Kap0, P.COMP_UNIT,
                      P.C_LIGHT, ts.dt, bcT=ts.bcT_eV, conv_type=2, conv_ho=1e-8, maxit_rte=30)
        host = []
        nm = len(ox)
        iavg = torch.empty((nt, clen * nm * prob.ng), dtype=torch.float32, device="cuda")
        for t in range(nt):
            s.tstep()
            # the snapshot store on the device: slot t of a time-last (clen, n_g, n_t) array, and the FP32
            # angular snapshot beside it
            assert pkg.lib().trt_snapshot_output(s.handle, b"fg_avg_xx", ctypes.c_void_p(snaps[t].data_ptr())) == 0
            assert pkg.lib().trt_snapshot_angular(s.handle, ctypes.c_void_p(iavg[t].data_ptr())) == 0
            s.sync()
            f = s.moments(["fg_avg_xx"])["fg_avg_xx"]            # (nx, ny, ng), for the host-side check
            host.append(f)
            assert np.array_equal(snaps[t].cpu().numpy().reshape(-1), f.reshape(-1, order="F"))
            I = s.angular(("I_avg",))["I_avg"]
            assert np.array_equal(iavg[t].cpu().numpy(), I.reshape(-1, order="F").astype(np.float32))
    data = np.stack([h.reshape(clen, prob.ng, order="F") for h in host], axis=2)   # (clen, ng, nt)
    g = 1
    k = min(clen, nt)
    outs = [torch.empty(n, dtype=torch.float64, device="cuda") for n in (clen, clen * k, k, k * nt)]
    L = pkg.lib()
    assert L.trt_pod_calc_device(ctypes.c_void_p(snaps.data_ptr()), nt, prob.ng, clen, g,
                                 *[ctypes.c_void_p(o.data_ptr()) for o in outs], None) == 0
    torch.cuda.synchronize()
    c, u, sg, vt = (o.cpu().numpy() for o in outs)
    u, vt = u.reshape(clen, k, order="F"), vt.reshape(k, nt, order="F")
    rc, ru, rs, rvt = oracle.pod_calc(data, nt, prob.ng, clen, g)
    assert np.array_equal(c, rc)
    np.testing.assert_allclose(sg, rs, rtol=0, atol=1e-12 * rs[0])
    r = 3
    X = data[:, g, :]
    approx = c[:, None] + (u[:, :r] * sg[:r]) @ vt[:r]
    assert np.linalg.norm(approx - X) == pytest.approx(np.sqrt(np.sum(rs[r:] ** 2)), rel=1e-6, abs=1e-13)


FACTORS = ("fg_avg_xx", "fg_avg_yy", "fg_edgV_xx", "fg_edgV_xy", "fg_edgH_yy", "fg_edgH_xy", "Cg_L", "Cg_B", "Cg_R",
           "Cg_T")


@pytest.mark.gpu
def test_pod_rom_drives_the_low_order_time_loop():
    """The reference's POD-ROM run (HO_Form 1: each step's QD and boundary factors from POD_RECONSTRUCT
    instead of a sweep): factors recorded from a full mlqd run, decomposed per group (trt_pod_calc) and
    rebuilt at every time level (trt_pod_reconstruct, all modes) drive an ho_form = 1 run, which lands on the
    full run's temperatures (both converge the same low-order problem to the iteration tolerances)."""
    from test_mlqd import device, setup_problem
    prob, ts, km, bcT, cv = setup_problem(8, 6, 10, "S8", 31)
    kw = dict(conv_ho=1e-9, maxit_rte=40, conv_lo=1e-10, maxit_mloqd=80)
    nt = 3
    snaps, T_full = {k: [] for k in FACTORS}, []
    with device(prob, ts, km, bcT, cv, **kw) as s:
        for _ in range(nt):
            s.mlqd_step()
            m = s.moments(list(FACTORS))
            for k in FACTORS:
                snaps[k].append(m[k])
            T_full.append(s.mlqd_field("Temp"))
    ng = prob.ng
    rom = {}
    for k in FACTORS:
        data = np.stack([a.reshape(-1, ng, order="F") for a in snaps[k]], axis=2)   # (clen, ng, nt)
        clen = data.shape[0]
        parts = [pkg.POD_Calc(data, nt, ng, clen, g) for g in range(ng)]
        rank = [len(p[2]) for p in parts]
        rom[k] = (clen * ng, np.concatenate([p[0] for p in parts]), np.concatenate([p[2] for p in parts]),
                  np.concatenate([p[1].ravel(order="F") for p in parts]),
                  np.concatenate([p[3].ravel(order="F") for p in parts]), rank)
    with device(prob, ts, km, bcT, cv, ho_form=1, **kw) as s:
        for t in range(1, nt + 1):
            for k in FACTORS:
                length, C, S, U, V, rank = rom[k]
                out = np.zeros(length)
                pkg.POD_RECONSTRUCT(out, C, S, U, V, rank, length, ng, nt, t, 0)
                assert np.abs(out - snaps[k][t - 1].ravel(order="F")).max() <= 1e-12 * max(1.0, np.abs(out).max())
                s.mlqd_put(k, out)
            st = s.mlqd_step()
            assert st["sweeps"] == 0 and st["mgqd_nonconv"] == 0
            T = s.mlqd_field("Temp")
            assert float(np.max(np.abs(T - T_full[t - 1])) / np.max(T_full[t - 1])) < 1e-7


def dmd_model(clen, n_blocks, ranks, seed):
    """Modes, amplitudes and complex exponents of a DMD expansion (conjugate pairs, as a real signal has)."""
    rng = np.random.default_rng(seed)
    L, B, W = [], [], []
    for g in range(n_blocks):
        for _ in range(ranks[g]):
            L.append(complex(rng.uniform(-5, 1), rng.uniform(-40, 40)))
            B.append(complex(rng.standard_normal(), rng.standard_normal()))
            W.append(rng.standard_normal(clen) + 1j * rng.standard_normal(clen))
    return np.array(L), np.array(B), np.concatenate(W), rng.standard_normal(clen * n_blocks)


def test_oracle_dmd_reconstruct_is_the_expansion(oracle):
    clen, ranks = 25, [3, 2]
    L, B, W, C = dmd_model(clen, 2, ranks, 4)
    t = 0.037
    r = oracle.dmd_reconstruct(L, B, W, C, ranks, 2 * clen, 2, 0, t)
    ref = np.empty(2 * clen)
    o = 0
    for g in range(2):
        Wg = W[clen * o:clen * (o + ranks[g])].reshape(clen, ranks[g], order="F")
        ref[g * clen:(g + 1) * clen] = (Wg @ (B[o:o + ranks[g]] * np.exp(L[o:o + ranks[g]] * t))).real + \
            C[g * clen:(g + 1) * clen]
        o += ranks[g]
    np.testing.assert_allclose(r, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


@pytest.mark.gpu
@pytest.mark.parametrize("gsum", [0, 1])
def test_device_dmd_reconstruct_bit_identical(oracle, gsum):
    clen, ng = 300, 3
    ranks = [4, 2, 6] if gsum == 0 else [9]
    nb = ng if gsum == 0 else 1
    L, B, W, C = dmd_model(clen * (1 if gsum == 0 else ng), nb, ranks, 8)
    length = clen * ng
    for t in (0.0, 0.013, 0.2):
        out = np.zeros(length)
        pkg.DMD_RECONSTRUCT(out, L, B, W, C, ranks, length, ng, gsum, t)
        assert np.array_equal(out, oracle.dmd_reconstruct(L, B, W, C, ranks, length, ng, gsum, t))


def dmd_data(clen, n_g, n_t, seed, base=0.0):
    """Snapshots that are an exact sum of a few discrete-time modes: one real decaying mode and two
    conjugate oscillating pairs per block, plus a constant base vector."""
    rng = np.random.default_rng(seed)
    out = np.empty((clen, max(n_g, 1), n_t), order="F")
    mus = [0.93, 0.97 * np.exp(0.3j), 0.85 * np.exp(1.1j)]
    for g in range(max(n_g, 1)):
        field = base * rng.standard_normal(clen)
        modes = [rng.standard_normal(clen) + 1j * rng.standard_normal(clen) for _ in mus]
        for t in range(n_t):
            x = field.copy()
            for mu, phi in zip(mus, modes):
                x = x + (phi * mu ** t).real if mu.imag else x + phi.real * mu.real ** t
            out[:, g, t] = x
    return out


def match(a, b):
    """Order of the entries of b that pairs them with a (nearest, one to one)."""
    used, idx = set(), []
    for x in a:
        j = min((j for j in range(len(b)) if j not in used), key=lambda j: abs(b[j] - x))
        used.add(j)
        idx.append(j)
    return np.array(idx)


def test_oracle_dmd_recovers_the_modes(oracle):
    data = dmd_data(60, 2, 14, 3)
    o = oracle.dmd_calc(data, 14, 2, 60, 1, svd_eps=1e-10, delt=0.1)
    assert len(o["lambda_"]) == 5
    mus = np.array([0.93, 0.97 * np.exp(0.3j), 0.97 * np.exp(-0.3j), 0.85 * np.exp(1.1j), 0.85 * np.exp(-1.1j)])
    np.testing.assert_allclose(o["lambda_"][match(mus, o["lambda_"])], mus, atol=1e-10)
    for t in (0, 5, 12):   # the expansion reproduces the snapshots (DMD_RECONSTRUCT's formula at Time = t delt)
        x = (o["wmat"] @ (o["b"] * np.exp(o["omega"] * 0.1 * t))).real + o["cvec"]
        np.testing.assert_allclose(x, data[:, 1, t], atol=1e-9 * np.abs(data).max())


@pytest.mark.gpu
@pytest.mark.parametrize("case", [(80, 0, 16, 0, 0), (50, 3, 12, 2, 0), (40, 0, 15, 0, 1)])
def test_device_dmd_matches_oracle(oracle, case):
    clen, ng, nt, g, base = case
    data = dmd_data(clen, ng, nt, 11 + clen, base=1.0 if base else 0.0)
    dev = pkg.DMD_Calc(data, nt, ng, clen, g, base_subtract=base, svd_eps=1e-10, delt=0.05)
    ref = oracle.dmd_calc(data, nt, ng, clen, g, base_subtract=base, svd_eps=1e-10, delt=0.05)
    assert len(dev["lambda_"]) == len(ref["lambda_"])
    idx = match(ref["lambda_"], dev["lambda_"])
    np.testing.assert_allclose(dev["lambda_"][idx], ref["lambda_"], atol=1e-10)
    np.testing.assert_allclose(dev["omega"][idx], ref["omega"], atol=1e-8)
    np.testing.assert_array_equal(dev["cvec"], ref["cvec"])
    # the eigenvectors are unique up to a phase, which the amplitudes b absorb: compare the products
    np.testing.assert_allclose(dev["wmat"][:, idx] * dev["b"][idx], ref["wmat"] * ref["b"], rtol=0,
                               atol=1e-8 * np.abs(ref["wmat"] * ref["b"]).max())
    if base:   # with the last snapshot as base the affine part is outside a linear fit: no exact expansion
        return
    # and the device expansion, evaluated by DMD_RECONSTRUCT on the device, reproduces the snapshots
    blk = data[:, g, :] if ng else data[:, 0, :]
    xr = len(dev["lambda_"])
    for t in (1, nt // 2, nt - 2):
        out = np.zeros(clen)
        pkg.DMD_RECONSTRUCT(out, dev["omega"], dev["b"], dev["wmat"], dev["cvec"], [xr], clen, 1, 1, 0.05 * t)
        np.testing.assert_allclose(out, blk[:, t], rtol=0, atol=1e-8 * np.abs(blk).max())


def grid_maps(nx1, ny1, nx2, ny2, seed):
    """A coarse data grid (grid 1) and a finer simulation grid (grid 2) on [0, 6]^2 with the four-corner maps
    FMAP reads (1-based): the grid-1 cells that bracket each grid-2 point; points on a grid-1 line collapse
    the bracket (the degenerate branches of BILINEAR_INTERPOLATE)."""
    x1, y1 = np.linspace(0, 6, nx1), np.linspace(0, 6, ny1)
    rng = np.random.default_rng(seed)
    x2 = np.sort(np.concatenate([rng.uniform(0, 6, nx2 - 2), [x1[1], 6.0]]))
    y2 = np.sort(np.concatenate([rng.uniform(0, 6, ny2 - 2), [y1[2], 0.0]]))
    G1 = np.array([[x, y] for y in y1 for x in x1]).reshape(-1)       # point p = ix + nx1 * iy, (x, y) pairs
    G2 = np.array([[x, y] for y in y2 for x in x2]).reshape(-1)
    pt = lambda ix, iy: ix + nx1 * iy
    GM, VM = [], []
    for y in y2:
        for x in x2:
            ia = min(np.searchsorted(x1, x, side="right") - 1, nx1 - 1)
            ja = min(np.searchsorted(y1, y, side="right") - 1, ny1 - 1)
            ib = ia if x1[ia] == x else min(ia + 1, nx1 - 1)
            jb = ja if y1[ja] == y else min(ja + 1, ny1 - 1)
            corners = [pt(ia, ja), pt(ia, jb), pt(ib, ja), pt(ib, jb)]           # f11, f12, f21, f22
            VM += [corners[0] + 1, corners[2] + 1, corners[1] + 1, corners[3] + 1]   # VMap order: 11, 21, 12, 22
            GM += [2 * corners[0] + 1, 0, 0, 2 * corners[3] + 1]
    GM = np.array(GM)
    GM[1::4], GM[2::4] = GM[0::4], GM[3::4]
    return G1, G2, GM, np.array(VM)


def test_oracle_fmap_reproduces_a_bilinear_field(oracle):
    G1, G2, GM, VM = grid_maps(7, 6, 11, 9, 1)
    n1, n2 = len(G1) // 2, len(G2) // 2
    f = lambda g: 1.0 + 2.0 * g[0::2] - 0.5 * g[1::2] + 0.25 * g[0::2] * g[1::2]
    f1 = np.concatenate([f(G1), 3.0 * f(G1)])                       # two blocks (groups)
    f2 = oracle.fmap(f1, G1, G2, GM, VM, n1, n2, 2 * n2)
    np.testing.assert_allclose(f2, np.concatenate([f(G2), 3.0 * f(G2)]), rtol=1e-13, atol=1e-13)


@pytest.mark.gpu
def test_device_fmap_and_time_interpolation_bit_identical(oracle):
    G1, G2, GM, VM = grid_maps(9, 8, 23, 17, 2)
    n1, n2 = len(G1) // 2, len(G2) // 2
    rng = np.random.default_rng(3)
    f1 = rng.standard_normal(3 * n1)
    f2 = pkg.FMAP(f1, G1, G2, GM, VM, n1, n2, 3 * n2)
    assert np.array_equal(f2, oracle.fmap(f1, G1, G2, GM, VM, n1, n2, 3 * n2))
    v1, v2 = rng.standard_normal(500), rng.standard_normal(500)
    out = v1.copy()
    pkg.LINEAR_INTERPOLATION(out, v2, 0.37, 0.2, 0.9, 500)
    assert np.array_equal(out, oracle.linear_interpolation(v1, v2, 0.37, 0.2, 0.9))
    bad = VM.copy()
    bad[5] = n1 + 1                                                   # a map entry outside grid 1
    with pytest.raises(pkg.TrtError):
        pkg.FMAP(f1, G1, G2, GM, bad, n1, n2, 3 * n2)


def test_grid_coordinates_and_maps_match_oracle(oracle):
    """GRIDMAP_GEN_* and MAP_GRIDS (host code of the library, no device needed) against their restatements, and
    the maps they build drive FMAP (the oracle's restatement) to reproduce a bilinear field on the finer grid."""
    rng = np.random.default_rng(6)
    dx1, dy1 = rng.uniform(0.5, 1.5, 6), rng.uniform(0.5, 1.5, 5)
    dx2, dy2 = np.full(13, dx1.sum() / 13), np.full(11, dy1.sum() / 11)
    for kind, (nx, ny) in ((0, (6, 5)), (1, (7, 5)), (2, (6, 6))):
        assert np.array_equal(pkg.GRIDMAP_GEN(kind, dx1, dy1, nx, ny), oracle.gridmap_gen(kind, dx1, dy1, nx, ny))
    # data on the cell-edge lattice of the coarse grid (corners included), mapped to the fine grid's centres
    xe = np.concatenate([[0.0], np.cumsum(dx1)])
    ye = np.concatenate([[0.0], np.cumsum(dy1)])
    G1 = np.array([[x, y] for y in ye for x in xe]).reshape(-1)
    G2 = pkg.GRIDMAP_GEN(0, dx2, dy2, 13, 11)
    gm, vm = pkg.MAP_GRIDS(G1, G2, 2 * len(xe))
    rgm, rvm = oracle.map_grids(G1, G2, 2 * len(xe))
    assert np.array_equal(gm, rgm) and np.array_equal(vm, rvm)
    f = lambda g: 2.0 - 0.3 * g[0::2] + 0.7 * g[1::2] + 0.05 * g[0::2] * g[1::2]
    n1, n2 = len(G1) // 2, len(G2) // 2
    f2 = oracle.fmap(f(G1), G1, G2, gm, vm, n1, n2, n2)
    np.testing.assert_allclose(f2, f(G2), rtol=1e-13, atol=1e-13)
    # a bracket that would reach outside grid 1's arrays is rejected, not read past them
    with pytest.raises(pkg.TrtError):
        pkg.MAP_GRIDS(G1, np.array([-1.0, 1.0]), 2 * len(xe))


def test_time_map_and_boundary_helpers_match_oracle(oracle):
    """GENERATE_GRIDS_T and the boundary helpers of the reconstruction (host code of the library, no device)."""
    import ctypes
    L = pkg.lib()
    D, I = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    for args in ((2e-3, 1e-3, 0.0, 0.0, 7, 15), (5e-3, 2e-3, 0.01, 0.0, 6, 20), (1e-3, 1e-3, 0.0, 0.0, 10, 10)):
        dN_t, N_t = args[4], args[5]
        sim, dat, tm = np.zeros(N_t), np.zeros(dN_t), np.zeros(2 * N_t, dtype=np.int32)
        assert L.trt_generate_grids_t(*args, sim.ctypes.data_as(D), dat.ctypes.data_as(D), tm.ctypes.data_as(I)) == 0
        rs, rd, rt = oracle.generate_grids_t(*args)
        assert np.array_equal(sim, rs) and np.array_equal(dat, rd) and np.array_equal(tm, rt)
    ng, ny, nx = 3, 5, 4
    f = np.random.default_rng(7).standard_normal(ng * ny * nx)
    fp = f.ctypes.data_as(D)
    for name, n in (("collect_lr_bnd", ng * ny * 2), ("collect_bt_bnd", ng * 2 * nx), ("collect_crn_bnd", ng * 4),
                    ("extnd_bt_bnd", ng * (ny + 2) * nx), ("extnd_lr_bnd", ng * ny * (nx + 2))):
        out = np.zeros(n)
        assert getattr(L, "trt_" + name)(out.ctypes.data_as(D), fp, ng, ny, nx) == 0
        assert np.array_equal(out, getattr(oracle, name)(f, ng, ny, nx)), name
    lr, bt, crn = oracle.collect_lr_bnd(f, ng, ny, nx), oracle.collect_bt_bnd(f, ng, ny, nx), \
        oracle.collect_crn_bnd(f, ng, ny, nx)
    out = np.zeros(ng * (ny + 2) * (nx + 2))
    assert L.trt_avg_apnd_bnd(out.ctypes.data_as(D), fp, lr.ctypes.data_as(D), bt.ctypes.data_as(D),
                              crn.ctypes.data_as(D), ng, ny, nx) == 0
    assert np.array_equal(out, oracle.avg_apnd_bnd(f, lr, bt, crn, ng, ny, nx))


def _map_linear_field(oracle, g, f, dN_x, dN_y, N_x, N_y):
    """FMAP (the oracle's) of the linear field f from every data point set to the simulation's, the four boundary
    sides one at a time with their own offsets, as the reconstructions call it (POD_ROUTINES.f08:335-347)."""
    for k in ("Avg", "EdgV", "EdgH"):
        G1, G2 = g["Dat_Grid_" + k], g["Sim_Grid_" + k]
        n1, n2 = G1.size // 2, G2.size // 2
        f2 = oracle.fmap(f(G1), G1, G2, g["GMap_xy" + k], g["VMap_xy" + k], n1, n2, n2)
        np.testing.assert_allclose(f2, f(G2), rtol=1e-12, atol=1e-12, err_msg=k)
    for do, so, mo, n1, n2 in ((0, 0, 0, dN_y + 2, N_y), (2 * dN_y + 4, 2 * N_y, 4 * N_y, dN_x + 2, N_x),
                               (2 * (dN_y + dN_x) + 8, 2 * (N_y + N_x), 4 * (N_y + N_x), dN_y + 2, N_y),
                               (4 * dN_y + 2 * dN_x + 12, 4 * N_y + 2 * N_x, 8 * N_y + 4 * N_x, dN_x + 2, N_x)):
        G1, G2 = g["Dat_Grid_Bnds"][do:do + 2 * n1], g["Sim_Grid_Bnds"][so:so + 2 * n2]
        f2 = oracle.fmap(f(G1), G1, G2, g["GMap_xyBnds"][mo:mo + 4 * n2], g["VMap_xyBnds"][mo:mo + 4 * n2], n1, n2,
                         n2)
        np.testing.assert_allclose(f2, f(G2), rtol=1e-12, atol=1e-12, err_msg="Bnds")


@pytest.mark.parametrize("dN,N", [(6, 9), (9, 5), (4, 4)])
def test_generate_grids_xy_matches_oracle(oracle, dN, N):
    """GENERATE_GRIDS_XY with GRIDMAP_GEN_LR/BT_BND (host code of the library, no device) against the restatement
    of the reference's calls on square grids of uneven widths, and the maps drive FMAP (the oracle's) to reproduce
    a linear field on every point set from the padded data grid."""
    rng = np.random.default_rng(dN * 10 + N)
    L = 2.0
    dxd, dyd = rng.uniform(0.5, 1.5, dN), rng.uniform(0.5, 1.5, dN)
    dxd, dyd = dxd * (L / dxd.sum()), dyd * (L / dyd.sum())
    dx, dy = rng.uniform(0.5, 1.5, N), rng.uniform(0.5, 1.5, N)
    dx, dy = dx * (L / dx.sum()), dy * (L / dy.sum())
    got = pkg.GENERATE_GRIDS_XY(dxd, dyd, dx, dy, dxd.sum(), dyd.sum(), dx.sum(), dy.sum())
    ref = oracle.generate_grids_xy(dxd, dyd, dx, dy, dxd.sum(), dyd.sum(), dx.sum(), dy.sum())
    assert set(got) == set(ref)
    for k in ref:
        assert got[k].shape == ref[k].shape and np.array_equal(got[k], ref[k]), k
    assert np.array_equal(pkg.GRIDMAP_GEN_BND(1, dx, 0.5, N), oracle.gridmap_gen_bnd(1, dx, 0.5, N))
    _map_linear_field(oracle, got, lambda g: 1.5 + 0.4 * g[0::2] - 0.9 * g[1::2], dN, dN, N, N)


def test_generate_grids_xy_rectangular_grids(oracle):
    """On grids with different x and y counts each boundary map uses its own side's counts (the reference's calls
    are defined on square grids only): every point set still maps a linear field exactly."""
    rng = np.random.default_rng(3)
    dxd, dyd, dx, dy = (rng.uniform(0.5, 1.5, n) for n in (7, 4, 5, 8))
    dyd, dx, dy = dyd * (dxd.sum() / dyd.sum()), dx * (dxd.sum() / dx.sum()), dy * (dxd.sum() / dy.sum())
    L = dxd.sum()
    got = pkg.GENERATE_GRIDS_XY(dxd, dyd, dx, dy, L, L, L, L)
    _map_linear_field(oracle, got, lambda g: -0.5 + 1.1 * g[0::2] + 0.3 * g[1::2], 7, 4, 5, 8)
    with pytest.raises(pkg.TrtError):
        pkg.GENERATE_GRIDS_XY(dxd, dyd, dx[:0], dy, L, L, L, L)


# ------------------------------------------------------------------------------------------------------------
# Reconstruction drivers POD_RECONSTRUCT_fg / _BCg, DMD_RECONSTRUCT_fg / _BCg
# ------------------------------------------------------------------------------------------------------------
def _widths(rng, n, length=1.0):
    d = rng.uniform(0.6, 1.4, n)
    return d * (length / d.sum())


def _driver_setup(oracle, dN, N, dN_g, seed):
    """Grids of trt_generate_grids_xy for a dN x dN data grid and an N x N simulation grid of uneven widths."""
    rng = np.random.default_rng(seed)
    dxd, dyd, dx, dy = _widths(rng, dN), _widths(rng, dN), _widths(rng, N), _widths(rng, N)
    if N == dN:
        dx, dy = dxd, dyd
    return pkg.GENERATE_GRIDS_XY(dxd, dyd, dx, dy, 1.0, 1.0, 1.0, 1.0)


def _pod_dec(rng, length, n_g, n_t, gsum):
    nb = n_g if gsum == 0 else 1
    glen = length // nb
    rank = rng.integers(1, min(4, n_t, glen) + 1, nb).astype(np.int32)
    tot = int(rank.sum())
    return (rng.standard_normal(length), rng.uniform(0.1, 1.0, tot), rng.standard_normal(glen * tot),
            rng.standard_normal(n_t * tot), rank)


def _dmd_dec(rng, length, n_g, gsum):
    nb = n_g if gsum == 0 else 1
    rank = rng.integers(1, 4, nb)
    L, B, W, C = dmd_model(length // nb, nb, rank, int(rng.integers(1 << 30)))
    return L, B, W, C, rank.astype(np.int32)


def _fg_lengths(dN_x, dN_y, dN_g):
    la, lv, lh = dN_x * dN_y * dN_g, (dN_x + 1) * dN_y * dN_g, dN_x * (dN_y + 1) * dN_g
    return {"avg_xx": la, "edgV_xx": lv, "avg_yy": la, "edgH_yy": lh, "edgV_xy": lv, "edgH_xy": lh}


def test_oracle_reconstruction_drivers_on_the_data_grid(oracle):
    """With the simulation grid equal to the data grid every mapped point coincides with a data point, so the
    drivers' padding and FMAP hand back the reconstructions themselves: at a data level, between two levels
    (linear time interpolation), and for the boundary factors side by side."""
    dN, dN_g, dN_t = 5, 3, 6
    g = _driver_setup(oracle, dN, dN, dN_g, 11)
    rng = np.random.default_rng(12)
    lens = _fg_lengths(dN, dN, dN_g)
    dec = {k: _pod_dec(rng, n, dN_g, dN_t, 0) for k, n in lens.items()}
    tg = oracle.generate_grids_t(2e-3, 1e-3, 0.0, 0.0, dN_t, 2 * dN_t)
    names = {"fg_avg_xx": "avg_xx", "fg_avg_yy": "avg_yy", "fg_edgV_xx": "edgV_xx", "fg_edgV_xy": "edgV_xy",
             "fg_edgH_yy": "edgH_yy", "fg_edgH_xy": "edgH_xy"}
    for t in (4, 5):                                   # level 4 sits on data level 2; level 5 between 2 and 3
        out = oracle.pod_reconstruct_fg(dec, (dN, dN, dN_g, dN_t), (dN, dN, dN_g), t, 0, g, tg)
        a, b = tg[2][2 * t - 2], tg[2][2 * t - 1]
        assert (a == b) == (t == 4)
        for o, k in names.items():
            f = oracle.pod_reconstruct(*dec[k][:4], dec[k][4], lens[k], dN_g, dN_t, a, 0)
            if a != b:
                f3 = oracle.pod_reconstruct(*dec[k][:4], dec[k][4], lens[k], dN_g, dN_t, b, 0)
                f = oracle.linear_interpolation(f, f3, tg[0][t - 1], tg[1][a - 1], tg[1][b - 1])
            assert np.array_equal(out[o], f), o
    bdec = _pod_dec(rng, dN_g * 4 * dN, dN_g, dN_t, 1)
    sides = oracle.pod_reconstruct_bcg(bdec, (dN, dN, dN_g, dN_t), (dN, dN, dN_g), 4, 1, g, tg)
    BC = oracle.pod_reconstruct(*bdec[:4], bdec[4], dN_g * 4 * dN, dN_g, dN_t, 2, 1).reshape(dN_g, 4, dN)
    for s in range(4):
        assert np.array_equal(sides[s], BC[:, s, :].reshape(-1))


@pytest.mark.gpu
@pytest.mark.parametrize("gsum,t", [(0, 4), (0, 5), (1, 7)])
def test_device_pod_reconstruct_drivers_bit_identical(oracle, gsum, t):
    """trt_pod_reconstruct_fg / _bcg against the oracle's restatement of the drivers, data grid 6 x 6 to a
    simulation grid 9 x 9 of other widths, 3 groups, bit for bit."""
    dN, N, dN_g, dN_t = 6, 9, 3, 5
    g = _driver_setup(oracle, dN, N, dN_g, 21)
    rng = np.random.default_rng(22 + t)
    dec = {k: _pod_dec(rng, n, dN_g, dN_t, gsum) for k, n in _fg_lengths(dN, dN, dN_g).items()}
    tg = oracle.generate_grids_t(2e-3, 1e-3, 0.0, 0.0, dN_t, 2 * dN_t)
    got = pkg.POD_RECONSTRUCT_fg(dec, (dN, dN, dN_g, dN_t), (N, N, dN_g, 2 * dN_t), t, gsum, g, tg)
    ref = oracle.pod_reconstruct_fg(dec, (dN, dN, dN_g, dN_t), (N, N, dN_g), t, gsum, g, tg)
    for k in ref:
        assert got[k].shape == ref[k].shape and np.array_equal(got[k], ref[k]), k
    bdec = _pod_dec(rng, dN_g * 4 * dN, dN_g, dN_t, gsum)
    got = pkg.POD_RECONSTRUCT_BCg(bdec, (dN, dN, dN_g, dN_t), (N, N, dN_g, 2 * dN_t), t, gsum, g, tg)
    ref = oracle.pod_reconstruct_bcg(bdec, (dN, dN, dN_g, dN_t), (N, N, dN_g), t, gsum, g, tg)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
    with pytest.raises(pkg.TrtError):                  # a simulation level beyond the time map
        pkg.POD_RECONSTRUCT_BCg(bdec, (dN, dN, dN_g, dN_t), (N, N, dN_g, 2 * dN_t), 2 * dN_t + 1, gsum, g, tg)


@pytest.mark.gpu
@pytest.mark.parametrize("gsum", [0, 1])
def test_device_dmd_reconstruct_drivers_bit_identical(oracle, gsum):
    """trt_dmd_reconstruct_fg / _bcg against the oracle's restatement of the drivers, bit for bit."""
    dN, N, dN_g = 5, 8, 2
    g = _driver_setup(oracle, dN, N, dN_g, 31)
    rng = np.random.default_rng(32 + gsum)
    dec = {k: _dmd_dec(rng, n, dN_g, gsum) for k, n in _fg_lengths(dN, dN, dN_g).items()}
    got = pkg.DMD_RECONSTRUCT_fg(dec, (dN, dN, dN_g), (N, N, dN_g), 0.037, gsum, g)
    ref = oracle.dmd_reconstruct_fg(dec, (dN, dN, dN_g), (N, N, dN_g), 0.037, gsum, g)
    for k in ref:
        assert got[k].shape == ref[k].shape and np.array_equal(got[k], ref[k]), k
    bdec = _dmd_dec(rng, dN_g * 4 * dN, dN_g, gsum)
    got = pkg.DMD_RECONSTRUCT_BCg(bdec, (dN, dN, dN_g), (N, N, dN_g), 0.037, gsum, g)
    ref = oracle.dmd_reconstruct_bcg(bdec, (dN, dN, dN_g), (N, N, dN_g), 0.037, gsum, g)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


@pytest.mark.gpu
def test_pod_rom_through_the_reconstruction_drivers():
    """The reference's POD-ROM run through its own drivers: per-group PODs of the recorded factors (the boundary
    factors as one vector per group, left, bottom, right, top, as the drivers read them), rebuilt at every step by
    trt_pod_reconstruct_fg / _bcg on the simulation's own grids and time levels (the maps then name the data
    points themselves), drive an ho_form = 1 run to the full run's temperatures."""
    from test_mlqd import device, setup_problem
    prob, ts, km, bcT, cv = setup_problem(8, 6, 10, "S8", 31)
    kw = dict(conv_ho=1e-9, maxit_rte=40, conv_lo=1e-10, maxit_mloqd=80)
    nt, nx, ny, ng = 3, prob.nx, prob.ny, prob.ng
    snaps, T_full = {k: [] for k in FACTORS}, []
    with device(prob, ts, km, bcT, cv, **kw) as s:
        for _ in range(nt):
            s.mlqd_step()
            m = s.moments(list(FACTORS))
            for k in FACTORS:
                snaps[k].append(m[k])
            T_full.append(s.mlqd_field("Temp"))

    def pod_of(data):                                   # data (clen, ng, nt) -> (C, S, U, V, rank), groupwise
        parts = [pkg.POD_Calc(data, nt, ng, data.shape[0], g) for g in range(ng)]
        return (np.concatenate([p[0] for p in parts]), np.concatenate([p[2] for p in parts]),
                np.concatenate([p[1].ravel(order="F") for p in parts]),
                np.concatenate([p[3].ravel(order="F") for p in parts]),
                np.array([len(p[2]) for p in parts], dtype=np.int32))

    dec = {k[3:]: pod_of(np.stack([a.reshape(-1, ng, order="F") for a in snaps[k]], axis=2)) for k in FACTORS[:6]}
    bc = np.stack([np.concatenate([snaps[k][t].reshape(-1, ng, order="F") for k in FACTORS[6:]], axis=0)
                   for t in range(nt)], axis=2)
    bdec = pod_of(bc)
    dx, dy = np.asarray(prob.delx, dtype=np.float64), np.asarray(prob.dely, dtype=np.float64)
    grids = pkg.GENERATE_GRIDS_XY(dx, dy, dx, dy, dx.sum(), dy.sum(), dx.sum(), dy.sum())
    tgrids = pkg.GENERATE_GRIDS_T(ts.dt, ts.dt, 0.0, 0.0, nt, nt)
    assert np.array_equal(tgrids[2], np.repeat(np.arange(1, nt + 1), 2))
    dims = (nx, ny, ng, nt)
    # the device-resident forms: decompositions, point sets, maps and outputs in HBM
    import torch
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    P = lambda x: ctypes.c_void_p(x.data_ptr())
    tg = [np.ascontiguousarray(a, dtype=np.float64) for a in tgrids[:2]]
    tm = np.ascontiguousarray(tgrids[2], dtype=np.int32)
    D = ctypes.POINTER(ctypes.c_double)
    I = ctypes.POINTER(ctypes.c_int)
    names = ("avg_xx", "edgV_xx", "avg_yy", "edgH_yy", "edgV_xy", "edgH_xy")
    ddec = {k: [dev(a) for a in dec[k][:4]] for k in names}
    dgr = {k: dev(v) for k, v in grids.items()}
    bd = [dev(a) for a in bdec[:4]]
    with device(prob, ts, km, bcT, cv, ho_form=1, **kw) as s:
        for t in range(1, nt + 1):
            fg = pkg.POD_RECONSTRUCT_fg(dec, dims, dims, t, 0, grids, tgrids)
            cg = dict(zip(FACTORS[6:], pkg.POD_RECONSTRUCT_BCg(bdec, dims, dims, t, 0, grids, tgrids)))
            dout = {k: torch.zeros(snaps[k][0].size, dtype=torch.float64, device="cuda") for k in FACTORS}
            rc = pkg.lib().trt_pod_reconstruct_fg_device(
                *[P(dout[k]) for k in FACTORS[:6]], *[P(a) for k in names for a in ddec[k]],
                *[dec[k][4].ctypes.data_as(I) for k in names], nx, ny, ng, nt, nx, ny, ng, nt, t, 0,
                *[P(dgr[p + k]) for p in ("Sim_Grid_", "Dat_Grid_") for k in ("Avg", "EdgV", "EdgH")],
                *[a.ctypes.data_as(D) for a in tg],
                *[P(dgr[p + k]) for p in ("GMap_xy", "VMap_xy") for k in ("Avg", "EdgV", "EdgH")], tm.ctypes.data_as(I),
                None)
            assert rc == 0
            rc = pkg.lib().trt_pod_reconstruct_bcg_device(
                *[P(dout[k]) for k in FACTORS[6:]], *[P(a) for a in bd], bdec[4].ctypes.data_as(I), nx, ny, ng, nt,
                nx, ny, ng, nt, t, 0, P(dgr["Sim_Grid_Bnds"]), P(dgr["Dat_Grid_Bnds"]), *[a.ctypes.data_as(D) for a in tg],
                P(dgr["GMap_xyBnds"]), P(dgr["VMap_xyBnds"]), tm.ctypes.data_as(I), None)
            assert rc == 0
            for k in FACTORS:
                out = fg[k] if k in fg else cg[k]
                ref = snaps[k][t - 1].ravel(order="F")
                assert out.shape == ref.shape
                assert np.abs(out - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()), k
                assert np.array_equal(dout[k].cpu().numpy(), out), k      # resident form = host form, bit for bit
                assert pkg.lib().trt_mlqd_put(s.handle, k.encode(), P(dout[k]), out.size, 1) == 0
            st = s.mlqd_step()
            assert st["sweeps"] == 0 and st["mgqd_nonconv"] == 0
            T = s.mlqd_field("Temp")
            assert float(np.max(np.abs(T - T_full[t - 1])) / np.max(T_full[t - 1])) < 1e-7
    # one bad entry in the last of the three map sets (checked together on the device, one verdict): the call is
    # refused before any FMAP reads through it, and the outputs are left untouched
    bad = dict(dgr)
    bad["VMap_xyEdgH"] = dgr["VMap_xyEdgH"].clone()
    bad["VMap_xyEdgH"][-1] = 0
    dout = {k: torch.full((snaps[k][0].size,), -7.0, dtype=torch.float64, device="cuda") for k in FACTORS[:6]}
    rc = pkg.lib().trt_pod_reconstruct_fg_device(
        *[P(dout[k]) for k in FACTORS[:6]], *[P(a) for k in names for a in ddec[k]],
        *[dec[k][4].ctypes.data_as(I) for k in names], nx, ny, ng, nt, nx, ny, ng, nt, 1, 0,
        *[P(bad[p + k]) for p in ("Sim_Grid_", "Dat_Grid_") for k in ("Avg", "EdgV", "EdgH")],
        *[a.ctypes.data_as(D) for a in tg],
        *[P(bad[p + k]) for p in ("GMap_xy", "VMap_xy") for k in ("Avg", "EdgV", "EdgH")], tm.ctypes.data_as(I), None)
    assert rc == pkg._lib.TRT_ERR_ARG
    for k in FACTORS[:6]:
        assert bool((dout[k] == -7.0).all()), k


def test_rrank_calc_matches_oracle(oracle):
    """RRANK_CALC (host code of the library) against the restatement: decaying spectra over error levels, the
    edge levels (0 keeps every mode, 1 keeps one) and trailing zeros; POD_TRUNCATE packs the truncated groups."""
    rng = np.random.default_rng(41)
    for n in (1, 2, 7, 20):
        sig = np.sort(rng.uniform(0.0, 1.0, n) ** 3)[::-1]
        for eps in (0.0, 1e-12, 1e-3, 0.05, 0.3, 1.0):
            assert pkg.RRANK_CALC(sig, eps) == oracle.rrank_calc(list(sig), eps), (n, eps)
        assert pkg.RRANK_CALC(sig, 1.0) == 1
    assert pkg.RRANK_CALC(np.array([3.0, 2.0, 0.0, 0.0]), 0.0) == 2
    assert pkg.RRANK_CALC(np.array([1.0, 1e-9, 1e-12]), 0.0) == 3
    with pytest.raises(pkg.TrtError):
        pkg.RRANK_CALC(np.zeros(0), 0.1)
    clen, nt = 9, 5
    parts = []
    for _ in range(3):
        u, sig, vt = rng.standard_normal((clen, nt)), np.array([4.0, 1.0, 0.1, 0.01, 0.001]), rng.standard_normal((nt, nt))
        parts.append((rng.standard_normal(clen), u, sig, vt))
    C, S, U, V, rank = pkg.POD_TRUNCATE(parts, 0.02)
    r = oracle.rrank_calc([4.0, 1.0, 0.1, 0.01, 0.001], 0.02)
    assert list(rank) == [r] * 3 and S.size == 3 * r and U.size == 3 * clen * r and V.size == 3 * nt * r
    # the packed arrays reconstruct what the truncated factors give, group by group (POD_RECONSTRUCT's layout)
    for t in (1, nt):
        dat = oracle.pod_reconstruct(C, S, U, V, rank, 3 * clen, 3, nt, t, 0)
        for g, (c, u, sig, vt) in enumerate(parts):
            ref = c + (u[:, :r] * sig[:r]) @ vt[:r, t - 1]
            np.testing.assert_allclose(dat[g * clen:(g + 1) * clen], ref, rtol=1e-13, atol=1e-13)
