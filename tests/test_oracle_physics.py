"""Oracle backflow, projection, Hubbard and sampler checks (CPU)."""

import json
import os

import numpy as np
import pytest

from oracle import backflow, hubbard, lattice, pfaffian, projection, sampler

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def params(L, channels=16, std=0.3, seed=0):
    rng = np.random.default_rng(seed)
    conv_w, conv_b = [], []
    cin = 2
    for _ in range(4):
        conv_w.append(rng.normal(0, std, (channels, cin, 3, 3)))
        conv_b.append(rng.normal(0, std, channels))
        cin = channels
    d = channels // 2
    W = rng.normal(0, 1, (3, L * L, d)) / np.sqrt(d)
    return dict(conv_w=conv_w, conv_b=conv_b, W=W, theta=0.55, Lx=L, Ly=L)


def test_displacement_tables():
    disp, neg, dist = lattice.displacement_tables(4, 6)
    N = 24
    assert disp.shape == (N, N) and np.all(disp[np.arange(N), np.arange(N)] == 0)
    assert np.all(neg[neg] == np.arange(N))
    assert np.allclose(dist[neg], dist)
    # disp[i, j] + disp[j, i] = 0 as displacements
    assert np.all(neg[disp] == disp.T)


def test_wtilde_exact_antisymmetry():
    p = params(6, channels=16)
    for dt in (np.float32, np.float64):
        W = p["W"].astype(dt)
        Wt = backflow.build_wtilde(W, 0.55, 6, 6, dt)
        _, neg, _ = lattice.displacement_tables(6, 6)
        # Wt[2 sq + sp, -r] == -Wt[2 sp + sq, r] bit for bit
        for sp in range(2):
            for sq in range(2):
                assert np.array_equal(Wt[2 * sq + sp][neg], -Wt[2 * sp + sq])


def test_conv_matches_direct_loop():
    rng = np.random.default_rng(1)
    x = rng.normal(size=(2, 3, 5, 4))
    w = rng.normal(size=(2, 3, 3, 3))
    b = rng.normal(size=2)
    out = backflow.conv3x3_periodic(x, w, b)
    ref = np.zeros_like(out)
    for bb in range(2):
        for o in range(2):
            for X in range(5):
                for Y in range(4):
                    acc = b[o]
                    for i in range(3):
                        for u in range(3):
                            for v in range(3):
                                acc += w[o, i, u, v] * x[bb, i, (X + u - 1) % 5, (Y + v - 1) % 4]
                    ref[bb, o, X, Y] = acc
    assert np.allclose(out, ref, atol=1e-12)


@pytest.mark.parametrize("L", [4, 8])
def test_gather_kernel_formula_equals_einsum_twin(L):
    """pf_kernel.py's gather and models.py's einsum path give the same occupied block."""
    p = params(L)
    N = L * L
    s = lattice.random_configs(np.random.default_rng(L), 3, N, 7 * N // 16, 7 * N // 16)
    y = backflow.cnn_forward(s, p["conv_w"], p["conv_b"], L, L)
    idx = backflow.fermion_idx(s)
    Wt = backflow.build_wtilde(p["W"], p["theta"], L, L)
    F = backflow.pairing_occ(backflow.occupied_features(y, idx), idx, Wt, L, L)
    for b in range(3):
        full = backflow.pairing_matrix_einsum(y[b], p["W"], p["theta"], L, L)
        Fe = full[np.ix_(idx[b], idx[b])]
        assert np.allclose(F[b], Fe, atol=1e-12 * np.abs(Fe).max())
        assert np.allclose(F[b], -F[b].T, atol=0)


def test_golden_oracle_amplitudes():
    g = np.load(os.path.join(GOLDEN, "oracle_amplitude_L4.npz"))
    rng = np.random.default_rng(7)
    conv_w, conv_b = [], []
    cin = 2
    for _ in range(4):
        conv_w.append(rng.normal(0, 0.3, (16, cin, 3, 3)))
        conv_b.append(rng.normal(0, 0.3, 16))
        cin = 16
    W = rng.normal(0, 1, (3, 16, 8)) / np.sqrt(8)
    p = dict(conv_w=conv_w, conv_b=conv_b, W=W, theta=0.55, Lx=4, Ly=4)
    sg, la = backflow.amplitude(g["spins"], p)
    assert np.array_equal(sg, g["sign"]) and np.allclose(la, g["logabs"], atol=1e-10)
    sgp, lap = projection.projected_amplitude(g["spins"], p)
    assert np.array_equal(sgp, g["sign_p"]) and np.allclose(lap, g["logabs_p"], atol=1e-10)


def _fock_apply_perm(s, perm):
    """U_g |s> by explicit creation operators: returns (sign, image configuration)."""
    occ = [int(m) for m in np.flatnonzero(s > 0)]
    bits, sign = 0, 1
    for m in reversed(occ):  # c+_{m1} ... c+_{mk}|0>: apply c+_{g(mk)} first
        gm = int(perm[m])
        if bin(bits & ((1 << gm) - 1)).count("1") % 2:
            sign = -sign
        bits |= 1 << gm
    img = -np.ones_like(s)
    for m in range(len(s)):
        if (bits >> m) & 1:
            img[m] = 1
    return sign, img


def test_image_signs_from_operators():
    L = 4
    maps = lattice.symmetry_mode_maps(L, L)
    for g in range(8):
        assert np.all(maps[g][maps[g]] == np.arange(2 * L * L))  # involutions
    s = lattice.random_configs(np.random.default_rng(3), 5, 16, 5, 4)
    eta = projection.image_signs(s, maps)
    imgs = projection.image_configs(s, maps)
    for b in range(5):
        for g in range(8):
            sg, img = _fock_apply_perm(s[b], maps[g])
            assert sg == eta[b, g]
            assert np.array_equal(img, imgs[b, g])


def test_projection_invariance():
    """The projected state is invariant: eta_g(s) psi_P(g s) = psi_P(s)."""
    L = 4
    p = params(L, channels=16, std=0.3)
    maps = lattice.symmetry_mode_maps(L, L)
    s = lattice.random_configs(np.random.default_rng(4), 3, 16, 7, 7)
    sg, la = projection.projected_amplitude(s, p)
    eta = projection.image_signs(s, maps)
    imgs = projection.image_configs(s, maps)
    for g in range(1, 8):
        sg2, la2 = projection.projected_amplitude(imgs[:, g], p)
        assert np.array_equal(sg2 * eta[:, g], sg)
        assert np.allclose(la2, la, atol=1e-9)


def test_hops_match_fock_golden():
    g = np.load(os.path.join(GOLDEN, "hubbard_4x4.npz"))
    off = 0
    for s, cnt in zip(g["spins"], g["counts"]):
        conn, vals = g["conn"][off : off + cnt], g["vals"][off : off + cnt]
        off += cnt
        want = {}
        for c, v in zip(conn, vals):
            if not np.array_equal(c, s):
                want[c.tobytes()] = v
        fr, to, hv = hubbard.hops(s, 4, 4, 1.0, -0.2)
        got = {}
        for f, t_, h in zip(fr, to, hv):
            got[hubbard.apply_hop(s, f, t_).tobytes()] = h
        assert got.keys() == want.keys()
        for k in got:
            assert got[k] == want[k]
        diag = [v for c, v in zip(conn, vals) if np.array_equal(c, s)]
        docc = hubbard.double_occupancy(s, 16)
        assert (diag[0] if diag else 0.0) == 8.0 * docc


def test_local_energy_bruteforce_and_hermiticity():
    L = 4
    basis = hubbard.fock_basis(16, 3, 1)  # 4 electrons: non-trivial Jordan-Wigner signs
    H = hubbard.hamiltonian_matrix(basis, L, L, 1.0, -0.2, 8.0)
    assert np.array_equal(H, H.T)
    p = params(L, channels=16, std=0.3, seed=2)

    def amp(c):
        return projection.projected_amplitude(c, p, symm=False)

    sg, la = amp(basis)
    psi = sg * np.exp(la - la.max())
    pick = np.random.default_rng(0).choice(len(basis), 12, replace=False)
    e = hubbard.local_energy(basis[pick], amp, L, L, 1.0, -0.2, 8.0)
    ref = (H[pick] @ psi) / psi[pick]
    assert np.allclose(e, ref, rtol=1e-9, atol=1e-9)
    cnt = hubbard.hop_counts(basis[pick], L, L)
    for b, a in enumerate(pick):
        assert cnt[b] == len(hubbard.hops(basis[a], L, L, 1.0, -0.2)[0])


def test_philox_golden():
    with open(os.path.join(GOLDEN, "philox_kat.json")) as f:
        kat = json.load(f)
    for k in kat:
        out = sampler.philox4x32([np.array([c]) for c in k["counter"]], k["key"])
        assert [int(o[0]) for o in out] == k["out"]


def test_detailed_balance_exact():
    """The plain proposal is symmetric, so P(s->s') pi(s) = P(s'->s) pi(s')."""
    L = 4
    basis = hubbard.fock_basis(16, 1, 1)
    key = {b.tobytes(): i for i, b in enumerate(basis)}
    p = params(L, channels=16, std=0.3, seed=3)
    sg, la = projection.projected_amplitude(basis, p, symm=False)
    pi = np.exp(2 * (la - la.max()))
    nbr = lattice.neighbour_table(L, L)
    D = len(basis)
    P = np.zeros((D, D))
    for a, s in enumerate(basis):
        occ = np.flatnonzero(s > 0)
        for m in occ:
            sigma, i = divmod(int(m), 16)
            for d in range(8):
                mj = sigma * 16 + int(nbr[i, d])
                if s[mj] > 0:
                    continue
                b = key[hubbard.apply_hop(s, m, mj).tobytes()]
                P[a, b] += (1 / len(occ)) * (1 / 8) * min(1.0, pi[b] / pi[a])
    flux = pi[:, None] * P
    assert np.allclose(flux, flux.T, atol=1e-15)


def test_tau_int_and_jackknife():
    rng = np.random.default_rng(0)
    T = 20000
    x = np.zeros(T)
    a = 0.8
    for t in range(1, T):
        x[t] = a * x[t - 1] + rng.normal()
    tau = sampler.tau_int(x)
    assert tau == pytest.approx((1 + a) / (2 * (1 - a)), rel=0.25)
    m, e = sampler.jackknife_mean(rng.normal(size=4096))
    assert abs(m) < 5 * e and e == pytest.approx(1 / 64, rel=0.3)
