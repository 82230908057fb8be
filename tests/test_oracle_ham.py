"""Pins the oracle's Hamiltonians, exact diagonalisation and exact-summation SR.

* Tests/TestHamTFI.cpp:7-20 with the mock state of Tests/HamiltonianHelper.hpp:
  the state form's requested flips equal the column form, for every column.
  Extended to XXZ and the 2D TFI model (no reference tests exist for those).
* Tests/TestHamJ1J2.cpp:7-55 (J1J2 N = 12, J2 in {-1, 0, 1, 2}, both sign rules;
  stoquasticity with the sign rule) and Tests/TestHamKitaev.cpp:7-45 (KitaevHex
  4 x 4: isotropic, anisotropic 0.2/0.4/0.6, field 0.2), plus XXX and XYZNNN.
* Lanczos ED against the closed form of the periodic TFI chain and scipy.
"""
import math

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def _column_from_state(orc, ham, col):
    n = ham.n
    s = np.array([1 - 2 * ((col >> i) & 1) for i in range(n)], np.int8)
    diag, masks, coeffs = orc.ham_enumerate(ham, s)
    out = {}
    out[col] = out.get(col, 0.0) + diag
    for mk, c in zip(masks, coeffs):
        r = col ^ int(mk)
        out[r] = out.get(r, 0.0) + c
    return out


HAMS = [
    ("tfi12", lambda o: o.Ham.tfi(12, 1.0, 0.2)),
    ("tfi12_ref_example", lambda o: o.Ham.tfi(12, -1.0, -1.0)),
    ("xxz10", lambda o: o.Ham.xxz(10, 1.0, 1.0)),
    ("xxz10_sign", lambda o: o.Ham.xxz(10, 1.0, 0.7, True)),
    ("tfi2d_3x4", lambda o: o.Ham.tfi2d(3, 4, -1.0, -3.0)),
    ("xxx12", lambda o: o.Ham.xxx(12)),
    ("xyznnn10", lambda o: o.Ham.xyznnn(10, 0.3, 0.7)),
] + [
    (f"j1j2_12_J2{d:+g}_{'sign' if sg else 'nosign'}", (lambda d, sg: lambda o: o.Ham.j1j2(12, 1.0, d, sg))(d, sg))
    for d in (-1.0, 0.0, 1.0, 2.0) for sg in (True, False)
]

# KitaevHex(4, 4, ...) has 2^16 columns; the reference walks all of them, here a
# fixed stride covers every bit pattern of the low sites and a spread of the rest.
KITAEV = [
    ("kitaev4x4_iso", lambda o: o.Ham.kitaev_hex(4, 4, 1.0, 1.0, 1.0)),
    ("kitaev4x4_aniso", lambda o: o.Ham.kitaev_hex(4, 4, 0.2, 0.4, 0.6)),
    ("kitaev4x4_field", lambda o: o.Ham.kitaev_hex(4, 4, 1.0, 1.0, 1.0, 0.2)),
]


@pytest.mark.parametrize("name,mk", HAMS, ids=[h[0] for h in HAMS])
def test_state_form_equals_column_form(orc, name, mk):
    ham = mk(orc)
    for col in range(1 << ham.n):
        want = dict(zip(*[list(map(int, orc.ham_column(ham, col)[0])), orc.ham_column(ham, col)[1]]))
        got = _column_from_state(orc, ham, col)
        # the reference's std::map keeps explicit zeros; compare non-zero content exactly
        want = {k: v for k, v in want.items() if v != 0.0}
        got = {k: v for k, v in got.items() if v != 0.0}
        assert got == want, col


@pytest.mark.parametrize("name,mk", KITAEV, ids=[h[0] for h in KITAEV])
def test_kitaev_state_form_equals_column_form(orc, name, mk):
    ham = mk(orc)
    for col in list(range(0, 1 << 16, 11)) + [0xFFFF, 0xAAAA, 0x5555]:
        r, v = orc.ham_column(ham, col)
        want = {int(k): x for k, x in zip(r, v) if x != 0.0}
        got = {k: x for k, x in _column_from_state(orc, ham, col).items() if x != 0.0}
        assert got == want, col


def test_kitaev_links_cover_each_site_once_per_axis(orc):
    # every site of the honeycomb has exactly one x, one y and one z neighbour
    ham = orc.Ham.kitaev_hex(4, 4, 1.0, 1.0, 1.0)
    for axis_mask in range(3):
        hx = orc.Ham.kitaev_hex(4, 4, *[1.0 if a == axis_mask else 0.0 for a in range(3)])
        diag, masks, coeffs = orc.ham_enumerate(hx, np.ones(16, np.int8))
        masks = [int(m) for m, c in zip(masks, coeffs) if c != 0.0]
        if axis_mask == 2:  # z-links are diagonal: 8 bonds, all satisfied at s = +1
            assert masks == [] and diag == 8.0
            continue
        assert len(masks) == 8 and all(bin(m).count("1") == 2 for m in masks)
        cover = 0
        for m in masks:
            assert cover & m == 0
            cover |= m
        assert cover == 0xFFFF
    assert ham.n == 16


def test_j1j2_stoquastic_with_sign_rule(orc):
    # Tests/TestHamJ1J2.cpp:39-55: J1J2(12, 1, 0, signRule) has no positive off-diagonal entry
    ham = orc.Ham.j1j2(12, 1.0, 0.0, True)
    s = 0.0
    for col in range(1 << 12):
        r, v = orc.ham_column(ham, col)
        s += sum(x for k, x in zip(r, v) if int(k) != col and x > 0)
    assert s < 1e-6


def test_j1j2_at_j2_zero_is_the_xxz_chain(orc):
    # J1J2(n, J1, 0, sign) and XXZ(n, J1, Delta = 1, sign) are the same operator
    for sg in (True, False):
        a = orc.ed_ground(orc.Ham.j1j2(12, 1.0, 0.0, sg), 1, 6)
        b = orc.ed_ground(orc.Ham.xxz(12, 1.0, 1.0, sg), 1, 6)
        assert a == pytest.approx(b, rel=1e-10)


def _dense_h(orc, ham, basis):
    idx = {int(b): i for i, b in enumerate(basis)}
    rows, cols, vals = [], [], []
    for j, b in enumerate(basis):
        r, v = orc.ham_column(ham, int(b))
        for rr, vv in zip(r, v):
            if int(rr) in idx:
                rows.append(idx[int(rr)])
                cols.append(j)
                vals.append(vv)
    return sp.csr_matrix((vals, (rows, cols)), shape=(len(basis), len(basis)))


def test_ed_tfi_closed_form(orc):
    # H = -sum ZZ - h sum X on a ring: E0 = -sum_k sqrt(1 + h^2 - 2 h cos k), k = (2j-1) pi / N
    for n, h in [(8, 0.5), (12, 1.0), (16, 1.0), (10, 1.7)]:
        ks = [(2 * j - 1) * math.pi / n for j in range(1, n + 1)]
        e0 = -sum(math.sqrt(1 + h * h - 2 * h * math.cos(k)) for k in ks)
        got = orc.ed_ground(orc.Ham.tfi(n, -1.0, -h))
        assert got == pytest.approx(e0, rel=1e-10)


@pytest.mark.parametrize("case", ["xxz12", "tfi2d_3x4", "xxz10_sign_full", "j1j2_12", "xyznnn10",
                                  "kitaev4x2_field", "kitaev4x4_aniso"])
def test_ed_matches_scipy(orc, case):
    if case == "xxz12":
        ham, bk, nup = orc.Ham.xxz(12, 1.0, 1.0, True), 1, 6
    elif case == "tfi2d_3x4":
        ham, bk, nup = orc.Ham.tfi2d(3, 4, -1.0, -3.0), 0, 0
    elif case == "j1j2_12":
        ham, bk, nup = orc.Ham.j1j2(12, 1.0, 0.5, True), 1, 6
    elif case == "xyznnn10":
        ham, bk, nup = orc.Ham.xyznnn(10, 0.3, 0.7), 0, 0
    elif case == "kitaev4x2_field":
        ham, bk, nup = orc.Ham.kitaev_hex(4, 2, 1.0, 1.0, 1.0, 0.2), 0, 0
    elif case == "kitaev4x4_aniso":
        ham, bk, nup = orc.Ham.kitaev_hex(4, 4, 0.2, 0.4, 0.6), 0, 0
    else:
        ham, bk, nup = orc.Ham.xxz(10, 1.0, 0.5), 0, 0
    basis = orc.basis(ham.n, bk, nup)
    H = _dense_h(orc, ham, basis)
    assert abs(H - H.T).max() < 1e-14
    want = spla.eigsh(H, k=1, which="SA")[0][0]
    assert orc.ed_ground(ham, bk, nup) == pytest.approx(want, rel=1e-9, abs=1e-9)


def test_basis_jz_order_and_size(orc):
    b = orc.basis(10, 1, 4)
    assert len(b) == math.comb(10, 4)
    assert np.all(np.diff(b.astype(np.int64)) > 0)
    assert all(bin(int(x)).count("1") == 4 for x in b)


def test_exact_sr_against_dense_numpy(orc):
    # GroundState/SRMatExact.hpp:97-132 restated vs a direct numpy evaluation
    n, m = 8, 8
    ham = orc.Ham.tfi(n, -1.0, -0.8)
    p = orc.init_params(n, m, 4, 0.3)
    res = orc.exact(ham, m, p)
    basis = orc.basis(n)
    psi = np.array([orc.psi(n, m, p, orc.sigma_of(b, n)) for b in basis])
    psi /= np.linalg.norm(psi)
    H = _dense_h(orc, ham, basis).toarray()
    E = np.vdot(psi, H @ psi).real
    assert res["energy"] == pytest.approx(E, rel=1e-12)
    O = np.array([orc.logderiv(n, m, p, s, orc.theta(n, m, p, s)) for s in
                  [orc.sigma_of(b, n) for b in basis]])
    w = np.abs(psi) ** 2
    ol = w @ O
    S = O.conj().T @ (w[:, None] * O) - np.outer(ol.conj(), ol)
    F = (psi[:, None] * O).conj().T @ (H @ psi) - np.vdot(psi, H @ psi) * ol.conj()
    assert np.allclose(res["oloc"], ol, rtol=1e-11, atol=1e-13)
    assert np.allclose(res["S"], S, rtol=1e-10, atol=1e-13)
    assert np.allclose(res["grad"], F, rtol=1e-10, atol=1e-13)
    # variational principle
    assert res["energy"] >= orc.ed_ground(ham) - 1e-10
