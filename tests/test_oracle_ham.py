"""Pins the oracle's Hamiltonians, exact diagonalisation and exact-summation SR.

* Tests/TestHamTFI.cpp:7-20 with the mock state of Tests/HamiltonianHelper.hpp:
  the state form's requested flips equal the column form, for every column.
  Extended to XXZ and the 2D TFI model (no reference tests exist for those).
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


@pytest.mark.parametrize("case", ["xxz12", "tfi2d_3x4", "xxz10_sign_full"])
def test_ed_matches_scipy(orc, case):
    if case == "xxz12":
        ham, bk, nup = orc.Ham.xxz(12, 1.0, 1.0, True), 1, 6
    elif case == "tfi2d_3x4":
        ham, bk, nup = orc.Ham.tfi2d(3, 4, -1.0, -3.0), 0, 0
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
