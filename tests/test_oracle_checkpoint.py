"""Pins the oracle's restatement of the reference's checkpoint format (the cereal
binary image of std::unique_ptr<RBM<T>> that Runners/RunRBM.hpp:155-164 writes and
Runners/AbstractRunner.hpp:83-94 reads; Serializers/SerializeRBM.hpp:20-82,
Serializers/SerializeEigen.hpp:8-35).  cereal is not vendored and the reference's
own serialisation test (Tests/TestSerializeRBM.cpp) only round-trips in memory,
so the byte layout is spelled out here field by field; the committed fixtures
under tests/golden/ are regenerated by tests/golden/make_rbm_archives.py."""
import os
import struct
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_rbm_archives as mk  # noqa: E402


def test_layout_field_by_field(orc):
    n, m = 3, 2
    p = mk.params(n, m, True, False)
    data = orc.rbm_archive(n, m, p, True, 1)
    # unique_ptr valid byte, class version, useBias, N, M
    assert data[:14] == bytes([1, 1, 0, 0, 0, 1, 3, 0, 0, 0, 2, 0, 0, 0])
    # W: rows = M, cols = N, then W(0,0), W(1,0), W(0,1), ... as (re, im) doubles
    assert struct.unpack_from("<ii", data, 14) == (2, 3)
    w = struct.unpack_from("<12d", data, 22)
    assert w[:4] == (0.125, -0.0, 0.25, -0.0625)
    # a: rows N, cols 1; b: rows M, cols 1
    at = 22 + 96
    assert struct.unpack_from("<ii", data, at) == (3, 1)
    assert struct.unpack_from("<2d", data, at + 8) == (p[6].real, p[6].imag)
    at += 8 + 48
    assert struct.unpack_from("<ii", data, at) == (2, 1)
    assert len(data) == at + 8 + 32


def test_without_bias_stops_after_w(orc):
    data = orc.rbm_archive(2, 4, mk.params(2, 4, False, False), False, 1)
    assert data[5] == 0
    assert len(data) == 14 + 8 + 8 * 16


@pytest.mark.parametrize("elem,esize", [(0, 8), (1, 16), (2, 8), (3, 4)])
def test_round_trip_and_sizes(orc, elem, esize):
    n, m = 5, 7
    p = mk.params(n, m, True, elem >= 2)
    data = orc.rbm_archive(n, m, p, True, elem)
    assert len(data) == 14 + 8 + n * m * esize + 8 + n * esize + 8 + m * esize
    n2, m2, b2, p2 = orc.rbm_unarchive(data, elem)
    assert (n2, m2, b2) == (n, m, True)
    np.testing.assert_array_equal(p2, p)


def test_golden_fixtures_are_current(orc):
    for name, n, m, bias, elem in mk.CASES:
        with open(os.path.join(HERE, "golden", name), "rb") as f:
            data = f.read()
        assert data == orc.rbm_archive(n, m, mk.params(n, m, bias, elem >= 2), bias, elem), name
