"""RBM checkpoints through the C ABI against the oracle's restatement of the
reference's cereal format (bit-exact bytes) and the committed fixtures; loading
restores the FP64 master parameters; RunRBM-style w%04d.dat files from the C++
adapter parse as the reference's archives."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_rbm_archives as mk  # noqa: E402


@pytest.fixture(scope="module")
def ctx():
    from yannq_b200 import api

    c = api.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("name,n,m,bias,elem", mk.CASES, ids=[c[0] for c in mk.CASES])
def test_device_archive_equals_fixture(ctx, orc, name, n, m, bias, elem):
    from yannq_b200 import api

    with open(os.path.join(HERE, "golden", name), "rb") as f:
        want = f.read()
    q = api.RBM(ctx, n, m, bias, api.C64 if elem == 0 else api.C128)
    p = mk.params(n, m, bias, elem >= 2)
    q.set_params(p)
    assert q.archive(elem) == want
    assert api.archive_shape(want) == (n, m, bias)
    q2 = api.RBM(ctx, n, m, bias, api.C64 if elem == 0 else api.C128)
    q2.load_archive(want, elem)
    np.testing.assert_array_equal(q2.get_params(), p)
    q.close()
    q2.close()


@pytest.mark.parametrize("dtype", [1, 0])
def test_random_machine_round_trip(ctx, orc, tmp_path, dtype):
    from yannq_b200 import api

    n, m = 144, 288
    q = api.RBM(ctx, n, m, True, dtype)
    q.init_random(20261203, 0.01)
    p = q.get_params()
    data = q.archive()
    elem = api.ARCHIVE_C128 if dtype == api.C128 else api.ARCHIVE_C64
    assert data == orc.rbm_archive(n, m, p if dtype == api.C128 else p.astype(np.complex64), True, elem)
    path = tmp_path / "w0000.dat"
    q.save(str(path))
    assert path.read_bytes() == data
    assert api.file_shape(str(path)) == (n, m, True)
    q2 = api.RBM(ctx, n, m, True, dtype)
    q2.load(str(path))
    got = q2.get_params()
    if dtype == api.C128:
        np.testing.assert_array_equal(got, p)
    else:  # std::complex<float> on disk
        np.testing.assert_array_equal(got, p.astype(np.complex64).astype(np.complex128))
    # a complex<double> archive of the complex64 machine keeps the FP64 masters
    if dtype == api.C64:
        q3 = api.RBM(ctx, n, m, True, dtype)
        q3.load_archive(q.archive(api.ARCHIVE_C128), api.ARCHIVE_C128)
        np.testing.assert_array_equal(q3.get_params(), p)
        q3.close()
    q.close()
    q2.close()


def test_archive_errors(ctx, orc, tmp_path):
    from yannq_b200 import api

    q = api.RBM(ctx, 4, 6, True, api.C128)
    q.init_random(1, 0.1)
    data = q.archive()
    other = api.RBM(ctx, 4, 8, True, api.C128)
    with pytest.raises(api.YQError):
        other.load_archive(data)  # shape differs
    with pytest.raises(api.YQError):
        q.load_archive(data[:-3])  # truncated
    with pytest.raises(api.YQError):
        q.archive(api.ARCHIVE_F64)  # complex parameters into a real archive
    with pytest.raises(api.YQError):
        q.load(str(tmp_path / "missing.dat"))
    nob = api.RBM(ctx, 4, 6, False, api.C128)
    with pytest.raises(api.YQError):
        nob.load_archive(data)  # useBias differs
    for x in (q, other, nob):
        x.close()
