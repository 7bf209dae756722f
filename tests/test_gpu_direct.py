"""The device direct sums (fmm_direct, the reference's accuracy check of
main.cpp:70-111) against the oracle's CPU direct sums, and their handling of
target indices outside [0, n).  Every call goes through the C ABI."""
import ctypes as C

import numpy as np
import pytest

import simplefmm_b200 as sf
from conftest import rel_err_per_target
from oracle import pyoracle
from simplefmm_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def ctx():
    return sf.Context(0)


@pytest.mark.parametrize("dist", ["plummer", "uniform"])
def test_direct_matches_oracle_scalar(ctx, dist):
    n = 30_000
    pos, q = W.points(dist, n, 5), W.charges(n, 5)
    tg = np.random.default_rng(6).choice(n, 3000, replace=False)
    pot, fld = sf.direct(pos, q, tg, ctx=ctx)
    opot = pyoracle.direct(pos, q, tg, "potential")
    ofld = pyoracle.direct(pos, q, tg, "field")
    sp, sfl = pyoracle.error_scales(pos, q, tg)
    assert rel_err_per_target(pot, opot, sp) < TOL
    assert rel_err_per_target(fld, ofld, sfl) < TOL
    # the plain relative error per target, where the sum does not cancel
    big = np.abs(opot) > 1e-3 * np.sqrt(np.mean(opot ** 2))
    assert np.max(np.abs(pot[big] - opot[big]) / np.abs(opot[big])) < 1e-10


def test_direct_matches_oracle_vector(ctx):
    n = 20_000
    pos = W.points("plummer", n, 8)
    q3 = np.random.default_rng(9).uniform(-1, 1, (n, 3))
    tg = np.random.default_rng(10).choice(n, 2000, replace=False)
    pot, bio = sf.direct(pos, q3, tg, ctx=ctx)
    opot = pyoracle.direct(pos, q3, tg, "potential")
    obio = pyoracle.direct(pos, q3, tg, "biot")
    sp, sfl = pyoracle.error_scales(pos, np.abs(q3).sum(axis=1), tg)
    for b in range(3):
        assert rel_err_per_target(pot[:, b], opot[:, b], sp) < TOL
    assert rel_err_per_target(bio, obio, sfl) < TOL


def test_direct_rejects_out_of_range_targets(ctx):
    torch = pytest.importorskip("torch")
    L = sf.load_library()
    n = 5000
    pos, q = W.points("uniform", n, 3), W.charges(n, 3)
    # host targets: refused before any copy
    for bad in (n, -1):
        tg = np.array([0, 1, bad, 3], dtype=np.int64)
        pot = np.zeros(4)
        rc = L.fmm_direct(ctx._h, C.c_void_p(pos.ctypes.data), n, C.c_void_p(q.ctypes.data), 1,
                          C.c_void_p(tg.ctypes.data), 4, C.c_void_p(pot.ctypes.data), None, sf.HOST)
        assert rc == 1 and "out of range" in L.fmm_last_error().decode()
    # device targets: skipped and flagged on the device
    pos_d = torch.from_numpy(pos).cuda()
    q_d = torch.from_numpy(q).cuda()
    tg_d = torch.tensor([0, 1, n + 7, 3], dtype=torch.int64, device="cuda")
    pot_d = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = L.fmm_direct(ctx._h, C.c_void_p(pos_d.data_ptr()), n, C.c_void_p(q_d.data_ptr()), 1,
                      C.c_void_p(tg_d.data_ptr()), 4, C.c_void_p(pot_d.data_ptr()), None, sf.DEVICE)
    assert rc == 1 and "out of range" in L.fmm_last_error().decode()
    got = pot_d.cpu().numpy()
    assert np.isnan(got[2]) and np.all(np.isfinite(got[[0, 1, 3]]))
    ref, _ = sf.direct(pos, q, np.array([0, 1, 3]), field=False, ctx=ctx)
    np.testing.assert_allclose(got[[0, 1, 3]], ref, rtol=1e-14)
