"""fmm_direct_noalloc -- direct sums with fixed device scratch, no allocation --
against fmm_direct, through the C ABI, on calls in a row.  Collected last so it
also runs after every other test in the same process."""
import ctypes as C

import numpy as np
import pytest

import simplefmm_b200 as sf
from simplefmm_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-12          # relative, as the parity tests


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _noalloc(torch, pos_d, q_d, qdim, tg, want_field):
    L = sf.load_library()
    nt = tg.size
    t_d = _dev(torch, tg.astype(np.int64))
    pot = torch.full((nt, qdim), float("nan"), dtype=torch.float64, device="cuda")
    fld = torch.full((nt, 3), float("nan"), dtype=torch.float64, device="cuda") if want_field else None
    st = torch.cuda.current_stream()
    rc = L.fmm_direct_noalloc(C.c_void_p(pos_d.data_ptr()), pos_d.shape[0], C.c_void_p(q_d.data_ptr()), qdim,
                              C.c_void_p(t_d.data_ptr()), nt, C.c_void_p(pot.data_ptr()),
                              C.c_void_p(fld.data_ptr()) if want_field else None, C.c_void_p(st.cuda_stream))
    assert rc == 0, L.fmm_last_error().decode()
    torch.cuda.synchronize()
    return pot.cpu().numpy(), (fld.cpu().numpy() if want_field else None)


def _close(got, ref):
    scale = np.abs(ref).max()
    np.testing.assert_allclose(got, ref, rtol=TOL, atol=TOL * scale)


def test_noalloc_matches_fmm_direct_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    n = 200_000
    pos = W.points("plummer", n, 11)
    q1 = W.charges(n, 11)
    q3 = np.random.default_rng(12).uniform(-1, 1, (n, 3))
    pos_d, q1_d, q3_d = _dev(torch, pos), _dev(torch, q1), _dev(torch, q3)
    rng = np.random.default_rng(13)
    tg_a = rng.choice(n, 5000, replace=False)
    tg_b = rng.choice(n, 20000, replace=False)
    # scalar charges, potential + field; then vector charges (Biot-Savart); then the first again
    ref_a = sf.direct(pos, q1, tg_a)
    ref_b = sf.direct(pos, q3, tg_b)
    for (q_d, qdim, tg, ref) in [(q1_d, 1, tg_a, ref_a), (q3_d, 3, tg_b, ref_b), (q1_d, 1, tg_a, ref_a)]:
        pot, fld = _noalloc(torch, pos_d, q_d, qdim, tg, True)
        _close(pot.reshape(ref[0].shape), ref[0])
        _close(fld, ref[1])


def test_noalloc_rejects_sizes_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    L = sf.load_library()
    n, nt = 1000, 174_763
    pos_d = _dev(torch, W.points("uniform", n, 3))
    q_d = _dev(torch, W.charges(n, 3))
    t_d = torch.zeros(nt, dtype=torch.int64, device="cuda")
    pot = torch.zeros(nt, dtype=torch.float64, device="cuda")
    before = sf.launch_count()
    rc = L.fmm_direct_noalloc(C.c_void_p(pos_d.data_ptr()), n, C.c_void_p(q_d.data_ptr()), 1,
                              C.c_void_p(t_d.data_ptr()), nt, C.c_void_p(pot.data_ptr()), None, None)
    assert rc == 6            # FMM_ERR_OVER_BUDGET
    assert "174762" in L.fmm_last_error().decode()
    assert sf.launch_count() == before
