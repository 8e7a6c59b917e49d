"""The allocation-free dot product (sevp_inprod_noalloc) against the existing
p_inprod_ entry point and the CPU oracle's p_inprod.

It exists for callers that cannot let the library allocate GPU memory (a
model whose pool owns the device, or one that overlaps solver calls with
other streams, where cudaFree would synchronise the device).  Its scratch is
a static device array shared by every call, so this test makes calls in a
row on different grids: a later call must not see an earlier one's rows.
Tolerance: the same as the p_inprod_ test, 1e-13 of sum |r*p|.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from musoc_solver_b200 import build, native

    build.build()
    return torch, native.lib()


def _ref_inprod(L, r, p):
    j0, i0 = r.shape
    tp = C.c_double()
    L.p_inprod_(r.ctypes.data_as(C.c_void_p), p.ctypes.data_as(C.c_void_p), C.byref(tp),
                C.byref(C.c_int(i0 - 2)), C.byref(C.c_int(j0 - 2)))
    assert L.sevp_last_status() == 0
    return tp.value


def _call(torch, L, r, p, out, stream=None):
    j2, i2 = r.shape[0] - 2, r.shape[1] - 2
    rd = torch.from_numpy(r).cuda()
    pd = torch.from_numpy(p).cuda()
    torch.cuda.synchronize()
    h = None if stream is None else C.c_void_p(stream.cuda_stream)
    st = L.sevp_inprod_noalloc(C.c_void_p(rd.data_ptr()), C.c_void_p(pd.data_ptr()), i2, j2,
                               C.c_void_p(out.data_ptr()), h)
    assert st == 0, L.sevp_last_error().decode()
    torch.cuda.synchronize()
    return float(out.item())


def test_noalloc_inprod_two_calls_match_p_inprod(env, oracle):
    torch, L = env
    rng = np.random.default_rng(11)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    # the second call covers fewer rows; the third is the largest allowed
    # grid (its last partial sum sits next to the arrival counter)
    for i2, j2 in ((300, 2000), (180, 90), (7, 16384)):
        r = rng.standard_normal((j2 + 2, i2 + 2))
        p = rng.standard_normal((j2 + 2, i2 + 2))
        got = _call(torch, L, r, p, out)
        ref = _ref_inprod(L, r, p)
        orc = oracle.inprod(r, p)
        scale = np.abs(r[1:-1, 1:-1] * p[1:-1, 1:-1]).sum()
        assert abs(got - ref) <= 1e-13 * scale, (i2, j2, got, ref)
        assert abs(got - orc) <= 1e-13 * scale, (i2, j2, got, orc)


def test_noalloc_on_a_side_stream_allocates_nothing(env):
    """Calls on a non-default stream give the p_inprod_ value, and 100 calls
    leave the device's free memory unchanged."""
    torch, L = env
    rng = np.random.default_rng(12)
    i2, j2 = 240, 120
    r = rng.standard_normal((j2 + 2, i2 + 2))
    p = rng.standard_normal((j2 + 2, i2 + 2))
    ref = _ref_inprod(L, r, p)
    scale = np.abs(r[1:-1, 1:-1] * p[1:-1, 1:-1]).sum()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    side = torch.cuda.Stream()
    got = _call(torch, L, r, p, out, stream=side)
    assert abs(got - ref) <= 1e-13 * scale
    rd = torch.from_numpy(r).cuda()
    pd = torch.from_numpy(p).cuda()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(100):
        assert L.sevp_inprod_noalloc(C.c_void_p(rd.data_ptr()), C.c_void_p(pd.data_ptr()), i2,
                                     j2, C.c_void_p(out.data_ptr()),
                                     C.c_void_p(side.cuda_stream)) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert abs(float(out.item()) - ref) <= 1e-13 * scale


def test_noalloc_rejects_too_many_rows(env):
    torch, L = env
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    st = L.sevp_inprod_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()), 10, 16385,
                               C.c_void_p(x.data_ptr()), None)
    assert st == 5  # SEVP_BAD_ARG
    assert "16384" in L.sevp_last_error().decode()
