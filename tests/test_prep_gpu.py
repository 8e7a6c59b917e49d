"""PREP's coefficient assembly on the GPU (sevp_prep_assemble, device arrays,
and sevp_prep_assemble_host) against the oracle's restatement of
P/prep_GLOBAL.f90:170-261, bit for bit: both DIMEN branches, closed
(NBIR = 1, side walls and the pressure pin) and periodic (NBIR = 2) grids,
a single layer, and the reference's idealised test stencil."""
import ctypes as C

import numpy as np
import pytest

from musoc_solver_b200 import problems as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from musoc_solver_b200 import build, native

    build.build()
    return torch, native.lib()


def _inputs(i2, j2, k1, seed, periodic):
    p = P.prep_grid(i2, j2, k1=k1, seed=seed, periodic=periodic)
    m = p.meta
    j1 = j2 + 1
    # the reference's INTEGER*2 masks: IU (I0, J0, K1), IV (I0, J1, K1)
    iu = np.ascontiguousarray(m["iu"][:k1], np.int16)
    iv = np.ascontiguousarray(m["iv"][:k1, :j1, :], np.int16)
    return p, m, iu, iv


def _gpu(torch, L, i2, j2, k1, dimen, m, iu, iv, nbir, gamma, idealised):
    dev = "cuda"
    t = {k: torch.from_numpy(np.ascontiguousarray(m[k], np.float32)).to(dev)
         for k in ("odx", "ody", "csv", "ocs", "odyv", "odz")}
    tu = torch.from_numpy(iu).to(dev)
    tv = torch.from_numpy(iv).to(dev)
    out = [torch.full((j2, i2), np.nan, dtype=torch.float32, device=dev) for _ in range(5)]
    st = L.sevp_prep_assemble(i2, j2, k1, dimen, *[t[k].data_ptr() for k in
                                                   ("odx", "ody", "csv", "ocs", "odyv", "odz")],
                              tu.data_ptr(), tv.data_ptr(), nbir, gamma, idealised,
                              *[o.data_ptr() for o in out], None)
    assert st == 0, L.sevp_last_error().decode()
    torch.cuda.synchronize()
    al, ar, ab, at, ac = (o.cpu().numpy() for o in out)
    return al, ab, ac, ar, at


@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("dimen", [3, 2])
def test_prep_assemble_bit_exact(env, oracle, periodic, dimen):
    torch, L = env
    i2, j2, k1 = 182, 93, 6
    p, m, iu, iv = _inputs(i2, j2, k1, seed=3, periodic=periodic)
    nbir = m["nbir"]
    gamma = float(m["gamma"])
    got = _gpu(torch, L, i2, j2, k1, dimen, m, iu, iv, nbir, gamma, 0)
    ref = oracle.assemble_dim(i2, j2, k1, dimen, m["odx"], m["ody"], m["csv"], m["ocs"], m["odyv"],
                              m["odz"], m["iu"], m["iv"], nbir, gamma, 0)
    for name, a, b in zip("AL AB AC AR AT".split(), got, ref):
        assert np.array_equal(a.view(np.int32), b.view(np.int32)), name
    if dimen == 3:
        # and the numpy statement the generators use
        for a, b in zip(got, p.coeffs()):
            assert np.array_equal(a, b)
    if not periodic:
        al, ab, ac, ar, at = got
        assert (al[:, 0] == 0).all() and (ar[:, -1] == 0).all()
        assert ab[0, i2 // 2 - 1] == ab[1, i2 // 2 - 1] != 0


def test_prep_assemble_one_layer_and_idealised(env, oracle):
    torch, L = env
    i2, j2 = 64, 1
    _, m, iu, iv = _inputs(i2, 40, 4, seed=4, periodic=False)
    for k1, j2, ideal in ((1, 40, 0), (4, 40, 1), (4, 1, 1), (4, 2, 0)):
        got = _gpu(torch, L, i2, j2, k1, 3, m, np.ascontiguousarray(iu[:k1, :j2 + 2]),
                   np.ascontiguousarray(iv[:k1, :j2 + 1]), 1, 0.0, ideal)
        ref = oracle.assemble_dim(i2, j2, k1, 3, m["odx"], m["ody"], m["csv"], m["ocs"],
                                  m["odyv"], m["odz"], m["iu"][:, :j2 + 2, :i2 + 2].copy(),
                                  m["iv"][:, :j2 + 2, :i2 + 2].copy(), 1, 0.0, ideal)
        for a, b in zip(got, ref):
            assert np.array_equal(a, b), (k1, j2, ideal)


def test_prep_assemble_host_and_arguments(env, oracle):
    torch, L = env
    i2, j2, k1 = 50, 30, 5
    _, m, iu, iv = _inputs(i2, j2, k1, seed=6, periodic=True)
    out = [np.zeros((j2, i2), np.float32) for _ in range(5)]
    f = [np.ascontiguousarray(m[k], np.float32) for k in ("odx", "ody", "csv", "ocs", "odyv", "odz")]
    st = L.sevp_prep_assemble_host(i2, j2, k1, 3, *[a.ctypes.data for a in f], iu.ctypes.data,
                                   iv.ctypes.data, 2, float(m["gamma"]), 0,
                                   *[o.ctypes.data for o in out])
    assert st == 0, L.sevp_last_error().decode()
    al, ar, ab, at, ac = out
    ref = oracle.assemble_dim(i2, j2, k1, 3, m["odx"], m["ody"], m["csv"], m["ocs"], m["odyv"],
                              m["odz"], m["iu"], m["iv"], 2, float(m["gamma"]), 0)
    for a, b in zip((al, ab, ac, ar, at), ref):
        assert np.array_equal(a, b)
    # refused: bad dimen, bad nbir, missing masks
    assert L.sevp_prep_assemble_host(i2, j2, k1, 4, *[a.ctypes.data for a in f], iu.ctypes.data,
                                     iv.ctypes.data, 2, 0.0, 0, *[o.ctypes.data for o in out]) == 5
    assert L.sevp_prep_assemble_host(i2, j2, k1, 3, *[a.ctypes.data for a in f], iu.ctypes.data,
                                     iv.ctypes.data, 3, 0.0, 0, *[o.ctypes.data for o in out]) == 5
    assert L.sevp_prep_assemble_host(i2, j2, k1, 3, *[a.ctypes.data for a in f], None, None, 2,
                                     0.0, 0, *[o.ctypes.data for o in out]) == 5
