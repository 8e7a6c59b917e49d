"""The barotropic correction loop of FS on the GPU against the oracle: each
kernel bit for bit, and the whole ITMASK loop (oracle PCG inside) to FP32
rounding."""
import numpy as np
import pytest

from musoc_solver_b200 import problems as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda_b():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from musoc_solver_b200 import build

    build.build()
    return torch


def test_fs_kernels_bit_exact(torch_cuda_b, oracle):
    torch = torch_cuda_b
    from musoc_solver_b200.barotropic import BarotropicCorrection

    st = P.fs_state(70, 36, 5, seed=4)
    bc = BarotropicCorrection(st)
    u, v, p0, scr = bc.upload()
    i0, j0, k0 = st.dims
    # masking
    uo, vo = st.u.copy(), st.v.copy()
    oracle.fs_mask(uo, vo, st.iu0, st.iv0)
    bc.mask(u, v)
    assert np.array_equal(u.cpu().numpy(), uo) and np.array_equal(v.cpu().numpy(), vo)
    # right-hand side (REAL*4) and its scaled FP64 copy
    s = torch.zeros((j0 - 2, i0 - 2), dtype=torch.float32, device="cuda")
    b = torch.zeros((j0 - 2, i0 - 2), dtype=torch.float64, device="cuda")
    bc.rhs(u, v, s=s, b=b)
    so = oracle.fs_rhs(uo, vo, st.odx, st.ody, st.ocs, st.csv, st.odz)
    assert np.array_equal(s.cpu().numpy(), so)
    assert np.array_equal(b.cpu().numpy(), so.astype(np.float64) * st.rscale[:, None].astype(np.float64))
    # correction with a random X
    x = np.random.default_rng(1).standard_normal((j0 - 2, i0 - 2)) * 1e3
    p0o, scro = st.p0.copy(), st.scr.copy()
    p0o[:] = np.random.default_rng(2).standard_normal(p0o.shape).astype(np.float32)
    p0.copy_(torch.from_numpy(p0o))
    scro[2:] = 0.5
    scr.copy_(torch.from_numpy(scro))
    vm_o = oracle.fs_correct(x, st.odt, st.odx, st.odyv, st.iu, st.iv, st.iu0, st.iv0, p0o, uo, vo,
                             scro)
    vm = bc.correct(torch.from_numpy(x).cuda(), u, v, p0, scr)
    assert np.array_equal(p0.cpu().numpy(), p0o)
    assert np.array_equal(u.cpu().numpy(), uo) and np.array_equal(v.cpu().numpy(), vo)
    assert np.array_equal(scr.cpu().numpy(), scro)
    assert vm == vm_o and vm > 0
    bc.close()


@pytest.mark.parametrize("schwarz", [False, True])
def test_fs_loop_matches_oracle_loop(torch_cuda_b, oracle, schwarz):
    torch = torch_cuda_b
    from musoc_solver_b200.barotropic import BarotropicCorrection
    from musoc_solver_b200.solver import tile_sub_blocks

    st = P.fs_state(64, 32, 4, seed=6)
    bc = BarotropicCorrection(st, tile_m=16, tile_h=8, schwarz=schwarz)
    assert bool(bc.solver.schwarz_shift) == schwarz
    u, v, p0, scr = bc.upload()
    tolerance, mxmask = 1e-6, 5
    passes, vm, iters = bc.run(u, v, p0, scr, tolerance=tolerance, mxmask=mxmask, precision=0)
    assert 1 <= passes <= mxmask and iters > 0
    # the oracle loop with the oracle PCG on the same operator
    pc = oracle.TilePC(st.problem, 16, 8, tile_nb=tile_sub_blocks(st.problem, 16, 8, 1e10))
    uo, vo, p0o, scro = st.u.copy(), st.v.copy(), st.p0.copy(), st.scr.copy()
    k = 0
    while True:
        k += 1
        oracle.fs_mask(uo, vo, st.iu0, st.iv0)
        so = oracle.fs_rhs(uo, vo, st.odx, st.ody, st.ocs, st.csv, st.odz)
        bo = so.astype(np.float64) * st.rscale[:, None].astype(np.float64)
        xo, _, rel = pc.pcg(bo, tol=1e-12)
        assert rel <= 1e-12
        vmo = oracle.fs_correct(xo, st.odt, st.odx, st.odyv, st.iu, st.iv, st.iu0, st.iv0, p0o, uo,
                                vo, scro)
        if vmo <= tolerance or k == mxmask:
            break
    assert passes == k
    scale = lambda a: np.abs(a).max()
    for g, o in ((p0, p0o), (u, uo), (v, vo), (scr, scro)):
        g = g.cpu().numpy()
        assert np.abs(g - o).max() <= 1e-5 * scale(o), (np.abs(g - o).max(), scale(o))
    assert abs(vm - vmo) <= 1e-5 * max(vmo, 1e-30) + 1e-7
    bc.close()
