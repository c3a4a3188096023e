"""GPU: the tensor-core DFT-as-GEMM path (tcgen05.mma, kind::tf32)."""
import numpy as np
import pytest

import qbgpu

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def tf32(x):
    """round FP32 values to TF32 (10 explicit mantissa bits), nearest, ties away from zero"""
    b = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x1000) & 0xFFFFE000
    return b.astype(np.uint32).view(np.float32)


def test_umma_selftest_layouts():
    """one 128 x 64 x 64 TF32 GEMM through K-major shared-memory descriptors
    and a tensor-memory accumulator"""
    L = qbgpu.lib()
    rng = np.random.default_rng(11)
    A = rng.standard_normal((128, 64)).astype(np.float32)
    Bt = rng.standard_normal((64, 64)).astype(np.float32)
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(Bt).cuda()
    dD = torch.zeros((128, 64), dtype=torch.float32, device="cuda")
    rc = L.qb_umma_selftest(dA.data_ptr(), dB.data_ptr(), dD.data_ptr(), qbgpu._stream())
    assert rc == 0, L.qb_last_error().decode()
    torch.cuda.synchronize()
    want = tf32(A).astype(np.float64) @ tf32(Bt).astype(np.float64).T
    got = dD.cpu().numpy().astype(np.float64)
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err < 1e-5, err


L_, R_ = 6.0, 3.75


def rel_l2(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


@pytest.mark.parametrize("J,M,ncells", [(4, 3, 3), (16, 16, 2)])
def test_i3_dft_gemm_variant_against_oracle(J, M, ncells):
    """FP32 form at N = 16 with the I3 sums as tensor-core DFT-GEMMs
    (variant 1): Cc and Cd within the FP32 form's bound (1e-5 relative L2) of
    the CPU oracle, no bounded wait ran out, and the result is not the FFT
    kernels' under another name"""
    import orc
    N = 16
    o = orc.Oracle(N, J, M, L_, R_)
    q = qbgpu.Quad(N, J, M, L_, R_)
    Wv = qbgpu.gaussian_mixture_state(N, L_, seed=81, ncells=ncells)
    Wf = np.stack([orc.to_fourier(w) for w in Wv])
    W = torch.from_numpy(Wf).cuda()
    ws = qbgpu.Workspace(N, precision=32)
    ws.set_i3_variant(1)
    cc, cd = qbgpu.collision_operators(ws, q, W)
    assert ws.device_errors() == 0
    ref_cd = np.stack([o.cd(w) for w in Wf])
    ref_cc = np.stack([o.cc(w) for w in Wf])
    e_cd = rel_l2(cd.cpu().numpy(), ref_cd)
    assert e_cd <= 1e-5, e_cd
    assert rel_l2(cc.cpu().numpy(), ref_cc) <= 1e-5
    ws0 = qbgpu.Workspace(N, precision=32)
    _, cd0 = qbgpu.collision_operators(ws0, q, W)
    assert not torch.equal(cd0, cd)
