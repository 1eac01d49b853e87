"""The tensor-core (tcgen05, 3xTF32) product of the mixed-precision projection
against an FP64 reference on the same padded block workspaces.

The product C_i = op(A_i) diag(d_i) op(B_i) of the large-block projection
(the F_DGEMM pair of Update_xz, v2rdm_solver.cc:3273,3286, and the refinement
residuals) runs on the tensor cores while the projection only needs FP32
accuracy.  Tolerance: 1e-5 of the largest |C| (FP32 accumulation over K up to
832; a layout or descriptor error gives O(1) differences).  The FP64 kernel
of the same entry point is checked at 1e-12."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIMS = [100, 200, 65, 800, 64, 130]


def _blocks(rng, dims, fill):
    out = []
    for n in dims:
        np_ = (n + 63) // 64 * 64
        m = np.zeros((np_, np_))
        m[:n, :n] = fill(rng, n)
        out.append(m)
    return out


def _flat(blocks):
    return np.concatenate([b.reshape(-1) for b in blocks])


@pytest.mark.parametrize("ta,tb,use_d", [(False, False, False), (True, False, False), (False, True, True),
                                         (True, True, True)])
def test_tc_block_gemm_matches_fp64(v2g, ta, tb, use_d):
    import torch

    rng = np.random.default_rng(11 + 2 * ta + tb)
    A = _blocks(rng, DIMS, lambda r, n: r.standard_normal((n, n)))
    B = _blocks(rng, DIMS, lambda r, n: r.standard_normal((n, n)))
    D = [np.concatenate([rng.uniform(-1, 2, n), np.zeros((n + 63) // 64 * 64 - n)]) for n in DIMS]
    dev = torch.device("cuda:0")
    dA = torch.from_numpy(_flat(A)).to(dev)
    dB = torch.from_numpy(_flat(B)).to(dev)
    dD = torch.from_numpy(np.concatenate(D)).to(dev)
    for tc in (True, False):
        dC = torch.full_like(dA, float("nan"))
        v2g.block_gemm_device(DIMS, dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), trans_a=ta, trans_b=tb,
                              d_d=dD.data_ptr() if use_d else None, tensor_cores=tc)
        C = dC.cpu().numpy()
        off = 0
        for a, b, d in zip(A, B, D):
            np_ = a.shape[0]
            ref = (a.T if ta else a) @ (np.diag(d) if use_d else np.eye(np_)) @ (b.T if tb else b)
            got = C[off:off + np_ * np_].reshape(np_, np_)
            off += np_ * np_
            assert np.isfinite(got).all()
            tol = (1e-5 if tc else 1e-12) * np.abs(ref).max()
            assert np.abs(got - ref).max() <= tol, (tc, np_, np.abs(got - ref).max() / np.abs(ref).max())


def test_tc_block_gemm_is_more_accurate_than_one_tf32_product(v2g):
    """3xTF32 keeps FP32 accuracy: its error is far below a single TF32 product's."""
    import torch

    rng = np.random.default_rng(5)
    dims = [256]
    A = _blocks(rng, dims, lambda r, n: r.standard_normal((n, n)))
    B = _blocks(rng, dims, lambda r, n: r.standard_normal((n, n)))
    dev = torch.device("cuda:0")
    dA = torch.from_numpy(_flat(A)).to(dev)
    dB = torch.from_numpy(_flat(B)).to(dev)
    dC = torch.empty_like(dA)
    v2g.block_gemm_device(dims, dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), tensor_cores=True)
    ref = A[0] @ B[0]
    err = np.abs(dC.cpu().numpy().reshape(256, 256) - ref).max() / np.abs(ref).max()
    # one TF32 product (10-bit mantissa) is off by ~1e-3 relative on these inputs
    assert err < 2e-6, err


def test_timed_products_leave_the_same_result(v2g):
    """The timing entry point runs the same product: after it, C holds A B."""
    import torch

    rng = np.random.default_rng(9)
    dims = [300, 130]
    A = _blocks(rng, dims, lambda r, n: r.standard_normal((n, n)))
    B = _blocks(rng, dims, lambda r, n: r.standard_normal((n, n)))
    dev = torch.device("cuda:0")
    dA = torch.from_numpy(_flat(A)).to(dev)
    dB = torch.from_numpy(_flat(B)).to(dev)
    for tc in (True, False):
        dC = torch.full_like(dA, float("nan"))
        sec = v2g.time_block_gemm(dims, dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), tensor_cores=tc, reps=3)
        assert 0.0 < sec < 1.0
        C, off = dC.cpu().numpy(), 0
        for a, b in zip(A, B):
            np_ = a.shape[0]
            ref = a @ b
            got = C[off:off + np_ * np_].reshape(np_, np_)
            off += np_ * np_
            assert np.abs(got - ref).max() <= (1e-5 if tc else 1e-12) * np.abs(ref).max()


@pytest.mark.parametrize("ta,tb,use_d", [(False, False, False), (True, False, True), (False, True, False),
                                         (True, True, True)])
def test_fp64_small_grid_split_k_matches_numpy(v2g, ta, tb, use_d):
    """Blocks of one instance's size (30 tiles of 64 x 64): the FP64 product runs
    as split-K clusters whose partial tiles are summed through distributed shared
    memory; same 1e-12 bound as the other FP64 forms."""
    import torch

    dims = [100, 64, 130, 200]
    rng = np.random.default_rng(21 + 2 * ta + tb)
    A = _blocks(rng, dims, lambda r, n: r.standard_normal((n, n)))
    B = _blocks(rng, dims, lambda r, n: r.standard_normal((n, n)))
    D = [np.concatenate([rng.uniform(-1, 2, n), np.zeros((n + 63) // 64 * 64 - n)]) for n in dims]
    dev = torch.device("cuda:0")
    dA = torch.from_numpy(_flat(A)).to(dev)
    dB = torch.from_numpy(_flat(B)).to(dev)
    dD = torch.from_numpy(np.concatenate(D)).to(dev)
    for rep in range(2):
        dC = torch.full_like(dA, float("nan"))
        v2g.block_gemm_device(dims, dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), trans_a=ta, trans_b=tb,
                              d_d=dD.data_ptr() if use_d else None, tensor_cores=False)
        C, off = dC.cpu().numpy(), 0
        for a, b, d in zip(A, B, D):
            np_ = a.shape[0]
            ref = (a.T if ta else a) @ (np.diag(d) if use_d else np.eye(np_)) @ (b.T if tb else b)
            got = C[off:off + np_ * np_].reshape(np_, np_)
            off += np_ * np_
            assert np.isfinite(got).all()
            assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
