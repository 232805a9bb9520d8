"""Device adjoints through the C ABI: bit for bit against the adjoint oracle
(FP64, same summation orders), and the torch autograd wrappers against
central finite differences of the device forward."""
import numpy as np
import pytest
from scipy import sparse

from oracle import adjoint_oracle
from parallellocallyoptimalapproximatesparsematrixinverses_b200 import adjoint, backward_error, global_spai, problems

pytestmark = pytest.mark.gpu


def _m_from_mr(A, topk):
    r = global_spai.mr(A, M0=problems.diagonal_inverse(A), max_iterations=4, tolerance=1e-14,
                       max_density=topk / A.shape[0], topk_per_column=topk)
    return adjoint_oracle.canonical_csc(r.M)


CASES = {
    # a built SPAI M: non-symmetric pattern, top-5 per column
    "laplacian_16_mr": lambda: (problems.laplacian_2d(16), 5),
    # variable coefficients
    "diffusion_20_mr": lambda: (problems.diffusion_2d(20, 1.0, 4), 7),
    # long-range couplings: windows wider than the bitmap kernels take
    "banded_wide": lambda: (problems.random_banded_spd(20_000, half_width=2, extra=2, seed=9), 0),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_residual_adjoint_bit_exact(require_gpu, case):
    A, topk = CASES[case]()
    A = adjoint_oracle.canonical_csc(A)
    M = _m_from_mr(A, topk) if topk else adjoint_oracle.canonical_csc(problems.diagonal_inverse(A))
    loss, grad_m, grad_a = adjoint.residual_adjoint(A, M)
    want_loss, want_m, want_a = adjoint_oracle.residual_adjoint(A, M)
    assert loss == want_loss
    assert np.array_equal(grad_m.indices, M.indices) and np.array_equal(grad_a.indices, A.indices)
    assert np.array_equal(grad_m.data, want_m)
    assert np.array_equal(grad_a.data, want_a)
    assert np.abs(grad_m.data).max() > 0


def test_pcg_adjoint_bit_exact(require_gpu):
    A = sparse.csr_matrix(problems.diffusion_2d(24, 1.0, 5))
    A.sort_indices()
    M = sparse.csr_matrix(problems.diagonal_inverse(A))
    rng = np.random.default_rng(2)
    x_t = rng.standard_normal(A.shape[0])
    b = A @ x_t
    _, status, x = backward_error.pcg(A.data, A.indices, A.indptr, M.data, M.indices, M.indptr, b, 3000, 1, 1e-10,
                                      return_x=True)
    assert status == 1
    g = 2.0 * (x - x_t)
    grad_b, grad_a, history, status = adjoint.pcg_adjoint(A.data, A.indices, A.indptr, M.data, M.indices,
                                                          M.indptr, x, g, 3000, 1e-10)
    want_b, want_a, want_history, want_status = adjoint_oracle.pcg_adjoint(A, M, x, g, 3000, 1e-10)
    assert status == want_status == 1
    assert np.array_equal(history.view(np.int64), want_history.view(np.int64))
    assert np.array_equal(grad_b, want_b)
    assert np.array_equal(grad_a, want_a)
    # the adjoint solve is the forward's own arithmetic with b = grad_x
    _, _, lam = backward_error.pcg(A.data, A.indices, A.indptr, M.data, M.indices, M.indptr, g, 3000, 1, 1e-10,
                                   return_x=True)
    assert np.array_equal(grad_b, lam)


def _symmetric_direction(A_csr, rng):
    upper = sparse.triu(A_csr, format="csr")
    upper.data = rng.standard_normal(upper.nnz)
    d = sparse.csr_matrix(upper + sparse.triu(upper, k=1).T)
    d.sort_indices()
    assert np.array_equal(d.indices, A_csr.indices) and np.array_equal(d.indptr, A_csr.indptr)
    return d.data


def test_pcg_autograd_matches_finite_differences(require_gpu):
    # variable-coefficient 5-point operator; x_t ~ N(0, 1), b = A x_t + 0.01 N(0, 1); L = ||x - x_t||^2
    import torch
    A = sparse.csr_matrix(problems.diffusion_2d(64, 1.0, 11))
    A.sort_indices()
    M = sparse.csr_matrix(problems.diagonal_inverse(A))
    rng = np.random.default_rng(12)
    x_t = torch.from_numpy(rng.standard_normal(A.shape[0]))
    b0 = A @ x_t.numpy() + 0.01 * rng.standard_normal(A.shape[0])
    solve = dict(a_indices=A.indices, a_offsets=A.indptr, m_values=M.data, m_indices=M.indices,
                 m_offsets=M.indptr, max_iterations=20_000, tolerance=1e-13)

    def loss(a_values, b):
        x = adjoint.pcg_solve(a_values, b, **solve)
        return torch.sum((x - x_t) ** 2)

    a = torch.from_numpy(A.data.copy()).requires_grad_(True)
    b = torch.from_numpy(b0.copy()).requires_grad_(True)
    loss(a, b).backward()
    scale = np.abs(A.data).max()
    for _ in range(16):
        da = torch.from_numpy(_symmetric_direction(A, rng))
        db = torch.from_numpy(rng.standard_normal(A.shape[0]))
        # the step where truncation (h^2) and solve error balance, found with the
        # oracle PCG (the device's arithmetic): worst relative gap 5e-8 over these 16
        h = 1e-8 * scale
        with torch.no_grad():
            fd = (loss(a + h * da, b + h * db) - loss(a - h * da, b - h * db)).item() / (2 * h)
        got = (a.grad @ da + b.grad @ db).item()
        assert got == pytest.approx(fd, rel=1e-6)


def test_residual_objective_autograd(require_gpu):
    import torch
    A = adjoint_oracle.canonical_csc(problems.diffusion_2d(12, 1.0, 3))
    M = _m_from_mr(A, 6)
    a = torch.from_numpy(A.data.copy()).requires_grad_(True)
    m = torch.from_numpy(M.data.copy()).requires_grad_(True)
    a_pattern, m_pattern = (A.indptr, A.indices), (M.indptr, M.indices)
    f = adjoint.residual_objective(a, m, a_pattern, m_pattern)
    (3.0 * f).backward()
    _, want_m, want_a = adjoint_oracle.residual_adjoint(A, M)
    assert np.array_equal(m.grad.numpy(), 3.0 * want_m)
    assert np.array_equal(a.grad.numpy(), 3.0 * want_a)
    rng = np.random.default_rng(5)
    for _ in range(4):
        da = torch.from_numpy(rng.standard_normal(A.nnz))
        dm = torch.from_numpy(rng.standard_normal(M.nnz))
        h = 1e-6
        with torch.no_grad():
            fp = adjoint.residual_objective(a + h * da, m + h * dm, a_pattern, m_pattern).item()
            fm = adjoint.residual_objective(a - h * da, m - h * dm, a_pattern, m_pattern).item()
        got = ((a.grad @ da + m.grad @ dm) / 3.0).item()
        assert got == pytest.approx((fp - fm) / (2 * h), rel=1e-6)


def test_autograd_on_cuda_tensors_stays_on_the_device_and_matches_the_host_path(require_gpu):
    """CUDA tensors go through the device entry points (no host copies of the
    values): the same bits as the host path, gradients on the device."""
    import torch
    dev = torch.device("cuda:0")
    A = adjoint_oracle.canonical_csc(problems.diffusion_2d(14, 1.0, 6))
    M = _m_from_mr(A, 6)
    a_pattern, m_pattern = (A.indptr, A.indices), (M.indptr, M.indices)
    grads = {}
    for where in ("cpu", dev):
        a = torch.from_numpy(A.data.copy()).to(where).requires_grad_(True)
        m = torch.from_numpy(M.data.copy()).to(where).requires_grad_(True)
        f = adjoint.residual_objective(a, m, a_pattern, m_pattern)
        (2.0 * f).backward()
        assert f.device.type == a.grad.device.type == m.grad.device.type == torch.device(where).type
        grads[str(where)] = (f.item(), a.grad.cpu().numpy(), m.grad.cpu().numpy())
    assert grads["cpu"][0] == grads["cuda:0"][0]
    assert np.array_equal(grads["cpu"][1], grads["cuda:0"][1]) and np.array_equal(grads["cpu"][2], grads["cuda:0"][2])

    R = sparse.csr_matrix(problems.diffusion_2d(20, 1.0, 7))
    R.sort_indices()
    P = sparse.csr_matrix(problems.diagonal_inverse(R))
    rng = np.random.default_rng(4)
    x_t = rng.standard_normal(R.shape[0])
    b0 = R @ x_t
    solve = dict(a_indices=R.indices, a_offsets=R.indptr, m_values=P.data, m_indices=P.indices, m_offsets=P.indptr,
                 max_iterations=4000, tolerance=1e-12, refresh_period=9)
    out = {}
    for where in ("cpu", dev):
        a = torch.from_numpy(R.data.copy()).to(where).requires_grad_(True)
        b = torch.from_numpy(b0.copy()).to(where).requires_grad_(True)
        x = adjoint.pcg_solve(a, b, **solve)
        assert x.device.type == torch.device(where).type
        loss = torch.sum((x - torch.from_numpy(x_t).to(where)) ** 2)
        loss.backward()
        out[str(where)] = (x.detach().cpu().numpy(), a.grad.cpu().numpy(), b.grad.cpu().numpy())
    for h, d in zip(out["cpu"], out["cuda:0"]):
        assert np.array_equal(h, d)


def test_device_entry_points_reject_host_pointers_and_aliases(require_gpu):
    import ctypes

    import torch
    from parallellocallyoptimalapproximatesparsematrixinverses_b200 import _lib
    A = sparse.csr_matrix(problems.laplacian_2d(8))
    n = A.shape[0]
    dev = torch.device("cuda:0")
    t = lambda v: torch.from_numpy(np.ascontiguousarray(v)).to(dev)  # noqa: E731
    av, ai, ao = t(A.data), t(A.indices.astype(np.int64)), t(A.indptr.astype(np.int64))
    b = torch.ones(n, dtype=torch.float64, device=dev)
    p = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    params = _lib.PcgParams(100, 1e-10, 0, 0, 0, 0)
    hist = np.zeros(100)
    status = ctypes.c_int64(0)
    err = _lib.error_buffer()
    lib = _lib.load()
    torch.cuda.synchronize()
    rc = lib.spai_pcg_device(n, av.numel(), p(av), p(ai), p(ao), av.numel(), p(av), p(ai), p(ao), p(b), params,
                             hist.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(status), p(b), err,
                             len(err))
    assert rc == -1 and b"x overlaps b" in err.value
    host_b = np.ones(n)
    x = torch.empty(n, dtype=torch.float64, device=dev)
    rc = lib.spai_pcg_device(n, av.numel(), p(av), p(ai), p(ao), av.numel(), p(av), p(ai), p(ao),
                             ctypes.c_void_p(host_b.ctypes.data), params,
                             hist.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(status), p(x), err,
                             len(err))
    assert rc == -1 and b"b must point to device memory" in err.value
    bad = ao.clone()
    bad[3] = bad[4] + 1
    rc = lib.spai_pcg_device(n, av.numel(), p(av), p(ai), p(bad), av.numel(), p(av), p(ai), p(ao), p(b), params,
                             hist.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(status), p(x), err,
                             len(err))
    assert rc == -1 and b"CSR offsets" in err.value


def test_residual_adjoint_512_against_the_oracle_and_64_finite_differences(require_gpu):
    """Config 5, L1 = ||I - A M||_F^2 on the 512^2 log-normal (sigma 1) 5-point
    operator with M from 5 Global MR iterations (top-8): the device gradient,
    through CUDA tensors, is the FP64 oracle's bit for bit, and 64 random
    central differences (step 1e-6) agree with it; measured worst relative
    gap over 16 of them on a B200: 5.8e-9."""
    import torch
    dev = torch.device("cuda:0")
    A = adjoint_oracle.canonical_csc(problems.diffusion_2d(512, 1.0, 11))
    n = A.shape[0]
    M = adjoint_oracle.canonical_csc(global_spai.mr(A, M0=problems.diagonal_inverse(A), max_iterations=5,
                                                    tolerance=1e-14, max_density=8.0 / n, topk_per_column=8).M)
    want_loss, want_m, want_a = adjoint_oracle.residual_adjoint(A, M)
    a = torch.from_numpy(A.data.copy()).to(dev).requires_grad_(True)
    m = torch.from_numpy(M.data.copy()).to(dev).requires_grad_(True)
    a_pattern, m_pattern = (A.indptr, A.indices), (M.indptr, M.indices)
    f = adjoint.residual_objective(a, m, a_pattern, m_pattern)
    f.backward()
    assert f.item() == want_loss
    assert np.array_equal(a.grad.cpu().numpy(), want_a) and np.array_equal(m.grad.cpu().numpy(), want_m)
    rng = np.random.default_rng(5)
    h = 1e-6
    worst = 0.0
    for _ in range(64):
        da = torch.from_numpy(rng.standard_normal(A.nnz)).to(dev)
        dm = torch.from_numpy(rng.standard_normal(M.nnz)).to(dev)
        with torch.no_grad():
            fp = adjoint.residual_objective(a + h * da, m + h * dm, a_pattern, m_pattern).item()
            fm = adjoint.residual_objective(a - h * da, m - h * dm, a_pattern, m_pattern).item()
        fd = (fp - fm) / (2 * h)
        worst = max(worst, abs((a.grad @ da + m.grad @ dm).item() - fd) / abs(fd))
    assert worst <= 1e-6, worst


def test_pcg_adjoint_512_against_the_direct_solve_gradient_and_64_finite_differences(require_gpu):
    """Config 5, L2 = ||x - x_t||^2 with x = PCG(A, M, b) on the 512^2
    operator, x_t ~ N(0, 1), b = A x_t + 0.01 N(0, 1), Jacobi M, PCG to 1e-14
    (about 2,800 iterations), all on CUDA tensors.  The FP64 reference gradient
    comes from a direct solve (scipy splu): x = A^-1 b, lambda = A^-1 2(x - x_t),
    dL/db = lambda, dL/dA_ij = -lambda_i x_j.  Measured on a B200: gradients
    within 7e-13 (b) and 4.7e-12 (A) relative in norm.  Central differences
    along 64 random symmetric perturbations of A's values and b, with step
    1e-8 x max|A|, where truncation and the solve's rounding balance: worst
    relative gap 1.0e-6 over 16 measured."""
    import torch
    from scipy.sparse import linalg as spla
    dev = torch.device("cuda:0")
    A = sparse.csr_matrix(problems.diffusion_2d(512, 1.0, 11))
    A.sort_indices()
    n = A.shape[0]
    M = sparse.csr_matrix(problems.diagonal_inverse(A))
    rng = np.random.default_rng(12)
    x_t = rng.standard_normal(n)
    b0 = A @ x_t + 0.01 * rng.standard_normal(n)
    lu = spla.splu(sparse.csc_matrix(A))
    x_ref = lu.solve(b0)
    lam_ref = lu.solve(2.0 * (x_ref - x_t))
    coo = A.tocoo()
    grad_a_ref = -lam_ref[coo.row] * x_ref[coo.col]
    solve = dict(a_indices=A.indices, a_offsets=A.indptr, m_values=M.data, m_indices=M.indices, m_offsets=M.indptr,
                 max_iterations=60_000, tolerance=1e-14)
    xt = torch.from_numpy(x_t).to(dev)

    def loss(a_values, b):
        return torch.sum((adjoint.pcg_solve(a_values, b, **solve) - xt) ** 2)

    a = torch.from_numpy(A.data.copy()).to(dev).requires_grad_(True)
    b = torch.from_numpy(b0.copy()).to(dev).requires_grad_(True)
    loss(a, b).backward()
    gb, ga = b.grad.cpu().numpy(), a.grad.cpu().numpy()
    assert np.linalg.norm(gb - lam_ref) <= 1e-10 * np.linalg.norm(lam_ref)
    assert np.linalg.norm(ga - grad_a_ref) <= 1e-10 * np.linalg.norm(grad_a_ref)
    h = 1e-8 * np.abs(A.data).max()
    rng2 = np.random.default_rng(3)
    worst = 0.0
    for _ in range(64):
        da = torch.from_numpy(_symmetric_direction(A, rng2)).to(dev)
        db = torch.from_numpy(rng2.standard_normal(n)).to(dev)
        with torch.no_grad():
            fd = (loss(a + h * da, b + h * db) - loss(a - h * da, b - h * db)).item() / (2 * h)
        worst = max(worst, abs((a.grad @ da + b.grad @ db).item() - fd) / abs(fd))
    assert worst <= 1e-5, worst
