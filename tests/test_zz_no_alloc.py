"""pastix_gpu_solve_noalloc: the solve for callers that cannot let the library
allocate device memory (their own pool allocator owns the GPU's memory, or a
cudaMalloc in the middle of their solve loop would stall it).  Called through
the C ABI, its result must match pastix_gpu_solve's on the same factors, on
two calls in a row (the second reuses the scratch array the first one left
behind).  Collected last on purpose (file name) so that a run stopping at the
first failure has run every other test before this one."""
import ctypes as C

import numpy as np
import pytest

from pastix_b200 import matrices as M

pytestmark = pytest.mark.gpu

TOL = 1e-12          # FP64 solves, relative max-norm (the tolerance of the GPU parity tests)
TOL_MIXED = 1e-6     # FP32 factors: both entry points run the same FP32 solve


def _solver(system, mixed=False):
    from pastix_b200 import analysis
    from pastix_b200 import gpu as G
    st = analysis.analyze(system)
    s = G.Solver()
    s.set_iparm(G.IPARM_FACTORIZATION, G.FACT["potrf"])
    s.set_iparm(G.IPARM_MIXED, 1 if mixed else 0)
    s.set_structure(st)
    s.set_spm(system)
    s.numfact(system.values)
    return s


def _lib():
    from pastix_b200 import gpu as G
    L = G.load()
    L.pastix_gpu_solve_noalloc.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64]
    return L


@pytest.mark.parametrize("mixed", [False, True])
def test_noalloc_solve_matches_solve_on_two_calls(mixed):
    import torch
    from pastix_b200 import matrices as M
    A = M.diffusion_lognormal(14, 13, 12, 1.0, np.random.default_rng(8))
    s = _solver(A, mixed)
    L = _lib()
    nrhs = 3
    for call in range(2):
        b = np.random.default_rng(100 + call).uniform(-1.0, 1.0, (A.n, nrhs))
        flat = np.asfortranarray(b).ravel(order="F")
        ref = torch.from_numpy(flat.copy()).cuda()
        new = torch.from_numpy(flat.copy()).cuda()
        torch.cuda.synchronize()
        assert L.pastix_gpu_solve(s._h, nrhs, C.c_void_p(ref.data_ptr()), A.n) == 0
        assert L.pastix_gpu_solve_noalloc(s._h, nrhs, C.c_void_p(new.data_ptr()), A.n) == 0
        torch.cuda.synchronize()
        err = (new - ref).abs().max().item() / ref.abs().max().item()
        assert err <= (TOL_MIXED if mixed else TOL), (call, err)
        # and it solves the system (to the accuracy of the factors: single
        # precision factors whose large updates ran on TF32 tensor cores leave
        # residuals around 1e-3 before refinement)
        x = new.cpu().numpy().reshape(A.n, nrhs, order="F")
        r = b - A.to_scipy_full() @ x
        assert np.abs(r).max() <= (2e-2 if mixed else 1e-10) * np.abs(b).max()
    s.close()


@pytest.mark.parametrize("fact,make", [
    ("getrf", lambda: M.convdiff_upwind(10, 9, 8, 10.0)),
    ("potrf", lambda: M.magnetic_laplacian(8, 7, 6, -0.5, np.random.default_rng(4))),
], ids=["getrf_real", "potrf_complex"])
def test_noalloc_many_rhs_in_chunks(fact, make):
    """20 right-hand sides: two chunks of the scratch (16, then 4, the second
    starting 16 columns into B), on LU factors and on complex factors (solved
    8 columns at a time), against pastix_gpu_solve, twice in a row."""
    import torch
    from pastix_b200 import analysis
    from pastix_b200 import gpu as G
    A = make()
    st = analysis.analyze(A)
    s = G.Solver()
    s.set_iparm(G.IPARM_FACTORIZATION, G.FACT[fact])
    s.set_structure(st)
    s.set_spm(A)
    s.numfact(A.values)
    L = _lib()
    nrhs = 20
    cplx = np.iscomplexobj(A.values)
    for call in range(2):
        rng = np.random.default_rng(200 + call)
        b = rng.uniform(-1.0, 1.0, (A.n, nrhs))
        if cplx:
            b = b + 1j * rng.uniform(-1.0, 1.0, (A.n, nrhs))
        flat = np.asfortranarray(b).ravel(order="F")
        ref = torch.from_numpy(flat.copy()).cuda()
        new = torch.from_numpy(flat.copy()).cuda()
        torch.cuda.synchronize()
        assert L.pastix_gpu_solve(s._h, nrhs, C.c_void_p(ref.data_ptr()), A.n) == 0
        assert L.pastix_gpu_solve_noalloc(s._h, nrhs, C.c_void_p(new.data_ptr()), A.n) == 0
        torch.cuda.synchronize()
        err = (new - ref).abs().max().item() / ref.abs().max().item()
        assert err <= TOL, (call, err)
        x = new.cpu().numpy().reshape(A.n, nrhs, order="F")
        assert np.abs(b - A.to_scipy_full() @ x).max() <= 1e-10 * np.abs(b).max()
    s.close()


def test_noalloc_rejects_sizes_beyond_scratch():
    import torch
    from pastix_b200 import gpu as G
    from pastix_b200 import matrices as M
    A = M.laplacian_7pt(400, 400, 1)          # n = 160000: 16 FP64 columns need 20.5 MB > 16 MiB
    s = _solver(A)
    L = _lib()
    big = torch.zeros(A.n * 16, dtype=torch.float64, device="cuda")
    PASTIX_ERR_BADPARAMETER = 7
    assert L.pastix_gpu_solve_noalloc(s._h, 16, C.c_void_p(big.data_ptr()), A.n) == PASTIX_ERR_BADPARAMETER
    assert G.ERRORS[PASTIX_ERR_BADPARAMETER] == "PASTIX_ERR_BADPARAMETER"
    # one column fits (1.28 MB) and solves
    b = np.random.default_rng(3).uniform(-1.0, 1.0, A.n)
    one = torch.from_numpy(b.copy()).cuda()
    assert L.pastix_gpu_solve_noalloc(s._h, 1, C.c_void_p(one.data_ptr()), A.n) == 0
    x = one.cpu().numpy()
    assert np.abs(b - A.to_scipy_full() @ x).max() <= 1e-10 * np.abs(b).max()
    s.close()
