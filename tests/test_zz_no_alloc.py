"""`sdot_linear_solve_noalloc` (the CG with its work vectors in the library's static device array) against
`sdot_linear_solve` (method 0, per-call device memory), both through the C ABI on device arrays.

The Laplacian is a weighted 250 x 200 grid graph (50,000 rows, random positive couplings).  Two calls in a row
must match the allocating entry point within |x - x_ref| <= 1e-9 max|x_ref| (the rhs mean is summed in a
different order), use the same CG iteration counts (+-1), leave the device's free memory unchanged, and a size past
SDOT_NOALLOC_MAX_ROWS is refused with SDOT_ERR_CAPACITY.  Also: a right-hand side with a nonzero mean on a grid whose
row count is not a multiple of the CG's 256-row chunks (the last chunk partial), a system with no coupling at all
(cols and vals NULL), and host memory refused before any launch."""
import ctypes

import numpy as np
import pytest
import torch

from sdot import _lib

pytestmark = pytest.mark.gpu

MAX_ROWS = 262144


def _grid_laplacian(nx, ny, seed):
    rng = np.random.default_rng(seed)
    n = nx * ny
    idx = np.arange(n).reshape(ny, nx)
    a = np.r_[idx[:, :-1].ravel(), idx[:-1, :].ravel()]
    b = np.r_[idx[:, 1:].ravel(), idx[1:, :].ravel()]
    c = rng.uniform(0.5, 2.0, size=len(a))
    rows = np.r_[a, b]
    cols = np.r_[b, a]
    vals = np.r_[c, c]
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    row_ptr = np.zeros(n + 1, np.int64)
    np.add.at(row_ptr, rows + 1, 1)
    row_ptr = np.cumsum(row_ptr)
    dia = np.zeros(n)
    np.add.at(dia, rows, vals)
    return n, row_ptr, cols.astype(np.int32), vals, dia


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _both(n, rp, cols, vals, dia, rhs, calls=2):
    """the allocating solve once, then the no-alloc one `calls` times in a row: (reference, [solutions], iterations)"""
    L = _lib.load()
    ctx = _lib.context()
    k = rhs.shape[0]
    d_rp, d_dia, d_rhs = _dev(rp), _dev(dia), _dev(rhs)
    d_cols = _dev(cols) if cols is not None else None
    d_vals = _dev(vals) if vals is not None else None
    pc = d_cols.data_ptr() if d_cols is not None else None
    pv = d_vals.data_ptr() if d_vals is not None else None
    x_ref = torch.empty(k, n, dtype=torch.float64, device="cuda")
    its_ref = (ctypes.c_int32 * k)()
    st = _lib.Status()
    code = L.sdot_linear_solve(ctx, n, d_rp.data_ptr(), pc, pv, d_dia.data_ptr(), k, d_rhs.data_ptr(), x_ref.data_ptr(), 0, 1e-10, 100000,
                               _lib.SDOT_DEVICE, its_ref, ctypes.byref(st))
    assert code == 0, st.message
    got = []
    for _ in range(calls):
        x = torch.full((k, n), np.nan, dtype=torch.float64, device="cuda")
        its = (ctypes.c_int32 * k)()
        code = L.sdot_linear_solve_noalloc(ctx, n, d_rp.data_ptr(), pc, pv, d_dia.data_ptr(), k, d_rhs.data_ptr(), x.data_ptr(), 1e-10,
                                           100000, its, ctypes.byref(st))
        assert code == 0, st.message
        got.append((x.cpu().numpy(), list(its)))
    return x_ref.cpu().numpy(), got, list(its_ref)


def test_the_static_work_area_solve_matches_the_allocating_one():
    L = _lib.load()
    ctx = _lib.context()
    n, rp, cols, vals, dia = _grid_laplacian(250, 200, 5)
    rng = np.random.default_rng(6)
    k = 2
    rhs = rng.standard_normal((k, n))
    rhs -= rhs.mean(axis=1, keepdims=True)
    d_rp, d_cols, d_vals, d_dia, d_rhs = _dev(rp), _dev(cols), _dev(vals), _dev(dia), _dev(rhs)
    x_ref = torch.empty(k, n, dtype=torch.float64, device="cuda")
    its_ref = (ctypes.c_int32 * k)()
    st = _lib.Status()
    torch.cuda.synchronize()
    code = L.sdot_linear_solve(ctx, n, d_rp.data_ptr(), d_cols.data_ptr(), d_vals.data_ptr(), d_dia.data_ptr(), k, d_rhs.data_ptr(),
                               x_ref.data_ptr(), 0, 1e-10, 100000, _lib.SDOT_DEVICE, its_ref, ctypes.byref(st))
    assert code == 0, st.message
    ref = x_ref.cpu().numpy()
    assert np.isfinite(ref).all() and np.abs(ref[:, 0]).max() == 0.0
    scale = np.abs(ref).max()
    for call in range(2):
        x = torch.full((k, n), np.nan, dtype=torch.float64, device="cuda")
        its = (ctypes.c_int32 * k)()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        code = L.sdot_linear_solve_noalloc(ctx, n, d_rp.data_ptr(), d_cols.data_ptr(), d_vals.data_ptr(), d_dia.data_ptr(), k,
                                           d_rhs.data_ptr(), x.data_ptr(), 1e-10, 100000, its, ctypes.byref(st))
        assert code == 0, st.message
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        if call == 1:
            # the second call allocates nothing (the first one may load the library's device code)
            assert free_after == free_before
        got = x.cpu().numpy()
        assert np.isfinite(got).all()
        assert np.abs(got - ref).max() <= 1e-9 * scale, (call, np.abs(got - ref).max(), scale)
        assert all(abs(a - b) <= 1 for a, b in zip(its, its_ref)) and min(its) > 0
    # the residual of the solution itself
    import scipy.sparse as sp
    A = sp.diags(dia) - sp.csr_matrix((vals, cols, rp), shape=(n, n))
    for q in range(k):
        r = A @ got[q] - rhs[q]
        assert np.linalg.norm(r) <= 1e-8 * np.linalg.norm(rhs[q])


def test_a_size_past_the_static_work_area_is_refused():
    L = _lib.load()
    ctx = _lib.context()
    n = MAX_ROWS + 1
    rp = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    dia = torch.ones(n, dtype=torch.float64, device="cuda")
    rhs = torch.zeros(n, dtype=torch.float64, device="cuda")
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    its = (ctypes.c_int32 * 1)()
    st = _lib.Status()
    code = L.sdot_linear_solve_noalloc(ctx, n, rp.data_ptr(), None, None, dia.data_ptr(), 1, rhs.data_ptr(), x.data_ptr(), 1e-10, 100,
                                       its, ctypes.byref(st))
    assert code == 4 and st.needed == n and b"past the static work area" in st.message


def test_a_nonzero_mean_rhs_on_a_partial_last_chunk():
    n, rp, cols, vals, dia = _grid_laplacian(123, 77, 8)          # 9,471 rows: the last 256-row chunk is partial
    assert n % 256 != 0
    rng = np.random.default_rng(9)
    rhs = rng.standard_normal((2, n)) + np.array([[3.0], [-0.5]])  # nonzero means: both solves project them out
    ref, got, its_ref = _both(n, rp, cols, vals, dia, rhs)
    scale = np.abs(ref).max()
    assert np.isfinite(ref).all() and scale > 0
    for x, its in got:
        assert np.isfinite(x).all()
        assert np.abs(x - ref).max() <= 1e-9 * scale
        assert all(abs(a - b) <= 1 for a, b in zip(its, its_ref))


def test_a_system_without_couplings():
    n = 3000
    rp = np.zeros(n + 1, np.int64)
    dia = np.random.default_rng(10).uniform(0.5, 2.0, size=n)
    rhs = np.random.default_rng(11).standard_normal((1, n))
    ref, got, its_ref = _both(n, rp, None, None, dia, rhs)
    scale = max(np.abs(ref).max(), 1e-300)
    for x, its in got:
        assert np.isfinite(x).all()
        assert np.abs(x - ref).max() <= 1e-9 * scale
        assert list(its) == list(its_ref) or all(abs(a - b) <= 1 for a, b in zip(its, its_ref))


def test_host_memory_is_refused_before_any_launch():
    L = _lib.load()
    ctx = _lib.context()
    n = 1000
    rp = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    dia = torch.ones(n, dtype=torch.float64, device="cuda")
    host_rhs = np.zeros(n)                                          # pageable host memory
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    its = (ctypes.c_int32 * 1)()
    st = _lib.Status()
    launches = _lib.kernel_launches()
    code = L.sdot_linear_solve_noalloc(ctx, n, rp.data_ptr(), None, None, dia.data_ptr(), 1, host_rhs.ctypes.data, x.data_ptr(), 1e-10,
                                       100, its, ctypes.byref(st))
    assert code == 1 and b"device memory of the context's device" in st.message
    assert _lib.kernel_launches() == launches
