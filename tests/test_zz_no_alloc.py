"""afl_solve_cg_noalloc: the pressure solve for callers that may not allocate
device memory (real-time threads that must not block on the driver's
allocator, hosts with one budgeted device pool).  It runs the streaming FP64 CG
kernel, on device buffers the caller owns, with its working memory taken from a
fixed array inside the library.  These checks call it through the C ABI twice
in a row and compare each result with the handle-based afl_solve_cg run on the
same kernel (AFL_POISSON_KERNEL_STREAMING) and inputs: on a small grid, on the
largest grid the array holds (64^3, all four CG vectors fill it), and on a grid
whose x extent is not a multiple of 4 (narrower runs per thread)."""
import ctypes

import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu

SHAPES = [(40, 36, 30), (64, 64, 64), (37, 45, 29)]


def compatible_rhs(shape, seed):
    """Zero off the interior, zero-mean on it: solvable by the Neumann operator."""
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    b = np.zeros((nz, ny, nx))
    inner = rng.standard_normal((nz - 2, ny - 2, nx - 2)) * 0.01
    b[1:-1, 1:-1, 1:-1] = inner - inner.mean()
    return b.ravel()


def handle_solve(af, shape, b, p0, iters, rel_tol):
    nx, ny, nz = shape
    h = af.FluidSolver3D(nx, ny, nz, poisson_kernel=1, cg_rel_tol=rel_tol)
    h.set_field("divergence", b)
    h.set_field("pressure", p0)
    info = h.solve_poisson_conjugate_gradient(iters)
    out = h.get_field("pressure")
    h.close()
    return out, info


@pytest.mark.parametrize("shape", SHAPES, ids=["x".join(map(str, s)) for s in SHAPES])
def test_noalloc_solve_matches_handle_solve_twice(af, shape):
    import torch
    from aether_fluid import _lib
    lib = _lib.load()
    nx, ny, nz = shape
    stream = torch.cuda.current_stream()
    p_start = np.random.default_rng(7).standard_normal(nx * ny * nz) * 0.01
    d_p = torch.from_numpy(p_start.copy()).cuda()
    for call, (seed, iters, rel_tol) in enumerate(((1, 150, 1e-6), (2, 60, 0.0))):
        b = compatible_rhs(shape, seed)
        p0 = d_p.cpu().numpy().copy()  # the second call warm-starts from the first
        ref, ref_info = handle_solve(af, shape, b, p0, iters, rel_tol)
        d_b = torch.from_numpy(b).cuda()
        info = _lib.AflSolveInfo()
        st = lib.afl_solve_cg_noalloc(d_b.data_ptr(), d_p.data_ptr(), nx, ny, nz, iters,
                                      rel_tol, stream.cuda_stream, ctypes.byref(info))
        assert st == 0, lib.afl_last_error()
        got = d_p.cpu().numpy()
        assert info.iterations == ref_info.iterations, (call, info.iterations)
        assert bool(info.converged) == ref_info.converged
        assert rel_l2(got, ref) <= 1e-11, (call, rel_l2(got, ref))
        assert abs(info.final_residual - ref_info.final_residual) <= 1e-9 * ref_info.rhs_norm


def test_noalloc_rejects_grids_beyond_its_limit(af):
    import torch
    from aether_fluid import _lib
    lib = _lib.load()
    d = torch.zeros(65 * 64 * 64, dtype=torch.float64, device="cuda")
    info = _lib.AflSolveInfo()
    # one cell too many, and a grid whose cell count wraps around to 0 in 64 bits
    for dims in ((65, 64, 64), (1 << 22, 1 << 21, 1 << 21)):
        st = lib.afl_solve_cg_noalloc(d.data_ptr(), d.data_ptr(), *dims, 10, 0.0, None,
                                      ctypes.byref(info))
        assert st == 1, dims
        assert b"no-allocation limit" in lib.afl_last_error()
