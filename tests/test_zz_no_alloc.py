"""The allocation-free grid sweep (wos_solve_grid_device_noalloc) against the
regular device entry point (wos_solve_grid_device), called twice in a row
through the C ABI.

Callers that cannot allocate device memory while they solve (a pool that owns
the device budget, code that must not synchronise the device) use it; its
temporaries live in a fixed static array in the library.  Same per-walk
random streams as the regular entry point; only the order in which walk
statistics are summed differs, so means agree to 1e-10 relative and step
counts exactly.  This file is collected last on purpose."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from walk_on_spheres_b200 import _lib, meshes

pytestmark = pytest.mark.gpu


def _noalloc_fn():
    f = _lib.lib().wos_solve_grid_device_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.POINTER(_lib.Params), C.POINTER(_lib.Grid)] + [C.c_void_p] * 5 + \
        [C.POINTER(_lib.Counters)]
    return f


def _outputs(torch, n):
    dev = torch.device("cuda", 0)
    return [torch.full((n,), float("nan"), dtype=torch.float64, device=dev) for _ in range(4)] + \
        [torch.zeros(n, dtype=torch.uint8, device=dev)]


@pytest.mark.parametrize("method", ["fast", "plain"])
def test_noalloc_matches_device_entry_point(solver, method):
    torch = pytest.importorskip("torch")
    solver.set_mesh(meshes.annulus())
    grid = solver.grid_over_mesh(40, 40, 1)
    n = 40 * 40
    walks = 2000 if method == "fast" else 300
    params = solver.params("laplace", N_walks=walks, seed=99, method=method)
    ref = _outputs(torch, n)
    solver.solve_grid_device("laplace", grid, *[t.data_ptr() for t in ref], N_walks=walks,
                             seed=99, method=method)
    torch.cuda.synchronize()
    f = _noalloc_fn()
    free_before = None
    for call in range(2):
        out = _outputs(torch, n)
        torch.cuda.synchronize()
        if call == 1:
            free_before = torch.cuda.mem_get_info(0)[0]
        cnt = _lib.Counters()
        rc = f(solver._ctx, C.byref(params), C.byref(grid), *[t.data_ptr() for t in out],
               C.byref(cnt))
        assert rc == 0, _lib.lib().wos_last_error(solver._ctx)
        torch.cuda.synchronize()
        if call == 1:
            # the second call reserves nothing new on the device
            assert torch.cuda.mem_get_info(0)[0] == free_before
        loc = out[4].cpu().numpy()
        assert np.array_equal(loc, ref[4].cpu().numpy())
        ins = loc == 1
        for a, b in zip(out[:3], ref[:3]):
            a, b = a.cpu().numpy()[ins], b.cpu().numpy()[ins]
            assert np.allclose(a, b, rtol=1e-10, atol=1e-12)
        assert np.array_equal(out[3].cpu().numpy()[ins], ref[3].cpu().numpy()[ins])
        assert cnt.total_walks == int(ins.sum()) * walks


@pytest.mark.parametrize("method", ["fast", "plain"])
def test_first_noalloc_call_on_a_new_context_reserves_nothing(method):
    """The static array is reserved when a context is created (the context
    takes its address then), so not even the first call on a context changes
    the device's free memory.  The kernels are loaded beforehand by one regular
    solve, whose own buffers are allocated then."""
    torch = pytest.importorskip("torch")
    from walk_on_spheres_b200 import Solver
    with Solver(0) as s:
        s.set_mesh(meshes.annulus())
        grid = s.grid_over_mesh(24, 24, 1)
        n = 24 * 24
        walks = 500 if method == "fast" else 100
        warm = _outputs(torch, n)
        s.solve_grid_device("laplace", grid, *[t.data_ptr() for t in warm], N_walks=walks,
                            seed=5, method=method)
        out = _outputs(torch, n)
        params = s.params("laplace", N_walks=walks, seed=5, method=method)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(0)[0]
        cnt = _lib.Counters()
        rc = _noalloc_fn()(s._ctx, C.byref(params), C.byref(grid), *[t.data_ptr() for t in out],
                           C.byref(cnt))
        assert rc == 0, _lib.lib().wos_last_error(s._ctx)
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info(0)[0] == free_before
        assert np.array_equal(out[4].cpu().numpy(), warm[4].cpu().numpy())


def test_noalloc_checks_arguments_like_the_device_entry_point(solver):
    """Non-finite grid bounds, a non-finite alpha and a bad source mode are
    rejected by both entry points with the same rule."""
    solver.set_mesh(meshes.annulus())
    f = _noalloc_fn()
    good = solver.grid_over_mesh(8, 8, 1)
    bad_grid = _lib.Grid(8, 8, 1, float("nan"), 1.0, -1.0, 1.0, 0.0, 0.0)
    cases = [(solver.params("laplace", N_walks=10, method="fast"), bad_grid),
             (solver.params("screened_poisson", N_walks=10, alpha=float("inf"), method="fast"),
              good),
             (solver.params("poisson", N_walks=10, source_mode=2, method="fast"), good)]
    L = _lib.lib()
    for params, grid in cases:
        rc_ref = L.wos_solve_grid_device(solver._ctx, C.byref(params), C.byref(grid), None, None,
                                         None, None, None, None)
        rc = f(solver._ctx, C.byref(params), C.byref(grid), None, None, None, None, None, None)
        assert rc_ref == rc == 1
    # laplace ignores the source mode on both
    params = solver.params("laplace", N_walks=10, source_mode=2, method="fast")
    assert f(solver._ctx, C.byref(params), C.byref(good), None, None, None, None, None, None) == 0


def test_noalloc_rejects_grids_beyond_the_scratch(solver):
    solver.set_mesh(meshes.annulus())
    grid = solver.grid_over_mesh(400, 400, 1)  # 160 000 points > about 94 000
    params = solver.params("laplace", N_walks=10, seed=1, method="fast")
    rc = _noalloc_fn()(solver._ctx, C.byref(params), C.byref(grid), None, None, None, None, None,
                       None)
    assert rc == 1
    assert b"static" in _lib.lib().wos_last_error(solver._ctx)
