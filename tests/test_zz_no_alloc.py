"""bsn_cfl_dt_3d_f64_noalloc: the CFL time step for callers that may not
allocate GPU memory (a host runtime that owns a fixed device-memory pool, or
a job that sizes all of its memory at start-up), whose scratch is a static
device array inside libbsn instead of a cudaMalloc'd workspace.

Called through the C ABI with ctypes and compared with the regular
bsn_cfl_dt_3d_f64 on the same states, two calls in a row; dt is a maximum
followed by one division, so the two must agree exactly (the tolerance the
other dt tests use).  This file is collected last so that a failure here
cannot stop the rest of the GPU suite from running first.
"""
import ctypes as C

import numpy as np
import pytest

from gpu_util import dev, random_state

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _ctx_and_lib():
    import bsn
    from bsn._lib import load
    return bsn.context(), load()


def _dt(L, fn, ctx, U, n, d, gamma=1.4, cfl=0.4):
    out = C.c_double(-1.0)
    rc = getattr(L, fn)(ctx, C.c_void_p(U.data_ptr()), *n, *d, gamma, cfl, C.byref(out))
    assert rc == 0, L.bsn_last_error(ctx).decode()
    return out.value


def test_noalloc_cfl_matches_regular_entry_two_calls_in_a_row():
    ctx, L = _ctx_and_lib()
    cases = [((24, 9, 17), (0.1, 0.07, 0.13), random_state(24, 9, 17, seed=11)),
             ((40, 33, 21), (0.05, 0.05, 0.05), random_state(40, 33, 21, seed=12, jumps=False))]
    for n, d, U in cases:
        Ud = dev(U)
        first = _dt(L, "bsn_cfl_dt_3d_f64_noalloc", ctx, Ud, n, d)
        second = _dt(L, "bsn_cfl_dt_3d_f64_noalloc", ctx, Ud, n, d)
        ref = _dt(L, "bsn_cfl_dt_3d_f64", ctx, Ud, n, d)
        assert np.isfinite(ref) and ref > 0
        assert first == ref and second == ref


def test_noalloc_cfl_reserves_no_device_memory():
    # A fresh context has no workspace yet.  After one warm-up call (which,
    # under lazy module loading, lets the driver place the static array),
    # further calls must leave the device's free memory unchanged: no
    # cudaMalloc, and no workspace slot created behind the caller's back.
    import bsn
    from bsn._lib import load
    L = load()
    bsn.context()
    torch.cuda.set_device(0)
    U = dev(random_state(32, 24, 16, seed=15))
    torch.cuda.synchronize()
    ctx = C.c_void_p()
    assert L.bsn_ctx_create(C.byref(ctx), 0, C.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
    try:
        n, d = (32, 24, 16), (0.1, 0.1, 0.1)
        warm = _dt(L, "bsn_cfl_dt_3d_f64_noalloc", ctx, U, n, d)
        free_before, _ = torch.cuda.mem_get_info()
        got = [_dt(L, "bsn_cfl_dt_3d_f64_noalloc", ctx, U, n, d) for _ in range(4)]
        free_after, _ = torch.cuda.mem_get_info()
        assert free_after == free_before, (free_before, free_after)
        assert all(g == warm for g in got)
        assert got[0] == _dt(L, "bsn_cfl_dt_3d_f64", ctx, U, n, d)
    finally:
        L.bsn_ctx_destroy(ctx)


def test_noalloc_cfl_nan_state_gives_inf_like_the_reference():
    ctx, L = _ctx_and_lib()
    U = random_state(16, 8, 8, seed=13)
    U[0, 5, 5, 5] = np.nan
    Ud = dev(U)
    assert _dt(L, "bsn_cfl_dt_3d_f64_noalloc", ctx, Ud, (16, 8, 8), (0.1, 0.1, 0.1)) == np.inf
    assert _dt(L, "bsn_cfl_dt_3d_f64", ctx, Ud, (16, 8, 8), (0.1, 0.1, 0.1)) == np.inf


def test_noalloc_cfl_rejects_grids_beyond_its_capacity():
    # rejected on the host before any launch, so the small buffer is never read
    ctx, L = _ctx_and_lib()
    U = dev(random_state(8, 8, 8, seed=14))
    out = C.c_double(-1.0)
    rc = L.bsn_cfl_dt_3d_f64_noalloc(ctx, C.c_void_p(U.data_ptr()), 1024, 1024, 1024, 0.1, 0.1, 0.1, 1.4, 0.4,
                                     C.byref(out))
    assert rc == 5  # BSN_ERR_UNSUPPORTED
    assert b"capacity" in L.bsn_last_error(ctx)
