"""The no-allocation dense solve (v3dba_dense_cholesky_solve_noalloc) against the allocating
v3dba_dense_cholesky_solve, through the C-ABI, on two calls in a row.

The entry point exists for callers that cannot allocate device memory where they solve (a loop
that reserved its memory up front, or a framework that owns every device allocation): it works
in a fixed array compiled into the library, so the second call must not see stale state from
the first.  This file is collected last so that a failure here stops a -x run only after every
other test has run."""
import ctypes as C

import numpy as np
import pytest

from v3dsfmtoolkit_b200 import capi
from tests.helpers import rel

pytestmark = pytest.mark.gpu


def _noalloc():
    lib = capi.library()
    f = lib.v3dba_dense_cholesky_solve_noalloc
    f.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def _spd(n, seed):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(n, n))
    return A @ A.T + n * np.eye(n), rng.normal(size=n)


def test_noalloc_solve_matches_allocating_solve_twice():
    import torch
    f = _noalloc()
    # two calls in a row: a larger system first, then a smaller one, so that leftovers of the
    # first call in the shared scratch would show up in the second
    for n, seed in ((200, 1), (77, 2)):
        S, b = _spd(n, seed)
        x_ref, fail_ref = capi.dense_cholesky_solve(S, b)
        assert not fail_ref
        dS = torch.tensor(S, dtype=torch.float64, device="cuda")
        db = torch.tensor(b, dtype=torch.float64, device="cuda")
        dx = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        dfail = torch.ones(1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        rc = f(n, dS.data_ptr(), db.data_ptr(), dx.data_ptr(), dfail.data_ptr(), None)
        torch.cuda.synchronize()
        assert rc == capi.OK
        assert int(dfail.item()) == 0
        assert rel(dx.cpu().numpy(), x_ref) < 1e-10


def test_noalloc_solve_rejects_sizes_beyond_its_scratch():
    import torch
    f = _noalloc()
    n = 257
    d = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    v = torch.zeros(n, dtype=torch.float64, device="cuda")
    fl = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert f(n, d.data_ptr(), v.data_ptr(), v.data_ptr(), fl.data_ptr(), None) == capi.ERR_INVALID_ARGUMENT


def _call(f, S, b, stream=None):
    """One call through the C-ABI on device copies of S and b; x starts as NaN and fail as 1 so
    that a call which writes neither is caught.  Returns (rc, x, fail)."""
    import torch
    n = len(b)
    ctx = torch.cuda.stream(stream) if stream is not None else torch.cuda.stream(torch.cuda.current_stream())
    with ctx:
        dS = torch.tensor(S, dtype=torch.float64, device="cuda")
        db = torch.tensor(b, dtype=torch.float64, device="cuda")
        dx = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        dfail = torch.ones(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = f(n, dS.data_ptr(), db.data_ptr(), dx.data_ptr(), dfail.data_ptr(),
           stream.cuda_stream if stream is not None else None)
    torch.cuda.synchronize()
    return rc, dx.cpu().numpy(), int(dfail.item())


def test_noalloc_solve_reports_indefinite_then_recovers():
    """A matrix with a negative pivot sets the failure flag; the next call, on an SPD matrix in
    the same scratch, clears it and solves as the allocating entry point does."""
    f = _noalloc()
    S, b = _spd(150, 3)
    S_bad = S.copy()
    S_bad[120, 120] = -5.0
    x_ref_bad, fail_ref = capi.dense_cholesky_solve(S_bad, b)
    assert fail_ref
    rc, _, fail = _call(f, S_bad, b)
    assert rc == capi.OK and fail == 1
    x_ref, fail_ref = capi.dense_cholesky_solve(S, b)
    assert not fail_ref
    rc, x, fail = _call(f, S, b)
    assert rc == capi.OK and fail == 0
    assert rel(x, x_ref) < 1e-10


def test_noalloc_solve_on_a_caller_stream():
    """The work is enqueued on the stream the caller passes (here a non-default torch stream)."""
    import torch
    f = _noalloc()
    s = torch.cuda.Stream()
    for n, seed in ((256, 4), (64, 5)):
        S, b = _spd(n, seed)
        x_ref, _ = capi.dense_cholesky_solve(S, b)
        rc, x, fail = _call(f, S, b, stream=s)
        assert rc == capi.OK and fail == 0
        assert rel(x, x_ref) < 1e-10
