"""The allocation-free residual norm (q2d_gpu_residual_norm_noalloc) against the residual that
the regular step entry point reports.

That entry point exists for callers that cannot allocate device memory when they need the
norm (their device memory is owned by their own pool, or they sit on a path that cannot take
an allocation's synchronisation): it takes only their input and output pointers and keeps its
scratch in a fixed device array. This file is collected last so that a run stopping at the
first failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12   # the per-step parity tolerance of the GPU tests


def _planes(prim, torch):
    """(nj, ni, 4) primitive state -> device tensor of 4 planes (rho, u, v, p)."""
    return torch.tensor(np.ascontiguousarray(prim.reshape(-1, 4).T), dtype=torch.float64, device="cuda")


def test_noalloc_norm_matches_step_residual_two_calls():
    import torch
    from q2d_b200 import _abi, cases, make_options
    from q2d_b200.solver import Q2DSolver

    lib = _abi.load_library()
    cs = cases.ramp(96, 40, seed=3)
    s = Q2DSolver(make_options(cs), [cs])
    try:
        stream = torch.cuda.current_stream().cuda_stream
        for _ in range(2):   # two calls in a row, each against the step it follows
            old = s.prim()
            ref = np.array(s.step(1)[0]["residual"])
            new = s.prim()
            pn, po = _planes(new, torch), _planes(old, torch)
            out = torch.full((4,), -1.0, dtype=torch.float64, device="cuda")
            st = lib.q2d_gpu_residual_norm_noalloc(pn.data_ptr(), po.data_ptr(), cs.cells, cs.cells,
                                                   out.data_ptr(), C.c_void_p(stream))
            assert st == 0
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert np.all(ref > 0)
            assert np.allclose(got, ref, rtol=RTOL, atol=0.0), (got, ref)
    finally:
        s.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    from q2d_b200 import _abi

    lib = _abi.load_library()
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    limit = 8192 * 2048   # Q2D_NOALLOC_MAX_PARTIALS * Q2D_NOALLOC_CELLS_PER_PARTIAL
    # rejected on the host before anything is launched
    assert lib.q2d_gpu_residual_norm_noalloc(x.data_ptr(), x.data_ptr(), limit + 1, limit + 1,
                                             x.data_ptr(), None) == _abi.ERR_CAPACITY
    assert lib.q2d_gpu_residual_norm_noalloc(x.data_ptr(), x.data_ptr(), 0, 1, x.data_ptr(), None) == _abi.ERR_BADARG


def _numpy_norms(new, old, n):
    d = new[:, :n] - old[:, :n]
    return np.sqrt((d * d).sum(axis=1))


@pytest.mark.parametrize("ncells,stride", [
    (3 * 2048, 3 * 2048 + 37),        # padded planes: the padding holds garbage
    (5 * 2048, 5 * 2048),             # last chunk exactly full
    (5 * 2048 + 1, 5 * 2048 + 64),    # one cell in the last chunk, padded
    (8192 * 2048, 8192 * 2048),       # the largest accepted size
])
def test_noalloc_sizes_and_strides_against_numpy(ncells, stride):
    import torch
    from q2d_b200 import _abi

    lib = _abi.load_library()
    rng = np.random.default_rng(ncells)
    old = rng.standard_normal((4, stride))
    new = old + rng.standard_normal((4, stride)) * np.array([[1e-3], [1.0], [0.5], [1e3]])
    old[:, ncells:] = np.nan   # padding beyond ncells is never read
    new[:, ncells:] = 1e300
    pn = torch.tensor(new, dtype=torch.float64, device="cuda")
    po = torch.tensor(old, dtype=torch.float64, device="cuda")
    ref = _numpy_norms(new, old, ncells)
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):   # two calls in a row share the scratch array
        out = torch.full((4,), -1.0, dtype=torch.float64, device="cuda")
        st = lib.q2d_gpu_residual_norm_noalloc(pn.data_ptr(), po.data_ptr(), ncells, stride,
                                               out.data_ptr(), C.c_void_p(stream))
        assert st == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.allclose(got, ref, rtol=RTOL, atol=0.0), (got, ref)
