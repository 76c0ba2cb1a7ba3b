"""Serving context (q2d_serve_*): continuous batching on the GPU.

* Each result is the same alone and in the mix: cases admitted at different times into a
  running context, next to other cases, end bit-for-bit where they end when served alone
  (tolerance 0: every cell update, time step and residual of a case reads only that case's
  data, and admissions compute time steps only for the new cases).
* Served results equal the batch path's (q2d_gpu_* context with the same options and steps).
* Memory-budget admission: a full context refuses with Q2D_ERR_CAPACITY and keeps running;
  retirement frees the slot and the memory for the next request.
* The request loop serves a small stream to completion and retires every case on its residual
  drop or its iteration cap.
"""
import numpy as np
import pytest

from q2d_b200 import _abi, cases
from q2d_b200.serve import Request, ServeContext, serve, serve_options
from q2d_b200.solver import Q2DSolver

pytestmark = pytest.mark.gpu

BUDGET = 256 << 20


def small_requests():
    rng = np.random.default_rng(123)
    return [cases.request_case("ramp", 800, rng), cases.request_case("nozzle", 640, rng),
            cases.request_case("ramp", 1500, rng), cases.request_case("nozzle", 2000, rng)]


def run_alone(case, opts, steps):
    with ServeContext(opts, BUDGET, 4) as sc:
        cid = sc.admit(case)
        assert cid is not None
        sc.step_async(steps)
        infos = sc.wait()
        return [sc.prim(cid, b) for b in range(len(case.blocks))], infos[cid]


@pytest.mark.parametrize("precision", [_abi.PREC_FP64, _abi.PREC_FP32_FLUX])
def test_alone_equals_in_mix(precision):
    reqs = small_requests()
    steps = 24
    opts = serve_options(precision=precision, itermax=steps, drop=1e-30)
    alone = [run_alone(c, opts, steps + 10) for c in reqs]
    # mix: admissions staggered over the run; every case stops at its own itermax
    with ServeContext(opts, BUDGET, 8) as sc:
        ids = [sc.admit(reqs[0])]
        sc.step_async(5); sc.wait()
        ids.append(sc.admit(reqs[1]))
        ids.append(sc.admit(reqs[2]))
        sc.step_async(7); sc.wait()
        ids.append(sc.admit(reqs[3]))
        for _ in range(6):
            sc.step_async(6)
            infos = sc.wait()
        for k, (cid, c) in enumerate(zip(ids, reqs)):
            inf = infos[cid]
            assert inf.iter == steps and inf.todo == _abi.TODO_END and inf.err == 0
            a_state, a_inf = alone[k]
            for b in range(len(c.blocks)):
                m = sc.prim(cid, b)
                assert np.array_equal(m, a_state[b]), f"case {k} block {b}: in-mix result differs from alone"
            assert inf.residual[0] == a_inf.residual[0] and inf.dtglobal == a_inf.dtglobal


def test_multiblock_axisymmetric_alone_equals_in_mix():
    a = cases.nozzle_axi(ni=40, nj=12, nblocks=2, seed=21)
    b = cases.nozzle_axi(ni=32, nj=10, nblocks=3, seed=22)
    opts = _abi.default_options(**dict(a.options, itermax=15, res_threshold=0.0, sol_diter=10 ** 9))
    alone_b = run_alone(b, opts, 20)
    with ServeContext(opts, BUDGET, 4) as sc:
        ia = sc.admit(a)
        sc.step_async(4); sc.wait()
        ib = sc.admit(b)
        for _ in range(4):
            sc.step_async(5)
            infos = sc.wait()
        assert infos[ia].iter == 15 and infos[ib].iter == 15
        for k in range(3):
            assert np.array_equal(sc.prim(ib, k), alone_b[0][k])


def test_served_equals_batch_path():
    reqs = small_requests()[:2]
    opts = serve_options(precision=_abi.PREC_FP32_FLUX, itermax=12, drop=1e-30)
    g = Q2DSolver(opts, reqs)
    try:
        g.step(12)
        batch = [g.prim(c, 0) for c in range(len(reqs))]
    finally:
        g.close()
    with ServeContext(opts, BUDGET, 4) as sc:
        ids = [sc.admit(c) for c in reqs]
        sc.step_async(12)
        sc.wait()
        for k, cid in enumerate(ids):
            assert np.array_equal(sc.prim(cid, 0), batch[k])


def test_capacity_admission_and_retire():
    rng = np.random.default_rng(5)
    big = cases.request_case("nozzle", 60000, rng)
    opts = serve_options(itermax=5)
    # a budget for about 1.5 of these cases
    budget = int(1.5 * big.cells * 306)
    with ServeContext(opts, budget, 4) as sc:
        c0 = sc.admit(big)
        assert c0 is not None
        assert sc.admit(big) is None            # memory exhausted: refused, nothing kept
        sc.step_async(5)
        infos = sc.wait()
        assert infos[c0].iter == 5 and infos[c0].todo == _abi.TODO_END
        sc.retire(c0)
        c1 = sc.admit(big)
        assert c1 is not None
        sc.step_async(5)
        infos = sc.wait()
        assert infos[c1].iter == 5 and infos[c1].err == 0
    # slots exhausted
    small = cases.request_case("ramp", 500, rng)
    with ServeContext(opts, BUDGET, 2) as sc:
        assert sc.admit(small) is not None and sc.admit(small) is not None
        assert sc.admit(small) is None


def test_request_loop_small_stream():
    rng = np.random.default_rng(9)
    reqs = [Request(k, 0.002 * k, kind, cells, int(rng.integers(1 << 31)))
            for k, (kind, cells) in enumerate([("ramp", 900), ("nozzle", 1200), ("ramp", 3000),
                                               ("nozzle", 700), ("ramp", 2000), ("nozzle", 5000)])]
    opts = serve_options(itermax=300, drop=1e-3)
    st = serve(reqs, opts, device_bytes=int(2 * 5000 * 306 + (1 << 20)), max_cases=3, steps_per_call=10,
               realtime=False)
    assert st["served"] == len(reqs) and st["errors"] == 0 and st["rejected"] == 0
    for r in reqs:
        assert r.iters <= 300 and (r.iters == 300 or r.residual_drop <= 1e-3)
    assert st["cell_updates"] > 0 and st["p99_latency_s"] >= st["p50_latency_s"] > 0


@pytest.mark.parametrize("precision", [_abi.PREC_FP64, _abi.PREC_FP32_FLUX])
@pytest.mark.parametrize("kw", [dict(shock_detector=1, riemann="HLLE", irs_beta=0.5), dict(riemann="HLLC+"),
                                dict(riemann="AUSM+")])
def test_serving_with_sensor_and_other_solvers(precision, kw):
    """The serving context on the shock-sensor instantiations, HLLC+ and a run-time selected
    solver (with IRS for the first): every case in the mix, admitted while others run, ends
    with the state it reaches alone."""
    reqs = small_requests()
    steps = 12
    opts = serve_options(precision=precision, itermax=steps, drop=1e-30, **kw)
    alone = [run_alone(c, opts, steps + 4) for c in reqs]
    with ServeContext(opts, BUDGET, 8) as sc:
        ids = [sc.admit(reqs[0]), sc.admit(reqs[1])]
        sc.step_async(4); sc.wait()
        ids += [sc.admit(reqs[2]), sc.admit(reqs[3])]
        for _ in range(4):
            sc.step_async(4)
            infos = sc.wait()
        for k, (cid, c) in enumerate(zip(ids, reqs)):
            assert infos[cid].iter == steps and infos[cid].err == 0
            for b in range(len(c.blocks)):
                assert np.array_equal(sc.prim(cid, b), alone[k][0][b]), (kw, k, b)


def test_case_end_inside_a_multi_step_call():
    """q2d_gpu_set_case_end: a served case with its own end stops at exactly that iteration
    inside a 20-step call, its state equal to the same case served alone for that many steps,
    while the case next to it runs the whole call; the request loop's end budget lands on the
    first iteration at which cells x iterations reach it."""
    rng = np.random.default_rng(31)
    a, b = cases.request_case("ramp", 900, rng), cases.request_case("nozzle", 1200, rng)
    opts = serve_options(itermax=1000, drop=1e-12)
    ref, _ = run_alone(a, opts, 7)
    with ServeContext(opts, BUDGET, 4) as sc:
        ca, cb = sc.admit(a), sc.admit(b)
        sc.set_end(ca, 7)
        sc.step_async(20)
        infos = sc.wait()
        assert infos[ca].iter == 7 and infos[ca].todo == _abi.TODO_END and infos[ca].err == 0
        assert infos[cb].iter == 20 and infos[cb].todo != _abi.TODO_END
        assert np.array_equal(sc.prim(ca, 0), ref[0])
    reqs = [Request(k, 0.0, kind, cells, int(rng.integers(1 << 31)))
            for k, (kind, cells) in enumerate([("ramp", 900), ("nozzle", 1300), ("ramp", 2100)])]
    st = serve(reqs, opts, device_bytes=int(3 * 2100 * 306 + (1 << 20)), max_cases=3, steps_per_call=50,
               realtime=False, end_cell_updates=40000)
    for r in reqs:
        cells = r.build().cells   # the built grid's cells (near the requested number)
        end = -(-40000 // cells)
        assert r.rule == "end" and r.iters == end == r.meta["end_iter"], (cells, r.iters, end)
    assert st["retired_by"]["end"] == 1.0


def test_admission_and_retirement_while_steps_run():
    """Admissions during a step call copy their images on the context's copy stream while the
    steps run, retirements during a call wait for it; cases admitted while others run, and after
    a retirement that frees a slot, end bitwise where they end alone."""
    a, b, c, d = small_requests()
    opts = serve_options(itermax=1000, drop=1e-30)
    ref_c, _ = run_alone(c, opts, 20)
    ref_d, _ = run_alone(d, opts, 12)
    ref_a, _ = run_alone(a, opts, 32)
    budget = int((a.cells + b.cells + max(c.cells, d.cells)) * 306 * 1.3 + (1 << 20))
    with ServeContext(opts, budget, 3) as sc:
        ca, cb = sc.admit(a), sc.admit(b)
        sc.step_async(12)
        cc = sc.admit(c)                     # images copied while the 12 steps run
        assert cc is not None
        sc.wait()
        sc.step_async(8)
        sc.retire(cb)                        # waits for the 8 steps
        cd = sc.admit(d)                     # into the slot b left
        assert cd is not None
        sc.step_async(12)
        infos = sc.wait()
        assert infos[ca].iter == 32 and infos[cc].iter == 20 and infos[cd].iter == 12
        assert np.array_equal(sc.prim(ca, 0), ref_a[0])
        assert np.array_equal(sc.prim(cc, 0), ref_c[0])
        assert np.array_equal(sc.prim(cd, 0), ref_d[0])


def test_upload_after_admission_before_the_first_step():
    """q2d_gpu_upload_prim on an admitted case before its first step (its images are already
    on the copy stream) replaces the admitted state: the case then runs as if admitted with
    the uploaded state."""
    import copy
    from q2d_b200 import _abi as abi
    a = small_requests()[0]
    b = copy.deepcopy(a)
    b.blocks[0].prim[..., 3] *= 1.02
    b.blocks[0].prim[..., 1] *= 0.97
    opts = serve_options(itermax=1000, drop=1e-30)
    ref, _ = run_alone(b, opts, 6)
    with ServeContext(opts, BUDGET, 4) as sc:
        cid = sc.admit(a)
        import ctypes as C
        bid = C.c_int()
        assert sc.lib.q2d_serve_block_id(sc.ctx, cid, 1, C.byref(bid)) == abi.OK
        P = b.blocks[0].prim_ghost(ghosts=None)
        assert sc.lib.q2d_gpu_upload_prim(sc.ctx, bid.value, abi.dptr(P)) == abi.OK
        sc.step_async(6)
        sc.wait()
        assert np.array_equal(sc.prim(cid, 0), ref[0])
