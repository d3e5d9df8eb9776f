"""Solve server: continuous batching of requests that arrive while others run.

Every request's result must be the same whether it is served alone or in a
mix with others that join and leave around it: FP64 bit for bit, and equal to
the oracle's rho and u after the same number of steps (the reference's
Lattice after perform_lbm(steps)); the shifted FP32 form within 1e-6 relative
L2 of its own result alone.  Admission keeps the device bytes in use under the
budget, and requests that arrive while others run are admitted before those
finish (their work overlaps).
"""
import threading
import time

import numpy as np
import pytest

import harness as H

pytestmark = pytest.mark.gpu


def requests():
    """(name, lists, params, inlet spec, outlet spec, steps): sizes, BGK/TRT,
    velocity/pressure/open outlets, a time-varying lid, uneven step counts."""
    out = []
    cav = H.classify(H.cavity_types(64))
    out.append(("cavity64_bgk", cav, H.Params(tau=0.7), "const:0.08:0", "const:0:0", 240))
    ch = H.classify(H.channel_types(48, 96, discs=[(24, 30, 6), (12, 60, 4)]))
    out.append(("channel_trt_pressure", ch, H.Params.trt_magic(0.56, outlet_bc=H.BC_ZH_PRESSURE),
                "parabolic:0.05:1:46", "pressure", 333))
    ch2 = H.classify(H.channel_types(40, 200, discs=[(20, 25, 5), (15, 120, 6)]))
    out.append(("channel_bgk_open", ch2, H.Params(tau=1.2, outlet_bc=H.BC_OPEN), "const:0.04:0", "const:0:0", 57))
    por = H.classify(H.porous_types(128, 160, seed=11))
    out.append(("porous_bgk_pressure", por, H.Params(tau=0.8, outlet_bc=H.BC_ZH_PRESSURE), "const:0.02:0",
                "pressure", 410))
    cav2 = H.classify(H.cavity_types(96))
    out.append(("cavity96_trt_ramp", cav2, H.Params.trt_magic(0.6), "lidramp:0.15:0.001", "const:0:0", 175))
    out.append(("cavity64_two_steps", cav, H.Params(tau=0.9), "const:0.05:0", "const:0:0", 2))
    return out


REQS = requests()


def table(req):
    name, lists, p, ins, outs, steps = req
    t = H.open_values(lists, ins, outs, steps + 2)
    if p.inlet_bc == H.BC_ZH_PRESSURE:
        t[:, : len(lists.inlet)] = (p.rho_out, p.tangential_u)
    if p.outlet_bc == H.BC_ZH_PRESSURE:
        t[:, len(lists.inlet):] = (p.rho_out, p.tangential_u)
    return t


def submit(server, req):
    name, lists, p, ins, outs, steps = req
    return server.submit(lists.rows, lists.cols, lists.fluid, lists.wall, lists.inlet, lists.inlet_side,
                         lists.outlet, lists.outlet_side, lists.obstacle, lists.obstacle_dirs, steps=steps,
                         collision=p.collision, tau=p.tau, tau_even=p.tau_even, tau_odd=p.tau_odd,
                         inlet_bc=p.inlet_bc, outlet_bc=p.outlet_bc, open_values=table(req))


def serve_alone(L, storage, mode=None):
    out = []
    mode = L.SERVE_BATCHED if mode is None else mode
    with L.CudaServer(storage=storage, mode=mode, budget_bytes=8 << 30) as s:
        for req in REQS:
            rid = submit(s, req)
            s.wait(rid, 120)
            out.append(s.result(rid))
    return out


def serve_mix(L, storage, budget, gap_s=0.004, order=None):
    """Submits every request from a second thread, gap_s apart; returns the
    results in REQS order and the peak device bytes seen by a poller."""
    order = list(range(len(REQS))) if order is None else order
    ids = {}
    peak = [0]
    with L.CudaServer(storage=storage, budget_bytes=budget, max_chunk_steps=32) as s:
        def feeder():
            for q in order:
                ids[q] = submit(s, REQS[q])
                time.sleep(gap_s)
        th = threading.Thread(target=feeder)
        th.start()
        done = False
        while not done:
            st = s.stats()
            peak[0] = max(peak[0], st["bytes_in_use"])
            done = not th.is_alive() and st["completed"] + st["failed"] == len(REQS)
            time.sleep(0.0005)
        th.join()
        res = {}
        for q in order:
            s.wait(ids[q], 120)
            res[q] = s.result(ids[q])
        stats = s.stats()
    return [res[q] for q in range(len(REQS))], peak[0], stats


def test_served_f64_equals_oracle_alone_and_in_the_mix():
    import llalbm_cuda as L

    alone = serve_alone(L, L.STORE_F64)
    for (rho, u, _), req in zip(alone, REQS):
        name, lists, p, ins, outs, steps = req
        ref = H.run_oracle(lists, p, steps, H.open_values(lists, ins, outs, steps))
        np.testing.assert_array_equal(rho, ref["rho"], err_msg=name)
        np.testing.assert_array_equal(u, ref["u"], err_msg=name)
    # budget for about two of the larger lattices (admission reserves an upper
    # bound of a lattice's bytes, compacted planes included: 5.6 MiB for the
    # porous one, 3.3 MiB for the next): admission is gated, the rest queue
    mixed, peak, stats = serve_mix(L, L.STORE_F64, budget=9 << 20, order=[3, 0, 4, 1, 5, 2])
    assert stats["completed"] == len(REQS) and stats["failed"] == 0
    assert 0 < peak <= 9 << 20
    for (rho_a, u_a, _), (rho_m, u_m, _), req in zip(alone, mixed, REQS):
        np.testing.assert_array_equal(rho_m, rho_a, err_msg=req[0])
        np.testing.assert_array_equal(u_m, u_a, err_msg=req[0])


def test_served_f32s_alone_equals_mix():
    import llalbm_cuda as L

    alone = serve_alone(L, L.STORE_F32S)
    mixed, _, stats = serve_mix(L, L.STORE_F32S, budget=1 << 30)
    assert stats["failed"] == 0
    for (rho_a, u_a, _), (rho_m, u_m, _), req in zip(alone, mixed, REQS):
        err = np.sqrt(((u_m - u_a) ** 2).sum() / max((u_a ** 2).sum(), 1e-30))
        assert err <= 1e-6, (req[0], err)
        assert np.abs(rho_m - rho_a).max() <= 1e-6, req[0]


def test_sequential_plain_f64_equals_batched():
    import llalbm_cuda as L

    seq = serve_alone(L, L.STORE_F64, mode=L.SERVE_SEQUENTIAL)
    bat = serve_alone(L, L.STORE_F64)
    for (rho_s, u_s, _), (rho_b, u_b, _), req in zip(seq, bat, REQS):
        np.testing.assert_array_equal(rho_s, rho_b, err_msg=req[0])
        np.testing.assert_array_equal(u_s, u_b, err_msg=req[0])


def test_arrivals_overlap_running_requests():
    """A request submitted while a long one runs is admitted and finished
    before the long one ends, when the budget has room."""
    import llalbm_cuda as L

    long_req = REQS[3][:5] + (20000,)
    short_req = REQS[0]
    with L.CudaServer(storage=L.STORE_F32S, budget_bytes=1 << 30, max_chunk_steps=64) as s:
        a = submit(s, long_req)
        while s.state(a) != L.REQ_RUNNING:
            time.sleep(0.0005)
        b = submit(s, short_req)
        s.wait(b, 120)
        s.wait(a, 120)
        _, _, ta = s.result(a, fields=False)
        _, _, tb = s.result(b, fields=False)
    assert tb[1] < ta[2] and tb[2] < ta[2]


def test_budget_gates_admission_and_rejects_oversize():
    import llalbm_cuda as L

    big = REQS[3]
    with L.CudaServer(storage=L.STORE_F64, budget_bytes=1 << 20) as s:
        with pytest.raises(L.LLBError) as e:
            submit(s, big)
        assert e.value.code == -3
    # budget for one lattice at a time (5.6 MiB reserved for each, about as
    # much held once created): the second waits for the first
    with L.CudaServer(storage=L.STORE_F64, budget_bytes=8 << 20) as s:
        a = submit(s, big)
        b = submit(s, big)
        s.wait(a, 120)
        s.wait(b, 120)
        _, _, ta = s.result(a, fields=False)
        _, _, tb = s.result(b, fields=False)
    assert tb[1] >= ta[2]


def test_destroy_with_queued_requests_returns():
    import llalbm_cuda as L

    s = L.CudaServer(storage=L.STORE_F32S, budget_bytes=8 << 20)
    ids = [submit(s, REQS[3]) for _ in range(6)]
    s.close()
    assert len(ids) == 6


def test_small_lane_is_not_held_to_the_large_lattices_step_rate():
    """Lattices of 2^20 nodes or more run in their own lane: a small request
    with more steps than a large one that runs beside it still finishes
    first, and both results are bit for bit those of each request alone (and,
    for the large one, of the plain path)."""
    import llalbm_cuda as L

    big = ("cavity1024", H.classify(H.cavity_types(1024)), H.Params(tau=0.8), "const:0.05:0", "const:0:0", 10000)
    small = ("cavity64_long", REQS[0][1], H.Params(tau=0.7), "const:0.08:0", "const:0:0", 12000)
    alone = {}
    with L.CudaServer(storage=L.STORE_F64, budget_bytes=8 << 30) as s:
        for req in (big, small):
            rid = submit(s, req)
            s.wait(rid, 300)
            alone[req[0]] = s.result(rid)
    with L.CudaServer(storage=L.STORE_F64, mode=L.SERVE_SEQUENTIAL, budget_bytes=8 << 30) as s:
        rid = submit(s, big)
        s.wait(rid, 300)
        plain_big = s.result(rid)
    with L.CudaServer(storage=L.STORE_F64, budget_bytes=8 << 30) as s:
        a = submit(s, big)
        while s.state(a) != L.REQ_RUNNING:
            time.sleep(0.0005)
        b = submit(s, small)
        s.wait(b, 300)
        s.wait(a, 300)
        rb, ub, tb = s.result(b)
        ra, ua, ta = s.result(a)
    assert tb[2] < ta[2]
    np.testing.assert_array_equal(ra, alone["cavity1024"][0])
    np.testing.assert_array_equal(ua, alone["cavity1024"][1])
    np.testing.assert_array_equal(rb, alone["cavity64_long"][0])
    np.testing.assert_array_equal(ub, alone["cavity64_long"][1])
    np.testing.assert_array_equal(ra, plain_big[0])
    np.testing.assert_array_equal(ua, plain_big[1])


@pytest.mark.parametrize("order", ["shortest_first", "fifo"])
def test_admission_order_under_the_node_cap(order):
    """With room for one lattice at a time (resident-node cap), requests that
    queue behind a running one are admitted shortest work first (lattice
    nodes x steps) -- or in arrival order with ADMIT_FIFO."""
    import llalbm_cuda as L

    base = REQS[3]
    first, longer, shorter = base[:5] + (50000,), base[:5] + (3000,), base[:5] + (300,)
    nodes = base[1].rows * base[1].cols
    with L.CudaServer(storage=L.STORE_F32S, budget_bytes=1 << 30, max_chunk_steps=64) as s:
        s.set_admission(nodes, L.ADMIT_SHORTEST_FIRST if order == "shortest_first" else L.ADMIT_FIFO)
        a = submit(s, first)
        while s.state(a) != L.REQ_RUNNING:
            time.sleep(0.0005)
        b = submit(s, longer)
        c = submit(s, shorter)
        assert s.state(b) == L.REQ_QUEUED and s.state(c) == L.REQ_QUEUED
        for r in (a, b, c):
            s.wait(r, 120)
        ta, tb, tc = (s.result(r, fields=False)[2] for r in (a, b, c))
    assert tb[1] >= ta[2] and tc[1] >= ta[2]   # one lattice resident at a time
    if order == "shortest_first":
        assert tc[1] < tb[1] and tb[1] >= tc[2]
    else:
        assert tb[1] < tc[1] and tc[1] >= tb[2]
