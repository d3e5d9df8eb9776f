"""Batches: many lattices advanced by one persistent launch per step.

Every lattice of a batch must end exactly where it would alone: FP64 bit for
bit against the oracle (through the single-lattice path's semantics), under
every launch shape, with lattices joining and leaving at different times, and
after the autotuner has picked a shape.  The shifted FP32 form is compared
with its own single-lattice run within a tolerance.
"""
import numpy as np
import pytest

import harness as H

pytestmark = pytest.mark.gpu


def problems():
    """A mixed set: sizes, BGK/TRT, velocity/pressure/open outlets, time-varying lid."""
    out = []
    cav = H.classify(H.cavity_types(64))
    out.append(("cavity64_bgk", cav, H.Params(tau=0.7), "const:0.08:0", "const:0:0"))
    ch = H.classify(H.channel_types(48, 96, discs=[(24, 30, 6), (12, 60, 4)]))
    out.append(("channel_trt_pressure", ch, H.Params.trt_magic(0.56, outlet_bc=H.BC_ZH_PRESSURE),
                "parabolic:0.05:1:46", "pressure"))
    ch2 = H.classify(H.channel_types(40, 200, discs=[(20, 25, 5), (15, 120, 6)]))
    out.append(("channel_bgk_open", ch2, H.Params(tau=1.2, outlet_bc=H.BC_OPEN), "const:0.04:0", "const:0:0"))
    odd = H.channel_types(37, 53, discs=[(18, 20, 4)])
    odd[1:-1, 0] = H.BOUNDARY
    odd[:, 0] = H.INLET
    out.append(("odd_corners", H.classify(odd), H.Params.trt_magic(0.9), "const:0.03:0.01", "const:0:0"))
    cav2 = H.classify(H.cavity_types(96))
    out.append(("cavity96_trt_ramp", cav2, H.Params.trt_magic(0.6), "lidramp:0.15:0.001", "const:0:0"))
    return out


PROBLEMS = problems()


def gpu_table(lists, p, ins, outs, rows):
    t = H.open_values(lists, ins, outs, rows)
    if p.inlet_bc == H.BC_ZH_PRESSURE:
        t[:, : len(lists.inlet)] = (p.rho_out, p.tangential_u)
    if p.outlet_bc == H.BC_ZH_PRESSURE:
        t[:, len(lists.inlet):] = (p.rho_out, p.tangential_u)
    return t


def add(batch, prob, rows):
    name, lists, p, ins, outs = prob
    tab = gpu_table(lists, p, ins, outs, rows)
    return batch.add(lists.rows, lists.cols, lists.fluid, lists.wall, lists.inlet, lists.inlet_side, lists.outlet,
                     lists.outlet_side, lists.obstacle, lists.obstacle_dirs, collision=p.collision, tau=p.tau,
                     tau_even=p.tau_even, tau_odd=p.tau_odd, inlet_bc=p.inlet_bc, outlet_bc=p.outlet_bc,
                     open_values=tab)


def check_against_oracle(view, prob, steps):
    """After `steps` collisions the lattice's populations are the oracle's S_steps."""
    name, lists, p, ins, outs = prob
    ref = H.run_oracle(lists, p, steps, H.open_values(lists, ins, outs, steps))
    pop = view.populations()
    act = H.active_mask(lists)
    np.testing.assert_array_equal(pop[:, act], ref["populations"][:, act], err_msg=name)


@pytest.mark.parametrize("block_y,spl", [(1, 1), (4, 1), (8, 1), (2, 8), (4, 5)])
def test_batch_f64_bit_exact_every_shape(block_y, spl):
    import llalbm_cuda as L

    steps = 300
    with L.CudaBatch(storage=L.STORE_F64) as b:
        slots = [add(b, prob, steps + 2) for prob in PROBLEMS]
        b.set_config(block_y, spl)
        b.step(steps - 1)
        b.synchronize()
        for slot, prob in zip(slots, PROBLEMS):
            view = b.lattice(slot)
            assert view.t == steps
            check_against_oracle(view, prob, steps)


def test_batch_lattices_join_and_leave():
    import llalbm_cuda as L

    P = PROBLEMS
    with L.CudaBatch(storage=L.STORE_F64) as b:
        a = add(b, P[0], 400)
        b.step(49)                                  # a at step 50
        c = add(b, P[1], 400)
        b.step(100)                                 # a 150, c 101
        check_against_oracle(b.lattice(a), P[0], 150)
        b.remove(a)
        d = add(b, P[4], 400)                       # time-varying lid joins late
        b.step(70)                                  # c 171, d 71
        # one lattice stepped on its own, then back in the batch
        vd = b.lattice(d)
        vd.step(5)                                  # d 76
        b.step(24)                                  # c 195, d 100
        b.synchronize()
        check_against_oracle(b.lattice(c), P[1], 195)
        check_against_oracle(b.lattice(d), P[4], 100)


def test_batch_autotune_keeps_results():
    import llalbm_cuda as L

    with L.CudaBatch(storage=L.STORE_F64) as b:
        slots = [add(b, prob, 1000) for prob in PROBLEMS]
        by, spl, ms = b.tune(16)
        assert 1 <= by <= 8 and spl >= 1 and ms > 0
        t = b.t + 1                                 # steps done by every lattice (init + batch steps)
        b.step(50)
        b.synchronize()
        for slot, prob in zip(slots, PROBLEMS):
            check_against_oracle(b.lattice(slot), prob, t + 50)


def test_compute_macro_is_next_steps_macro():
    import llalbm_cuda as L

    prob = PROBLEMS[1]
    name, lists, p, ins, outs = prob
    with L.CudaBatch(storage=L.STORE_F64) as b:
        s = add(b, prob, 10)
        b.step(99)                                  # 100 collisions done
        rho, u = b.lattice(s).compute_macro()
    ref = H.run_oracle(lists, p, 101, H.open_values(lists, ins, outs, 101))  # macro of step 100
    np.testing.assert_array_equal(u, ref["u"])
    np.testing.assert_array_equal(rho, ref["rho"])


def test_batch_f32s_matches_single_lattice():
    import llalbm_cuda as L

    steps = 500
    singles = []
    for name, lists, p, ins, outs in PROBLEMS:
        tab = gpu_table(lists, p, ins, outs, steps + 2)
        with L.CudaLattice(lists.rows, lists.cols, lists.fluid, lists.wall, lists.inlet, lists.inlet_side,
                           lists.outlet, lists.outlet_side, lists.obstacle, lists.obstacle_dirs, collision=p.collision,
                           tau=p.tau, tau_even=p.tau_even, tau_odd=p.tau_odd, inlet_bc=p.inlet_bc,
                           outlet_bc=p.outlet_bc, storage=L.STORE_F32S, open_table_rows=tab.shape[0]) as g:
            g.set_open_values(tab)
            g.init()
            g.step(steps - 1)
            singles.append(g.compute_macro()[1])
    with L.CudaBatch(storage=L.STORE_F32S) as b:
        slots = [add(b, prob, steps + 2) for prob in PROBLEMS]
        b.step(steps - 1)
        for slot, u1, prob in zip(slots, singles, PROBLEMS):
            u = b.lattice(slot).compute_macro()[1]
            err = np.sqrt(((u - u1) ** 2).sum() / max((u1 ** 2).sum(), 1e-30))
            assert err <= 1e-6, (prob[0], err)


def test_large_lattices_are_items_of_the_one_work_list():
    """Lattices of 2^20 nodes or more are tiles or slot blocks of the same work
    list as the small ones (one launch per batch step): the porous channel on
    its compacted planes (its single-lattice default too), the cavity on the
    dense ones, joining at different step parities and crossing graph
    replays and single steps; every lattice stays bit-exact."""
    import llalbm_cuda as L

    por = H.classify(H.porous_types(1024, 1024, seed=5))
    cav = H.classify(H.cavity_types(1024))
    big_por = ("porous1024", por, H.Params(tau=0.8, outlet_bc=H.BC_ZH_PRESSURE), "const:0.02:0", "pressure")
    big_cav = ("cavity1024", cav, H.Params.trt_magic(0.7), "const:0.05:0", "const:0:0")
    with L.CudaLattice(por.rows, por.cols, por.fluid, por.wall, por.inlet, por.inlet_side, por.outlet,
                       por.outlet_side, por.obstacle, por.obstacle_dirs) as g:
        assert g.pipeline == -3                     # compacted planes by default
    with L.CudaLattice(cav.rows, cav.cols, cav.fluid, cav.wall, cav.inlet, cav.inlet_side, cav.outlet,
                       cav.outlet_side, cav.obstacle, cav.obstacle_dirs) as g:
        assert g.pipeline == -1                     # one thread per node
    with L.CudaBatch(storage=L.STORE_F64) as b:
        a = add(b, big_por, 200)
        s = add(b, PROBLEMS[1], 200)
        b.step(40)                                  # a, s at 41 (graph + 8 single steps)
        c = add(b, big_cav, 200)
        b.step(37)                                  # a, s 78; c 38
        b.step(33)                                  # odd batch step: the other parity's graph
        b.synchronize()
        check_against_oracle(b.lattice(a), big_por, 111)
        check_against_oracle(b.lattice(s), PROBLEMS[1], 111)
        check_against_oracle(b.lattice(c), big_cav, 71)


def test_batch_f16s_matches_single_lattice():
    import llalbm_cuda as L

    steps = 300
    singles = []
    for name, lists, p, ins, outs in PROBLEMS:
        tab = gpu_table(lists, p, ins, outs, steps + 2)
        with L.CudaLattice(lists.rows, lists.cols, lists.fluid, lists.wall, lists.inlet, lists.inlet_side,
                           lists.outlet, lists.outlet_side, lists.obstacle, lists.obstacle_dirs, collision=p.collision,
                           tau=p.tau, tau_even=p.tau_even, tau_odd=p.tau_odd, inlet_bc=p.inlet_bc,
                           outlet_bc=p.outlet_bc, storage=L.STORE_F16S, open_table_rows=tab.shape[0]) as g:
            g.set_open_values(tab)
            g.init()
            g.step(steps - 1)
            singles.append(g.compute_macro()[1])
    with L.CudaBatch(storage=L.STORE_F16S) as b:
        slots = [add(b, prob, steps + 2) for prob in PROBLEMS]
        b.step(steps - 1)
        for slot, u1, prob in zip(slots, singles, PROBLEMS):
            u = b.lattice(slot).compute_macro()[1]
            err = np.sqrt(((u - u1) ** 2).sum() / max((u1 ** 2).sum(), 1e-30))
            assert err <= 1e-6, (prob[0], err)


def test_batch_barrier_timeout_reports_and_recovers():
    """A cooperative multi-step launch whose grid barrier gives up at once
    (wait limit 0: every block but the last to arrive) reports LLB_E_TIMEOUT
    on synchronisation and leaves the barrier cleared: fresh lattices added
    to the same batch then run bit-exact with the default limit."""
    import llalbm_cuda as L

    steps = 120
    with L.CudaBatch(storage=L.STORE_F64) as b:
        slots = [add(b, prob, steps + 2) for prob in PROBLEMS]
        b.set_config(4, 8)
        b.set_wait_limit(0)
        b.step(16)
        with pytest.raises(L.LLBError) as e:
            b.synchronize()
        assert e.value.code == -9
        for s in slots:
            b.remove(s)
        b.set_wait_limit(-1)
        slots = [add(b, prob, steps + 2) for prob in PROBLEMS]
        b.step(steps - 1)
        b.synchronize()
        for slot, prob in zip(slots, PROBLEMS):
            check_against_oracle(b.lattice(slot), prob, steps)


def test_batch_stop_step_holds_a_lattice():
    """A lattice given a stop step is left as it is by later batch steps (its
    state is the oracle's at that step) while the others run on; the stop is
    set mid-run and reached inside a graph-replayed stretch."""
    import llalbm_cuda as L

    with L.CudaBatch(storage=L.STORE_F64) as b:
        slots = [add(b, prob, 400) for prob in PROBLEMS]
        b.step(10)
        b.set_stop(slots[1], 47)
        b.set_stop(slots[3], 200)
        b.step(150)
        b.set_stop(slots[3], -1)   # lifted before it was reached: runs on
        b.step(9)
        b.synchronize()
        want = {slots[1]: 47}
        for slot, prob in zip(slots, PROBLEMS):
            view = b.lattice(slot)
            steps = want.get(slot, 170)
            assert view.t == steps, (prob[0], view.t)
            check_against_oracle(view, prob, steps)


@pytest.mark.parametrize("layout", ["auto", "compact", "dense"])
def test_batch_layouts_bit_exact_and_switchable(layout):
    """Every lattice equals the oracle bit for bit whichever planes the batch
    steps it on (compacted or dense), including after the layout of the
    attached lattices changes in the middle of the run."""
    import llalbm_cuda as L

    first = {"auto": L.LAYOUT_AUTO, "compact": L.LAYOUT_COMPACT, "dense": L.LAYOUT_DENSE}[layout]
    then = L.LAYOUT_DENSE if first != L.LAYOUT_DENSE else L.LAYOUT_COMPACT
    steps = 150
    with L.CudaBatch(storage=L.STORE_F64) as b:
        b.set_layout(first)
        slots = [add(b, prob, steps + 2) for prob in PROBLEMS]
        assert b.layout == first
        b.step(61)
        b.set_layout(then)
        b.step(steps - 62)
        b.synchronize()
        for slot, prob in zip(slots, PROBLEMS):
            view = b.lattice(slot)
            assert view.t == steps
            check_against_oracle(view, prob, steps)
