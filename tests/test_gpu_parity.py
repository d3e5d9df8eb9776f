"""Parity of the CUDA path (through the C ABI) with the C oracle.

The FP64 path must equal the oracle bit for bit on populations of fluid, inlet
and outlet nodes, on u and rho, and on the post-collision state; the oracle is
itself pinned bit for bit to the reference (tests/test_oracle.py).
"""
import numpy as np
import pytest

import harness as H

pytestmark = pytest.mark.gpu


def make_gpu(lists: H.NodeLists, p: H.Params, storage=0, table_rows=1, pipeline=None):
    import llalbm_cuda as L

    g = L.CudaLattice(lists.rows, lists.cols, lists.fluid, lists.wall, lists.inlet, lists.inlet_side,
                         lists.outlet, lists.outlet_side, lists.obstacle, lists.obstacle_dirs,
                         collision=p.collision, tau=p.tau, tau_even=p.tau_even, tau_odd=p.tau_odd,
                         inlet_bc=p.inlet_bc, outlet_bc=p.outlet_bc, storage=storage,
                         open_table_rows=table_rows, obstacle_bc=p.obstacle_bc, ps_tau=p.ps_tau,
                         obstacle_b=p.obstacle_b)
    if pipeline is not None:
        g.set_pipeline(pipeline)
    return g


def pressure_table(table: np.ndarray, lists: H.NodeLists, p: H.Params) -> np.ndarray:
    """Pressure-policy nodes take (rho0, tangential u) instead of a velocity."""
    t = table.copy()
    if p.inlet_bc == H.BC_ZH_PRESSURE:
        t[:, : len(lists.inlet)] = (p.rho_out, p.tangential_u)
    if p.outlet_bc == H.BC_ZH_PRESSURE:
        t[:, len(lists.inlet):] = (p.rho_out, p.tangential_u)
    return t


def run_gpu(lists, p, steps, table, storage=0, pipeline=None):
    tab = pressure_table(table, lists, p)
    rows = tab.shape[0]
    with make_gpu(lists, p, storage=storage, table_rows=max(rows, 1), pipeline=pipeline) as g:
        if lists.n_open:
            g.set_open_values(tab, 0)
        g.init(macro=(steps == 1))
        if steps > 1:
            g.step(steps - 1, macro=True)
        pop = g.populations()
        rho, u = g.macro()
        post = g.post_collision()
        g.check_numerics()
        return {"populations": pop, "rho": rho, "u": u, "post": post, "t": g.t}


def cases():
    cav = H.classify(H.cavity_types(129))
    yield "cavity129_bgk", cav, H.Params(tau=0.884), "const:0.1:0", "const:0:0"
    cav64 = H.classify(H.cavity_types(64))
    yield "cavity64_trt_ramp", cav64, H.Params.trt_magic(0.58), "lidramp:0.15:0.001", "const:0:0"
    ch = H.classify(H.channel_types(48, 96, discs=[(24, 30, 6), (12, 60, 4)]))
    yield ("channel_trt_parabolic_pressure", ch,
           H.Params.trt_magic(0.53, outlet_bc=H.BC_ZH_PRESSURE), "parabolic:0.05:1:46", "pressure")
    ch2 = H.classify(H.channel_types(40, 80, discs=[(20, 25, 5)]))
    yield "channel_bgk_open_outlet", ch2, H.Params(tau=0.7, outlet_bc=H.BC_OPEN), "const:0.04:0", "const:0:0"
    yield "channel_trt_zh_outlet", ch2, H.Params.trt_magic(0.7), "const:0.04:0", "const:0.04:0"
    odd = H.channel_types(37, 53, discs=[(18, 20, 4)])
    odd[1:-1, 0] = H.BOUNDARY
    odd[:, 0] = H.INLET               # inlet column including both corner nodes (no closure there)
    odd[20, 30] = H.SOLID             # file-SOLID node next to fluid: its sources keep their initial value
    yield "odd_corners_solid", H.classify(odd), H.Params(tau=0.8), "const:0.03:0.01", "const:0:0"
    pres_in = H.classify(H.channel_types(30, 60, discs=[(15, 20, 4)]))
    yield ("pressure_inlet_velocity_outlet", pres_in, H.Params(tau=0.9, inlet_bc=H.BC_ZH_PRESSURE,
           rho_out=1.01), "pressure", "const:0.02:0")


CASES = list(cases())


@pytest.mark.parametrize("steps", [1, 2, 7, 100, 1000])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_f64_bit_exact(case, steps):
    name, lists, p, ins, outs = case
    table = H.open_values(lists, ins, outs, steps)
    ref = H.run_oracle(lists, p, steps, table)
    got = run_gpu(lists, p, steps, table)
    act = H.active_mask(lists)
    assert got["t"] == steps
    np.testing.assert_array_equal(got["populations"][:, act], ref["populations"][:, act])
    np.testing.assert_array_equal(got["post"][:, act], ref["post"][:, act])
    np.testing.assert_array_equal(got["u"], ref["u"])
    np.testing.assert_array_equal(got["rho"], ref["rho"])


@pytest.mark.parametrize("pipeline", [-4, -3, -2, 3, 4, 5])
@pytest.mark.parametrize("steps", [2, 7, 300])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_f64_list_and_two_step_kernels_bit_exact(case, steps, pipeline):
    """The lattice resident in one thread-block cluster (-4), the
    compacted-plane kernel (-3), the active-sector list kernel (-2) and the
    two-steps-per-launch configurations (3-5; odd step counts end with a lone
    step, 300 steps run through graph replays) on every case."""
    name, lists, p, ins, outs = case
    table = H.open_values(lists, ins, outs, steps)
    ref = H.run_oracle(lists, p, steps, table)
    got = run_gpu(lists, p, steps, table, pipeline=pipeline)
    act = H.active_mask(lists)
    np.testing.assert_array_equal(got["populations"][:, act], ref["populations"][:, act])
    np.testing.assert_array_equal(got["post"][:, act], ref["post"][:, act])
    np.testing.assert_array_equal(got["u"], ref["u"])
    np.testing.assert_array_equal(got["rho"], ref["rho"])


@pytest.mark.parametrize("pipeline", [-4, -3, -2, -1, 0, 1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("case", [CASES[2], CASES[5], CASES[6]], ids=[CASES[2][0], CASES[5][0], CASES[6][0]])
def test_f64_every_step_kernel_bit_exact(case, pipeline):
    """The cluster-resident lattice (-4), the compacted planes (-3), the
    active-sector list (-2), the one-thread-per-node kernel (-1) and every TMA
    pipeline configuration."""
    name, lists, p, ins, outs = case
    steps = 150
    table = H.open_values(lists, ins, outs, steps)
    ref = H.run_oracle(lists, p, steps, table)
    got = run_gpu(lists, p, steps, table, pipeline=pipeline)
    act = H.active_mask(lists)
    np.testing.assert_array_equal(got["populations"][:, act], ref["populations"][:, act])
    np.testing.assert_array_equal(got["u"], ref["u"])


def test_f64_pipeline_large_lattice_bit_exact():
    """A lattice with many tiles per CTA (porous 512 x 640, several tile rows and
    columns, ragged last tiles) through the pipelined kernel vs the simple one."""
    lists = H.classify(H.porous_types(500, 640, seed=3))
    p = H.Params(tau=0.8, outlet_bc=H.BC_ZH_PRESSURE)
    table = H.open_values(lists, "const:0.02:0", "pressure", 1)
    outs = []
    for pipeline in (-1, -3, -2, 0, 1, 2, 3, 4, 5, 6):
        outs.append(run_gpu(lists, p, 60, table, pipeline=pipeline))
    act = H.active_mask(lists)
    for o in outs[1:]:
        np.testing.assert_array_equal(o["populations"][:, act], outs[0]["populations"][:, act])
        np.testing.assert_array_equal(o["post"][:, act], outs[0]["post"][:, act])


def test_cavity129_10k_steps_bit_exact():
    """Config 1 (129x129 lid cavity, BGK tau 0.884, lid u = (0.1, 0)) after 10 000 steps."""
    lists = H.classify(H.cavity_types(129))
    p = H.Params(tau=0.884)
    table = H.open_values(lists, "const:0.1:0", "const:0:0", 1)
    ref = H.run_oracle(lists, p, 10000, table)
    got = run_gpu(lists, p, 10000, table)
    act = H.active_mask(lists)
    diff = np.abs(got["populations"][:, act] - ref["populations"][:, act]).max()
    assert diff <= 1e-12
    np.testing.assert_array_equal(got["populations"][:, act], ref["populations"][:, act])
    np.testing.assert_array_equal(got["u"], ref["u"])


@pytest.mark.parametrize("n,default", [(96, True), (129, False)], ids=["cavity96", "cavity129"])
@pytest.mark.parametrize("storage", [0, 1, 2], ids=["f64", "f32s", "f16s"])
def test_cluster_resident_cavity_equals_the_grid(storage, n, default):
    """A lid cavity resident in one thread-block cluster (-4; the default for
    96 x 96, chosen explicitly for config 1): runs that cross launch
    boundaries (4096 steps per launch), odd and even step counts and output
    steps in between equal the one-thread-per-node kernel bit for bit in
    every storage form."""
    lists = H.classify(H.cavity_types(n))
    p = H.Params(tau=0.884)
    table = H.open_values(lists, "const:0.1:0", "const:0:0", 1)
    plan = [(1, False), (4097, False), (3, True), (8192, False), (33, True)]
    outs = []
    for pipeline in (None if default else -4, -1):
        with make_gpu(lists, p, storage=storage, pipeline=pipeline) as g:
            assert g.pipeline == (-4 if pipeline != -1 else -1)
            g.set_open_values(table, 0)
            g.init()
            for k, macro in plan:
                g.step(k, macro=macro)
            outs.append((g.t, g.post_collision(), g.macro()))
    act = H.active_mask(lists)
    assert outs[0][0] == outs[1][0] == 1 + sum(k for k, _ in plan)
    np.testing.assert_array_equal(outs[0][1][:, act], outs[1][1][:, act])
    np.testing.assert_array_equal(outs[0][2][0], outs[1][2][0])
    np.testing.assert_array_equal(outs[0][2][1], outs[1][2][1])


@pytest.mark.parametrize("storage", [1, 2], ids=["f32s", "f16s"])
def test_cluster_resident_porous_shifted_equals_every_kernel(storage):
    """A porous channel whose slabs fit the cluster in the shifted forms
    (96 x 160, TRT, pressure outlet, uneven slab widths): the cluster-resident
    lattice gives the bits of every other kernel."""
    lists = H.classify(H.porous_types(96, 157, fraction=0.25, rmin=2, rmax=5, seed=21))
    p = H.Params.trt_magic(0.6, outlet_bc=H.BC_ZH_PRESSURE)
    table = H.open_values(lists, "const:0.03:0", "pressure", 1)
    outs = [run_gpu(lists, p, 203, table, storage=storage, pipeline=cfg) for cfg in (-1, -4, -3, -2, 0, 3, 6)]
    act = H.active_mask(lists)
    for o in outs[1:]:
        np.testing.assert_array_equal(o["post"][:, act], outs[0]["post"][:, act])
        np.testing.assert_array_equal(o["u"], outs[0]["u"])


def test_cluster_resident_refuses_what_does_not_fit():
    """A lattice whose slabs do not fit one cluster's shared memory refuses
    pipeline -4 (LLB_E_UNSUPPORTED) and keeps stepping on its kernel."""
    import llalbm_cuda as L

    lists = H.classify(H.porous_types(300, 400, seed=11))
    p = H.Params(tau=0.8, outlet_bc=H.BC_ZH_PRESSURE)
    table = H.open_values(lists, "const:0.02:0", "pressure", 1)
    with make_gpu(lists, p) as g:
        before = g.pipeline
        with pytest.raises(L.LLBError) as e:
            g.set_pipeline(-4)
        assert e.value.code == -8 and g.pipeline == before
        g.set_open_values(pressure_table(table, lists, p), 0)
        g.init()
        g.step(20, macro=True)
        got = g.post_collision()
    ref = H.run_oracle(lists, p, 21, table)
    act = H.active_mask(lists)
    np.testing.assert_array_equal(got[:, act], ref["post"][:, act])


def rel_l2(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.mark.parametrize("pipeline", [-4, -3, -2, -1, 0, 1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("storage,tol", [(1, 1e-5), (2, 5e-3)], ids=["f32s", "f16s"])
def test_shifted_storage_velocity_error(storage, tol, pipeline):
    lists = H.classify(H.channel_types(64, 160, discs=[(32, 40, 8)]))
    p = H.Params.trt_magic(0.56, outlet_bc=H.BC_ZH_PRESSURE)
    table = H.open_values(lists, "parabolic:0.05:1:62", "pressure", 1)
    steps = 2000
    ref = H.run_oracle(lists, p, steps, table)
    got = run_gpu(lists, p, steps, table, storage=storage, pipeline=pipeline)
    err = rel_l2(got["u"], ref["u"])
    assert err <= tol, err


@pytest.mark.parametrize("storage", [1, 2], ids=["f32s", "f16s"])
def test_shifted_forms_equal_across_kernels(storage):
    """Shifted storage: every step kernel (list, grid, TMA, two steps per pass)
    writes the same multiply-adds and keeps the two-step intermediate in the
    storage type, so all of them give the same bits."""
    lists = H.classify(H.porous_types(200, 300, fraction=0.25, rmin=2, rmax=6, seed=9))
    p = H.Params.trt_magic(0.6, outlet_bc=H.BC_ZH_PRESSURE)
    table = H.open_values(lists, "const:0.03:0", "pressure", 1)
    outs = [run_gpu(lists, p, 101, table, storage=storage, pipeline=cfg) for cfg in (-1, -3, -2, 0, 1, 2, 3, 4, 5, 6)]
    act = H.active_mask(lists)
    for o in outs[1:]:
        np.testing.assert_array_equal(o["post"][:, act], outs[0]["post"][:, act])
        np.testing.assert_array_equal(o["u"], outs[0]["u"])


@pytest.mark.parametrize("storage", [0, 1])
def test_tune_pipeline_steps_are_ordinary_steps(storage):
    """The autotuner runs real steps under every configuration it tries and
    keeps the fastest; the lattice then holds exactly the state of that many
    ordinary steps (FP64: the oracle's bits; FP32: a run without tuning)."""
    lists = H.classify(H.porous_types(300, 400, seed=11))
    p = H.Params(tau=0.8, outlet_bc=H.BC_ZH_PRESSURE)
    table = H.open_values(lists, "const:0.02:0", "pressure", 1)
    with make_gpu(lists, p, storage=storage) as g:
        g.set_open_values(pressure_table(table, lists, p), 0)
        g.init()
        cfg, ms = g.tune_pipeline(8)
        assert cfg in (-3, -2, -1, 0, 1, 2, 3, 4, 5, 6) and ms > 0.0 and g.pipeline == cfg
        assert g.t == 1 + 2 * 8 * 10  # init + warm-up and timed steps of all 10 configurations
        g.step(5, macro=True)
        steps = g.t
        got_pop, (got_rho, got_u) = g.post_collision(), g.macro()
    ref = H.run_oracle(lists, p, steps, table) if storage == 0 else run_gpu(lists, p, steps, table, storage=storage)
    act = H.active_mask(lists)
    np.testing.assert_array_equal(got_pop[:, act], ref["post"][:, act])
    np.testing.assert_array_equal(got_u, ref["u"])
    np.testing.assert_array_equal(got_rho, ref["rho"])


@pytest.mark.parametrize("storage", [0, 1, 2], ids=["f64", "f32s", "f16s"])
def test_compact_state_moves_between_layouts(storage):
    """Steps on the compacted planes (-3) interleaved with everything that reads
    the dense planes (populations, forces, mass, output steps) and with
    switches to other kernels and back: the state is copied across whenever
    needed, so the run equals one without switches (FP64: the oracle)."""
    lists = H.classify(H.porous_types(150, 210, seed=5))
    p = H.Params.trt_magic(0.6, outlet_bc=H.BC_ZH_PRESSURE)
    table = H.open_values(lists, "const:0.03:0", "pressure", 1)
    plan = [(-3, 7, False), (-3, 40, True), (-1, 3, False), (-3, 33, False), (1, 5, False), (-3, 1, True),
            (-3, 64, False), (-2, 2, False)]
    with make_gpu(lists, p, storage=storage) as g:
        g.set_open_values(pressure_table(table, lists, p), 0)
        g.init()
        g.set_force_points(lists.obstacle, lists.obstacle_dirs)
        for cfg, n, macro in plan:
            g.set_pipeline(cfg)
            g.step(n, macro=macro)
            g.flow_forces()
            g.mass_momentum()
        g.set_pipeline(-3)
        g.step(9, macro=True)
        steps = g.t
        got_pop, got_post, (got_rho, got_u) = g.populations(), g.post_collision(), g.macro()
    ref = H.run_oracle(lists, p, steps, table) if storage == 0 else run_gpu(lists, p, steps, table, storage=storage,
                                                                            pipeline=-1)
    act = H.active_mask(lists)
    np.testing.assert_array_equal(got_pop[:, act], ref["populations"][:, act])
    np.testing.assert_array_equal(got_post[:, act], ref["post"][:, act])
    np.testing.assert_array_equal(got_u, ref["u"])
    np.testing.assert_array_equal(got_rho, ref["rho"])


def test_flow_forces_and_gather():
    lists = H.classify(H.channel_types(48, 96, discs=[(24, 30, 6)]))
    p = H.Params.trt_magic(0.6, outlet_bc=H.BC_ZH_PRESSURE)
    table = H.open_values(lists, "parabolic:0.05:1:46", "pressure", 1)
    steps = 300
    ref = H.run_oracle(lists, p, steps, table)
    lift_ref, drag_ref = H.oracle_flow_properties(lists.rows, lists.cols, ref["post"], lists.obstacle,
                                                  lists.obstacle_dirs)
    with make_gpu(lists, p) as g:
        g.set_open_values(pressure_table(table, lists, p))
        g.init()
        g.step(steps - 1)
        g.set_force_points(lists.obstacle, lists.obstacle_dirs)
        lift, drag = g.flow_forces()
        vals = g.gather_force_inputs()
        post = g.post_collision()
    assert abs(lift - lift_ref) <= 1e-12 * max(1.0, abs(lift_ref))
    assert abs(drag - drag_ref) <= 1e-12 * max(1.0, abs(drag_ref))
    # gathered inputs are exactly the post-collision values the analyzer reads
    opp = [0, 3, 4, 1, 2, 7, 8, 5, 6]
    for q, ((i, j), b) in enumerate(zip(lists.obstacle, lists.obstacle_dirs)):
        for k in range(1, 9):
            want = ref["post"][opp[k], j + H.DJ[k], i + H.DI[k]] if (int(b) >> k) & 1 else 0.0
            assert vals[q, k - 1] == want
    np.testing.assert_array_equal(post[:, H.active_mask(lists)], ref["post"][:, H.active_mask(lists)])


def test_mass_momentum_compensated():
    lists = H.classify(H.cavity_types(96))
    p = H.Params(tau=0.7)
    table = H.open_values(lists, "const:0.08:0", "const:0:0", 1)
    ref = H.run_oracle(lists, p, 500, table)
    with make_gpu(lists, p) as g:
        g.set_open_values(table)
        g.init()
        g.step(499)
        mm = g.mass_momentum()
    act = H.active_mask(lists)
    f = ref["post"][:, act]
    import math
    mass = math.fsum(f.sum(axis=0).tolist())
    mx = math.fsum(((f[1] + f[5] + f[8]) - (f[3] + f[6] + f[7])).tolist())
    my = math.fsum(((f[2] + f[5] + f[6]) - (f[4] + f[7] + f[8])).tolist())
    assert abs(mm[0] - mass) <= 1e-12 * abs(mass)
    assert abs(mm[1] - mx) <= 1e-12 * max(1.0, abs(mx))
    assert abs(mm[2] - my) <= 1e-12 * max(1.0, abs(my))


def test_graph_replay_matches_single_launches():
    """Multi-step calls replay CUDA graphs; results must not depend on the chunking."""
    lists = H.classify(H.channel_types(40, 80, discs=[(20, 25, 5)]))
    p = H.Params(tau=0.7, outlet_bc=H.BC_OPEN)
    table = H.open_values(lists, "const:0.04:0", "const:0:0", 1)
    outs = []
    for chunks in ([199], [1] * 199, [31, 64, 33, 71]):
        with make_gpu(lists, p) as g:
            g.set_open_values(table)
            g.init()
            for c in chunks:
                g.step(c)
            outs.append(g.populations())
    np.testing.assert_array_equal(outs[0], outs[1])
    np.testing.assert_array_equal(outs[0], outs[2])


@pytest.mark.parametrize("pipeline", [-4, -1])
def test_numerics_flag(pipeline):
    """An unstable run (tau near 0.5, strong lid) is reported as LLB_E_NUMERIC."""
    import llalbm_cuda as L

    lists = H.classify(H.cavity_types(32))
    p = H.Params(tau=0.5001)
    table = H.open_values(lists, "const:0.6:0", "const:0:0", 1)
    with make_gpu(lists, p, pipeline=pipeline) as g:
        g.set_open_values(table)
        g.init()
        g.step(5000)
        with pytest.raises(L.LLBError) as e:
            g.check_numerics()
        assert e.value.code == -7


def test_cylinder_drag_lift_shifted_f32_within_a_thousandth():
    """The 1024 x 256 cylinder street (TRT magic 1/4, parabolic inlet u_max
    0.05, pressure outlet): drag and lift of the FP32-shifted form, sampled
    every 100 steps with the compensated FP64 reduction once the flow has
    developed, stay within 0.1 % of the FP64 run (drag relative to itself,
    lift relative to its amplitude)."""
    import llalbm_cuda as L

    types = H.cylinder_types()
    n = L.classify(types)
    R, C = types.shape
    ni, no = len(n["inlet"]), len(n["outlet"])
    tab = np.zeros((1, ni + no, 2))
    tab[0, :ni, 0] = [H.parabolic_u(int(i), 0.05, 1, R - 2) for i in n["inlet"][:, 0]]
    tab[0, ni:] = (1.0, 0.0)
    te = 3.0 * (0.05 * 40 / 200) + 0.5
    hist = {}
    for storage in (L.STORE_F64, L.STORE_F32S):
        with L.CudaLattice(R, C, n["fluid"], n["wall"], n["inlet"], n["inlet_side"], n["outlet"], n["outlet_side"],
                           n["obstacle"], n["obstacle_dirs"], collision=L.TRT, tau_even=te,
                           tau_odd=0.25 / (te - 0.5) + 0.5, outlet_bc=L.BC_ZH_PRESSURE, storage=storage) as g:
            g.set_open_values(tab)
            g.init()
            g.set_force_points(n["obstacle"], n["obstacle_dirs"])
            h = []
            for _ in range(160):
                g.step(100)
                h.append(g.flow_forces())
            hist[storage] = np.array(h)[80:]          # steps 8001..16001: the street has formed
    lift64, drag64 = hist[L.STORE_F64][:, 0], hist[L.STORE_F64][:, 1]
    lift32, drag32 = hist[L.STORE_F32S][:, 0], hist[L.STORE_F32S][:, 1]
    assert np.max(np.abs(drag32 - drag64) / np.abs(drag64)) <= 1e-3
    assert np.max(np.abs(lift32 - lift64)) <= 1e-3 * max(np.abs(lift64).max(), 1e-12)


@pytest.mark.parametrize("pipeline", [1, 6, 3])
def test_pipelined_wait_timeout_reports_and_recovers(pipeline):
    """The TMA (1, 6) and two-steps-per-pass (3) kernels with their stage
    waits limited to 0 polls give up at once: the flag comes back as
    LLB_E_TIMEOUT, the kernel returns after its copies in flight have landed
    (that wait keeps its full limit), and the same handle, re-initialised with
    the default limit, runs bit-exact."""
    import llalbm_cuda as L

    lists = H.classify(H.porous_types(300, 400, seed=4))
    p = H.Params(tau=0.8, outlet_bc=H.BC_ZH_PRESSURE)
    table = H.open_values(lists, "const:0.02:0", "pressure", 1)
    steps = 64
    ref = H.run_oracle(lists, p, steps, table)
    with make_gpu(lists, p, pipeline=pipeline) as g:
        g.set_open_values(pressure_table(table, lists, p), 0)
        g.init()
        g.set_wait_limit(0)
        g.step(4)
        with pytest.raises(L.LLBError) as e:
            g.check_numerics()
        assert e.value.code == -9
        g.set_wait_limit(-1)
        g.init()
        g.step(steps - 1, macro=True)
        g.check_numerics()
        pop, (rho, u) = g.populations(), g.macro()
    act = H.active_mask(lists)
    np.testing.assert_array_equal(pop[:, act], ref["populations"][:, act])
    np.testing.assert_array_equal(u, ref["u"])


def test_split_numerics_check():
    """llb_check_numerics_begin/_end report what llb_check_numerics reports,
    per slot, while later steps are already queued."""
    import llalbm_cuda as L

    lists = H.classify(H.cavity_types(32))
    with make_gpu(lists, H.Params(tau=0.7)) as g:
        g.set_open_values(H.open_values(lists, "const:0.05:0", "const:0:0", 1))
        g.init()
        for q in range(6):
            g.step(1)
            g.check_numerics_begin(q % 2)
            if q:
                g.check_numerics_end((q - 1) % 2)
        g.check_numerics_end(1)
    with make_gpu(lists, H.Params(tau=0.5001)) as g:
        g.set_open_values(H.open_values(lists, "const:0.6:0", "const:0:0", 1))
        g.init()
        g.step(5000)
        g.check_numerics_begin(3)
        g.step(10)
        with pytest.raises(L.LLBError) as e:
            g.check_numerics_end(3)
        assert e.value.code == -7
