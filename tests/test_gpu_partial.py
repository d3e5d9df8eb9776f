"""Partially saturated bounce-back (PSBounceBackPolicy<2>) on wet obstacles.

Walls keep plain bounce-back; every wet obstacle mixes the relaxed reflection
of the population it receives with the previous value of its fluid
neighbour's slot.  The FP64 CUDA path equals the C oracle bit for bit (the
oracle itself equals the reference, tests/test_oracle.py), with the
reference's b = 1 and with per-obstacle b values.
"""
import numpy as np
import pytest

import harness as H
from test_gpu_parity import run_gpu

pytestmark = pytest.mark.gpu


def cases():
    ch = H.classify(H.channel_types(40, 90, discs=[(20, 30, 7), (12, 62, 4)]))
    yield ("channel_bgk_pressure", ch, H.Params(tau=0.7, outlet_bc=H.BC_ZH_PRESSURE, obstacle_bc=1, ps_tau=0.55),
           "parabolic:0.04:1:38", "pressure")
    yield ("channel_trt_zh", ch, H.Params.trt_magic(0.6, obstacle_bc=1, ps_tau=0.8), "const:0.03:0", "const:0.03:0")
    cav = H.cavity_types(48)
    ii, jj = np.mgrid[0:48, 0:48]
    cav[((ii - 24) ** 2 + (jj - 24) ** 2 <= 64) & (cav == H.FLUID)] = H.OBSTACLE
    cl = H.classify(cav)
    yield "cavity_disc_trt_ramp", cl, H.Params.trt_magic(0.6, obstacle_bc=1, ps_tau=0.51), "lidramp:0.1:0.002", \
        "const:0:0"
    por = H.classify(H.porous_types(64, 96, fraction=0.25, rmin=2, rmax=5, seed=4))
    b = np.random.default_rng(7).uniform(0.0, 1.0, len(por.obstacle))
    yield ("porous_bgk_open_b", por, H.Params(tau=0.8, outlet_bc=H.BC_OPEN, obstacle_bc=1, ps_tau=0.6, obstacle_b=b),
           "const:0.02:0", "const:0:0")


CASES = list(cases())


@pytest.mark.parametrize("steps", [1, 2, 7, 100, 400])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_partially_saturated_f64_bit_exact(case, steps):
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


def test_partially_saturated_limits():
    """FP64 storage, the one-thread-per-node kernel and single lattices only."""
    import llalbm_cuda as L

    name, lists, p, ins, outs = CASES[0]
    kw = dict(collision=p.collision, tau=p.tau, outlet_bc=p.outlet_bc, obstacle_bc=1, ps_tau=p.ps_tau)
    args = (lists.rows, lists.cols, lists.fluid, lists.wall, lists.inlet, lists.inlet_side, lists.outlet,
            lists.outlet_side, lists.obstacle, lists.obstacle_dirs)
    with pytest.raises(L.LLBError) as e:
        L.CudaLattice(*args, storage=L.STORE_F32S, **kw)
    assert e.value.code == -8
    with L.CudaLattice(*args, **kw) as g:
        assert g.pipeline == -1
        for cfg in (1, -2):
            with pytest.raises(L.LLBError) as e:
                g.set_pipeline(cfg)
            assert e.value.code == -8
    with L.CudaBatch(storage=L.STORE_F64) as b:
        with pytest.raises(L.LLBError) as e:
            b.add(*args, **kw)
        assert e.value.code == -8
