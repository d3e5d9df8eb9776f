"""The C oracle, pinned against the reference.

Two anchors:
  * golden fixtures written by the reference itself (tests/golden/make_golden.py
    runs LLALBM's unmodified headers); these always run;
  * the live reference runner (oracle/_ref/ref_runner) on further seeded cases,
    when it has been built.
Every comparison is bit for bit on fluid, inlet and outlet populations, u, rho.
"""
import glob
import os

import numpy as np
import pytest

import harness as H

GOLDEN = sorted(glob.glob(os.path.join(H.GOLDEN, "*.npz")))


def params_from_args(args):
    """Params and update-function specs from a ref_runner argument list."""
    a = dict(zip(args[::2], args[1::2]))
    bc = {"zh": H.BC_ZH_VELOCITY, "open": H.BC_OPEN, "zhp": H.BC_ZH_PRESSURE}
    kw = dict(inlet_bc=bc[a.get("--inlet", "zh")], outlet_bc=bc[a.get("--outlet", "zh")],
              rho_out=float(a.get("--rho-out", 1.0)),
              obstacle_bc=1 if a.get("--obstacle", "bb") == "ps" else 0, ps_tau=float(a.get("--ps-tau", 0.6)))
    if a.get("--collision", "bgk") == "trt":
        p = H.Params.trt_magic(float(a["--tau-even"]), float(a.get("--magic", 0.25)), **kw)
    else:
        p = H.Params(tau=float(a.get("--tau", 0.6)), **kw)
    return p, a.get("--inlet-u", "const:0:0"), a.get("--outlet-u", "const:0:0")


def golden_lists(g) -> H.NodeLists:
    return H.NodeLists(int(g["rows"]), int(g["cols"]), g["fluid"], g["wall"][:, :2],
                       g["inlet"][:, :2], g["inlet"][:, 2].astype(np.int32),
                       g["outlet"][:, :2], g["outlet"][:, 2].astype(np.int32),
                       g["obstacle"][:, :2], g["obstacle"][:, 2].astype(np.uint16))


def assert_lists_equal(a: H.NodeLists, b: H.NodeLists):
    for f in ("fluid", "wall", "inlet", "inlet_side", "outlet", "outlet_side", "obstacle", "obstacle_dirs"):
        np.testing.assert_array_equal(np.asarray(getattr(a, f)), np.asarray(getattr(b, f)), err_msg=f)


def assert_fields_equal(lists, got, want_pop, want_u, want_rho):
    act = H.active_mask(lists)
    np.testing.assert_array_equal(got["populations"][:, act], want_pop[:, act])
    np.testing.assert_array_equal(got["u"], want_u)
    np.testing.assert_array_equal(got["rho"], want_rho)


@pytest.mark.parametrize("path", [p for p in GOLDEN if "args" in np.load(p).files],
                         ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_matches_reference_golden(path):
    g = np.load(path)
    lists = H.classify(g["types"])
    assert_lists_equal(lists, golden_lists(g))          # classification parity
    p, ins, outs = params_from_args([str(x) for x in g["args"]])
    steps = int(g["steps"])
    table = H.open_values(lists, ins, outs, steps)
    got = H.run_oracle(lists, p, steps, table)
    assert_fields_equal(lists, got, g["populations"], g["u"], g["rho"])


def test_oracle_lid129_10k_matches_reference():
    """Config 1 on the reference's own fixture test/assets/lid-lattice.txt."""
    g = np.load(os.path.join(H.GOLDEN, "lid129_bgk_10k.npz"))
    lists = H.classify(H.cavity_types(129))
    assert_lists_equal(lists, golden_lists(g))
    table = H.open_values(lists, "const:0.1:0", "const:0:0", 1)
    got = H.run_oracle(lists, H.Params(tau=0.884), 10000, table)
    assert_fields_equal(lists, got, g["populations"], g["u"], g["rho"])


def test_oracle_construction_info_golden():
    g = np.load(os.path.join(H.GOLDEN, "construct60x80_omp_trt.npz"))
    lists = H.classify(g["types"])
    assert_lists_equal(lists, golden_lists(g))
    p = H.Params.trt_magic(0.7, outlet_bc=H.BC_OPEN)
    table = H.open_values(lists, "const:0.03:0", "const:0:0", 1)
    got = H.run_oracle(lists, p, int(g["steps"]), table)
    assert_fields_equal(lists, got, g["populations"], g["u"], g["rho"])


def test_oracle_flow_analyzer_golden():
    g = np.load(os.path.join(H.GOLDEN, "cylinder64x160_flow_analyzer.npz"))
    lists = H.classify(g["types"])
    assert_lists_equal(lists, golden_lists(g))
    p = H.Params.trt_magic(0.56, outlet_bc=H.BC_ZH_PRESSURE)
    table = H.open_values(lists, "parabolic:0.05:1:62", "pressure", 1)
    got = H.run_oracle(lists, p, int(g["steps"]), table, analyzer_every=int(g["every"]))
    np.testing.assert_array_equal(got["lift_drag"], g["lift_drag"])
    assert_fields_equal(lists, got, g["populations"], g["u"], g["rho"])


# ---------------------------------------------------------------------------
# live reference runner
# ---------------------------------------------------------------------------
needs_ref = pytest.mark.skipif(not H.have_ref(), reason="oracle/_ref/ref_runner not built")


def ref_vs_oracle(types, args, steps, tmp_path, extra=()):
    tmp_path.mkdir(parents=True, exist_ok=True)
    path = str(tmp_path / "lattice.txt")
    H.write_lattice_file(path, types)
    res = H.run_ref(["--lattice-file", path, *args, "--steps", str(steps), "--dump-nodes", *extra],
                    str(tmp_path / "out"))
    lists = H.ref_lists(res)
    assert_lists_equal(lists, H.classify(types))
    p, ins, outs = params_from_args(args)
    if "--ps-b" in args:  # the runner's per-obstacle weight pattern
        p.obstacle_b = np.array([((37 * q + 11) % 101) / 100.0 for q in range(len(lists.obstacle))])
    table = H.open_values(lists, ins, outs, steps)
    got = H.run_oracle(lists, p, steps, table)
    R, C = lists.rows, lists.cols
    assert_fields_equal(lists, got, res["populations"].reshape(9, C, R), res["u"].reshape(2, C, R),
                        res["rho"].reshape(C, R))


@needs_ref
@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("coll", ["bgk", "trt"])
def test_live_reference_porous(seed, coll, tmp_path):
    types = H.porous_types(56, 72, fraction=0.25, rmin=2, rmax=5, seed=seed)
    args = (["--collision", "bgk", "--tau", "0.75"] if coll == "bgk" else
            ["--collision", "trt", "--tau-even", "0.62", "--magic", "0.1875"])
    args += ["--inlet", "zh", "--outlet", "zhp", "--inlet-u", "const:0.03:0", "--outlet-u", "pressure"]
    ref_vs_oracle(types, args, 120, tmp_path)


@needs_ref
def test_live_reference_omp_trt_threads(tmp_path):
    """The reference's OpenMP TRT policies are race-free; with 4 threads they
    must reproduce the serial run (and the oracle) exactly."""
    types = H.channel_types(40, 70, discs=[(20, 30, 6)])
    args = ["--policy", "omp", "--threads", "4", "--collision", "trt", "--tau-even", "0.65", "--magic", "0.25",
            "--inlet", "zh", "--outlet", "zh", "--inlet-u", "parabolic:0.04:1:38", "--outlet-u", "const:0.03:0"]
    ref_vs_oracle(types, args, 150, tmp_path)


@needs_ref
def test_live_reference_lid_ramp(tmp_path):
    """Time-dependent update function (examples/1_LidDrivenCavity.cpp:80)."""
    ref_vs_oracle(H.cavity_types(40), ["--collision", "trt", "--tau-even", "0.58", "--magic", "0.25",
                                       "--inlet", "zh", "--outlet", "zh", "--inlet-u", "lidramp:0.15:0.001"],
                  250, tmp_path)


@needs_ref
@pytest.mark.parametrize("coll", ["bgk", "trt"])
def test_live_reference_partially_saturated_obstacles(coll, tmp_path):
    """PSBounceBackPolicy on wet obstacles (walls keep plain bounce-back): a
    channel with discs and a pressure outlet, and a cavity with a disc as in
    test/unit/LidWithPSObstacle.cpp.  The oracle equals the reference bit for
    bit."""
    col = (["--collision", "bgk", "--tau", "0.7"] if coll == "bgk" else
           ["--collision", "trt", "--tau-even", "0.6", "--magic", "0.25"])
    ch = H.channel_types(40, 90, discs=[(20, 30, 7), (12, 62, 4)])
    ref_vs_oracle(ch, col + ["--obstacle", "ps", "--ps-tau", "0.55", "--inlet", "zh", "--outlet", "zhp",
                             "--inlet-u", "parabolic:0.04:1:38", "--outlet-u", "pressure"], 160, tmp_path / "ch")
    cav = H.cavity_types(48)
    ii, jj = np.mgrid[0:48, 0:48]
    cav[((ii - 24) ** 2 + (jj - 24) ** 2 <= 64) & (cav == H.FLUID)] = H.OBSTACLE
    ref_vs_oracle(cav, col + ["--obstacle", "ps", "--ps-tau", "0.51", "--inlet", "zh", "--outlet", "zh",
                              "--inlet-u", "lidramp:0.1:0.002"], 200, tmp_path / "cav")


@needs_ref
def test_live_reference_partially_saturated_per_obstacle_b(tmp_path):
    """PSBounceBackPolicy with a weight b in [0, 1] set on each obstacle node
    (ObstaclePoint::set_b) before the run: the oracle's per-obstacle b path
    equals the reference bit for bit."""
    ch = H.channel_types(40, 90, discs=[(20, 30, 7), (12, 62, 4)])
    ref_vs_oracle(ch, ["--collision", "trt", "--tau-even", "0.6", "--magic", "0.25", "--obstacle", "ps",
                       "--ps-tau", "0.7", "--ps-b", "pattern", "--inlet", "zh", "--outlet", "zhp",
                       "--inlet-u", "parabolic:0.04:1:38", "--outlet-u", "pressure"], 150, tmp_path / "ch")
