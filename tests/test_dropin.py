"""The C++ drop-in: LLALBM programs built with CUDAPolicy instead of SerialPolicy.

The example programs (package examples/) use LLALBM's own Lattice API; each is
built twice from the same source, differing only in the parallelization-policy
template argument.  The CUDA build must reproduce the reference's serial build
bit for bit: populations of fluid/inlet/outlet nodes, u, rho, the saved u files
and the FlowAnalyzer lift/drag series.  The serial build is itself checked
against the C oracle.
"""
import filecmp
import os
import subprocess

import numpy as np
import pytest

import harness as H

BIN = os.path.join(H.ROOT, "latticeboltzmannmethod-fonnesu-grassi-guffanti_b200", "examples", "_bin")
needs_bins = pytest.mark.skipif(not os.path.exists(os.path.join(BIN, "lid_driven_cavity_serial")),
                                reason="example programs not built (the reference headers were absent)")


def run(exe, args, cwd):
    os.makedirs(cwd, exist_ok=True)
    p = subprocess.run([os.path.join(BIN, exe), *args], cwd=cwd, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stdout[-1000:] + p.stderr[-1000:]
    return {n: np.fromfile(os.path.join(cwd, n + ".f64")) for n in ("populations", "u", "rho", "lift_drag")
            if os.path.exists(os.path.join(cwd, n + ".f64"))}


def active_flat(lists):
    a = H.active_mask(lists)  # (C, R)
    return np.tile(a.reshape(-1), 9)


@needs_bins
def test_serial_example_matches_oracle(tmp_path):
    lists = H.classify(H.cavity_types(129))
    lat = str(tmp_path / "lid.txt")
    H.write_lattice_file(lat, H.cavity_types(129))
    out = run("lid_driven_cavity_serial", [lat, "200", "0", str(tmp_path / "s")], str(tmp_path / "s"))
    ref = H.run_oracle(lists, H.Params(tau=0.884), 200, H.open_values(lists, "const:0.1:0", "const:0:0", 1))
    act = active_flat(lists)
    np.testing.assert_array_equal(out["populations"][act], ref["populations"].reshape(-1)[act])
    np.testing.assert_array_equal(out["u"], ref["u"].reshape(-1))


@needs_bins
@pytest.mark.gpu
@pytest.mark.parametrize("steps,save,ramp", [(1000, 0, False), (600, 150, True)], ids=["const", "ramp_saves"])
def test_cuda_policy_matches_serial_policy_lid(tmp_path, steps, save, ramp):
    lat = str(tmp_path / "lid.txt")
    H.write_lattice_file(lat, H.cavity_types(129))
    lists = H.classify(H.cavity_types(129))
    extra = ["ramp"] if ramp else []
    outs = {}
    for pol in ("serial", "cuda"):
        d = str(tmp_path / pol)
        outs[pol] = run(f"lid_driven_cavity_{pol}", [lat, str(steps), str(save), d, *extra], d)
    act = active_flat(lists)
    np.testing.assert_array_equal(outs["cuda"]["populations"][act], outs["serial"]["populations"][act])
    np.testing.assert_array_equal(outs["cuda"]["u"], outs["serial"]["u"])
    np.testing.assert_array_equal(outs["cuda"]["rho"], outs["serial"]["rho"])
    if save:
        files = sorted(os.listdir(tmp_path / "serial" / "results"))
        assert len(files) == 2 * (steps // save)
        for f in files:
            assert filecmp.cmp(tmp_path / "serial" / "results" / f, tmp_path / "cuda" / "results" / f, shallow=False), f


@needs_bins
@pytest.mark.gpu
def test_cuda_policy_matches_serial_policy_cylinder_with_analyzer(tmp_path):
    types = H.cylinder_types(64, 160, x0=40, y0=33, r=8)
    lat = str(tmp_path / "cyl.txt")
    H.write_lattice_file(lat, types)
    lists = H.classify(types)
    outs = {}
    for pol in ("serial", "cuda"):
        d = str(tmp_path / pol)
        outs[pol] = run(f"cylinder_flow_{pol}", [lat, "400", "0.56", "0.05", d], d)
    act = active_flat(lists)
    np.testing.assert_array_equal(outs["cuda"]["populations"][act], outs["serial"]["populations"][act])
    np.testing.assert_array_equal(outs["cuda"]["u"], outs["serial"]["u"])
    assert len(outs["serial"]["lift_drag"]) == 2 * 39
    np.testing.assert_array_equal(outs["cuda"]["lift_drag"], outs["serial"]["lift_drag"])


def ps_cavity(n=64, r=7):
    t = H.cavity_types(n)
    ii, jj = np.mgrid[0:n, 0:n]
    t[((ii - n // 2) ** 2 + (jj - n // 2) ** 2 <= r * r) & (t == H.FLUID)] = H.OBSTACLE
    return t


@needs_bins
def test_serial_ps_example_matches_oracle(tmp_path):
    """PSBounceBackPolicy obstacle (test/unit/LidWithPSObstacle.cpp's set-up,
    compute_obstacle_weight included) through the reference's SerialPolicy."""
    types = ps_cavity()
    lists = H.classify(types)
    lat = str(tmp_path / "ps.txt")
    H.write_lattice_file(lat, types)
    out = run("lid_ps_obstacle_serial", [lat, "300", "0.6", "0.55", str(tmp_path / "s")], str(tmp_path / "s"))
    p = H.Params.trt_magic(0.6, obstacle_bc=1, ps_tau=0.55)
    ref = H.run_oracle(lists, p, 300, H.open_values(lists, "lidramp:0.1:0.002", "const:0:0", 300))
    act = active_flat(lists)
    np.testing.assert_array_equal(out["populations"][act], ref["populations"].reshape(-1)[act])
    np.testing.assert_array_equal(out["u"], ref["u"].reshape(-1))


@needs_bins
@pytest.mark.gpu
def test_cuda_policy_matches_serial_policy_ps_obstacle(tmp_path):
    types = ps_cavity(96, 10)
    lists = H.classify(types)
    lat = str(tmp_path / "ps.txt")
    H.write_lattice_file(lat, types)
    outs = {}
    for pol in ("serial", "cuda"):
        d = str(tmp_path / pol)
        outs[pol] = run(f"lid_ps_obstacle_{pol}", [lat, "800", "0.6", "0.55", d], d)
    act = active_flat(lists)
    np.testing.assert_array_equal(outs["cuda"]["populations"][act], outs["serial"]["populations"][act])
    np.testing.assert_array_equal(outs["cuda"]["u"], outs["serial"]["u"])
    np.testing.assert_array_equal(outs["cuda"]["rho"], outs["serial"]["rho"])


REF_LID_BINS = [os.path.join(BIN, f"ref_lid_exec_{p}") for p in ("serial", "cuda")]
needs_ref_lid = pytest.mark.skipif(not all(os.path.exists(b) for b in REF_LID_BINS),
                                   reason="the reference's LidExecTest was not built (reference headers absent)")


@needs_ref_lid
@pytest.mark.gpu
def test_reference_lid_exec_program_with_one_token_swapped(tmp_path):
    """The reference's own program test/unit/LidExecTest.cpp (Lattice from
    ../test/assets/lid-lattice.txt, BGK tau 0.6, lid u 0.2, perform_lbm(100)
    saving u on every step), built as shipped and with only its
    `using Parallel = SerialPolicy<2, Config>;` line switched to CUDAPolicy:
    all 200 saved files are byte-identical.  The lattice file is written from
    the config-1 generator, which equals the reference's asset token for
    token."""
    results = {}
    for exe in REF_LID_BINS:
        root = tmp_path / os.path.basename(exe)
        (root / "test" / "assets").mkdir(parents=True)
        H.write_lattice_file(str(root / "test" / "assets" / "lid-lattice.txt"), H.cavity_types(129))
        (root / "build").mkdir()
        p = subprocess.run([exe], cwd=root / "build", capture_output=True, text=True, timeout=900)
        assert p.returncode == 0, p.stdout[-1000:] + p.stderr[-1000:]
        results[exe] = root / "build" / "results"
    ser, cud = (results[b] for b in REF_LID_BINS)
    files = sorted(os.listdir(ser))
    assert len(files) == 200 and sorted(os.listdir(cud)) == files
    for f in files:
        assert filecmp.cmp(ser / f, cud / f, shallow=False), f


OMP_BINS = [os.path.join(BIN, f"lid_trt_omp_{p}") for p in ("omp", "cuda")]


@pytest.mark.skipif(not all(os.path.exists(b) for b in OMP_BINS), reason="OpenMP-family example not built")
@pytest.mark.gpu
def test_cuda_policy_matches_omp_policy_trt(tmp_path):
    """A program on the reference's OpenMP policy family (OMPTRT collision,
    OMPBounceBack, OMPZouHe lid with a ramp, OMPDefaultEquilibrium) built with
    OMPPolicy and run on 4 threads, and built with CUDAPolicy: populations,
    u, rho and the saved u files are identical."""
    lat = str(tmp_path / "lid.txt")
    H.write_lattice_file(lat, H.cavity_types(129))
    lists = H.classify(H.cavity_types(129))
    outs = {}
    for exe in OMP_BINS:
        d = tmp_path / os.path.basename(exe)
        d.mkdir()
        env = dict(os.environ, OMP_NUM_THREADS="4")
        p = subprocess.run([exe, lat, "800", "200", str(d)], cwd=d, capture_output=True, text=True, timeout=900,
                           env=env)
        assert p.returncode == 0, p.stdout[-1000:] + p.stderr[-1000:]
        outs[exe] = {n: np.fromfile(d / (n + ".f64")) for n in ("populations", "u", "rho")}
        outs[exe]["dir"] = d / "results"
    omp, cud = (outs[b] for b in OMP_BINS)
    act = active_flat(lists)
    np.testing.assert_array_equal(cud["populations"][act], omp["populations"][act])
    np.testing.assert_array_equal(cud["u"], omp["u"])
    np.testing.assert_array_equal(cud["rho"], omp["rho"])
    files = sorted(os.listdir(omp["dir"]))
    assert len(files) == 8
    for f in files:
        assert filecmp.cmp(omp["dir"] / f, cud["dir"] / f, shallow=False), f


READ_BINS = [os.path.join(BIN, f"read_lattice_{p}") for p in ("serial", "cuda")]
needs_read = pytest.mark.skipif(not all(os.path.exists(b) for b in READ_BINS), reason="read_lattice not built")


def read_structure(exe, path, out):
    p = subprocess.run([exe, path, out], capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-1000:]
    secs = float([ln for ln in p.stderr.splitlines() if ln.startswith("read seconds")][-1].split()[-1])
    return open(out).read(), secs


@needs_read
@pytest.mark.parametrize("geom", ["cavity129", "channel_discs", "odd_corners_solid", "porous"])
def test_fast_reader_equals_reference_reader(tmp_path, geom):
    """Lattice<CUDAPolicy>(path) reads the lattice file with the library's
    O(R*C) classification; its node vectors (print_lattice_structure with
    nodes) equal those of the reference's reader, Lattice<SerialPolicy>(path)."""
    if geom == "cavity129":
        types = H.cavity_types(129)
    elif geom == "channel_discs":
        types = H.channel_types(60, 140, discs=[(30, 40, 8), (12, 90, 5), (45, 100, 6)])
    elif geom == "odd_corners_solid":
        types = H.channel_types(37, 53, discs=[(18, 20, 4)])
        types[1:-1, 0] = H.BOUNDARY
        types[:, 0] = H.INLET
        types[20, 30] = H.SOLID
    else:
        types = H.porous_types(120, 150, seed=7)
    lat = str(tmp_path / "lattice.txt")
    H.write_lattice_file(lat, types)
    ref, _ = read_structure(READ_BINS[0], lat, str(tmp_path / "serial.txt"))
    got, _ = read_structure(READ_BINS[1], lat, str(tmp_path / "cuda.txt"))
    assert len(ref) > 0 and got == ref


@needs_read
def test_fast_reader_loads_a_4096_lattice_in_seconds(tmp_path):
    """The 4096 x 4096 porous channel (about 5.2 million listed nodes): the
    reference's reader classifies it in O(N^2) (std::find per obstacle
    neighbour); the fast reader takes seconds."""
    lat = str(tmp_path / "porous4096.txt")
    types = H.porous_types(4096, 4096)
    R, C = types.shape
    counts = [int((types == c).sum()) for c in range(6)]
    i, j = np.nonzero(types != H.FLUID)
    with open(lat, "w") as f:
        f.write("2\n%d %d\n%s\n" % (R, C, " ".join(str(c) for c in counts)))
        np.savetxt(f, np.stack([i, j, types[i, j]], axis=1), fmt="%d")
    text, secs = read_structure(READ_BINS[1], lat, str(tmp_path / "cuda.txt"))
    assert secs < 30.0, secs
    n_fluid = text.count("\n")  # one line per node and a few header lines
    assert n_fluid > counts[0]
