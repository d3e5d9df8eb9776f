"""The output writer (llb_writer_*): the reference's velocity text files
(utils/writers/LatticeWriter.hpp:60-92) written by a native thread.

CPU tests: the text format against printf "%.6g" (the reference's
`ostream << double`), the files against the ones the reference's own writer
wrote in a SerialPolicy run, ordering with one slot, and errors.  GPU tests:
a save enqueued on the lattice's stream captures u of its step even when the
next steps are enqueued at once.
"""
import filecmp
import os
import subprocess

import numpy as np
import pytest

import harness as H

L = pytest.importorskip("llalbm_cuda")

BIN = os.path.join(H.ROOT, "latticeboltzmannmethod-fonnesu-grassi-guffanti_b200", "examples", "_bin")


def printf_text(u):
    """The reference's file contents for u[i, j, d], one string per component."""
    R, C, _ = u.shape
    return ["".join("".join("%.6g " % u[i, j, d] for j in range(C)) + "\n" for i in range(R)) for d in (0, 1)]


def read_pair(directory, n):
    out = []
    for c in ("x", "y"):
        with open(os.path.join(directory, f"output-{n}u_{c}.txt")) as f:
            out.append(f.read())
    return out


def sample_values(rng, shape):
    """Magnitudes 1e-25..1e13 (both the writer's integer fast path and its
    fallback), exact ties of the sixth digit, powers of ten and their
    neighbours, tiny, huge and subnormal values, signed zeros."""
    u = rng.standard_normal(shape) * 10.0 ** rng.integers(-25, 13, shape)
    flat = u.reshape(-1)
    special = [0.0, -0.0, 1.0, -1.0, 0.1, 1e-5, 9.999995e-5, 123456.5, 123457.5, 1234567.0, 0.5e-4, 1e300,
               -1e-300, 5e-324, 2.5, 1.0 / 3.0, 999999.5, 9.9999995, 0.0001, 0.00001, 1e-17, 1e-18, 99999.95,
               np.nextafter(1e-4, 0.0), np.nextafter(1e6, 0.0), np.nextafter(1e6, 2e6), 2.0 ** -20, 3 * 2.0 ** -30]
    flat[: len(special)] = special
    return u


def test_format_matches_printf(tmp_path):
    rng = np.random.default_rng(3)
    u = sample_values(rng, (157, 211, 2))
    with L.OutputWriter(str(tmp_path), slots=2, threads=4) as w:
        w.save_host(u, 7)
        w.flush()
        assert w.stats()["files"] == 1
    assert read_pair(tmp_path, 7) == printf_text(u)


def test_non_finite_values(tmp_path):
    """A diverged run prints what ostream prints: nan, -nan, inf, -inf, -0."""
    u = np.zeros((1, 5, 2))
    u[0, :, 0] = [np.nan, -np.nan, np.inf, -np.inf, -0.0]
    u[0, :, 1] = [1.0, 2.5, -3.25, 1e-7, 123456789.0]
    assert np.signbit(u[0, 1, 0])
    with L.OutputWriter(str(tmp_path)) as w:
        w.save_host(u, 0)
    assert read_pair(tmp_path, 0) == ["nan -nan inf -inf -0 \n", "1 2.5 -3.25 1e-07 1.23457e+08 \n"]


def test_many_saves_one_slot_in_order(tmp_path):
    rng = np.random.default_rng(5)
    us = [rng.standard_normal((9, 5, 2)) for _ in range(12)]
    with L.OutputWriter(str(tmp_path), slots=1, threads=1) as w:
        for n, u in enumerate(us):
            w.save_host(u, n)  # the slot is reused: each call waits for the previous file
    for n, u in enumerate(us):
        assert read_pair(tmp_path, n) == printf_text(u)


def test_errors(tmp_path):
    with pytest.raises(L.LLBError) as e:
        L.OutputWriter(str(tmp_path), slots=65)
    assert e.value.code == -1
    w = L.OutputWriter(str(tmp_path / "missing"))
    w.save_host(np.zeros((3, 3, 2)), 0)
    with pytest.raises(L.LLBError) as e:
        w.flush()
    assert e.value.code == -1 and "cannot open" in str(e.value)
    w.flush()  # the error was reported once
    w.close()


@pytest.mark.skipif(not os.path.exists(os.path.join(BIN, "lid_driven_cavity_serial")),
                    reason="example programs not built (the reference headers were absent)")
def test_files_equal_reference_writer(tmp_path):
    """The reference's SerialPolicy lid cavity saves every 150 steps; its last
    file holds the final u, which the writer turns into the same bytes."""
    lat = str(tmp_path / "lid.txt")
    H.write_lattice_file(lat, H.cavity_types(65))
    run_dir = tmp_path / "serial"
    run_dir.mkdir()
    p = subprocess.run([os.path.join(BIN, "lid_driven_cavity_serial"), lat, "301", "150", str(run_dir), "ramp"],
                       cwd=run_dir, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    u = np.fromfile(run_dir / "u.f64").reshape((65, 65, 2), order="F")
    out = tmp_path / "mine"
    out.mkdir()
    with L.OutputWriter(str(out)) as w:
        w.save_host(u, 2)
    for c in ("x", "y"):
        name = f"output-2u_{c}.txt"
        assert filecmp.cmp(run_dir / "results" / name, out / name, shallow=False), name


@pytest.mark.gpu
def test_device_saves_capture_their_step(tmp_path):
    """save_u after a macro step, then further macro steps enqueued at once:
    each file holds u of its own step (the oracle's, formatted as the
    reference does)."""
    lists = H.classify(H.channel_types(40, 80, discs=[(20, 25, 5)]))
    p = H.Params(tau=0.7, outlet_bc=H.BC_OPEN)
    table = H.open_values(lists, "const:0.04:0", "const:0:0", 1)
    marks = [1, 40, 41, 200]
    with L.CudaLattice(lists.rows, lists.cols, lists.fluid, lists.wall, lists.inlet, lists.inlet_side,
                       lists.outlet, lists.outlet_side, lists.obstacle, lists.obstacle_dirs, tau=p.tau,
                       outlet_bc=p.outlet_bc) as g, L.OutputWriter(str(tmp_path), slots=2) as w:
        g.set_open_values(table, 0)
        g.init(macro=True)
        done = 1
        for n, m in enumerate(marks):
            if m > done:
                g.step(m - done, macro=True)
                done = m
            w.save_u(g, n)
        w.flush()
    for n, m in enumerate(marks):
        ref = H.run_oracle(lists, p, m, table)
        u = ref["u"].reshape(2, lists.cols, lists.rows).transpose(2, 1, 0)
        assert read_pair(tmp_path, n) == printf_text(u), (n, m)
