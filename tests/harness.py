"""Test harness: lattice cases, the C oracle (ctypes) and the reference runner.

Array conventions follow the reference's Eigen tensors (column-major, row index i
fastest).  In numpy (C order) a populations tensor (R, C, 9) is viewed as
``pop[k, j, i]``, u (R, C, 2) as ``u[c, j, i]`` and rho (R, C) as ``rho[j, i]``.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
import tempfile
from dataclasses import dataclass

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "liblbm_oracle.so")
REF_RUNNER = os.path.join(ORACLE_DIR, "_ref", "ref_runner")
REF_RUNNER_FAST = os.path.join(ORACLE_DIR, "_ref", "ref_runner_fast")
GOLDEN = os.path.join(ROOT, "tests", "golden")

# InputNodeType codes (llalbm/src/utils/aliases.hpp:41-48)
FLUID, SOLID, BOUNDARY, INLET, OUTLET, OBSTACLE = range(6)
# btypes (aliases.hpp:28-38)
BT_NONE, BT_TOP, BT_RIGHT, BT_BOTTOM, BT_LEFT = range(5)
BC_ZH_VELOCITY, BC_OPEN, BC_ZH_PRESSURE = range(3)
BGK, TRT = 0, 1
DI = [0, 0, -1, 0, 1, -1, -1, 1, 1]
DJ = [0, 1, 0, -1, 0, 1, -1, -1, 1]


# --------------------------------------------------------------------------
# node lists (the reference's classification, restated for test inputs)
# --------------------------------------------------------------------------
@dataclass
class NodeLists:
    rows: int
    cols: int
    fluid: np.ndarray            # (n, 2) int64
    wall: np.ndarray             # (n, 2)
    inlet: np.ndarray            # (n, 2)
    inlet_side: np.ndarray       # (n,) int32
    outlet: np.ndarray
    outlet_side: np.ndarray
    obstacle: np.ndarray         # (n, 2)
    obstacle_dirs: np.ndarray    # (n,) uint16

    @property
    def n_open(self) -> int:
        return len(self.inlet) + len(self.outlet)


def side_of(i: int, j: int, R: int, C: int) -> int:
    """identify_node_type (NodeIdentification.hpp:45-110) for one node."""
    if i == 0:
        return 8 if j == 0 else (5 if j == C - 1 else BT_TOP)          # LEFT_TOP_C / RIGHT_TOP_C
    if i == R - 1:
        return 7 if j == 0 else (6 if j == C - 1 else BT_BOTTOM)       # LEFT_BOTTOM_C / RIGHT_BOTTOM_C
    if j == 0:
        return BT_LEFT
    if j == C - 1:
        return BT_RIGHT
    return BT_NONE


def classify(types: np.ndarray) -> NodeLists:
    """Node vectors from an (R, C) grid of InputNodeType codes, in the reference's
    order (row-major (i, j), LatticeReader.hpp:108-204) with wet obstacles only."""
    R, C = types.shape
    ii, jj = np.nonzero(types >= 0)          # row-major order
    t = types[ii, jj]
    def pick(code):
        sel = t == code
        return np.stack([ii[sel], jj[sel]], axis=1).astype(np.int64)
    fluid, wall, inlet, outlet, obst = (pick(c) for c in (FLUID, BOUNDARY, INLET, OUTLET, OBSTACLE))
    active = np.isin(types, (FLUID, INLET, OUTLET))
    dirs = np.zeros(len(obst), dtype=np.uint16)
    for k in range(1, 9):
        ni, nj = obst[:, 0] + DI[k], obst[:, 1] + DJ[k]
        ok = (ni >= 0) & (nj >= 0) & (ni < R) & (nj < C)
        hit = np.zeros(len(obst), dtype=bool)
        hit[ok] = active[ni[ok], nj[ok]]
        dirs |= (hit.astype(np.uint16) << k)
    wet = dirs != 0
    sides = lambda a: np.array([side_of(int(i), int(j), R, C) for i, j in a], dtype=np.int32)
    return NodeLists(R, C, fluid, wall, inlet, sides(inlet), outlet, sides(outlet), obst[wet], dirs[wet])


# --------------------------------------------------------------------------
# geometries: the package's seeded workload generators
# --------------------------------------------------------------------------
import sys as _sys  # noqa: E402

_PKG_PY = os.path.join(ROOT, "latticeboltzmannmethod-fonnesu-grassi-guffanti_b200", "python")
if _PKG_PY not in _sys.path:
    _sys.path.insert(0, _PKG_PY)
from llb_workloads import cavity_types, channel_types, cylinder_types, porous_types, parabolic_u  # noqa: E402,F401


# --------------------------------------------------------------------------
# boundary values (the update functions of VelocityInitializer)
# --------------------------------------------------------------------------
def open_values(lists: NodeLists, inlet_spec: str, outlet_spec: str, steps: int) -> np.ndarray:
    """Table [rows][n_open][2] of update-function values (inlets then outlets).
    Specs as in oracle/ref_runner.cpp: const:ux:uy, parabolic:umax:i0:i1,
    lidramp:a:b, pressure:rho0:ut.  A table with one row means constant in time."""
    specs = ((lists.inlet, inlet_spec), (lists.outlet, outlet_spec))
    timevarying = any(s.startswith("lidramp") for _, s in specs)
    nrow = steps if timevarying else 1
    table = np.zeros((max(nrow, 1), lists.n_open, 2), dtype=np.float64)
    base = 0
    for nodes, spec in specs:
        f = spec.split(":")
        for q, (i, j) in enumerate(nodes):
            for t in range(table.shape[0]):
                if f[0] == "const":
                    v = (float(f[1]), float(f[2]))
                elif f[0] == "parabolic":
                    v = (parabolic_u(int(i), float(f[1]), int(f[2]), int(f[3])), 0.0)
                elif f[0] == "lidramp":
                    a, b = float(f[1]), float(f[2])
                    v = (a * (1.0 - math.exp(-float(t) * b)), 0.0)
                elif f[0] == "pressure":
                    v = (float(f[1]) if len(f) > 1 else 1.0, float(f[2]) if len(f) > 2 else 0.0)
                else:
                    raise ValueError(spec)
                table[t, base + q] = v
        base += len(nodes)
    return table


# --------------------------------------------------------------------------
# C oracle (ctypes)
# --------------------------------------------------------------------------
class _Problem(ctypes.Structure):
    _fields_ = [
        ("rows", ctypes.c_int64), ("cols", ctypes.c_int64),
        ("n_fluid", ctypes.c_int64), ("fluid", ctypes.c_void_p),
        ("n_wall", ctypes.c_int64), ("wall", ctypes.c_void_p),
        ("n_inlet", ctypes.c_int64), ("inlet", ctypes.c_void_p), ("inlet_side", ctypes.c_void_p),
        ("n_outlet", ctypes.c_int64), ("outlet", ctypes.c_void_p), ("outlet_side", ctypes.c_void_p),
        ("n_obst", ctypes.c_int64), ("obst", ctypes.c_void_p), ("obst_dirs", ctypes.c_void_p),
        ("collision", ctypes.c_int32), ("tau", ctypes.c_double), ("tau_even", ctypes.c_double),
        ("tau_odd", ctypes.c_double), ("inlet_bc", ctypes.c_int32), ("outlet_bc", ctypes.c_int32),
        ("rho_out", ctypes.c_double), ("tangential_u", ctypes.c_double),
        ("obstacle_bc", ctypes.c_int32), ("ps_tau", ctypes.c_double), ("obst_b", ctypes.c_void_p),
    ]


_oracle = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_LIB):
            subprocess.check_call(["make", "-C", ORACLE_DIR, "liblbm_oracle.so"], stdout=subprocess.DEVNULL)
        _oracle = ctypes.CDLL(ORACLE_LIB)
        _oracle.lbo_run.restype = ctypes.c_int
        _oracle.lbo_flow_properties.restype = None
    return _oracle


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None and a.size else None


@dataclass
class Params:
    collision: int = BGK
    tau: float = 0.6
    tau_even: float = 0.6
    tau_odd: float = 0.6
    inlet_bc: int = BC_ZH_VELOCITY
    outlet_bc: int = BC_ZH_VELOCITY
    rho_out: float = 1.0
    tangential_u: float = 0.0
    obstacle_bc: int = 0          # 0 bounce-back, 1 partially saturated (PSBounceBackPolicy)
    ps_tau: float = 0.6
    obstacle_b: object = None     # per obstacle b (ObstaclePoint::get_b), None: 1.0

    @staticmethod
    def trt_magic(tau_even: float, magic: float = 0.25, **kw) -> "Params":
        """TRTCollisionPolicy::enforce_magic_parameter (TRTCollision.hpp:128-134)."""
        return Params(collision=TRT, tau_even=tau_even, tau_odd=(magic) * (1.0 / (tau_even - 0.5)) + 0.5, **kw)


def run_oracle(lists: NodeLists, params: Params, steps: int, table: np.ndarray,
               analyzer_every: int = 0, analyzer_pts=None, analyzer_dirs=None):
    lib = oracle_lib()
    arrs = {
        "fluid": np.ascontiguousarray(lists.fluid, dtype=np.int64),
        "wall": np.ascontiguousarray(lists.wall, dtype=np.int64),
        "inlet": np.ascontiguousarray(lists.inlet, dtype=np.int64),
        "inlet_side": np.ascontiguousarray(lists.inlet_side, dtype=np.int32),
        "outlet": np.ascontiguousarray(lists.outlet, dtype=np.int64),
        "outlet_side": np.ascontiguousarray(lists.outlet_side, dtype=np.int32),
        "obst": np.ascontiguousarray(lists.obstacle, dtype=np.int64),
        "obst_dirs": np.ascontiguousarray(lists.obstacle_dirs, dtype=np.uint16),
    }
    if params.obstacle_b is not None:
        arrs["obst_b"] = np.ascontiguousarray(params.obstacle_b, dtype=np.float64)
    pr = _Problem(lists.rows, lists.cols,
                  len(arrs["fluid"]), _ptr(arrs["fluid"]), len(arrs["wall"]), _ptr(arrs["wall"]),
                  len(arrs["inlet"]), _ptr(arrs["inlet"]), _ptr(arrs["inlet_side"]),
                  len(arrs["outlet"]), _ptr(arrs["outlet"]), _ptr(arrs["outlet_side"]),
                  len(arrs["obst"]), _ptr(arrs["obst"]), _ptr(arrs["obst_dirs"]),
                  params.collision, params.tau, params.tau_even, params.tau_odd,
                  params.inlet_bc, params.outlet_bc, params.rho_out, params.tangential_u,
                  params.obstacle_bc, params.ps_tau, _ptr(arrs["obst_b"]) if "obst_b" in arrs else None)
    R, C = lists.rows, lists.cols
    pop = np.zeros((9, C, R)); u = np.zeros((2, C, R)); rho = np.zeros((C, R)); post = np.zeros((9, C, R))
    table = np.ascontiguousarray(table, dtype=np.float64)
    apts = np.ascontiguousarray(analyzer_pts if analyzer_pts is not None else lists.obstacle, dtype=np.int64)
    adirs = np.ascontiguousarray(analyzer_dirs if analyzer_dirs is not None else lists.obstacle_dirs, dtype=np.uint16)
    ld = np.zeros((max(steps, 1), 2))
    nld = ctypes.c_int64(0)
    rc = lib.lbo_run(ctypes.byref(pr), ctypes.c_int64(steps), _ptr(table), ctypes.c_int64(table.shape[0]),
                     ctypes.c_int64(analyzer_every), _ptr(apts), _ptr(adirs), ctypes.c_int64(len(apts)),
                     _ptr(ld), ctypes.byref(nld), _ptr(pop), _ptr(u), _ptr(rho), _ptr(post))
    if rc != 0:
        raise RuntimeError(f"lbo_run failed: {rc}")
    return {"populations": pop, "u": u, "rho": rho, "post": post, "lift_drag": ld[: nld.value]}


def oracle_flow_properties(rows: int, cols: int, densities: np.ndarray, pts: np.ndarray, dirs: np.ndarray):
    lib = oracle_lib()
    out = (ctypes.c_double * 2)()
    d = np.ascontiguousarray(densities, dtype=np.float64)
    p = np.ascontiguousarray(pts, dtype=np.int64)
    q = np.ascontiguousarray(dirs, dtype=np.uint16)
    lib.lbo_flow_properties(ctypes.c_int64(rows), ctypes.c_int64(cols), _ptr(d), _ptr(p), _ptr(q),
                            ctypes.c_int64(len(p)), out)
    return out[0], out[1]


# --------------------------------------------------------------------------
# reference runner (LLALBM's own headers; oracle/_ref)
# --------------------------------------------------------------------------
def have_ref() -> bool:
    return os.path.exists(REF_RUNNER)


def write_lattice_file(path: str, types: np.ndarray) -> None:
    """The reference's lattice file format (LatticeReader.hpp:300-360): dims,
    extensions, per-type counts, then `i j type` for every non-fluid node."""
    R, C = types.shape
    counts = [int((types == c).sum()) for c in range(6)]
    with open(path, "w") as f:
        f.write("2\n%d %d\n%s\n" % (R, C, " ".join(str(c) for c in counts)))
        for i, j in zip(*np.nonzero(types != FLUID)):
            f.write("%d %d %d\n" % (i, j, types[i, j]))


def run_ref(args: list[str], workdir: str | None = None, fast: bool = False, timeout: float = 600):
    """Runs the reference runner; returns its dumps as numpy arrays."""
    exe = REF_RUNNER_FAST if fast else REF_RUNNER
    out = workdir or tempfile.mkdtemp(prefix="llb_ref_")
    os.makedirs(out, exist_ok=True)
    proc = subprocess.run([exe, *args, "--out", out], cwd=out, capture_output=True, text=True, timeout=timeout)
    if proc.returncode != 0:
        raise RuntimeError(f"ref_runner failed ({proc.returncode}): {proc.stderr[-2000:]}")
    res = {"stdout": proc.stdout, "dir": out}
    dims = os.path.join(out, "dims.i64")
    if os.path.exists(dims):
        R, C = np.fromfile(dims, dtype=np.int64)
        res["rows"], res["cols"] = int(R), int(C)
        rd = lambda n, w: np.fromfile(os.path.join(out, n), dtype=np.int64).reshape(-1, w)
        res["fluid"] = rd("fluid.i64", 2)
        res["wall"] = rd("boundary.i64", 3)
        res["inlet"] = rd("inlet.i64", 3)
        res["outlet"] = rd("outlet.i64", 3)
        res["obstacle"] = rd("obstacle.i64", 3)
    for name in ("populations", "u", "rho", "lift_drag"):
        p = os.path.join(out, name + ".f64")
        if os.path.exists(p):
            res[name] = np.fromfile(p)
    return res


def ref_lists(res) -> NodeLists:
    """NodeLists from the reference runner's node dumps."""
    return NodeLists(res["rows"], res["cols"], res["fluid"], res["wall"][:, :2],
                     res["inlet"][:, :2].copy(), res["inlet"][:, 2].astype(np.int32),
                     res["outlet"][:, :2].copy(), res["outlet"][:, 2].astype(np.int32),
                     res["obstacle"][:, :2].copy(), res["obstacle"][:, 2].astype(np.uint16))


def active_mask(lists: NodeLists) -> np.ndarray:
    """(C, R) boolean view of fluid, inlet and outlet nodes."""
    m = np.zeros((lists.cols, lists.rows), dtype=bool)
    for a in (lists.fluid, lists.inlet, lists.outlet):
        if len(a):
            m[a[:, 1], a[:, 0]] = True
    return m
