"""ctypes binding of libllalbm_cuda.so (C ABI in include/llalbm_cuda.h).

This is the Python face of the CUDA parallelization policy: a `CudaLattice`
holds one lattice resident on a GPU and exposes the same operations the C++
`CUDAPolicy` drives (init, steps, macroscopic output, populations, flow forces).
Arrays use the reference's Eigen layouts; in numpy (C order) a populations
tensor (R, C, 9) is `pop[k, j, i]`, u (R, C, 2) is `u[c, j, i]`, rho is `rho[j, i]`.

The library is loaded from the package directory; a missing or unloadable
library raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libllalbm_cuda.so")

LLB_OK = 0
ERRORS = {
    -1: "LLB_E_INVALID", -2: "LLB_E_GEOMETRY", -3: "LLB_E_NOMEM", -4: "LLB_E_CUDA", -5: "LLB_E_NODEVICE",
    -6: "LLB_E_STATE", -7: "LLB_E_NUMERIC", -8: "LLB_E_UNSUPPORTED", -9: "LLB_E_TIMEOUT",
}
BGK, TRT = 0, 1
STORE_F64, STORE_F32S, STORE_F16S = 0, 1, 2
PATTERN_AB, PATTERN_AA = 0, 1
BC_ZH_VELOCITY, BC_OPEN, BC_ZH_PRESSURE = 0, 1, 2
OBSTACLE_BOUNCE_BACK, OBSTACLE_PARTIAL = 0, 1
STEP_MACRO = 1
SERVE_BATCHED, SERVE_SEQUENTIAL = 0, 1
ADMIT_SHORTEST_FIRST, ADMIT_FIFO = 0, 1
LAYOUT_AUTO, LAYOUT_COMPACT, LAYOUT_DENSE = 0, 1, 2
REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = 0, 1, 2, 3
STORAGE_BYTES = {STORE_F64: 8, STORE_F32S: 4, STORE_F16S: 2}


class LLBError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class _Desc(ctypes.Structure):
    _fields_ = [
        ("rows", ctypes.c_int64), ("cols", ctypes.c_int64),
        ("n_fluid", ctypes.c_int64), ("fluid_ij", ctypes.c_void_p),
        ("n_wall", ctypes.c_int64), ("wall_ij", ctypes.c_void_p),
        ("n_inlet", ctypes.c_int64), ("inlet_ij", ctypes.c_void_p), ("inlet_side", ctypes.c_void_p),
        ("n_outlet", ctypes.c_int64), ("outlet_ij", ctypes.c_void_p), ("outlet_side", ctypes.c_void_p),
        ("n_obstacle", ctypes.c_int64), ("obstacle_ij", ctypes.c_void_p), ("obstacle_dirs", ctypes.c_void_p),
        ("inlet_bc", ctypes.c_int32), ("outlet_bc", ctypes.c_int32),
        ("collision", ctypes.c_int32), ("tau", ctypes.c_double),
        ("tau_even", ctypes.c_double), ("tau_odd", ctypes.c_double),
        ("storage", ctypes.c_int32), ("pattern", ctypes.c_int32),
        ("device", ctypes.c_int32), ("open_table_rows", ctypes.c_int32),
        ("obstacle_bc", ctypes.c_int32), ("ps_tau", ctypes.c_double), ("obstacle_b", ctypes.c_void_p),
    ]


class _NodeLists(ctypes.Structure):
    _fields_ = [
        ("n_fluid", ctypes.c_int64), ("n_wall", ctypes.c_int64), ("n_inlet", ctypes.c_int64),
        ("n_outlet", ctypes.c_int64), ("n_obstacle", ctypes.c_int64),
        ("fluid_ij", ctypes.c_void_p), ("wall_ij", ctypes.c_void_p),
        ("inlet_ij", ctypes.c_void_p), ("inlet_side", ctypes.c_void_p),
        ("outlet_ij", ctypes.c_void_p), ("outlet_side", ctypes.c_void_p),
        ("obstacle_ij", ctypes.c_void_p), ("obstacle_dirs", ctypes.c_void_p),
    ]


_lib = None

# every exported function: (name, argtypes)
_H = ctypes.c_void_p
_P = ctypes.c_void_p
SIGNATURES = {
    "llb_abi_version": [],
    "llb_last_error": [_H],
    "llb_classify_count": [ctypes.c_int64, ctypes.c_int64, _P, _P],
    "llb_classify_fill": [ctypes.c_int64, ctypes.c_int64, _P, ctypes.POINTER(_NodeLists)],
    "llb_create": [ctypes.POINTER(_Desc), ctypes.POINTER(_H)],
    "llb_destroy": [_H],
    "llb_set_open_values": [_H, ctypes.c_int64, ctypes.c_int32, _P],
    "llb_init": [_H, ctypes.c_uint32],
    "llb_step": [_H, ctypes.c_int32, ctypes.c_uint32],
    "llb_get_step": [_H, ctypes.POINTER(ctypes.c_int64)],
    "llb_get_macro": [_H, _P, _P],
    "llb_get_populations": [_H, _P],
    "llb_get_post_collision": [_H, _P],
    "llb_set_force_points": [_H, _P, _P, ctypes.c_int64],
    "llb_flow_forces": [_H, _P],
    "llb_gather_force_inputs": [_H, _P],
    "llb_flow_forces_noalloc": [_H, _P, _P, ctypes.c_int64, _P],
    "llb_mass_momentum": [_H, _P],
    "llb_synchronize": [_H],
    "llb_check_numerics": [_H],
    "llb_event_record": [_H, ctypes.c_int32],
    "llb_event_elapsed_ms": [_H, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_float)],
    "llb_set_pipeline": [_H, ctypes.c_int32],
    "llb_get_pipeline": [_H, ctypes.POINTER(ctypes.c_int32)],
    "llb_tune_pipeline": [_H, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_float)],
    "llb_set_launch_shape": [_H, ctypes.c_int32],
    "llb_set_wait_limit": [_H, ctypes.c_int64],
    "llb_check_numerics_begin": [_H, ctypes.c_int32],
    "llb_check_numerics_end": [_H, ctypes.c_int32],
    "llb_compute_macro": [_H, _P, _P],
    "llb_batch_create": [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(_H)],
    "llb_batch_destroy": [_H],
    "llb_batch_add": [_H, ctypes.POINTER(_Desc), _P, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)],
    "llb_batch_remove": [_H, ctypes.c_int32],
    "llb_batch_attach": [_H, _H, ctypes.POINTER(ctypes.c_int32)],
    "llb_batch_detach": [_H, ctypes.c_int32, ctypes.POINTER(_H)],
    "llb_batch_step": [_H, ctypes.c_int32],
    "llb_batch_lattice": [_H, ctypes.c_int32, ctypes.POINTER(_H)],
    "llb_batch_set_config": [_H, ctypes.c_int32, ctypes.c_int32],
    "llb_batch_get_config": [_H, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)],
    "llb_batch_tune": [_H, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                       ctypes.POINTER(ctypes.c_float)],
    "llb_batch_get_step": [_H, ctypes.POINTER(ctypes.c_int64)],
    "llb_batch_synchronize": [_H],
    "llb_batch_query": [_H, ctypes.POINTER(ctypes.c_int32)],
    "llb_batch_set_stream_priority": [_H, ctypes.c_int32],
    "llb_batch_set_wait_limit": [_H, ctypes.c_int64],
    "llb_batch_set_stop": [_H, ctypes.c_int32, ctypes.c_int64],
    "llb_batch_set_layout": [_H, ctypes.c_int32],
    "llb_batch_get_layout": [_H, ctypes.POINTER(ctypes.c_int32)],
    "llb_batch_event_record": [_H, ctypes.c_int32],
    "llb_batch_event_elapsed_ms": [_H, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_float)],
    "llb_batch_info": [_H, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                       ctypes.POINTER(ctypes.c_int64)],
    "llb_batch_last_error": [_H],
    "llb_device_bytes": [_H, ctypes.POINTER(ctypes.c_int64)],
    "llb_server_create": [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32,
                          ctypes.POINTER(_H)],
    "llb_server_destroy": [_H],
    "llb_server_set_admission": [_H, ctypes.c_int64, ctypes.c_int32],
    "llb_server_submit": [_H, ctypes.POINTER(_Desc), _P, ctypes.c_int32, ctypes.c_int64,
                          ctypes.POINTER(ctypes.c_int64)],
    "llb_server_poll": [_H, ctypes.c_int64, ctypes.POINTER(ctypes.c_int32)],
    "llb_server_wait": [_H, ctypes.c_int64, ctypes.c_double],
    "llb_server_result": [_H, ctypes.c_int64, _P, _P, _P],
    "llb_server_stats": [_H, _P],
    "llb_server_last_error": [_H],
    "llb_writer_create": [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(_H)],
    "llb_writer_save_u": [_H, _H, ctypes.c_int64],
    "llb_writer_save_host": [_H, _P, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64],
    "llb_writer_flush": [_H],
    "llb_writer_stats": [_H, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_double),
                         ctypes.POINTER(ctypes.c_double)],
    "llb_writer_destroy": [_H],
    "llb_writer_last_error": [_H],
}


def lib() -> ctypes.CDLL:
    """Loads the in-tree library (raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with build.py (no CPU fallback exists)")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_char_p if name.endswith("last_error") else ctypes.c_int
        _lib = L
    return _lib


def _check(rc: int, h=None):
    if rc != LLB_OK:
        msg = lib().llb_last_error(h)
        raise LLBError(rc, msg.decode() if msg else "")


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None and a.size else None


def _ij(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64).reshape(-1, 2))


def classify(types: np.ndarray) -> dict:
    """Reference node vectors from an (R, C) grid of InputNodeType codes
    (read_lattice_file's classification, in O(R*C))."""
    R, C = types.shape
    grid = np.ascontiguousarray(np.asarray(types, dtype=np.uint8).T)  # column-major (i fastest)
    counts = np.zeros(5, dtype=np.int64)
    _check(lib().llb_classify_count(R, C, _ptr(grid), _ptr(counts)))
    nf, nw, ni, no, nb = (int(c) for c in counts)
    out = {
        "fluid": np.zeros((nf, 2), np.int64), "wall": np.zeros((nw, 2), np.int64),
        "inlet": np.zeros((ni, 2), np.int64), "inlet_side": np.zeros(ni, np.int32),
        "outlet": np.zeros((no, 2), np.int64), "outlet_side": np.zeros(no, np.int32),
        "obstacle": np.zeros((nb, 2), np.int64), "obstacle_dirs": np.zeros(nb, np.uint16),
    }
    nl = _NodeLists(nf, nw, ni, no, nb, _ptr(out["fluid"]), _ptr(out["wall"]), _ptr(out["inlet"]),
                    _ptr(out["inlet_side"]), _ptr(out["outlet"]), _ptr(out["outlet_side"]),
                    _ptr(out["obstacle"]), _ptr(out["obstacle_dirs"]))
    _check(lib().llb_classify_fill(R, C, _ptr(grid), ctypes.byref(nl)))
    return out


def _desc(rows, cols, fluid, wall, inlet, inlet_side, outlet, outlet_side, obstacle, obstacle_dirs, *,
          collision, tau, tau_even, tau_odd, inlet_bc, outlet_bc, storage, pattern, device, open_table_rows,
          obstacle_bc=OBSTACLE_BOUNCE_BACK, ps_tau=0.6, obstacle_b=None):
    """Descriptor plus the arrays it points into (keep them alive while it is used)."""
    keep = {
        "fluid": _ij(fluid), "wall": _ij(wall), "inlet": _ij(inlet), "outlet": _ij(outlet),
        "obstacle": _ij(obstacle),
        "inlet_side": np.ascontiguousarray(np.asarray(inlet_side, dtype=np.int32).reshape(-1)),
        "outlet_side": np.ascontiguousarray(np.asarray(outlet_side, dtype=np.int32).reshape(-1)),
    }
    keep["obstacle_dirs"] = (None if obstacle_dirs is None else
                             np.ascontiguousarray(np.asarray(obstacle_dirs, dtype=np.uint16).reshape(-1)))
    d = _Desc(int(rows), int(cols),
              len(keep["fluid"]), _ptr(keep["fluid"]), len(keep["wall"]), _ptr(keep["wall"]),
              len(keep["inlet"]), _ptr(keep["inlet"]), _ptr(keep["inlet_side"]),
              len(keep["outlet"]), _ptr(keep["outlet"]), _ptr(keep["outlet_side"]),
              len(keep["obstacle"]), _ptr(keep["obstacle"]), _ptr(keep["obstacle_dirs"]),
              inlet_bc, outlet_bc, collision, tau, tau_even, tau_odd, storage, pattern, device, open_table_rows,
              obstacle_bc, ps_tau, None)
    if obstacle_b is not None:
        keep["obstacle_b"] = np.ascontiguousarray(np.asarray(obstacle_b, dtype=np.float64).reshape(-1))
        d.obstacle_b = _ptr(keep["obstacle_b"])
    return d, keep


class CudaLattice:
    """One D2Q9 lattice resident on a GPU (the engine behind CUDAPolicy)."""

    @classmethod
    def _wrap(cls, handle, rows, cols, storage, n_inlet, n_outlet, n_active):
        """Non-owning view of a handle that belongs to a batch."""
        obj = cls.__new__(cls)
        obj.rows, obj.cols, obj.storage = rows, cols, storage
        obj.n_inlet, obj.n_outlet = n_inlet, n_outlet
        obj.n_open, obj.n_active = n_inlet + n_outlet, n_active
        obj._h, obj._owner, obj._force_n = handle, False, 0
        return obj

    def __init__(self, rows: int, cols: int, fluid, wall, inlet, inlet_side, outlet, outlet_side,
                 obstacle, obstacle_dirs=None, *, collision: int = BGK, tau: float = 0.6,
                 tau_even: float = 0.6, tau_odd: float = 0.6, inlet_bc: int = BC_ZH_VELOCITY,
                 outlet_bc: int = BC_ZH_VELOCITY, storage: int = STORE_F64, pattern: int = PATTERN_AB,
                 device: int = 0, open_table_rows: int = 1, obstacle_bc: int = OBSTACLE_BOUNCE_BACK,
                 ps_tau: float = 0.6, obstacle_b=None):
        self.rows, self.cols = int(rows), int(cols)
        self.storage = storage
        self._owner = True
        d, keep = _desc(rows, cols, fluid, wall, inlet, inlet_side, outlet, outlet_side, obstacle, obstacle_dirs,
                        collision=collision, tau=tau, tau_even=tau_even, tau_odd=tau_odd, inlet_bc=inlet_bc,
                        outlet_bc=outlet_bc, storage=storage, pattern=pattern, device=device,
                        open_table_rows=open_table_rows, obstacle_bc=obstacle_bc, ps_tau=ps_tau,
                        obstacle_b=obstacle_b)
        self.n_inlet, self.n_outlet = len(keep["inlet"]), len(keep["outlet"])
        self.n_open = self.n_inlet + self.n_outlet
        self.n_active = len(keep["fluid"]) + self.n_open
        h = ctypes.c_void_p()
        _check(lib().llb_create(ctypes.byref(d), ctypes.byref(h)))
        self._h = h
        self._force_n = 0

    # -- lifetime --------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            if getattr(self, "_owner", True):
                lib().llb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    # -- stepping ----------------------------------------------------------------
    def set_open_values(self, values: np.ndarray, t_first: int = 0):
        """values: [rows][n_open][2] boundary values for steps t_first.. (inlets first)."""
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1, self.n_open, 2)
        _check(lib().llb_set_open_values(self._h, t_first, v.shape[0], _ptr(v)), self._h)

    def init(self, macro: bool = False):
        _check(lib().llb_init(self._h, STEP_MACRO if macro else 0), self._h)

    def step(self, n: int = 1, macro: bool = False):
        _check(lib().llb_step(self._h, n, STEP_MACRO if macro else 0), self._h)

    @property
    def t(self) -> int:
        s = ctypes.c_int64()
        _check(lib().llb_get_step(self._h, ctypes.byref(s)), self._h)
        return s.value

    def synchronize(self):
        _check(lib().llb_synchronize(self._h), self._h)

    def check_numerics(self):
        _check(lib().llb_check_numerics(self._h), self._h)

    def check_numerics_begin(self, slot: int = 0):
        """Queues the numerics check of the steps so far (slot in [0, 8))."""
        _check(lib().llb_check_numerics_begin(self._h, slot), self._h)

    def check_numerics_end(self, slot: int = 0):
        """Waits for the check queued on `slot`; raises as check_numerics."""
        _check(lib().llb_check_numerics_end(self._h, slot), self._h)

    # -- results -----------------------------------------------------------------
    def macro(self):
        rho = np.empty((self.cols, self.rows)); u = np.empty((2, self.cols, self.rows))
        _check(lib().llb_get_macro(self._h, _ptr(rho), _ptr(u)), self._h)
        return rho, u

    def compute_macro(self):
        """rho, u of the current populations without stepping."""
        rho = np.empty((self.cols, self.rows)); u = np.empty((2, self.cols, self.rows))
        _check(lib().llb_compute_macro(self._h, _ptr(rho), _ptr(u)), self._h)
        return rho, u

    def populations(self) -> np.ndarray:
        out = np.empty((9, self.cols, self.rows))
        _check(lib().llb_get_populations(self._h, _ptr(out)), self._h)
        return out

    def post_collision(self) -> np.ndarray:
        out = np.empty((9, self.cols, self.rows))
        _check(lib().llb_get_post_collision(self._h, _ptr(out)), self._h)
        return out

    def set_force_points(self, pts, dirs):
        p = _ij(pts); q = np.ascontiguousarray(np.asarray(dirs, dtype=np.uint16).reshape(-1))
        if len(q) != len(p):
            raise ValueError(f"{len(p)} force points but {len(q)} direction words")
        _check(lib().llb_set_force_points(self._h, _ptr(p), _ptr(q), len(p)), self._h)
        self._force_n = len(p)

    def flow_forces(self):
        out = np.zeros(2)
        _check(lib().llb_flow_forces(self._h, _ptr(out)), self._h)
        return float(out[0]), float(out[1])

    def flow_forces_noalloc(self, pts, dirs):
        """Lift and drag without device allocation (static scratch, <= 65536 points)."""
        p = _ij(pts); q = np.ascontiguousarray(np.asarray(dirs, dtype=np.uint16).reshape(-1))
        if len(q) != len(p):
            raise ValueError(f"{len(p)} force points but {len(q)} direction words")
        out = np.zeros(2)
        _check(lib().llb_flow_forces_noalloc(self._h, _ptr(p), _ptr(q), len(p), _ptr(out)), self._h)
        return float(out[0]), float(out[1])

    def gather_force_inputs(self) -> np.ndarray:
        out = np.zeros((self._force_n, 8))
        _check(lib().llb_gather_force_inputs(self._h, _ptr(out)), self._h)
        return out

    def mass_momentum(self) -> np.ndarray:
        out = np.zeros(3)
        _check(lib().llb_mass_momentum(self._h, _ptr(out)), self._h)
        return out

    # -- timing --------------------------------------------------------------------
    def record(self, slot: int):
        _check(lib().llb_event_record(self._h, slot), self._h)

    def elapsed_ms(self, a: int, b: int) -> float:
        ms = ctypes.c_float()
        _check(lib().llb_event_elapsed_ms(self._h, a, b, ctypes.byref(ms)), self._h)
        return float(ms.value)

    def set_pipeline(self, config: int):
        """-1: one thread per node; -2: the active-sector list; -3: compacted
        planes (active nodes only); -4: the lattice resident in one
        thread-block cluster's shared memory, a chunk of steps per launch;
        0..2 and 6: TMA pipeline configurations (6 also loads the tile's
        bounce bytes); 3..5: two steps per pass through shared memory."""
        _check(lib().llb_set_pipeline(self._h, config), self._h)

    @property
    def pipeline(self) -> int:
        c = ctypes.c_int32()
        _check(lib().llb_get_pipeline(self._h, ctypes.byref(c)), self._h)
        return c.value

    def tune_pipeline(self, trial_steps: int = 32):
        """Runs every plain-step configuration for 2 x trial_steps real steps
        and keeps the fastest; returns (configuration, ms per step)."""
        cfg, ms = ctypes.c_int32(), ctypes.c_float()
        _check(lib().llb_tune_pipeline(self._h, trial_steps, ctypes.byref(cfg), ctypes.byref(ms)), self._h)
        return cfg.value, ms.value

    def set_launch_shape(self, block_y: int):
        _check(lib().llb_set_launch_shape(self._h, block_y), self._h)

    def set_wait_limit(self, polls: int):
        """Polls of the pipelined kernels' stage waits before they give up
        (-1: default); for tests of the timeout path."""
        _check(lib().llb_set_wait_limit(self._h, polls), self._h)

    def device_bytes(self) -> int:
        b = ctypes.c_int64()
        _check(lib().llb_device_bytes(self._h, ctypes.byref(b)), self._h)
        return b.value


def from_types(types: np.ndarray, **kw) -> CudaLattice:
    """CudaLattice from an (R, C) InputNodeType grid, classified like the reference."""
    n = classify(types)
    R, C = types.shape
    return CudaLattice(R, C, n["fluid"], n["wall"], n["inlet"], n["inlet_side"], n["outlet"], n["outlet_side"],
                       n["obstacle"], n["obstacle_dirs"], **kw)


def _bcheck(rc: int, b):
    if rc != LLB_OK:
        msg = lib().llb_batch_last_error(b) if b else b""
        raise LLBError(rc, msg.decode() if msg else "")


class CudaBatch:
    """Many lattices advanced together (persistent batched launch, CUDA graphs)."""

    def __init__(self, storage: int = STORE_F32S, device: int = 0):
        b = ctypes.c_void_p()
        _check(lib().llb_batch_create(device, storage, ctypes.byref(b)))
        self._b, self.storage, self.device = b, storage, device
        self._meta = {}

    def close(self):
        if getattr(self, "_b", None):
            lib().llb_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add(self, rows, cols, fluid, wall, inlet, inlet_side, outlet, outlet_side, obstacle, obstacle_dirs=None, *,
            collision=BGK, tau=0.6, tau_even=0.6, tau_odd=0.6, inlet_bc=BC_ZH_VELOCITY, outlet_bc=BC_ZH_VELOCITY,
            open_values=None, obstacle_bc=OBSTACLE_BOUNCE_BACK, ps_tau=0.6, obstacle_b=None) -> int:
        vals = None if open_values is None else np.ascontiguousarray(open_values, dtype=np.float64)
        nrows = 0 if vals is None else vals.reshape(-1, len(inlet) + len(outlet), 2).shape[0]
        d, keep = _desc(rows, cols, fluid, wall, inlet, inlet_side, outlet, outlet_side, obstacle, obstacle_dirs,
                        collision=collision, tau=tau, tau_even=tau_even, tau_odd=tau_odd, inlet_bc=inlet_bc,
                        outlet_bc=outlet_bc, storage=self.storage, pattern=PATTERN_AB, device=self.device,
                        open_table_rows=max(nrows, 1), obstacle_bc=obstacle_bc, ps_tau=ps_tau,
                        obstacle_b=obstacle_b)
        slot = ctypes.c_int32()
        _bcheck(lib().llb_batch_add(self._b, ctypes.byref(d), _ptr(vals), nrows, ctypes.byref(slot)), self._b)
        n_in, n_out = len(keep["inlet"]), len(keep["outlet"])
        self._meta[slot.value] = (int(rows), int(cols), n_in, n_out, len(keep["fluid"]) + n_in + n_out)
        return slot.value

    def add_types(self, types, **kw) -> int:
        n = classify(types)
        R, C = types.shape
        return self.add(R, C, n["fluid"], n["wall"], n["inlet"], n["inlet_side"], n["outlet"], n["outlet_side"],
                        n["obstacle"], n["obstacle_dirs"], **kw)

    def remove(self, slot: int):
        _bcheck(lib().llb_batch_remove(self._b, slot), self._b)
        self._meta.pop(slot, None)

    def step(self, n: int = 1):
        _bcheck(lib().llb_batch_step(self._b, n), self._b)

    def lattice(self, slot: int) -> CudaLattice:
        h = ctypes.c_void_p()
        _bcheck(lib().llb_batch_lattice(self._b, slot, ctypes.byref(h)), self._b)
        R, C, ni, no, na = self._meta[slot]
        return CudaLattice._wrap(h, R, C, self.storage, ni, no, na)

    def set_config(self, block_y: int, steps_per_launch: int = 1):
        _bcheck(lib().llb_batch_set_config(self._b, block_y, steps_per_launch), self._b)

    @property
    def config(self):
        a, b = ctypes.c_int32(), ctypes.c_int32()
        _bcheck(lib().llb_batch_get_config(self._b, ctypes.byref(a), ctypes.byref(b)), self._b)
        return a.value, b.value

    def tune(self, trial_steps: int = 32):
        by, spl, ms = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_float()
        _bcheck(lib().llb_batch_tune(self._b, trial_steps, ctypes.byref(by), ctypes.byref(spl), ctypes.byref(ms)),
                self._b)
        return by.value, spl.value, ms.value

    @property
    def t(self) -> int:
        s = ctypes.c_int64()
        _bcheck(lib().llb_batch_get_step(self._b, ctypes.byref(s)), self._b)
        return s.value

    def synchronize(self):
        _bcheck(lib().llb_batch_synchronize(self._b), self._b)

    def set_wait_limit(self, polls: int):
        """Polls of the cooperative launches' grid barrier before a block
        gives up (-1: default); for tests of the timeout path."""
        _bcheck(lib().llb_batch_set_wait_limit(self._b, polls), self._b)

    def set_layout(self, layout: int):
        """LAYOUT_AUTO (compacted planes for obstacle-rich lattices),
        LAYOUT_COMPACT (for every lattice that has them) or LAYOUT_DENSE."""
        _bcheck(lib().llb_batch_set_layout(self._b, layout), self._b)

    @property
    def layout(self) -> int:
        v = ctypes.c_int32()
        _bcheck(lib().llb_batch_get_layout(self._b, ctypes.byref(v)), self._b)
        return v.value

    def set_stop(self, slot: int, stop_step: int):
        """The lattice in `slot` stops before step index stop_step (-1: never)."""
        _bcheck(lib().llb_batch_set_stop(self._b, slot, stop_step), self._b)

    def record(self, slot: int):
        _bcheck(lib().llb_batch_event_record(self._b, slot), self._b)

    def elapsed_ms(self, a: int, b: int) -> float:
        ms = ctypes.c_float()
        _bcheck(lib().llb_batch_event_elapsed_ms(self._b, a, b, ctypes.byref(ms)), self._b)
        return float(ms.value)

    def info(self):
        n, nodes, by = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _bcheck(lib().llb_batch_info(self._b, ctypes.byref(n), ctypes.byref(nodes), ctypes.byref(by)), self._b)
        return n.value, nodes.value, by.value


class _ServerCounters(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in ("completed", "failed", "node_steps", "queued", "running",
                                             "bytes_in_use", "chunks", "batch_steps")] + [(k, ctypes.c_double) for k in ("clock_s", "admit_s", "wait_s",
                                                                          "retire_s")]


def _scheck(rc: int, s):
    if rc != LLB_OK:
        msg = lib().llb_server_last_error(s) if s else b""
        raise LLBError(rc, msg.decode() if msg else "")


class CudaServer:
    """Solve server: requests (lattice, boundary values, step count) submitted
    from any thread are admitted under a device-memory budget and served by a
    native worker thread -- batched (continuous batching over one CudaBatch) or
    sequential (the plain single-lattice path, one request at a time).

    A request of `steps` steps returns the rho and u that the reference's
    Lattice holds after perform_lbm(steps)."""

    def __init__(self, storage: int = STORE_F32S, mode: int = SERVE_BATCHED, budget_bytes: int = 120 * 10**9,
                 max_chunk_steps: int = 256, device: int = 0):
        s = ctypes.c_void_p()
        _check(lib().llb_server_create(device, storage, mode, int(budget_bytes), max_chunk_steps, ctypes.byref(s)))
        self._s, self.storage, self.mode, self.device = s, storage, mode, device
        self._shape = {}

    def set_admission(self, max_resident_nodes: int = 0, order: int = 0):
        """Batched mode: at most max_resident_nodes lattice nodes resident (0:
        default) and the admission order (ADMIT_SHORTEST_FIRST or ADMIT_FIFO)."""
        rc = lib().llb_server_set_admission(self._s, int(max_resident_nodes), order)
        if rc != 0:
            raise LLBError(rc, "llb_server_set_admission")

    def close(self):
        if getattr(self, "_s", None):
            lib().llb_server_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, rows, cols, fluid, wall, inlet, inlet_side, outlet, outlet_side, obstacle, obstacle_dirs=None,
               *, steps: int, collision=BGK, tau=0.6, tau_even=0.6, tau_odd=0.6, inlet_bc=BC_ZH_VELOCITY,
               outlet_bc=BC_ZH_VELOCITY, open_values=None) -> int:
        """Queues one request; returns its id.  open_values: [rows][n_open][2]
        for steps 0.. (the last row repeats for later steps)."""
        vals = None if open_values is None else np.ascontiguousarray(open_values, dtype=np.float64)
        nrows = 0 if vals is None else vals.reshape(-1, len(inlet) + len(outlet), 2).shape[0]
        d, keep = _desc(rows, cols, fluid, wall, inlet, inlet_side, outlet, outlet_side, obstacle, obstacle_dirs,
                        collision=collision, tau=tau, tau_even=tau_even, tau_odd=tau_odd, inlet_bc=inlet_bc,
                        outlet_bc=outlet_bc, storage=self.storage, pattern=PATTERN_AB, device=self.device,
                        open_table_rows=max(nrows, 1))
        rid = ctypes.c_int64()
        _scheck(lib().llb_server_submit(self._s, ctypes.byref(d), _ptr(vals), nrows, int(steps), ctypes.byref(rid)),
                self._s)
        self._shape[rid.value] = (int(rows), int(cols))
        return rid.value

    def submit_types(self, types, **kw) -> int:
        n = classify(types)
        R, C = types.shape
        return self.submit(R, C, n["fluid"], n["wall"], n["inlet"], n["inlet_side"], n["outlet"], n["outlet_side"],
                           n["obstacle"], n["obstacle_dirs"], **kw)

    def state(self, rid: int) -> int:
        st = ctypes.c_int32()
        _scheck(lib().llb_server_poll(self._s, rid, ctypes.byref(st)), self._s)
        return st.value

    def wait(self, rid: int, timeout_s: float = 600.0):
        _scheck(lib().llb_server_wait(self._s, rid, float(timeout_s)), self._s)

    def result(self, rid: int, fields: bool = True):
        """(rho, u, times): rho[j, i], u[c, j, i] (None unless fields) and
        times = (submitted, admitted, done) in seconds; releases the request."""
        R, C = self._shape[rid]
        rho = np.empty((C, R)) if fields else None
        u = np.empty((2, C, R)) if fields else None
        times = np.zeros(3)
        _scheck(lib().llb_server_result(self._s, rid, _ptr(rho), _ptr(u), _ptr(times)), self._s)
        del self._shape[rid]
        return rho, u, tuple(float(x) for x in times)

    def stats(self) -> dict:
        c = _ServerCounters()
        _scheck(lib().llb_server_stats(self._s, ctypes.byref(c)), self._s)
        return {k: getattr(c, k) for k, _ in c._fields_}


def _wcheck(rc: int, w):
    if rc != LLB_OK:
        msg = lib().llb_writer_last_error(w) if w else b""
        raise LLBError(rc, msg.decode() if msg else "")


class OutputWriter:
    """The reference's velocity output files (LatticeWriter.hpp:60-92:
    <dir>/output-<n>u_x.txt, u_y.txt) written by a native thread while the
    caller keeps stepping.  save_u(lattice, n) enqueues the copy of the last
    macro step's u on the lattice's stream and returns; flush() waits for every
    queued file."""

    def __init__(self, directory: str, slots: int = 3, threads: int = 0):
        h = _H()
        rc = lib().llb_writer_create(str(directory).encode(), slots, threads, ctypes.byref(h))
        if rc != LLB_OK:
            raise LLBError(rc, "llb_writer_create")
        self._w = h

    def save_u(self, lattice: "CudaLattice", index: int):
        _wcheck(lib().llb_writer_save_u(self._w, lattice._h, index), self._w)

    def save_host(self, u: np.ndarray, index: int):
        """u: an (R, C, 2) array, u[i, j, d] as the reference's global_u(i, j, d)."""
        R, C = int(u.shape[0]), int(u.shape[1])
        flat = np.ascontiguousarray(np.ravel(np.asarray(u, dtype=np.float64), order="F"))
        _wcheck(lib().llb_writer_save_host(self._w, _ptr(flat), R, C, index), self._w)

    def flush(self):
        _wcheck(lib().llb_writer_flush(self._w), self._w)

    def stats(self) -> dict:
        n, a, b = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double()
        _wcheck(lib().llb_writer_stats(self._w, ctypes.byref(n), ctypes.byref(a), ctypes.byref(b)), self._w)
        return {"files": n.value, "wait_s": a.value, "write_s": b.value}

    def close(self):
        if self._w:
            w, self._w = self._w, None
            rc = lib().llb_writer_destroy(w)
            if rc != LLB_OK:
                raise LLBError(rc, "llb_writer_destroy")

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
