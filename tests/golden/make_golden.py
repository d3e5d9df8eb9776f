"""Generates the golden fixtures in this directory from the reference itself.

Every fixture is produced by oracle/_ref/ref_runner, i.e. LLALBM's own headers
(Lattice, policies, readers, ConstructionInfo, FlowAnalyzer) compiled unmodified
from the reference tree.  The reference ships no numeric golden vectors for this
path (its tests are smoke runs), so these files are the pinned answers the C
oracle and the CUDA path are checked against where the reference tree is absent.

    python tests/golden/make_golden.py --reference <LLALBM checkout>

Geometries are written in the reference's lattice-file format from the same
generators the tests use (tests/harness.py); config 1 uses the reference's own
fixture test/assets/lid-lattice.txt.
"""
from __future__ import annotations

import argparse
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import harness as H  # noqa: E402


def lattice_file(types: np.ndarray, d: str, name: str) -> str:
    p = os.path.join(d, name + ".txt")
    H.write_lattice_file(p, types)
    return p


def save(name: str, res: dict, extra: dict | None = None):
    R, C = res["rows"], res["cols"]
    out = {
        "rows": R, "cols": C,
        "fluid": res["fluid"], "wall": res["wall"], "inlet": res["inlet"], "outlet": res["outlet"],
        "obstacle": res["obstacle"],
    }
    if "populations" in res:
        out["populations"] = res["populations"].reshape(9, C, R)
        out["u"] = res["u"].reshape(2, C, R)
        out["rho"] = res["rho"].reshape(C, R)
    if "lift_drag" in res:
        out["lift_drag"] = res["lift_drag"].reshape(-1, 2)
    if extra:
        out.update(extra)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print("wrote", name, {k: getattr(v, "shape", v) for k, v in out.items() if k not in ("rows", "cols")})


# name -> (types generator, ref_runner args, steps)
def cases():
    yield ("cavity64_trt_lidramp", lambda: H.cavity_types(64),
           ["--collision", "trt", "--tau-even", "0.58", "--magic", "0.25", "--inlet", "zh", "--outlet", "zh",
            "--inlet-u", "lidramp:0.15:0.001"], 300)
    yield ("channel48x96_trt_parabolic_pressure",
           lambda: H.channel_types(48, 96, discs=[(24, 30, 6), (12, 60, 4)]),
           ["--collision", "trt", "--tau-even", "0.53", "--magic", "0.25", "--inlet", "zh", "--outlet", "zhp",
            "--inlet-u", "parabolic:0.05:1:46", "--outlet-u", "pressure", "--rho-out", "1.0"], 500)
    yield ("channel40x80_bgk_open_outlet", lambda: H.channel_types(40, 80, discs=[(20, 25, 5)]),
           ["--collision", "bgk", "--tau", "0.7", "--inlet", "zh", "--outlet", "open",
            "--inlet-u", "const:0.04:0"], 300)
    yield ("channel40x80_trt_zh_outlet", lambda: H.channel_types(40, 80, discs=[(20, 25, 5)]),
           ["--collision", "trt", "--tau-even", "0.7", "--magic", "0.25", "--inlet", "zh", "--outlet", "zh",
            "--inlet-u", "const:0.04:0", "--outlet-u", "const:0.04:0"], 300)

    def odd():
        t = H.channel_types(37, 53, discs=[(18, 20, 4)])
        t[1:-1, 0] = H.BOUNDARY
        t[:, 0] = H.INLET
        t[20, 30] = H.SOLID
        return t
    yield ("odd37x53_corners_solid", odd,
           ["--collision", "bgk", "--tau", "0.8", "--inlet", "zh", "--outlet", "zh",
            "--inlet-u", "const:0.03:0.01"], 300)
    yield ("porous96_bgk_pressure", lambda: H.porous_types(96, 96, seed=7),
           ["--collision", "bgk", "--tau", "0.8", "--inlet", "zh", "--outlet", "zhp",
            "--inlet-u", "const:0.02:0", "--outlet-u", "pressure"], 400)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the LLALBM checkout (test/assets/lid-lattice.txt)")
    a = ap.parse_args()
    if not H.have_ref():
        sys.exit("oracle/_ref/ref_runner is missing: run `make -C oracle` with the reference tree present")
    work = tempfile.mkdtemp(prefix="llb_golden_")

    # Config 1: the reference's own fixture, BGK tau 0.884, lid u = (0.1, 0), 10 000 steps.
    lid = os.path.join(a.reference, "test", "assets", "lid-lattice.txt")
    res = H.run_ref(["--lattice-file", lid, "--collision", "bgk", "--tau", "0.884", "--inlet", "zh",
                     "--outlet", "zh", "--inlet-u", "const:0.1:0", "--steps", "10000", "--dump-nodes"],
                    os.path.join(work, "lid"), timeout=3600)
    save("lid129_bgk_10k", res, {"steps": 10000})

    for name, gen, args, steps in cases():
        types = gen()
        d = os.path.join(work, name)
        os.makedirs(d, exist_ok=True)
        res = H.run_ref(["--lattice-file", lattice_file(types, d, name), *args, "--steps", str(steps),
                         "--dump-nodes"], d)
        save(name, res, {"steps": steps, "types": types, "args": np.array(args)})

    # ConstructionInfo + build_lattice (classification of the in-code geometry builder),
    # OpenMP policies with one thread.
    script = os.path.join(work, "construct.txt")
    with open(script, "w") as f:
        f.write("dims 60 80\nperimeter BOUNDARY\ninterval 1 0 58 0 INLET\ninterval 1 79 58 79 OUTLET\n"
                "rect 20 20 10 6\nsphere 30 55 8\n")
    d = os.path.join(work, "construct")
    os.makedirs(d, exist_ok=True)
    res = H.run_ref(["--construct", script, "--policy", "omp", "--threads", "1", "--collision", "trt",
                     "--tau-even", "0.7", "--magic", "0.25", "--inlet", "zh", "--outlet", "open",
                     "--inlet-u", "const:0.03:0", "--steps", "200", "--dump-nodes"], d)
    types = np.fromfile(os.path.join(d, "types.u8"), dtype=np.uint8).reshape(res["cols"], res["rows"]).T
    save("construct60x80_omp_trt", res, {"steps": 200, "script": open(script).read(), "types": types})

    # FlowAnalyzer every 10 steps on the wet obstacle nodes (Lattice.hpp:384-387).
    types = H.cylinder_types(64, 160, x0=40, y0=33, r=8)
    d = os.path.join(work, "flow")
    os.makedirs(d, exist_ok=True)
    res = H.run_ref(["--lattice-file", lattice_file(types, d, "flow"), "--collision", "trt", "--tau-even", "0.56",
                     "--magic", "0.25", "--inlet", "zh", "--outlet", "zhp", "--inlet-u", "parabolic:0.05:1:62",
                     "--outlet-u", "pressure", "--analyzer", "10", "--steps", "300", "--dump-nodes"], d)
    save("cylinder64x160_flow_analyzer", res, {"steps": 300, "types": types, "every": 10})


if __name__ == "__main__":
    main()
