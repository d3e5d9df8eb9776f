"""Host-side parts of the C ABI (no GPU needed): exported symbols, lattice
classification, and descriptor validation."""
import ctypes
import os
import re

import numpy as np
import pytest

import harness as H

HEADER = os.path.join(H.ROOT, "include", "llalbm_cuda.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(llb_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol(cuda_lib):
    import llalbm_cuda as L

    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(cuda_lib, n), n
        assert n in L.SIGNATURES, n
    assert cuda_lib.llb_abi_version() == 2


@pytest.mark.parametrize("types", [
    H.cavity_types(129),
    H.channel_types(48, 96, discs=[(24, 30, 6), (12, 60, 4)]),
    H.porous_types(96, 96, seed=7),
    H.cylinder_types(),
], ids=["cavity129", "channel", "porous96", "cylinder1024x256"])
def test_classify_matches_reference_rules(types):
    import llalbm_cuda as L

    got = L.classify(types)
    want = H.classify(types)
    for f in ("fluid", "wall", "inlet", "inlet_side", "outlet", "outlet_side", "obstacle", "obstacle_dirs"):
        np.testing.assert_array_equal(got[f], getattr(want, f), err_msg=f)


def test_classify_matches_reference_golden_lists():
    """Against node vectors the reference's own reader produced."""
    import llalbm_cuda as L

    for name in ("lid129_bgk_10k", "porous96_bgk_pressure", "odd37x53_corners_solid"):
        g = np.load(os.path.join(H.GOLDEN, name + ".npz"))
        types = H.cavity_types(129) if name.startswith("lid") else g["types"]
        got = L.classify(types)
        np.testing.assert_array_equal(got["fluid"], g["fluid"])
        np.testing.assert_array_equal(got["wall"], g["wall"][:, :2])
        np.testing.assert_array_equal(got["inlet"], g["inlet"][:, :2])
        np.testing.assert_array_equal(got["inlet_side"], g["inlet"][:, 2])
        np.testing.assert_array_equal(got["outlet"], g["outlet"][:, :2])
        np.testing.assert_array_equal(got["obstacle"], g["obstacle"][:, :2])
        np.testing.assert_array_equal(got["obstacle_dirs"], g["obstacle"][:, 2])


def test_classify_errors():
    import llalbm_cuda as L

    t = H.cavity_types(20)
    t[5, 5] = H.INLET               # inlet off the perimeter (verify_lattice_bounds)
    with pytest.raises(L.LLBError) as e:
        L.classify(t)
    assert e.value.code == -2
    t = H.cavity_types(20)
    t[3, 3] = 9                     # not an InputNodeType
    with pytest.raises(L.LLBError) as e:
        L.classify(t)
    assert e.value.code == -1


def _desc_kw(lists):
    return dict(rows=lists.rows, cols=lists.cols, fluid=lists.fluid, wall=lists.wall, inlet=lists.inlet,
                inlet_side=lists.inlet_side, outlet=lists.outlet, outlet_side=lists.outlet_side,
                obstacle=lists.obstacle, obstacle_dirs=lists.obstacle_dirs)


def test_create_validates_before_touching_a_device():
    import llalbm_cuda as L

    lists = H.classify(H.channel_types(30, 50, discs=[(15, 20, 4)]))
    # bad enum
    with pytest.raises(L.LLBError) as e:
        L.CudaLattice(**_desc_kw(lists), collision=7)
    assert e.value.code == -1
    # a node listed twice
    kw = _desc_kw(lists)
    kw["wall"] = np.concatenate([lists.wall, lists.fluid[:1]])
    with pytest.raises(L.LLBError) as e:
        L.CudaLattice(**kw)
    assert e.value.code == -2
    # fluid node on the lattice edge (the reference would stream it out of bounds)
    kw = _desc_kw(lists)
    kw["wall"] = lists.wall[1:]
    kw["fluid"] = np.concatenate([lists.fluid, lists.wall[:1]])
    with pytest.raises(L.LLBError) as e:
        L.CudaLattice(**kw)
    assert e.value.code == -2
    # a bad obstacle policy, and partially saturated b outside [0, 1]
    with pytest.raises(L.LLBError) as e:
        L.CudaLattice(**_desc_kw(lists), obstacle_bc=7)
    assert e.value.code == -1
    with pytest.raises(L.LLBError) as e:
        L.CudaLattice(**_desc_kw(lists), obstacle_bc=1, ps_tau=0.6,
                      obstacle_b=np.full(len(lists.obstacle), 1.5))
    assert e.value.code == -1
    # obstacle bits that are not the reference's neighbour rule
    kw = _desc_kw(lists)
    kw["obstacle_dirs"] = lists.obstacle_dirs ^ np.uint16(2)
    with pytest.raises(L.LLBError) as e:
        L.CudaLattice(**kw)
    assert e.value.code == -8


def test_create_without_gpu_reports_no_device():
    import llalbm_cuda as L

    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    lists = H.classify(H.cavity_types(16))
    with pytest.raises(L.LLBError) as e:
        L.CudaLattice(**_desc_kw(lists))
    assert e.value.code in (-5, -4)


def test_server_validates_arguments_and_device():
    import llalbm_cuda as L

    with pytest.raises(L.LLBError) as e:
        L.CudaServer(budget_bytes=0)
    assert e.value.code == -1
    with pytest.raises(L.LLBError) as e:
        L.CudaServer(mode=5)
    assert e.value.code == -1
    try:
        import torch
        if torch.cuda.is_available():
            return
    except ImportError:
        pass
    with pytest.raises(L.LLBError) as e:
        L.CudaServer()
    assert e.value.code == -5
