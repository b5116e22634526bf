"""The C-ABI library loads without a GPU and exports exactly the entry points
that include/fem_b200.h declares; the Python binding declares them all."""
import os
import re

import pytest

from tests.conftest import ROOT


def _header_symbols():
    txt = open(os.path.join(ROOT, "include", "fem_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return set(re.findall(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(fem_\w+)\s*\(", txt, flags=re.M))


def test_library_loads_and_exports_header_symbols():
    from jax_fem_cfd_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libfemb200.so not built")
    lib = _lib.load()
    syms = _header_symbols()
    assert len(syms) >= 30
    for s in syms:
        assert hasattr(lib, s), s
    assert syms == set(_lib.SIGNATURES), syms ^ set(_lib.SIGNATURES)


def test_no_gpu_compute_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from jax_fem_cfd_b200 import FemError
    from jax_fem_cfd_b200.setup import regular_mesh as rm
    with pytest.raises(FemError):
        rm.create_mesh_2d(4, 4, 1.0, 1.0)


def test_config_validation_matches_reference_rules():
    from jax_fem_cfd_b200.setup import simulation as sim
    mc = sim.SimpleMeshConfig(num_elem=[8, 8], domain_size=[1, 1], shape_func_ord=1, periodic=False)
    ok = sim.StandardSolverConfig([0], [], [], False, 1e-6, True, "multigrid", [2, 2])
    sim.Config(mesh="simple", solver="standard", mesh_config=mc, solver_config=ok)
    # final mesh larger than the mesh, and 12 // 4 = 3 (log2 not integral, simulation.py:87-93)
    mc12 = sim.SimpleMeshConfig(num_elem=[12, 12], domain_size=[1, 1], shape_func_ord=1, periodic=False)
    for m, bad in ((mc, [16, 16]), (mc12, [4, 4])):
        with pytest.raises(ValueError):
            sim.Config(mesh="simple", solver="standard", mesh_config=m,
                       solver_config=sim.StandardSolverConfig([0], [], [], False, 1e-6, True, "multigrid", bad))
    with pytest.raises(ValueError):
        sim.Config(mesh="simple", solver="standard", mesh_config=mc,
                   solver_config=sim.StandardSolverConfig([0], [], [], False, 1e-6, True, "multigrid", None))
    with pytest.raises(ValueError):
        sim.Config(mesh="grid", solver="standard", mesh_config=mc, solver_config=ok)
