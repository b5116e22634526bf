"""CPU oracle (FP64 numpy restatement) of jax_fem_cfd's matrix-free solver path.

TEST INFRASTRUCTURE ONLY. Nothing in the product (``jax_fem_cfd_b200``) imports
this package; only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline / ``--impl reference`` arm use it, and only as the checker or as the
timed CPU baseline.

Each function restates the reference algorithm it cites (paths relative to the
reference project root) operation for operation: same gathers, same element
products, scatter-adds in element order (``np.add.at``), same solver loop
conditions, initial values, mask/pin handling and mean removals.

Parity pinning: the reference ships no tests and its dependency (jax 0.4.13)
is absent here. The oracle is pinned instead against golden vectors produced by
executing the reference's own modules under a numpy stand-in for the JAX API
(``tests/golden/jax_shim.py``, ``tests/golden/make_golden.py``), and against
analytic known answers (element matrices, Taylor-Green decay).

Build-defined extensions (no reference counterpart, marked where they occur):
the 3D consistent mass (reference core/element_mult.py:23-26 raises NameError)
and the 3D u.n face integral on all six faces (core/element_calc.py:149 TODO).
"""
from . import mesh, shape, element, emult, multigrid, solvers, standard, transport, simulation  # noqa: F401
