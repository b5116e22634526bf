"""jax_fem_cfd_b200: B200-native (sm_100a) matrix-free FEM incompressible-flow
solver path with the call interface of jax_fem_cfd.

Subpackages mirror the reference: setup (regular_mesh, simulation), core
(shape_functions, element_calc, element_mult, multigrid), solvers (standard,
passive_transport), utils (iterative_solvers, running). All compute runs in
libfemb200.so (hand-written CUDA behind the C ABI of include/fem_b200.h)."""
from ._lib import FemError, LIB_PATH, launch_count, load  # noqa: F401

__version__ = "0.1.0"
