"""Config dataclasses, boundary-set assembly and setup (oracle restatement of
setup/simulation.py). Test infrastructure only."""
import time
from dataclasses import dataclass
from typing import Dict, List, Optional, Union

import numpy as np

from . import mesh as rm


@dataclass
class SimpleMeshConfig:
    """setup/simulation.py:10-18."""
    num_elem: List[int]
    domain_size: List[float]
    shape_func_ord: int
    periodic: bool
    partial_dirichlet: Dict = None


@dataclass
class StandardSolverConfig:
    """setup/simulation.py:20-29."""
    dirichlet_faces: List[int]
    symmetry_faces: List[int]
    outlet_faces: List[int]
    streamline_diff: bool
    solver_tol: float
    set_zeroP: bool
    pressure_precond: Optional[str] = None
    final_multigrid_mesh: Optional[List[int]] = None


@dataclass
class ADEConfig:
    phi_dirichlet_faces: List[int]
    phi_SUPG: bool


@dataclass
class PassiveTransportConfig:
    NS_config: StandardSolverConfig
    ADE_config: ADEConfig


@dataclass
class Config:
    """setup/simulation.py:41-93 (validation raises ValueError like the reference)."""
    mesh: str
    solver: str
    mesh_config: SimpleMeshConfig
    solver_config: Union[StandardSolverConfig, PassiveTransportConfig]

    def __post_init__(self):
        if self.mesh != "simple":
            raise ValueError(f"Unknown mesh type: {self.mesh}")
        if self.solver == "standard":
            if not isinstance(self.solver_config, StandardSolverConfig):
                raise ValueError("Solver type and config type must match")
        elif self.solver == "passive_transport":
            if not isinstance(self.solver_config, PassiveTransportConfig):
                raise ValueError("Solver type and config type must match")
        else:
            raise ValueError(f"Unknown solver type: {self.solver}")


def mesh_func_for(mc):
    """setup/simulation.py:104-119."""
    ndim = len(mc.num_elem)
    if mc.shape_func_ord == 1:
        if ndim == 2:
            return rm.create_periodic_mesh_2d if mc.periodic else rm.create_mesh_2d
        return rm.create_mesh_3d
    return rm.create_periodic_mesh_2d_quad9 if mc.periodic else rm.create_mesh_2d_quad9


def simple_mesh(mc, ns):
    """setup/simulation.py:96-183: gamma_d (all components, sorted), U_d = 0,
    gamma_p (outlet nodes, else scalar 0 = pin node 0), bconn/nvec of Dirichlet faces."""
    mesh_func = mesh_func_for(mc)
    node_coords, nconn, surfnodes, bconns, nvecs = mesh_func(*mc.num_elem, *mc.domain_size)
    ndim = len(mc.num_elem)
    if ndim == 3:
        # build-defined 3D boundary integral: on the geometric face quads (the
        # reference's D/T/F/B rows are not per-face quads, see mesh.create_mesh_3d)
        from .mesh import bconns_3d_faces
        bconns = bconns_3d_faces(*mc.num_elem)
    nn = node_coords.shape[0]
    h = mc.domain_size[0] / mc.num_elem[0]
    bconn = nvec = gamma_d = U_d = None
    dnodes, onodes, bl, nl = [], [], [], []
    if ns.dirichlet_faces:
        for f in ns.dirichlet_faces:
            dnodes.append(surfnodes[f])
            bl.append(bconns[f])
            nl.append(nvecs[f])
    if ns.outlet_faces:
        for f in ns.outlet_faces:
            onodes.append(surfnodes[f])
    if mc.partial_dirichlet:
        for f, (s, e, kind) in mc.partial_dirichlet.items():
            fn, fb, fv = surfnodes[f], bconns[f], nvecs[f]
            nfe = fb.shape[0]
            si, ei = round(s * nfe), round(e * nfe)
            bl.append(fb[si:ei])
            nl.append(fv[si:ei])
            if mc.shape_func_ord == 2:
                si, ei = 2 * si, 2 * ei
            surfnodes[f] = fn[si:ei + 1]
            dnodes.append(fn[si:ei + 1])
            if kind == "outlet":
                onodes.append(fn[:si])
                onodes.append(fn[ei + 1:])
    if dnodes:
        g = np.sort(np.unique(np.concatenate(dnodes)))
        gamma_d = np.concatenate([g + nn * i for i in range(ndim)])
        U_d = np.zeros(gamma_d.shape[0])
        bconn = np.concatenate(bl, axis=0)
        nvec = np.concatenate(nl, axis=0)
    gamma_p = np.unique(np.concatenate(onodes)) if onodes else 0
    return node_coords, nconn, surfnodes, nn, h, bconn, nvec, gamma_d, U_d, gamma_p, mesh_func


def setup(config):
    """setup/simulation.py:185-217."""
    from . import standard, transport
    ns = config.solver_config if config.solver == "standard" else config.solver_config.NS_config
    node_coords, nconn, surfnodes, nn, h, bconn, nvec, gamma_d, U_d, gamma_p, mesh_func = \
        simple_mesh(config.mesh_config, ns)
    if config.solver == "standard":
        compute, timestep = standard.setup_solver(node_coords, nconn, bconn, nvec, gamma_d, gamma_p, nn,
                                                  mesh_func, config)
        return compute, timestep, node_coords, surfnodes, h, nn, gamma_d, U_d
    mc = config.mesh_config
    nnx, nny = ((mc.num_elem[0] + 1, mc.num_elem[1] + 1) if mc.shape_func_ord == 1
                else (2 * mc.num_elem[0] + 1, 2 * mc.num_elem[1] + 1))
    faces = config.solver_config.ADE_config.phi_dirichlet_faces
    gamma_d_phi = None if not faces else np.sort(np.unique(np.concatenate([surfnodes[i] for i in faces])))
    compute, timestep = transport.setup_solver(node_coords, nconn, bconn, nvec, gamma_d, gamma_p, nn,
                                               gamma_d_phi, mesh_func, config)
    return compute, timestep, node_coords, surfnodes, h, nn, nnx, nny, gamma_d, U_d, gamma_d_phi


def set_face_velocity(U_d, nodes, gamma_d, values, nn, var):
    """setup/simulation.py:219-226."""
    idx = np.searchsorted(gamma_d, np.asarray(nodes) + nn * (var - 1))
    out = np.array(U_d, copy=True)
    out[idx] = values
    return out


def timestep_loop(num_steps, dt, compute_func, timestep_func, parameters, dirichlet_vals, initial_states):
    """Step loop of setup/simulation.py:229-347 without printing/HDF5: returns the
    final state and per-step iteration counts."""
    has_phi = len(initial_states) == 3
    U, P = initial_states[:2]
    phi = initial_states[2] if has_phi else None
    U_d = dirichlet_vals[0]
    phi_d = dirichlet_vals[1] if has_phi else None
    iters = []
    t0 = time.perf_counter()
    for step in range(1, num_steps + 1):
        F_p, F = compute_func(U_d, None, (step - 1) * dt, step * dt)
        if has_phi:
            U, P, phi, ui, pi, fi = timestep_func(U, P, phi, dt, *parameters, U_d, phi_d, F_p, F, None)
            iters.append((ui, pi, fi))
        else:
            U, P, ui, pi = timestep_func(U, P, dt, *parameters, U_d, F_p, F)
            iters.append((ui, pi))
    elapsed = time.perf_counter() - t0
    return (U, P, phi, iters, elapsed) if has_phi else (U, P, iters, elapsed)
