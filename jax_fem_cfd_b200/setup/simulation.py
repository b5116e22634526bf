"""Configuration, boundary sets, setup and time loops (drop-in for
jax_fem_cfd setup/simulation.py). Arrays are torch tensors on the CUDA device."""
import math
import time
from dataclasses import dataclass
from typing import Dict, List, Literal, Optional, Union

import numpy as np
import torch

from ..context import f64, i64, scatter_set
from . import regular_mesh as rm


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
    # Extension (no reference field): "mixed" runs the multigrid pressure solve
    # as FP64 refinement around FP32 multigrid-PCG iterations.
    precision: str = "fp64"


@dataclass
class ADEConfig:
    """setup/simulation.py:31-34."""
    phi_dirichlet_faces: List[int]
    phi_SUPG: bool


@dataclass
class PassiveTransportConfig:
    """setup/simulation.py:36-39."""
    NS_config: StandardSolverConfig
    ADE_config: ADEConfig


@dataclass
class Config:
    """setup/simulation.py:41-93: validated on construction (ValueError)."""
    mesh: Literal["simple"]
    solver: Literal["standard", "passive_transport"]
    mesh_config: SimpleMeshConfig
    solver_config: Union[StandardSolverConfig, PassiveTransportConfig]

    def __post_init__(self):
        self.validate()

    def validate(self):
        if self.mesh == "simple":
            if not isinstance(self.mesh_config, SimpleMeshConfig):
                raise ValueError("Mesh type and config type must match")
        else:
            raise ValueError(f"Unknown mesh type: {self.mesh}")
        if self.solver == "standard":
            if not isinstance(self.solver_config, StandardSolverConfig):
                raise ValueError("Solver type and config type must match")
        elif self.solver == "passive_transport":
            if not isinstance(self.solver_config, PassiveTransportConfig):
                raise ValueError("Solver type and config type must match")
        else:
            raise ValueError(f"Unknown solver type: {self.solver}")
        ns = self.solver_config if self.solver == "standard" else self.solver_config.NS_config
        if len(self.mesh_config.num_elem) == 3:
            if self.mesh_config.shape_func_ord == 2:
                raise ValueError("3D quadratic shape functions not yet implemented")
            if self.mesh_config.periodic:
                raise ValueError("3D periodic boundary conditions not yet implemented")
            # 3D multigrid is this package's extension (the reference raises
            # "3D multigrid not yet implemented"): all axes coarsen together,
            # pressure must be pinned
            if ns.pressure_precond == "multigrid":
                fm = ns.final_multigrid_mesh
                if fm is None or len(fm) != 3:
                    raise ValueError("3D multigrid needs a 3-entry final_multigrid_mesh")
                ratios = {n // f for n, f in zip(self.mesh_config.num_elem, fm) if f > 0}
                if len(ratios) != 1 or any(n % f for n, f in zip(self.mesh_config.num_elem, fm)):
                    raise ValueError("3D multigrid halves every axis together: num_elem / final_multigrid_mesh "
                                     "must be the same power of two on all axes")
                if not ns.set_zeroP:
                    raise ValueError("3D multigrid needs pinned pressure (set_zeroP=True)")
        if getattr(ns, "precision", "fp64") not in ("fp64", "mixed"):
            raise ValueError(f"Unknown precision: {ns.precision}")
        if getattr(ns, "precision", "fp64") == "mixed" and ns.pressure_precond != "multigrid":
            raise ValueError("precision='mixed' is implemented for the multigrid pressure solve")
        if ns.pressure_precond == "multigrid":
            num_elemf = ns.final_multigrid_mesh
            if num_elemf is None:
                raise ValueError("Must specify final_multigrid_mesh to use multigrid")
            for n, f in zip(self.mesh_config.num_elem, num_elemf):
                if f > n:
                    raise ValueError("final_multigrid_mesh is too large")
                lr = math.log2(n // f)
                if not math.isclose(lr, round(lr)):
                    raise ValueError(f"Invalid final_multigrid_mesh: log2({n}/{f}) is not an integer")


def mesh_func_for(mc):
    """setup/simulation.py:104-119."""
    ndim = len(mc.num_elem)
    if mc.shape_func_ord == 1:
        if ndim == 2:
            return rm.create_periodic_mesh_2d if mc.periodic else rm.create_mesh_2d
        return rm.create_mesh_3d
    return rm.create_periodic_mesh_2d_quad9 if mc.periodic else rm.create_mesh_2d_quad9


def simple_mesh(mesh_config: SimpleMeshConfig, NS_config: StandardSolverConfig):
    """setup/simulation.py:96-183: gamma_d (all components, sorted unique),
    U_d = 0, gamma_p (outlet nodes, else 0 = pin node 0), Dirichlet bconn/nvec."""
    mesh_func = mesh_func_for(mesh_config)
    node_coords, nconn, surfnodes, bconns, nvecs = mesh_func(*mesh_config.num_elem, *mesh_config.domain_size)
    ndim = len(mesh_config.num_elem)
    nn = node_coords.shape[0]
    h = mesh_config.domain_size[0] / mesh_config.num_elem[0]
    host = lambda t: t.cpu().numpy()
    bconn = nvec = gamma_d = U_d = None
    dnodes, onodes, bl, nl = [], [], [], []
    if NS_config.dirichlet_faces:
        for f in NS_config.dirichlet_faces:
            dnodes.append(host(surfnodes[f]))
            bl.append(host(bconns[f]))
            nl.append(host(nvecs[f]))
    if NS_config.outlet_faces:
        for f in NS_config.outlet_faces:
            onodes.append(host(surfnodes[f]))
    if mesh_config.partial_dirichlet:
        for f, (s0, e0, kind) in mesh_config.partial_dirichlet.items():
            fn, fb, fv = host(surfnodes[f]), host(bconns[f]), host(nvecs[f])
            nfe = fb.shape[0]
            si, ei = round(s0 * nfe), round(e0 * nfe)
            bl.append(fb[si:ei])
            nl.append(fv[si:ei])
            if mesh_config.shape_func_ord == 2:
                si, ei = 2 * si, 2 * ei
            surfnodes[f] = i64(fn[si:ei + 1])
            dnodes.append(fn[si:ei + 1])
            if kind == "outlet":
                onodes.append(fn[:si])
                onodes.append(fn[ei + 1:])
    if dnodes:
        g = np.sort(np.unique(np.concatenate(dnodes)))
        gamma_d = i64(np.concatenate([g + nn * i for i in range(ndim)]))
        U_d = torch.zeros(gamma_d.shape[0], dtype=torch.float64, device=node_coords.device)
        bconn = i64(np.concatenate(bl, axis=0)).view(-1, bl[0].shape[1])
        nvec = f64(np.concatenate(nl, axis=0)).view(-1, nl[0].shape[1])
    gamma_p = i64(np.unique(np.concatenate(onodes))) if onodes else 0
    return node_coords, nconn, surfnodes, nn, h, bconn, nvec, gamma_d, U_d, gamma_p, mesh_func


def setup(config: Config):
    """setup/simulation.py:185-217."""
    ns = config.solver_config if config.solver == "standard" else config.solver_config.NS_config
    node_coords, nconn, surfnodes, nn, h, bconn, nvec, gamma_d, U_d, gamma_p, mesh_func = simple_mesh(
        config.mesh_config, ns)
    if config.solver == "standard":
        from ..solvers.standard import setup_solver
        compute, timestep = setup_solver(node_coords, nconn, bconn, nvec, gamma_d, gamma_p, nn, mesh_func, config)
        return compute, timestep, node_coords, surfnodes, h, nn, gamma_d, U_d
    from ..solvers.passive_transport import setup_solver
    mc = config.mesh_config
    nnx, nny = ((mc.num_elem[0] + 1, mc.num_elem[1] + 1) if mc.shape_func_ord == 1
                else (2 * mc.num_elem[0] + 1, 2 * mc.num_elem[1] + 1))
    faces = config.solver_config.ADE_config.phi_dirichlet_faces
    gamma_d_phi = None
    if faces:
        gamma_d_phi = i64(np.sort(np.unique(np.concatenate([surfnodes[i].cpu().numpy() for i in faces]))))
    compute, timestep = setup_solver(node_coords, nconn, bconn, nvec, gamma_d, gamma_p, nn, gamma_d_phi, mesh_func,
                                     config)
    return compute, timestep, node_coords, surfnodes, h, nn, nnx, nny, gamma_d, U_d, gamma_d_phi


def set_face_velocity(U_d, nodes, gamma_d, values, nn, var):
    """setup/simulation.py:219-226: U_d.at[searchsorted(gamma_d, nodes + nn*(var-1))].set(values)."""
    g = gamma_d.cpu().numpy() if isinstance(gamma_d, torch.Tensor) else np.asarray(gamma_d)
    nd = nodes.cpu().numpy() if isinstance(nodes, torch.Tensor) else np.asarray(nodes)
    idx = np.searchsorted(g, nd + nn * (var - 1))
    out = f64(U_d).clone()
    if isinstance(values, (int, float)):
        return scatter_set(out, idx, float(values))
    return scatter_set(out, idx, values)


def timestep_loop(t_final, dt, save_interval, print_interval, compute_func, timestep_func, parameters,
                  dirichlet_vals, initial_states, S_func=None, phi_S_func=None, save2file=None, h5name=None):
    """setup/simulation.py:229-360 (same prints and return values). The HDF5
    streaming option needs h5py, which is not a dependency of this package."""
    if save2file:
        raise NotImplementedError("save2file needs h5py; save U_list with utils.running.save_sol instead")
    has_phi = len(initial_states) == 3
    U, P = f64(initial_states[0]), f64(initial_states[1])
    phi = f64(initial_states[2]) if has_phi else None
    U_d = dirichlet_vals[0]
    phi_d = dirichlet_vals[1] if has_phi else None
    U_iter_list, P_iter_list, step_list, U_list = [], [], [], []
    phi_iter_list, phi_list = [], []
    F_p, F = compute_func(U_d, S_func, 0, 0)
    t0 = time.perf_counter()
    if has_phi:
        _ = timestep_func(U, P, phi, dt, *parameters, U_d, phi_d, F_p, F, phi_S_func)
    else:
        _ = timestep_func(U, P, dt, *parameters, U_d, F_p, F)
    torch.cuda.synchronize()
    compile_time = time.perf_counter() - t0
    print(f"Run to compile took {compile_time:.2f} s\n")
    num_steps = int(t_final / dt)
    if num_steps * dt < t_final:
        num_steps += 1
    print("num steps:", num_steps)
    U_list, phi_list = [U.cpu()], [phi.cpu() if phi is not None else None]
    total_start = time.perf_counter()
    for step in range(1, num_steps + 1):
        U_n, P_n = U, P
        phi_n = phi
        t_n, t = (step - 1) * dt, step * dt
        start = time.perf_counter()
        F_p, F = compute_func(U_d, S_func, t_n, t)
        if has_phi:
            U, P, phi, U_iters, P_iters, phi_iters = timestep_func(U_n, P_n, phi_n, dt, *parameters, U_d, phi_d, F_p,
                                                                   F, phi_S_func)
        else:
            U, P, U_iters, P_iters = timestep_func(U_n, P_n, dt, *parameters, U_d, F_p, F)
        end = time.perf_counter()
        if step % save_interval == 0 or step == num_steps:
            U_list.append(U.cpu())
            U_iter_list.append(int(U_iters))
            P_iter_list.append(int(P_iters))
            step_list.append(step)
            if has_phi:
                phi_list.append(phi.cpu())
                phi_iter_list.append(int(phi_iters))
        if step <= 5 or step % print_interval == 0 or step == num_steps:
            diff = float(torch.linalg.vector_norm(U - U_n) / torch.linalg.vector_norm(U))
            if has_phi:
                print(f"End step {step}, time {t:.2f}, took {((end - start) * 1000):.2f} ms, {int(U_iters)} U iters, "
                      f"{int(P_iters)} P iters, {int(phi_iters)} phi iters, diff = {diff:.6f}")
            else:
                print(f"End step {step}, time {t:.2f}, took {((end - start) * 1000):.2f} ms, {int(U_iters)} U iters, "
                      f"{int(P_iters)} P iters, diff = {diff:.6f}")
    torch.cuda.synchronize()
    total_time = time.perf_counter() - total_start
    print(f"\nTotal timestepping time: {total_time:.2f} s")
    print(f"Avg of {((total_time / num_steps) * 1000):.2f} ms per timestep")
    print(f"Avg of {(((total_time + compile_time) / num_steps) * 1000):.2f} ms per timestep including compile time\n")
    U_iter_list, P_iter_list, step_list = np.array(U_iter_list), np.array(P_iter_list), np.array(step_list)
    U_list = torch.stack(U_list, dim=0)
    if has_phi:
        phi_list = torch.stack(phi_list, dim=0)
        return U, P, phi, U_iter_list, P_iter_list, np.array(phi_iter_list), step_list, U_list, phi_list
    return U, P, U_iter_list, P_iter_list, step_list, U_list


def timestep_loop_scan(dt, num_steps, compute_func, timestep_func, rho, mu, D, U_d, phi_d, U0, P0, phi0, S_func):
    """setup/simulation.py:362-374 with the step's argument order
    (U_d, phi_d, F_p, F) of solvers/passive_transport.py:177-178."""
    F_p, F = compute_func(U_d, S_func, 0, 0)
    U, P, phi = f64(U0), f64(P0), f64(phi0)
    for _ in range(int(num_steps)):
        U, P, phi, _, _, _ = timestep_func(U, P, phi, dt, rho, mu, D, U_d, phi_d, F_p, F, None)
    return U, P, phi
