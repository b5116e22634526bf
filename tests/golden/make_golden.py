"""Generate golden fixtures by executing the reference's own modules.

Run from the repository root:  python tests/golden/make_golden.py <path to the jax-fem-cfd checkout>

The reference (jax_fem_cfd) needs jax 0.4.13, which is not installable here; its
modules are executed under ``jax_shim`` (a numpy restatement of the JAX API subset
they call). Inputs are seeded with numpy.random.default_rng; outputs are written
as small .npz files next to this script. Nothing at test time imports the
reference: the tests read only these fixtures.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import jax_shim  # noqa: E402

if len(sys.argv) < 2:
    sys.exit("usage: python tests/golden/make_golden.py <path to the jax-fem-cfd checkout>")
REF = sys.argv[1]
R = jax_shim.load_reference(REF)
rm, sf, ec, em = R["regular_mesh"], R["shape_functions"], R["element_calc"], R["element_mult"]
mg, its, std, pt, sim = R["multigrid"], R["jax_iterative_solvers"], R["standard"], R["passive_transport"], R["simulation"]
W = jax_shim._wrap
A = np.asarray


def save(name, **arrs):
    out = {}
    for k, v in arrs.items():
        out[k] = np.asarray(v)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print("wrote", name, sorted(out))


# --- 1. meshes ---------------------------------------------------------------
def mesh_case(fn, args):
    nc, nconn, sn, bc, nv = fn(*args)
    d = dict(args=np.array(args, dtype=float), node_coords=nc, nconn=nconn)
    if sn is not None:
        for f in range(len(sn)):
            d[f"surf{f}"], d[f"bconn{f}"], d[f"nvec{f}"] = sn[f], bc[f], nv[f]
    return d


meshes = {
    "q1": (rm.create_mesh_2d, (4, 3, 2.0, 1.5)),
    "q2": (rm.create_mesh_2d_quad9, (3, 2, 1.0, 2.0)),
    "q1p": (rm.create_periodic_mesh_2d, (4, 4, 2 * np.pi, 2 * np.pi)),
    "q2p": (rm.create_periodic_mesh_2d_quad9, (3, 4, 1.0, 1.0)),
    "hex": (rm.create_mesh_3d, (3, 2, 2, 3.0, 1.0, 1.0)),
}
for key, (fn, args) in meshes.items():
    save(f"mesh_{key}", **mesh_case(fn, args))

# --- 2-5. shape functions, element matrices, Ce/SUPG, element mults ---------
rng = np.random.default_rng(1234)
elem_cases = {
    "q1": (rm.create_mesh_2d(5, 4, 2.0, 1.0), sf.quad4_shape_functions, 2),
    "q2": (rm.create_mesh_2d_quad9(4, 3, 1.0, 1.5), sf.quad9_shape_functions, 2),
    "q1p": (rm.create_periodic_mesh_2d(6, 4, 2 * np.pi, 2 * np.pi), sf.quad4_shape_functions, 2),
    "q2p": (rm.create_periodic_mesh_2d_quad9(4, 4, 2 * np.pi, 2 * np.pi), sf.quad9_shape_functions, 2),
    "hex": (rm.create_mesh_3d(3, 3, 2, 1.0, 1.0, 0.5), sf.hex8_shape_functions, 3),
}
for key, ((nc, nconn, sn, bc, nv), shp, ndim) in elem_cases.items():
    nn = nc.shape[0]
    wq, N, Nd = shp(nc[nconn[0]])
    Le = ec.laplacian_element_calc(wq, Nd)
    Ge = ec.gradient_element_calc(wq, N, Nd, ndim)
    Ld = ec.laplacian_diag(Le, nconn, nn)
    if ndim == 2:
        M, Me = ec.lumped_mass_matrix(nconn, wq, N, nn, ndim)
    else:  # reference lumped mass works in 3D (only consistent_mass_mult is broken)
        M, Me = ec.lumped_mass_matrix(nconn, wq, N, nn, ndim)
    U = W(rng.standard_normal(ndim * nn))
    P = W(rng.standard_normal(nn))
    phi = W(rng.standard_normal(nn))
    Ce05 = ec.conservative_convec_elem_calc(nconn, U, wq, N, Nd, nn, ndim, 0.5)
    Ce1 = ec.conservative_convec_elem_calc(nconn, U, wq, N, Nd, nn, ndim, 1)
    d = dict(nn=nn, ndim=ndim, nconn=nconn, node_coords=nc, wq=wq, N=N, Nderiv=Nd, Le=Le, Ge=Ge, L_diag=Ld,
             M=M, Me=Me, U=U, P=P, phi=phi, Ce05=Ce05, Ce1=Ce1,
             lap=em.laplacian_element_mult(P, Le, nconn, nn),
             grad=em.gradient_element_mult(P, Ge, nconn, nn, ndim),
             div=em.divergence_element_mult(U, Ge, nconn, nn, ndim),
             viscconv=em.visc_conv_mult(U, Ce05, Le, 0.013, 1.7, nconn, nn, ndim),
             scalar_vc=em.scalar_visc_conv_mult(phi, Ce1, Le, 1e-3, nconn, nn),
             mass1=em.consistent_mass_mult(phi, Me, nconn, nn, 1))
    if ndim == 2:
        Ct = ec.Ctau_tilde_elem_calc(nconn, U, wq, N, Nd, nn, ndim)
        tau = ec.calculate_tau(nconn, U, Ce1, Ct, N, nn, ndim, 1e-4, 1e-2, 2)
        Mtau = tau[:, None, None] * Ce1.transpose(0, 2, 1)
        d.update(mass=em.consistent_mass_mult(U, Me, nconn, nn, ndim), Ctau_tilde=Ct, tau=tau,
                 stab_vc=em.scalar_stabilized_visc_conv_mult(phi, Ce1, tau[:, None, None] * Ct, Le, 1e-3, nconn, nn),
                 supg_mass=em.scalar_consistent_mass_SUPG_mult(phi, Mtau, Me, nconn, nn))
    save(f"elem_{key}", **d)

# 1D boundary shape functions on a tilted edge
for key, shp, coords in [("lin2", sf.lin2_shape_functions, np.array([[0.0, 0.0], [0.3, 0.4]])),
                         ("lin3", sf.lin3_shape_functions, np.array([[0.0, 0.0], [0.15, 0.2], [0.3, 0.4]]))]:
    wq, N, Nd = shp(W(coords))
    save(f"shape_{key}", coords=coords, wq=wq, N=N, Nderiv=Nd)

# --- 6. multigrid ------------------------------------------------------------
for key, nel, order, periodic, fmg, setzero, dom in [
        ("q1", [16, 16], 1, False, [4, 4], True, [1.0, 1.0]),
        ("q2", [8, 8], 2, False, [2, 2], True, [1.0, 1.0]),
        ("q1p", [16, 16], 1, True, [4, 4], False, [2 * np.pi, 2 * np.pi]),
        ("q2p", [16, 16], 2, True, [4, 4], False, [2 * np.pi, 2 * np.pi])]:
    if order == 1:
        mf, shp = (rm.create_periodic_mesh_2d if periodic else rm.create_mesh_2d), sf.quad4_shape_functions
    else:
        mf, shp = (rm.create_periodic_mesh_2d_quad9 if periodic else rm.create_mesh_2d_quad9), sf.quad9_shape_functions
    lvl, Le_l, nconn_l, Ld_l, gp_l = mg.multigrid_setup(nel, fmg, dom, [], mf, shp, order, None)
    nn0 = lvl[1][0]
    r = rng.standard_normal(nn0)
    if not setzero:
        r = r - r.mean()
    else:
        r[0] = 0.0
    r = W(r)
    z = mg.v_cycle(r, lvl, Le_l, nconn_l, Ld_l, gp_l, 1e-8, periodic, setzero)
    # one transfer pair between levels 0 and 1
    xH = W(rng.standard_normal(lvl[2][0] - lvl[1][0]))
    xh = W(rng.standard_normal(nn0))
    P_ = mg.interpolation_operator(xH, lvl[2][1], lvl[2][2], lvl[1][1], lvl[1][2], periodic)
    R_ = mg.restriction_operator(xh, lvl[1][1], lvl[1][2], lvl[2][1], lvl[2][2], periodic)
    save(f"mg_{key}", lvl_nums=np.array(lvl), Le_lvls=Le_l, nconn_lvls=nconn_l, L_diag_lvls=Ld_l,
         gamma_p_lvls=gp_l, r=r, z=z, xH=xH, xh=xh, interp=P_, restrict=R_,
         nel=np.array(nel), order=order, periodic=periodic, fmg=np.array(fmg), setzero=setzero,
         dom=np.array(dom))

# --- 7. Krylov solvers on EBE operators --------------------------------------
nc, nconn, sn, bc, nv = rm.create_mesh_2d(10, 10, 1.0, 1.0)
nn = nc.shape[0]
wq, N, Nd = sf.quad4_shape_functions(nc[nconn[0]])
Le = ec.laplacian_element_calc(wq, Nd)
M, Me = ec.lumped_mass_matrix(nconn, wq, N, nn, 2)
gp = A(sn[0])
b = rng.standard_normal(nn)
b[gp] = 0.0
b = W(b)


def lap_op(x):
    return em.laplacian_element_mult(x, Le, nconn, nn).at[gp].set(0)


x_cg, k_cg = its.cg(lap_op, b, tol=1e-10, maxiter=1000)
Ld = ec.laplacian_diag(Le, nconn, nn)
x_pcg, k_pcg = its.cg(lap_op, b, tol=1e-10, maxiter=1000, M=lambda r: r / Ld)
U = W(0.3 * rng.standard_normal(2 * nn))
Ce = ec.conservative_convec_elem_calc(nconn, U, wq, N, Nd, nn, 2, 0.5)


def mom_op(x):
    return (1.0 / 0.01) * em.consistent_mass_mult(x, Me, nconn, nn, 2) + 0.5 * em.visc_conv_mult(
        x, Ce, Le, 0.01, 1.0, nconn, nn, 2)


bm = W(rng.standard_normal(2 * nn))
x_bi, k_bi = its.bicgstab(mom_op, bm, tol=1e-10)
save("krylov", b=b, gp=gp, x_cg=x_cg, k_cg=k_cg, x_pcg=x_pcg, k_pcg=k_pcg, U=U, bm=bm, x_bi=x_bi, k_bi=k_bi)


# --- 8-10. full steps through the reference API ------------------------------
def ns_config(nel, dom, order, periodic, dfaces, precond, setzero, tol, fmg, outlet=()):
    return sim.Config(mesh="simple", solver="standard",
                      mesh_config=sim.SimpleMeshConfig(num_elem=nel, domain_size=dom, shape_func_ord=order,
                                                       periodic=periodic),
                      solver_config=sim.StandardSolverConfig(dirichlet_faces=dfaces, symmetry_faces=[],
                                                             outlet_faces=list(outlet), streamline_diff=False,
                                                             solver_tol=tol, set_zeroP=setzero,
                                                             pressure_precond=precond, final_multigrid_mesh=fmg))


def run_ns(name, cfg, steps, dt, rho, mu, init, lid):
    compute, timestep, nc, sn, h, nn, gd, Ud = sim.setup(cfg)
    if lid is not None:
        Ud = sim.set_face_velocity(Ud, sn[2] if lid == "corners" else sn[2][1:-1], gd, 1.0, nn, var=1)
    ndim = len(cfg.mesh_config.num_elem)
    if init == "zero":
        U0, P0 = np.zeros(ndim * nn), np.zeros(nn)
    else:
        x, y = nc[:, 0], nc[:, 1]
        U0 = np.concatenate([np.sin(x) * np.cos(y), -np.cos(x) * np.sin(y)])
        P0 = (rho / 4) * (np.cos(2 * x) + np.cos(2 * y))
        P0 = P0 - (P0[0] if cfg.solver_config.set_zeroP else P0.mean())
    U, P = W(U0), W(P0)
    Ui, Pi, Fps = [], [], []
    for s in range(steps):
        Fp, F = compute(Ud, None, s * dt, (s + 1) * dt)
        U, P, ui, pi = timestep(U, P, dt, rho, mu, Ud, Fp, F)
        Ui.append(int(ui))
        Pi.append(int(pi))
        Fps.append(np.asarray(Fp) if not np.isscalar(Fp) else np.zeros(nn))
    save(name, U0=U0, P0=P0, U=U, P=P, U_iters=np.array(Ui), P_iters=np.array(Pi),
         U_d=(A(Ud) if Ud is not None else np.zeros(0)), gamma_d=(A(gd) if gd is not None else np.zeros(0, int)),
         F_p=Fps[-1], dt=dt, rho=rho, mu=mu, steps=steps)


run_ns("step_cavity_q1_mg", ns_config([16, 16], [1, 1], 1, False, [0, 1, 2, 3], "multigrid", True, 1e-8, [4, 4]),
       3, 0.01, 1.0, 0.01, "zero", "corners")
run_ns("step_cavity_q2_jacobi", ns_config([8, 8], [1, 1], 2, False, [0, 1, 2, 3], "jacobi", True, 1e-8, None),
       2, 0.01, 1.0, 0.01, "zero", "interior")
run_ns("step_cavity_q1_approxinv", ns_config([12, 12], [1, 1], 1, False, [0, 1, 2, 3], "approx_inv", True, 1e-8,
                                             None), 2, 0.01, 1.0, 0.01, "zero", "corners")
run_ns("step_tg_q2p_mg", ns_config([16, 16], [2 * np.pi, 2 * np.pi], 2, True, [], "multigrid", False, 1e-8, [4, 4]),
       3, 1e-3, 1.0, 0.01, "tg", None)
run_ns("step_tg_q1p_none", ns_config([16, 16], [2 * np.pi, 2 * np.pi], 1, True, [], None, False, 1e-8, None),
       2, 1e-2, 1.0, 0.01, "tg", None)
# channel with an outlet face (pinned gamma_p = outlet nodes) and inflow on the left
cfg = ns_config([16, 8], [2.0, 1.0], 1, False, [0, 2, 3], "multigrid", True, 1e-8, [4, 2], outlet=[1])
compute, timestep, nc, sn, h, nn, gd, Ud = sim.setup(cfg)
yL = nc[A(sn[3]), 1]
Ud = sim.set_face_velocity(Ud, sn[3], gd, W(4 * yL * (1 - yL)), nn, var=1)
U, P = W(np.zeros(2 * nn)), W(np.zeros(nn))
Fp, F = compute(Ud, None, 0.0, 0.01)
U1, P1, ui, pi = timestep(U, P, 0.01, 1.0, 0.02, Ud, Fp, F)
save("step_channel_q1_outlet", U_d=Ud, gamma_d=gd, F_p=Fp, U=U1, P=P1, U_iters=np.array([int(ui)]),
     P_iters=np.array([int(pi)]), dt=0.01, rho=1.0, mu=0.02, steps=1)

# passive transport (SUPG and plain)
for supg in (True, False):
    cfg = sim.Config(mesh="simple", solver="passive_transport",
                     mesh_config=sim.SimpleMeshConfig(num_elem=[12, 12], domain_size=[1, 1], shape_func_ord=1,
                                                      periodic=False),
                     solver_config=sim.PassiveTransportConfig(
                         sim.StandardSolverConfig(dirichlet_faces=[0, 1, 2, 3], symmetry_faces=[], outlet_faces=[],
                                                  streamline_diff=False, solver_tol=1e-8, set_zeroP=True,
                                                  pressure_precond="multigrid", final_multigrid_mesh=[3, 3]),
                         sim.ADEConfig(phi_dirichlet_faces=[], phi_SUPG=supg)))
    compute, timestep, nc, sn, h, nn, nnx, nny, gd, Ud, gdp = sim.setup(cfg)
    x, y = nc[:, 0], nc[:, 1]
    U0 = np.concatenate([-5 * (y - 0.5), 5 * (x - 0.5)])
    phi0 = ((x >= 0.4) & (x <= 0.6) & (y >= 0.2) & (y <= 0.4)).astype(float)
    U, P, phi = W(U0), W(np.zeros(nn)), W(phi0)
    its_ = []
    for s in range(2):
        Fp, F = compute(Ud, None, 0, 0)
        U, P, phi, ui, pi, fi = timestep(U, P, phi, 0.01, 1.0, 0.01, 1e-4, Ud, None, Fp, F, None)
        its_.append((int(ui), int(pi), int(fi)))
    save(f"step_transport_{'supg' if supg else 'plain'}", U0=U0, phi0=phi0, U=U, P=P, phi=phi,
         iters=np.array(its_), dt=0.01, rho=1.0, mu=0.01, D=1e-4, steps=2)
