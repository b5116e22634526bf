"""Serving path: request generator (CPU) and the continuous-batching loop (GPU):
a served request matches the oracle's 4-step projection, each result is the
same alone and in a mix, and the plain one-at-a-time path agrees."""
import numpy as np
import pytest
import torch

from tests.test_gpu_parity import SOLVE_TOL, rel


def test_fourier_velocity_is_divergence_free_and_normalised():
    from jax_fem_cfd_b200.serving import fourier_velocity
    n = 64
    U = fourier_velocity(n, 3)
    assert np.abs(np.hypot(U[:(n + 1) ** 2], U[(n + 1) ** 2:])).max() == pytest.approx(1.0, abs=1e-15)
    np.testing.assert_array_equal(U, fourier_velocity(n, 3))
    assert not np.array_equal(U, fourier_velocity(n, 4))
    u = U[:(n + 1) ** 2].reshape(n + 1, n + 1)
    v = U[(n + 1) ** 2:].reshape(n + 1, n + 1)
    h = 1.0 / n
    dudx = (u[1:-1, 2:] - u[1:-1, :-2]) / (2 * h)
    dvdy = (v[2:, 1:-1] - v[:-2, 1:-1]) / (2 * h)
    dudy = (u[2:, 1:-1] - u[:-2, 1:-1]) / (2 * h)
    # central differences of a curl: divergence is O(h^2) against the gradients
    assert np.abs(dudx + dvdy).max() < 0.1 * np.abs(dudy).max()


def test_request_stream_is_seeded():
    from jax_fem_cfd_b200.serving import SIZES, make_requests
    a = make_requests(12, seed=5, steps=7, rate=100.0)
    b = make_requests(12, seed=5, steps=7, rate=100.0)
    assert [(r.n, r.nu, r.arrival) for r in a] == [(r.n, r.nu, r.arrival) for r in b]
    assert all(r.n in SIZES and 1e-3 <= r.nu <= 1e-1 and r.steps == 7 for r in a)
    assert all(x.arrival < y.arrival for x, y in zip(a, a[1:]))
    assert all(r.dt == pytest.approx(0.25 / r.n) for r in a)
    assert all(r.arrival == 0.0 for r in make_requests(3, rate=None))


def test_cta_share():
    from jax_fem_cfd_b200.serving import ctas_for
    assert [ctas_for(n, 37) for n in (32, 64, 128, 256)] == [3, 9, 33, 37]
    assert ctas_for(256, 200) == 130


@pytest.fixture(scope="module")
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)


def _oracle_steps(req):
    import oracle.simulation as osim
    cfg = osim.Config(mesh="simple", solver="standard",
                      mesh_config=osim.SimpleMeshConfig(num_elem=[req.n, req.n], domain_size=[1.0, 1.0],
                                                        shape_func_ord=1, periodic=False),
                      solver_config=osim.StandardSolverConfig(dirichlet_faces=[0, 1, 2, 3], symmetry_faces=[],
                                                              outlet_faces=[], streamline_diff=False, solver_tol=1e-8,
                                                              set_zeroP=True, pressure_precond="multigrid",
                                                              final_multigrid_mesh=[4, 4]))
    compute, timestep, nc, sn, h, nn, gd, Ud = osim.setup(cfg)
    U, P = req.U0.copy(), np.zeros(nn)
    for s in range(req.steps):
        Fp, F = compute(Ud, None, s * req.dt, (s + 1) * req.dt)
        U, P, _, _ = timestep(U, P, req.dt, 1.0, req.nu, Ud, Fp, F)
    return U, P


@pytest.mark.gpu
def test_served_request_matches_oracle(_cuda):
    from jax_fem_cfd_b200.serving import Server, make_requests
    req = make_requests(1, seed=11, sizes=(32,), steps=3)[0]
    done, m = Server(chunk=2).run([req])
    assert m["requests"] == 1 and done[0]["status"] == 0
    U, P = _oracle_steps(req)
    assert rel(done[0]["U"], U) < SOLVE_TOL
    assert rel(done[0]["P"], P) < SOLVE_TOL


@pytest.mark.gpu
def test_each_result_same_alone_and_in_the_mix(_cuda):
    from jax_fem_cfd_b200.serving import Server, make_requests, run_plain
    reqs = make_requests(7, seed=2, sizes=(32, 64, 128), steps=6)
    srv = Server(chunk=2)
    mix, m = srv.run(reqs)
    assert m["requests"] == len(reqs)
    by_id = {d["rid"]: d for d in mix}
    for r in reqs:
        alone, _ = srv.run([r])
        assert by_id[r.rid]["status"] == 0
        np.testing.assert_array_equal(alone[0]["U"], by_id[r.rid]["U"])
        np.testing.assert_array_equal(alone[0]["P"], by_id[r.rid]["P"])
    # the plain path launches the same grids at these sizes (nodes / 512 CTAs
    # are under the share), so it reproduces the served results exactly
    plain, _ = run_plain(reqs, srv)
    for d in plain:
        np.testing.assert_array_equal(d["U"], by_id[d["rid"]]["U"])


@pytest.mark.gpu
def test_share_changes_grid_but_not_the_solution(_cuda):
    """256^2 requests run on their 37-CTA share when served and on the whole
    device when plain: different reduction orders, same solution to 1e-10."""
    from jax_fem_cfd_b200.serving import Server, make_requests, run_plain
    reqs = make_requests(2, seed=9, sizes=(256,), steps=2)
    srv = Server(chunk=1)
    served, _ = srv.run(reqs)
    plain, _ = run_plain(reqs, srv)
    s = {d["rid"]: d for d in served}
    for d in plain:
        assert rel(s[d["rid"]]["U"], d["U"]) < SOLVE_TOL
        assert rel(s[d["rid"]]["P"], d["P"]) < SOLVE_TOL


@pytest.mark.gpu
def test_autotuned_shares_and_graph_chunks(_cuda):
    """The autotuner picks a cap from its candidates; chunks replayed from
    captured graphs give the same bits as the same steps launched one by one."""
    from jax_fem_cfd_b200.serving import Server, make_requests
    srv = Server(chunk=2)
    reqs = make_requests(4, seed=4, sizes=(32, 64), steps=5)
    t = srv.autotune(reqs, caps=(4, 8), sample=3, sample_steps=2)
    assert t["picked"] in (4, 8) and srv.share == t["picked"]
    graphed, m = srv.run(reqs)
    assert m["graphs"], m["graph_error"]
    direct = Server(share=srv.share, chunk=2, graphs=False)
    plain, m2 = direct.run(reqs)
    assert not m2["graphs"]
    g = {d["rid"]: d for d in graphed}
    for d in plain:
        assert d["status"] == 0 and g[d["rid"]]["status"] == 0
        np.testing.assert_array_equal(d["U"], g[d["rid"]]["U"])
        np.testing.assert_array_equal(d["P"], g[d["rid"]]["P"])


@pytest.mark.gpu
def test_packed_members_equal_their_solo_runs(_cuda):
    """A Pack of four 32^2 members: three requests with their own viscosity and
    time step run 3 + 2, 2 + 3 and 1 + 4 steps over two packed launches (so
    they start the second launch from different buffers), the fourth stays
    idle. Each result equals its solver's solo fem_step4 steps on the same CTA
    count bit for bit, with zero statuses; the idle member's buffers are
    untouched."""
    from jax_fem_cfd_b200.serving import Pack, Slot, make_requests
    reqs = make_requests(3, seed=21, sizes=(32,), steps=5)
    ctas = 3
    pack = Pack(32, 4, ctas)
    st = torch.cuda.current_stream()
    for m, r in enumerate(reqs):
        pack.slots[m].U[0].copy_(torch.from_numpy(r.U0))
        pack.slots[m].P[0].zero_()
    idle = pack.slots[3]
    idle.U[0].fill_(0.25)
    idle.P[0].fill_(-0.5)
    dt = [r.dt for r in reqs] + [1.0]
    mu = [r.nu for r in reqs] + [0.0]
    first = [3, 2, 1, 0]
    pack.step(dt, mu, first, [0, 0, 0, 0], st)
    cur = [k & 1 for k in first]
    second = [2, 3, 4, 0]
    pack.step(dt, mu, second, cur, st)
    cur = [c ^ (k & 1) for c, k in zip(cur, second)]
    torch.cuda.synchronize()
    stat = pack.stat.cpu().numpy().reshape(4, 5)
    assert (stat[:3, 2:] == 0).all(), stat
    assert (stat[:3, :2] > 0).all(), stat
    assert torch.equal(idle.U[0], torch.full_like(idle.U[0], 0.25))
    assert torch.equal(idle.P[0], torch.full_like(idle.P[0], -0.5))
    solo = Slot(32)
    solo.set_ctas(ctas)
    for m, r in enumerate(reqs):
        solo.U[0].copy_(torch.from_numpy(r.U0))
        solo.P[0].zero_()
        c = solo.steps(0, 5, r.dt, r.nu, st)
        torch.cuda.synchronize()
        assert int(solo.solver.status.max()) == 0
        assert torch.equal(pack.slots[m].U[cur[m]], solo.U[c]), m
        assert torch.equal(pack.slots[m].P[cur[m]], solo.P[c]), m
    pack.close()


@pytest.mark.gpu
def test_packed_server_matches_the_stream_server(_cuda):
    """Seven requests of two sizes through packs of two members each (so
    members are reused) give the stream server's results on the same CTA
    shares, bit for bit."""
    from jax_fem_cfd_b200.serving import PackedServer, Server, make_requests
    reqs = make_requests(7, seed=4, sizes=(32, 64), steps=12)
    ps = PackedServer(share=16, chunk=4, members={32: 2, 64: 2})
    packed, m = ps.run(reqs, realtime=False)
    assert m["requests"] == len(reqs) and m["members"] == {32: 2, 64: 2}
    srv = Server(share=16, chunk=4)
    ref, _ = srv.run(reqs, realtime=False)
    by_id = {d["rid"]: d for d in ref}
    for d in packed:
        assert d["status"] == 0 and by_id[d["rid"]]["status"] == 0
        np.testing.assert_array_equal(d["U"], by_id[d["rid"]]["U"])
        np.testing.assert_array_equal(d["P"], by_id[d["rid"]]["P"])


@pytest.mark.gpu
@pytest.mark.parametrize("n", [64, 128, 256])
def test_served_and_packed_requests_match_the_oracle(_cuda, n):
    """One request of each larger mesh size, 10 steps, served on its own stream
    and served as a pack member, against the oracle's steps."""
    from jax_fem_cfd_b200.serving import PackedServer, Server, make_requests
    req = make_requests(1, seed=30 + n, sizes=(n,), steps=10)[0]
    U, P = _oracle_steps(req)
    served, _ = Server(chunk=2).run([req])
    ps = PackedServer(chunk=4, members={n: 1})
    packed, _ = ps.run([req], realtime=False)
    for p in ps.packs.values():
        p.close()
    for d in (served[0], packed[0]):
        assert d["status"] == 0
        assert rel(d["U"], U) < SOLVE_TOL and rel(d["P"], P) < SOLVE_TOL, (rel(d["U"], U), rel(d["P"], P))


@pytest.mark.gpu
def test_pack_launch_beyond_capacity_is_refused(_cuda):
    """Two 100-CTA members do not fit on the device together: a call with both
    active is refused on the host (nothing launched); one active member runs."""
    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.serving import Pack
    pack = Pack(256, 2, 100)
    st = torch.cuda.current_stream()
    with pytest.raises(_lib.FemError):
        pack.step([1e-3, 1e-3], [1e-2, 1e-2], [1, 1], [0, 0], st)
    pack.step([1e-3, 1e-3], [1e-2, 1e-2], [1, 0], [0, 0], st)
    torch.cuda.synchronize()
    stat = pack.stat.cpu().numpy().reshape(2, 5)
    assert (stat[0, 2:] == 0).all() and (stat[1] == 0).all(), stat
    pack.close()
