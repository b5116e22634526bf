"""Solution and iteration-history files keep the reference's .npy layouts
(utils/running.py:16-38): a solution is one 1-D array [len(U), U..., p...],
a history is the (3, n) stack of momentum iterations, pressure iterations and
steps. Files written here must read back with the reference's own slicing, and
files laid out by hand the reference's way must load here."""
import numpy as np
import torch

from jax_fem_cfd_b200.utils import running


def test_solution_file_layout_and_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    U, p = rng.standard_normal(2 * 25), rng.standard_normal(25)
    path = str(tmp_path / "sol.npy")
    running.save_sol(torch.from_numpy(U), torch.from_numpy(p), path)
    raw = np.load(path)
    assert raw.shape == (1 + U.size + p.size,)
    assert raw[0] == U.size
    np.testing.assert_array_equal(raw[1:1 + U.size], U)
    np.testing.assert_array_equal(raw[1 + U.size:], p)
    U2, p2 = running.load_sol(path)
    np.testing.assert_array_equal(U2, U)
    np.testing.assert_array_equal(p2, p)


def test_solution_written_the_reference_way_loads(tmp_path):
    U, p = np.arange(6.0), -np.arange(3.0)
    path = str(tmp_path / "ref_sol.npy")
    np.save(path, np.concatenate((np.array([U.shape[0]]), U, p)))  # utils/running.py:16-19
    U2, p2 = running.load_sol(path)
    np.testing.assert_array_equal(U2, U)
    np.testing.assert_array_equal(p2, p)


def test_iteration_history_round_trip(tmp_path):
    mom, prs, steps = np.array([3, 4, 3]), np.array([15, 14, 12]), np.array([1, 2, 3])
    path = str(tmp_path / "hist.npy")
    running.save_iter_hist(mom, prs, steps, path)
    raw = np.load(path)
    assert raw.shape == (3, 3)
    np.testing.assert_array_equal(raw, np.stack((mom, prs, steps)))
    m2, p2, s2 = running.load_iter_hist(path)
    np.testing.assert_array_equal(m2, mom)
    np.testing.assert_array_equal(p2, prs)
    np.testing.assert_array_equal(s2, steps)
