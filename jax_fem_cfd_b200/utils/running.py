"""Solution / iteration-history files (drop-in for jax_fem_cfd utils/running.py):
the same .npy layouts, [len(U), U, p] and stacked (momentum, pressure, steps)."""
import os

import numpy as np
import torch


def use_single_gpu(DEVICE_ID):
    """utils/running.py:4-10."""
    os.environ["CUDA_DEVICE_ORDER"] = "PCI_BUS_ID"
    os.environ["CUDA_VISIBLE_DEVICES"] = "" if DEVICE_ID is None else str(DEVICE_ID)


def _np(x):
    return x.detach().cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x)


def save_sol(U, p, sol_path):
    """utils/running.py:16-19."""
    U, p = _np(U), _np(p)
    np.save(sol_path, np.concatenate((np.array([U.shape[0]]), U, p)))
    print("Saved solution to", sol_path)


def load_sol(sol_path):
    """utils/running.py:21-26."""
    sol = np.load(sol_path)
    U = sol[1:(1 + int(sol[0]))]
    p = sol[(1 + int(sol[0])):]
    print("Loaded solution from", sol_path)
    return U, p


def save_iter_hist(momentum_list, pressure_list, steps, path):
    """utils/running.py:28-31."""
    np.save(path, np.stack((momentum_list, pressure_list, steps), axis=0))
    print("Saved linear solver iteration counts to", path)


def load_iter_hist(path):
    """utils/running.py:33-38."""
    hist = np.load(path)
    print("Loaded iteration counts from", path)
    return hist[0, :], hist[1, :], hist[2, :]
