"""Sharded permutation test across two CPU ranks (gloo) == one process."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from fastpls_b200 import replicas, workloads as W


def oracle_compute(x, y, folds, perms, prefixes, metric="q2"):
    from oracle import pls_oracle as O
    rows = [O.cv_regression(x, y, folds, prefixes, family=3)[metric]]
    for p in perms:
        rows.append(O.cv_regression(x, y[p], folds, prefixes, family=3)[metric])
    return np.stack(rows)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    x, y = W.latent_regression(60, 25, 2, 3, 0.4, 5, dtype=np.float64)
    folds = W.uneven_folds(60, 3, 5)
    perms = W.permutations(60, 5, 5)
    obs, permuted, pv = replicas.permutation_test(
        x, y, folds, perms, [1, 2, 3], world=world, rank=rank,
        compute=oracle_compute)
    np.savez(os.path.join(out_dir, f"r{rank}.npz"), obs=obs, permuted=permuted, pv=pv)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_covers_range():
    for count in (0, 1, 7, 200):
        for world in (1, 2, 3, 8):
            spans = [replicas.shard(count, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == count
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))


def test_two_rank_permutation_test_matches_single(tmp_path):
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2,
                       start_method="spawn")
    x, y = W.latent_regression(60, 25, 2, 3, 0.4, 5, dtype=np.float64)
    folds = W.uneven_folds(60, 3, 5)
    perms = W.permutations(60, 5, 5)
    obs, permuted, pv = replicas.permutation_test(
        x, y, folds, perms, [1, 2, 3], compute=oracle_compute)
    for r in range(2):
        got = np.load(tmp_path / f"r{r}.npz")
        assert np.allclose(got["obs"], obs)
        assert np.allclose(got["permuted"], permuted)
        assert np.allclose(got["pv"], pv, equal_nan=True)
