"""Sharding of the excited-state basis over ranks (optim_es_sharded), on CPU
with the gloo backend and world_size 2.

The per-column work (a nested CTMRG + pullback on the GPU) is replaced by a
deterministic column function, so the test checks what the sharding adds:
every column computed exactly once, by the rank shard_indices assigns it to,
and every rank ending with the full effH / effN after the all-reduce, equal
to the single-process assembly."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import load_package


def _columns(nb):
    rng = np.random.default_rng(42)
    H = rng.standard_normal((nb, nb)) + 1j * rng.standard_normal((nb, nb))
    N = rng.standard_normal((nb, nb)) + 1j * rng.standard_normal((nb, nb))
    return H, N


def _worker(rank, world, port, nb, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        drivers = load_package().drivers
        H, N = _columns(nb)
        calls = []

        def column_fn(i):
            calls.append(i)
            return H[:, i], N[:, i]

        effH, effN = drivers.optim_es_sharded(0.5, 0.5, None, None, np.zeros((nb * 2, nb)), column_fn=column_fn)
        np.savez(os.path.join(out_dir, "r%d.npz" % rank), effH=effH, effN=effN, calls=np.array(calls))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.parametrize("nb", [7, 161])
def test_sharded_es_matches_serial(tmp_path, nb):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), nb, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    H, N = _columns(nb)
    drivers = load_package().drivers
    seen = []
    for r in range(world):
        d = np.load(tmp_path / ("r%d.npz" % r))
        assert np.array_equal(d["effH"], H) and np.array_equal(d["effN"], N)
        assert list(d["calls"]) == drivers.shard_indices(nb, r, world)
        seen += list(d["calls"])
    assert sorted(seen) == list(range(nb))
    # the eigenproblem of the gathered matrices is the serial one
    w_serial = drivers.band_energies(H @ H.conj().T, N @ N.conj().T + np.eye(nb))
    d = np.load(tmp_path / "r1.npz")
    w_shard = drivers.band_energies(d["effH"] @ d["effH"].conj().T, d["effN"] @ d["effN"].conj().T + np.eye(nb))
    assert np.allclose(w_serial, w_shard)
