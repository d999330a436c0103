"""Multi-rank path on CPU: two gloo ranks shard a batch of pulses, each
propagates its shard (here with the CPU oracle standing in for the GPU), and
the gathered results equal a single-process run; timings reduce to the max."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from mpc_tdse.parallel import shard


def test_shard_partitions_exactly():
    for n in (0, 1, 7, 256, 257):
        for world in (1, 2, 3, 8):
            parts = [shard(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_path):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "mp-citdse_b200"))
    sys.path.insert(0, os.path.join(root, "oracle"))
    import datetime

    import torch.distributed as dist

    from mpc_tdse.parallel import propagate_sharded
    from mpc_tdse.systems import hydrogen_like_1e
    from oracle import Oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    o = Oracle()
    s = hydrogen_like_1e(12, 2, gauge="l", seed=1)
    ev, wc = o.units()
    pulses = [o.pulse_setup("sine", "l", I * wc, w * ev, 0.0, 1, 0.0)
              for I, w in [(1e14, 1.5), (2e14, 2.0), (5e13, 2.5), (3e14, 1.8), (1e14, 3.0)]]

    def run(items):
        rows = []
        for p in items:
            x0 = np.zeros(s.ntot, complex)
            x0[0] = 1
            x, *_ = o.propagate(s.n, s.eig, s.dip, "l", "sineEE", p, 0.0, 0.1, 50, x0)
            rows.append(x)
        rows = np.array(rows).reshape(len(items), s.ntot)
        return rows, 50 * len(items), 0.5 + rank

    allrows, units, sec = propagate_sharded(run, pulses, rank, world, dist)
    if rank == 0:
        np.savez(out_path, rows=allrows, units=units, sec=sec)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_equal_one_process(tmp_path):
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "oracle"))
    from mpc_tdse.systems import hydrogen_like_1e
    from oracle import Oracle

    out = tmp_path / "r.npz"
    mp.start_processes(_worker, args=(2, _free_port(), str(out)), nprocs=2, join=True,
                       start_method="spawn")
    z = np.load(out)
    o = Oracle()
    s = hydrogen_like_1e(12, 2, gauge="l", seed=1)
    ev, wc = o.units()
    want = []
    for I, w in [(1e14, 1.5), (2e14, 2.0), (5e13, 2.5), (3e14, 1.8), (1e14, 3.0)]:
        p = o.pulse_setup("sine", "l", I * wc, w * ev, 0.0, 1, 0.0)
        x0 = np.zeros(s.ntot, complex)
        x0[0] = 1
        want.append(o.propagate(s.n, s.eig, s.dip, "l", "sineEE", p, 0.0, 0.1, 50, x0)[0])
    assert np.array_equal(z["rows"], np.array(want))
    assert int(z["units"]) == 250 and float(z["sec"]) == 1.5
