"""The replica path of bench.py --gpus N on CPU: two gloo ranks (127.0.0.1)
each advance the same seeded two-mode Holstein chain one TDVP-PS2 step on
the test stand-in engine; the populations agree across ranks to the bit,
and the reduced time is the maximum over ranks (bench.reduce_max_ms), from
which the whole-job value world * steps / t_max follows."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import fake_engine
        from renormalizer_b200 import _native
        from renormalizer_b200.backend import Backend
        fake = fake_engine.FakeEngine()
        _native.Engine.get = classmethod(lambda cls, device=None: fake)
        Backend.device = property(lambda self: torch.device("cpu"))
        import bench
        from renormalizer_b200 import Mpo, backend
        backend.prec = "fp64"
        model = bench.holstein_2mode(2, 4)
        mpo = Mpo(model)
        mps = bench.initial_state(model, 6)
        mps = mps.evolve(mpo, 0.025)
        pops = torch.tensor(mps.e_occupations, dtype=torch.float64)
        gathered = [torch.zeros_like(pops) for _ in range(world)]
        dist.all_gather(gathered, pops)
        own = 10.0 * (rank + 1)             # a per-rank device time, ms
        tmax = bench.reduce_max_ms(own, dist, torch.device("cpu"))
        out[rank] = (tmax, [g.numpy() for g in gathered])
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_replicas_two_gloo_ranks():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        tmax, pops = res[rank]
        assert tmax == 20.0
        np.testing.assert_array_equal(pops[0], pops[1])
    assert abs(res[0][1][0].sum() - 1.0) < 1e-10
