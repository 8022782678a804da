"""The replica plumbing of bench.py on CPU: two gloo ranks, barrier, max over ranks and the whole-job rate."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import bench
    ranks = bench.Ranks(backend='gloo')
    ranks.barrier()
    slowest = ranks.max(10.0 + rank)          # each rank "took" 10 + rank ms
    out.put((rank, slowest, bench.replica_rate(ranks.world, 1000, 5, slowest)))
    ranks.close()


def test_two_gloo_ranks():
    torch = pytest.importorskip('torch')
    mp = torch.multiprocessing.get_context('spawn')
    out = mp.Queue()
    port = _free_port()
    procs = [mp.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in results] == [11.0, 11.0]
    assert results[0][2] == pytest.approx(2 * 1000 * 5 / 0.011)


def test_roofline_names_the_running_sweep(monkeypatch):
    """The bench line's roofline names the sweep kernel the library runs for the workload's precision form: the
    one-cell tile in FP64, the packed two-cell kernel in the mixed form, or what CAVITY_SWEEP selects."""
    import bench
    monkeypatch.delenv('CAVITY_SWEEP', raising=False)
    assert bench.sweep_kernel_name('fp64') == 'sweep_tile_kernel'
    assert bench.sweep_kernel_name('mixed') == 'sweep_pair_kernel'
    for kind, name in (('tile', 'sweep_tile_kernel'), ('face', 'momentum_kernel'), ('march', 'sweep_march_kernel')):
        monkeypatch.setenv('CAVITY_SWEEP', kind)
        assert bench.sweep_kernel_name('mixed') == name
