"""Host logic of the t-slab decomposition on the CPU: the slab bounds, and the NCCL id
handed over a world_size-2 gloo process group to every rank's slab handle."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from su2_b200 import slabs


@pytest.mark.parametrize("Lt,n", [(8, 1), (8, 2), (8, 4), (12, 3), (12, 6), (32, 16)])
def test_slab_bounds_cover_the_lattice_once(Lt, n):
    b = [slabs.slab_bounds(Lt, n, r) for r in range(n)]
    assert b[0][0] == 0 and b[-1][1] == Lt
    assert all(b[r][1] == b[r + 1][0] for r in range(n - 1))
    assert all((t1 - t0) % 2 == 0 and t1 > t0 for t0, t1 in b)


@pytest.mark.parametrize("Lt,n,r", [(8, 3, 0), (8, 8, 0), (8, 16, 0), (8, 2, 2), (8, 0, 0),
                                    (0, 1, 0), (-4, 2, 0)])
def test_slab_bounds_reject_what_the_library_rejects(Lt, n, r):
    with pytest.raises(ValueError):
        slabs.slab_bounds(Lt, n, r)


@pytest.mark.parametrize("L,Lt,n,first,count", [
    (4, 8, 3, 0, 3), (4, 8, 8, 0, 8), (4, 0, 1, 0, 1), (4, -4, 2, 0, 2), (4, 8, 2, 1, 2),
    (4, 8, 0, 0, 1), (1024, 1024, 512, 0, 1), (65536, 65536, 2, 0, 1)])
def test_slabs_create_refuses_before_touching_a_device(L, Lt, n, first, count):
    """su2b_slabs_create checks the decomposition and the whole lattice's volume (at most
    2^29 sites, also for extents whose product wraps 64 bits) before any CUDA call, so these
    run on a machine without a GPU."""
    import ctypes as C
    from su2_b200 import _abi
    lib = _abi.load()
    h = C.c_void_p()
    rc = lib.su2b_slabs_create(L, L, L, Lt, 4, 2.3, 1.0, _abi.PREC_FP64, n, first, count, 0,
                               C.byref(h))
    assert rc == _abi.ERR_INVALID and not h.value


class _Handle:
    """Stands in for a slab_lattice: records the connect call."""

    def __init__(self, nslabs, first, count=1):
        self.nslabs, self.first, self.count = nslabs, first, count
        self.connected = None

    def connect(self, uid, nranks, rank):
        self.connected = (uid, nranks, rank)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q, first):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        h = _Handle(world, first[rank])
        try:
            slabs.connect_process_group(h, dist, make_id=lambda: bytes(range(128)))
            q.put((rank, h.connected, None))
        except ValueError as e:
            q.put((rank, h.connected, str(e)))
    finally:
        dist.destroy_process_group()


def _run(first):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q, first)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


def test_two_ranks_join_with_rank_zeros_id():
    out = _run(first=[0, 1])
    for rank, connected, err in out:
        assert err is None
        assert connected == (bytes(range(128)), 2, rank)


def test_a_rank_holding_the_wrong_slab_raises_after_the_broadcast():
    """Rank 1 claims slab 0: it raises, rank 0 still connects (nobody waits forever)."""
    out = _run(first=[0, 0])
    assert out[0][2] is None and out[0][1] == (bytes(range(128)), 2, 0)
    assert out[1][2] is not None and out[1][1] is None
