"""The exchange steps of the distributed solve (ryoanji_b200/let.py) on CPU ranks over gloo: the global box and the
all-to-all of packed exports. The export and the traversal of the received trees run on the GPU
(tests/test_gpu_let.py)."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from ryoanji_b200.let import exchange, global_box
        rng = np.random.default_rng(rank)
        # each rank holds a different cloud; rank 2 holds nothing
        n = 0 if rank == 2 else 1000 * (rank + 1)
        pts = [torch.from_numpy(rng.uniform(-1 - rank, 1 + 2 * rank, n).astype(np.float32)) for _ in range(3)]
        box = global_box(*pts)
        # rank r sends to rank q a tensor of (r + 1) * q int32 words holding 1000 r + q; nothing to itself
        send = [None if q == rank else torch.full(((rank + 1) * q,), 1000 * rank + q, dtype=torch.int32)
                for q in range(world)]
        recv = exchange(send)
        got = [(t.numel(), sorted(set(t.tolist()))) for t in recv]
        out.put((rank, box, got, [float(p.min()) if n else None for p in pts],
                 [float(p.max()) if n else None for p in pts]))
    finally:
        dist.destroy_process_group()


def test_box_and_exchange_on_three_ranks():
    world = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        rank, box, got, lo, hi = q.get(timeout=180)
        res[rank] = (box, got, lo, hi)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # the same cube on every rank, enclosing every rank's points, lower corner at the global minimum
    boxes = {r: res[r][0] for r in res}
    assert len(set(boxes.values())) == 1
    box = boxes[0]
    lo = [min(res[r][2][d] for r in res if res[r][2][d] is not None) for d in range(3)]
    hi = [max(res[r][3][d] for r in res if res[r][3][d] is not None) for d in range(3)]
    ext = box[1] - box[0]
    assert all(abs((box[5] - box[4]) - ext) < 1e-9 and abs((box[3] - box[2]) - ext) < 1e-9 for _ in [0])
    for d in range(3):
        assert box[2 * d] == lo[d] and box[2 * d] + ext >= hi[d]
    assert ext >= max(h - l for h, l in zip(hi, lo))
    # rank q receives from rank r exactly what r sent it: (r + 1) q words of value 1000 r + q
    for q_ in range(world):
        got = res[q_][1]
        for r in range(world):
            n, vals = got[r]
            if r == q_:
                assert n == 0
            else:
                assert n == (r + 1) * q_ and (vals == [1000 * r + q_] if n else vals == [])
