"""The multi-GPU path of bench.py on CPU: world_size-2 `gloo` replicas.

Each rank renders its own seeded batch (weak scaling, no data-path
collective); the timing collectives are a barrier and max / sum reductions
of per-rank scalars.  Rendezvous on 127.0.0.1.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from pcr_b200 import workloads
    from pcr_b200.replicas import Replicas
    rep = Replicas("gloo", timeout_s=60)
    rep.barrier()
    seed = rep.seed(2026)
    batch = workloads.batch_requests(8, seed=seed)
    paths = sum(r["width"] * r["height"] * r["samples"] for r in batch)
    out = {"rank": rep.rank, "world": rep.world, "seed": seed,
           "max": rep.max(10.0 + rank), "sum": rep.sum(paths), "own": paths,
           "first": (batch[0]["variant"], batch[0]["width"], batch[0]["samples"])}
    rep.close()
    q.put(out)


def test_two_gloo_replicas_reduce_and_seed_apart():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=120) for _ in procs], key=lambda r: r["rank"])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r["world"] for r in res] == [2, 2]
    assert [r["seed"] for r in res] == [2026, 2027]          # each replica its own batch
    assert res[0]["first"] != res[1]["first"]
    assert all(r["max"] == 11.0 for r in res)                # time: max over ranks
    total = res[0]["own"] + res[1]["own"]
    assert all(r["sum"] == total for r in res)               # work: sum over ranks


def test_single_process_needs_no_process_group():
    from pcr_b200.replicas import Replicas
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        assert k not in os.environ or os.environ[k] in ("0", "1")
    rep = Replicas("gloo")
    assert rep.world == 1 and rep.dist is None
    assert rep.max(3.5) == 3.5 and rep.sum(2.0) == 2.0 and rep.seed(7) == 7
    rep.close()


class _FakeCtx:
    """Stands in for a GPU context: a 'render' of a sample range returns the
    range's sample count in every pixel (what a partial sum contributes)."""

    def render(self, sid, d, want_rgb=True):
        import numpy as np
        return np.full((d.height, d.width, 3), float(d.sample_end - d.sample_begin), np.float32), None, None

    def tonemap(self, hdr, aces=False, denoise=False):
        return (hdr * 0).astype("uint8") + 7


def _split_main(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from pcr_b200 import capi
    from pcr_b200.replicas import Replicas, sample_range, split_render
    rep = Replicas("gloo", timeout_s=60)
    desc = capi.render_desc(6, 4, samples=7)
    hdr, rgb = split_render(_FakeCtx(), 0, desc, rep)
    q.put({"rank": rank, "range": sample_range(7, rank, world), "hdr": float(hdr.mean()), "rgb": int(rgb.max())})
    rep.close()


def test_split_render_ranges_cover_samples_and_sum():
    from pcr_b200.replicas import sample_range
    for spp in (1, 2, 7, 64):
        for world in (1, 2, 3, 8):
            r = [sample_range(spp, k, world) for k in range(world)]
            assert r[0][0] == 0 and r[-1][1] == spp
            assert all(r[k][1] == r[k + 1][0] for k in range(world - 1))
            assert max(e - b for b, e in r) - min(e - b for b, e in r) <= 1
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=120) for _ in procs], key=lambda r: r["rank"])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r["range"] for r in res] == [(0, 4), (4, 7)]
    assert all(r["hdr"] == 7.0 for r in res)      # the partial sums add up to all 7 samples
    assert all(r["rgb"] == 7 for r in res)
