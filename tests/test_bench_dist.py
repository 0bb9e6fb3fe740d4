"""bench.py's multi-process plumbing on CPU: two gloo ranks (127.0.0.1) agree
on the max-over-ranks timing the benchmark reports, and the workload and form
tables are consistent."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    d = bench.Dist()
    d.init("gloo")
    d.barrier()
    got = d.max(10.0 + rank)
    d.close()
    q.put((rank, got))


def test_two_rank_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == {0: 11.0, 1: 11.0}


def test_single_process_dist_is_identity():
    d = bench.Dist()
    if d.world != 1:
        pytest.skip("running under a launcher")
    d.init("gloo")
    assert d.max(3.5) == 3.5
    d.close()


def test_form_bytes():
    assert bench.FORM_BYTES["fp64"] == 4 * 19 * 8 * 2
    assert bench.FORM_BYTES["fp32"] == 4 * 19 * 4 * 2
    assert bench.FORM_BYTES["fp16"] == 4 * 19 * 2 * 2 + 2 * 16 * 2


def test_workload_spec_geometry():
    spec = bench.workload_spec()
    assert spec.nodes() == 524288 and (spec.inx, spec.mnx, spec.mny) == (256, 64, 128)
    assert spec.tau == bench.WORKLOAD["tau_f"]


def test_measured_peaks_present_or_fallback():
    p = bench.measured_peaks()
    assert p["hbm_gbs"] > 1000 and p["source"] in ("measured", "fallback")
