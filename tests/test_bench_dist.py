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
    # interior nodes of the W=32 mixer (the library's count: 524,288 fluid
    # nodes less 57,608 boundary nodes)
    assert bench.interior_nodes(spec) == 466680


def test_measured_peaks_present_or_fallback():
    p = bench.measured_peaks()
    assert p["hbm_gbs"] > 1000 and p["source"] in ("measured", "fallback")


@pytest.mark.parametrize("W,u_max,tau_f,tau_c,k,rho", [(4, 0.05, 0.6, 0.6, 1e-3, 1.0), (8, 0.03, 0.7, 0.55, 5e-4, 1.0),
                                                     (32, 0.05, 0.6, 0.6, 1e-3, 1.0), (48, 0.08, 0.6, 0.52, 1e-2, 1.0)])
def test_w_layout_params_match_library(W, u_max, tau_f, tau_c, k, rho):
    """The reference arm's case constants, computed without the CUDA library,
    are bit for bit the library's tmx_case_wlayout (a host-only call)."""
    import tmixer_b200 as T

    want = bench.workload_ref_params(T.w_layout(W, u_max, tau_f, tau_c, k, rho))
    got = bench.w_layout_params(W, u_max, tau_f, tau_c, k, rho)
    assert got.keys() == want.keys()
    for key in want:
        assert float(got[key]).hex() == float(want[key]).hex(), key


def test_reference_arm_does_not_load_the_library():
    """The reference arm's case and config come from plain Python: building
    them in a fresh interpreter imports no tmixer_b200 module and maps no
    library of the package."""
    import json
    import subprocess
    import sys

    code = ("import sys, json, bench\n"
            "p = bench.workload_params(); c = bench.config_dict(p, 1)\n"
            "maps = open('/proc/self/maps').read()\n"
            "print(json.dumps({'mods': [m for m in sys.modules if m.startswith('tmixer_b200')],"
            " 'libtmx': 'libtmx' in maps, 'config': c}))\n")
    root = os.path.dirname(os.path.abspath(bench.__file__))
    out = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, check=True)
    r = json.loads(out.stdout.strip().splitlines()[-1])
    assert r["mods"] == [] and r["libtmx"] is False
    # the same config dict as our arm's (which builds it from the same params)
    assert r["config"] == json.loads(json.dumps(bench.config_dict(bench.workload_params(), 1)))
    assert r["config"]["fluid_nodes"] == 524288


def test_reference_arm_line():
    """`bench.py --impl reference` end to end on the CPU with a small budget:
    one JSON line with the driver's steps and warmup, our arm's config,
    metric and unit, an e2e object without copies, and no module or library
    of the package loaded in its process."""
    import json
    import subprocess
    import sys

    from oracle import build_ref

    binary = build_ref.binary_path("bench_w%d" % bench.WORKLOAD["W"], bench.workload_params())
    if not os.path.exists(binary) and not os.path.exists(build_ref.REF_SRC):
        pytest.skip("reference binary not built and reference source absent")
    root = os.path.dirname(os.path.abspath(bench.__file__))
    code = ("import sys, json, io, contextlib, bench\n"
            "buf = io.StringIO()\n"
            "with contextlib.redirect_stdout(buf):\n"
            "    rc = bench.main(['--impl', 'reference', '--steps', '1', '--warmup', '3', '--ref-budget', '1'])\n"
            "maps = open('/proc/self/maps').read()\n"
            "print(json.dumps({'rc': rc, 'line': buf.getvalue().strip().splitlines()[-1],"
            " 'mods': [m for m in sys.modules if m.startswith('tmixer_b200')], 'libtmx': 'libtmx' in maps}))\n")
    out = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, check=True,
                         timeout=600)
    r = json.loads(out.stdout.strip().splitlines()[-1])
    assert r["rc"] == 0 and r["mods"] == [] and r["libtmx"] is False
    line = json.loads(r["line"])
    assert line["impl"] == "reference" and "unavailable" not in line
    assert (line["steps"], line["warmup"]) == (1, 3)
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT and line["higher_is_better"] is True
    assert line["config"] == json.loads(json.dumps(bench.config_dict(bench.workload_params(), 1)))
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "reference" and line["steps_per_sample"] >= 1
