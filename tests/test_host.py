"""Host-side checks that need no GPU: the C-ABI library and its exports, the
state container, the multi-rank reduction of bench.py (gloo, two ranks), the
CPU reference arm of the benchmark and its roofline accounting."""
import ctypes
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT


def _declared_symbols():
    src = open(os.path.join(ROOT, "include", "mac_gpu.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(mac_\w+)\s*\(", src, re.M)))


def test_library_builds_and_exports_every_declared_symbol():
    from mac_b200 import build
    lib = build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (mac_\w+)", out))
    declared = _declared_symbols()
    assert declared, "no declarations found"
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    ctypes.CDLL(lib)  # loads without a GPU


def test_python_binding_covers_the_abi():
    from mac_b200 import gpu
    assert set(_declared_symbols()) <= set(gpu.EXPORTS) | {"mac_error_string"}


def test_state_roundtrip(tmp_path, golden):
    from mac_b200.state import State
    s = golden("c1_ref_t30")
    p = str(tmp_path / "s.state")
    s.write(p)
    t = State.read(p)
    assert np.array_equal(s.keys, t.keys) and np.array_equal(s.pos, t.pos)
    for n in s.f64:
        assert np.array_equal(s.f64[n], t.f64[n])


def test_no_device_reports_cleanly():
    """Without a GPU the context refuses with MAC_ERR_NO_DEVICE (no fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from mac_b200.gpu import Context, MacError
    from mac_b200.state import Params
    with pytest.raises(MacError) as e:
        Context(Params(), max_bricks=16, max_particles=16)
    assert e.value.code == -5


def _rank_main(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, ROOT)
    import bench
    sec, cnt = bench.reduce_over_ranks(1.0 + rank, 100.0 * (rank + 1), "cpu")
    q.put((rank, sec, cnt))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_reduction_two_ranks_gloo():
    import random

    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = random.randint(20000, 40000)
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert all(p.exitcode == 0 for p in procs)
    for _, sec, cnt in res:
        assert sec == 2.0 and cnt == 300.0


def test_cpu_reference_arm_runs(tmp_path):
    sys.path.insert(0, ROOT)
    import bench
    v, kind, secs, fcs, wall = bench.cpu_reference_run(1, 1, str(tmp_path))
    assert v > 0 and fcs > 0
    assert kind in ("reference", "port")


def test_roofline_models_count_cg_iterations():
    """The V-cycle phase's regions hold one V-cycle per CG iteration (with the
    update its first kernel applies) plus one update-only region per solve, so
    its launch is a CG iteration: bytes per launch (V-cycle + 48 B update per
    unknown) over the phase time divided by the iteration count."""
    sys.path.insert(0, ROOT)
    import bench
    stats = {"unknowns": 1_000_000}
    # 10 steps, 2 solves each, 18 iterations per solve: 360 V-cycles in 380 regions
    prof = {"vcycle": (150.0, 380), "spmv": (36.0, 360), "move": (40.0, 10)}
    rl = bench.roofline_models(stats, prof, 8_000_000, 2_000_000, mg_bytes=4, cg_iterations=360)
    vc = 117.0 * 8.0 / 7.0 * 0.5
    assert rl["vcycle"]["launches"] == 360
    assert abs(rl["vcycle"]["bytes_per_launch"] - (vc + 48.0) * 1e6) < 1e-3
    assert abs(rl["vcycle"]["gbs"] - (vc + 48.0) * 1e6 / (150.0 / 360 * 1e-3) / 1e9) < 1e-9
    # the other phases count their timed regions
    assert rl["spmv"]["launches"] == 360 and rl["move"]["launches"] == 10
    assert abs(rl["move"]["bytes_per_launch"] - 48.0 * 8_000_000) < 1e-3
    # the CG scalars move no bulk data and carry no bytes model
    assert "cg_vector" not in rl
