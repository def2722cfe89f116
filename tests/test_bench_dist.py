"""CPU: the N>1 path of bench.py (one process per GPU, replicas, max-over-ranks timing) with
two gloo ranks on the host.  Each rank joins the process group, the slowest rank's time is
taken by every rank, the whole-job throughput counts every rank's units, and the reference
arm's non-zero ranks leave without work or output."""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, str(ROOT))
    import bench

    w, r, local, pg = bench.dist_setup(world, backend="gloo")
    res = {"world": w, "rank": r}
    # every rank sees the slowest rank's time
    res["tmax"] = bench.max_over_ranks(pg, 1.0 + 0.5 * r, local)
    bench.barrier(pg)
    res["value"] = bench.aggregate(1000.0, w, res["tmax"])
    # the reference arm: rank 0 alone measures and prints; the others return 0 silently
    if r != 0:
        args = type("A", (), {"gpus": world, "steps": 1, "warmup": 0})()
        buf = io.StringIO()
        with redirect_stdout(buf):
            res["ref_rc"] = bench.run_reference_arm(args)
        res["ref_out"] = buf.getvalue()
    bench.barrier(pg)
    pg.destroy_process_group()
    Path(out_dir, f"rank{r}.json").write_text(json.dumps(res))


def test_two_gloo_ranks(tmp_path):
    world, port = 2, _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    res = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for r, d in enumerate(res):
        assert d["world"] == world and d["rank"] == r
        assert d["tmax"] == pytest.approx(1.5)          # max over ranks of 1.0, 1.5
        assert d["value"] == pytest.approx(1000.0 * world / 1.5)
    assert res[1]["ref_rc"] == 0 and res[1]["ref_out"] == ""


def test_single_process_needs_no_group():
    sys.path.insert(0, str(ROOT))
    import bench

    saved = {k: os.environ.pop(k, None) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    try:
        w, r, local, pg = bench.dist_setup(1)
        assert (w, r, local, pg) == (1, 0, 0, None)
        assert bench.max_over_ranks(pg, 3.25, 0) == 3.25
        assert bench.aggregate(10.0, 1, 2.0) == 5.0
    finally:
        for k, v in saved.items():
            if v is not None:
                os.environ[k] = v
