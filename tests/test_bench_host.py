"""Host-side logic of bench.py: clock summary, max-over-ranks on two gloo
ranks, workload scaling, and the CPU reference arm's JSON line."""

from __future__ import annotations

import json
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def test_summarise_clocks():
    s = bench.summarise_clocks([(1800.0, 1965.0, 0x4), (1700.0, 1965.0, 0x0), (1900.0, 1965.0, 0x1)])
    assert s["sm_mhz"] == 1800.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    assert bench.summarise_clocks([])["sm_mhz"] is None
    bad = bench.summarise_clocks([(900.0, 1965.0, 0x8 | 0x40)])
    assert bad["reasons"] == ["hw_slowdown", "hw_thermal_slowdown"]


def test_frame_config_scales_density():
    assert bench.frame_config(4096) == {"size": 4096, "n_stars": 20000, "n_transients": 50}
    small = bench.frame_config(1024)
    assert small["n_stars"] == 1250 and small["n_transients"] == 3


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench.barrier(None)
        got = bench.max_over_ranks(10.0 * (rank + 1), None)
        out[rank] = got
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
        assert dict(out) == {0: 20.0, 1: 20.0}


def test_max_over_ranks_without_group():
    assert bench.max_over_ranks(3.5) == 3.5


def test_reference_arm_line(capsys):
    from oracle import chain

    if not chain.available():
        pytest.skip("oracle/_ref not built")
    assert bench.main(["--impl", "reference", "--size", "512", "--steps", "1", "--warmup", "0"]) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "Mpix/s" and line["value"] > 0
    assert line["e2e"] == {"value": line["value"], "unit": "Mpix/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1


def test_reference_arm_other_ranks_exit_quietly(capsys, monkeypatch):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    assert bench.main(["--impl", "reference", "--gpus", "2"]) == 0
    assert capsys.readouterr().out == ""


def test_uneven_batch_specs_queue_and_dealing():
    specs = bench.uneven_specs(0)
    assert len(specs) == bench.UNEVEN_DISTINCT
    assert {(s["height"], s["width"]) for s in specs} == set(bench.UNEVEN_SHAPES)
    assert all(2.0 <= s["sci_fwhm"] <= 5.0 and 500 <= s["n_stars"] <= 20000 and 0 <= s["mask_fraction"] <= 0.03
               for s in specs)
    assert specs == bench.uneven_specs(0) and specs != bench.uneven_specs(1)
    q = bench.uneven_queue(0)
    assert len(q) == bench.UNEVEN_FRAMES
    assert all(sorted(q[i:i + 16]) == list(range(16)) for i in range(0, 64, 16))
    px = [specs[j]["height"] * specs[j]["width"] for j in q]
    assert bench.lpt_deal(px, 1) == [0] * len(px)
    for world in (2, 4, 8):
        owner = bench.lpt_deal(px, world)
        loads = [sum(p for p, r in zip(px, owner) if r == k) for k in range(world)]
        assert max(loads) - min(loads) <= max(px)
    # equal items alternate ranks in index order
    assert bench.lpt_deal([5, 5, 5, 5], 2) == [0, 1, 0, 1]
