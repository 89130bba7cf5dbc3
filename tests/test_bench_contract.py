"""Host-side rules of bench.py's timing contract, checked without a GPU: the
clock record that voids a run, the nvidia-smi sample parser, and the single
re-measurement of a voided timed region."""
import importlib.util
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_clock_rejections(bench):
    ok = {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": []}
    assert bench.clock_rejections(ok) == []
    # the power cap explains low clocks and is kept
    assert bench.clock_rejections({"sm_mhz": 1300.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"]}) == []
    for r in ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"):
        assert bench.clock_rejections({"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [r]}) == [r]
    # low clocks with nothing to explain them: a leftover lock
    assert bench.clock_rejections({"sm_mhz": 1000.0, "sm_max_mhz": 1965.0, "reasons": []}) == \
        ["sm_clock_low_without_reason"]
    assert bench.clock_rejections({"sm_mhz": 1000.0, "sm_max_mhz": 1965.0,
                                   "reasons": ["applications_clocks_setting"]}) == ["sm_clock_low_without_reason"]
    # no samples (no nvidia-smi): nothing to go by
    assert bench.clock_rejections({"sm_mhz": None, "sm_max_mhz": None, "reasons": []}) == []


def test_sampler_summary_parses_rows(bench):
    c = bench.ClockSampler(0)
    c.rows = [["1965", "1965", "500", "0x0000000000000004", "99"],
              ["1955", "1965", "510", "0x0000000000000000", "100"],
              ["210", "1965", "80", "0x0000000000000001", "0"],      # idle sample: not a load clock
              ["[N/A]", "1965", "80", "0x0", "0"]]                    # unreadable sample: skipped
    s = c.summary()
    assert s["sm_mhz"] == 1960.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"] and s["samples"] == 4


class _FakeSampler:
    """Stands in for ClockSampler: hands out prepared summaries in order."""
    queue = []

    def __init__(self, index):
        self.s = _FakeSampler.queue.pop(0)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def summary(self):
        return dict(self.s)


def test_timed_region_remeasures_once(bench, monkeypatch):
    monkeypatch.setattr(bench, "ClockSampler", _FakeSampler)
    import torch
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    calls = []

    def region():
        calls.append(1)
        return 10.0 * len(calls), len(calls)

    good = {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 5}
    hot = {"sm_mhz": 1700.0, "sm_max_mhz": 1965.0, "reasons": ["hw_thermal_slowdown"], "samples": 5}

    _FakeSampler.queue = [dict(good)]
    t, payload, s = bench.timed_region(region, 0)
    assert (t, payload) == (10.0, 1) and "rejected_first_run" not in s

    calls.clear()
    _FakeSampler.queue = [dict(hot), dict(good)]
    t, payload, s = bench.timed_region(region, 0)
    assert (t, payload) == (20.0, 2), "the second run is the one reported"
    assert s["rejected_first_run"]["reasons"] == ["hw_thermal_slowdown"]
    assert s["reasons"] == []

    # a second voided run is reported as it is (one re-measurement only)
    calls.clear()
    _FakeSampler.queue = [dict(hot), dict(hot)]
    t, payload, s = bench.timed_region(region, 0)
    assert len(calls) == 2 and s["reasons"] == ["hw_thermal_slowdown"]


def _rank_remeasure(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    import torch
    torch.cuda.synchronize = lambda *a, **k: None
    good = {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 5}
    hot = {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["hw_slowdown"], "samples": 5}
    # only rank 1 sees a slowdown in its first run
    _FakeSampler.queue = [dict(hot if rank == 1 else good), dict(good)]
    bench.ClockSampler = _FakeSampler
    calls = []

    def region():
        calls.append(1)
        dist.barrier()   # a collective inside the timed region, as the bench's ranks have
        return 1.0, None

    _, _, s = bench.timed_region(region, 0, dist, None)
    out[rank] = (len(calls), s.get("rejected_first_run", {}).get("reasons"))
    dist.destroy_process_group()


def test_two_gloo_ranks_remeasure_together():
    """A voided run on one rank makes every rank time the region again, so
    all ranks take the same collective steps."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = 30500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_remeasure, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0] == (2, ["another rank"])
    assert out[1] == (2, ["hw_slowdown"])
