"""Host-side logic of bench.py that runs without a GPU: the roofline denominator read from
the measured-peaks file, the clock record's parsing (median SM clock under load, throttle
reasons), the reference arm's non-zero ranks, and one workload config for both arms."""
import importlib.util
import json
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("rumi_bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("content,expect", [
    ('{"hbm_gbs": 7100.5, "bf16_tflops": 1590}', (7100.5, "measured")),
    ('{"b200": {"hbm_gbs": 6900}}', (6900.0, "measured")),
    ('{"hbm_gbs": "fast"}', (6650.0, "fallback")),
    ('{"bf16_tflops": 1590}', (6650.0, "fallback")),
    ("not json", (6650.0, "fallback")),
    (None, (6650.0, "fallback")),
])
def test_roofline_peak_from_the_measured_peaks_file(bench, tmp_path, monkeypatch, content, expect):
    if content is not None:
        (tmp_path / "MEASURED_PEAKS.json").write_text(content)
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    pk, kind = bench.peaks()
    assert (pk["hbm_gbs"], kind) == expect


class _FakeProc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0


def _sampled(bench, rows):
    cs = bench.ClockSampler(0)
    with open(cs.path, "w") as fh:
        fh.write("\n".join(rows) + "\n")
    cs.fh = open(cs.path, "a")
    cs.proc = _FakeProc()
    out = cs.stop()
    assert not os.path.exists(cs.path)
    return out


def test_clock_record_median_under_load_and_reasons(bench):
    idle = "0, 345, 1965, 140.2, 0x0000000000000001, Not Active, Not Active, Not Active, Not Active"
    busy = "0, {mhz}, 1965, 910.0, 0x0000000000000000, Not Active, Not Active, Not Active, {cap}"
    rows = [idle] + [busy.format(mhz=m, cap="Not Active") for m in (1965, 1950, 1965)] + \
           [busy.format(mhz=1890, cap="Active"), "garbage line", "0, [N/A], 1965, 0, 0, a, b, c, d"]
    out = _sampled(bench, rows)
    assert out["sm_mhz"] == 1957.5  # idle sample left out: median of 1965, 1950, 1965, 1890
    assert out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"]
    assert out["samples"] == 5


def test_clock_record_flags_hardware_slowdown(bench):
    row = "0, 1200, 1965, 700.0, 0x0000000000000008, Active, Not Active, Active, Not Active"
    out = _sampled(bench, [row, row])
    assert out["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]


def test_clock_record_without_nvidia_smi(bench):
    cs = bench.ClockSampler(0)
    cs.proc = None
    assert cs.stop()["reasons"] == ["nvidia-smi unavailable"]


def test_reference_arm_on_a_non_zero_rank_does_no_work(bench, monkeypatch, capsys):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setattr(bench, "RefPool", None)  # any use of the pool would raise
    args = bench.argparse.Namespace(impl="reference", gpus=2, steps=3, warmup=3, small=False)
    assert bench.reference_arm(args) == 0
    assert capsys.readouterr().out == ""


def test_both_arms_describe_the_same_workload(bench):
    w = bench.workload(bench.argparse.Namespace(small=False))
    cfg = bench.bench_config(w, 1)
    assert cfg["width"] == cfg["height"] == 1024 and cfg["spp"] == 64 and cfg["max_depth"] == 10
    assert cfg["triangles"] == 1048576
    json.dumps(cfg)
    # every key is a description of the workload, not a measurement
    assert set(cfg) == {"workload", "width", "height", "spp", "max_depth", "triangles", "parallelism", "l2"}
