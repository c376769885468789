"""The JSON line of `bench.py --impl reference` (the reference's own compiled code timed on the host
cores), on a small sample so that it runs in seconds: every key the benchmark contract names, the
reference-arm specifics, and silence on ranks other than 0."""
import argparse
import json

import pytest

EXPECTED = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
            "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e")


@pytest.fixture
def small_bench(monkeypatch):
    from oracle import oracle as O

    if not O.ref_available():
        O.build_ref()
    if not O.ref_available():
        pytest.skip("reference harness not built (needs the reference sources)")
    import bench

    monkeypatch.setattr(bench, "CPU_LOG2_HALF", 11)  # N = 4096
    monkeypatch.setattr(bench, "CPU_SAMPLE_STRIDE", 8)
    return bench


def test_reference_arm_json_line(small_bench, monkeypatch, capsys):
    monkeypatch.setenv("RANK", "0")
    args = argparse.Namespace(gpus=1, steps=1, warmup=0, err_tol_force_acc=5e-5)
    assert small_bench.reference_arm(args) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    for k in EXPECTED:
        assert k in line, k
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["unit"] == "particles/s" and line["higher_is_better"] is True
    assert line["steps"] == 1 and line["n_gpus"] == 1
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert "N=2^12" in cb["sample"] and cb["cores"] == cb["detail"]["procs"]
    assert line["ms_per_step"] == pytest.approx(1e3 * cb["detail"]["walk_s_timed"][0])
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert line["config"]["workload"].startswith("zoom box N=2^12")


def test_reference_arm_other_ranks_print_nothing(small_bench, monkeypatch, capsys):
    monkeypatch.setenv("RANK", "1")
    args = argparse.Namespace(gpus=2, steps=1, warmup=0, err_tol_force_acc=5e-5)
    assert small_bench.reference_arm(args) == 0
    assert capsys.readouterr().out == ""
