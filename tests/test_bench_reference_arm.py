"""bench.py's reference arm on the CPU: `--impl reference` times the oracle
port of the reference's integrate + ray-cast path (the reference has no CPU
implementation of it) on a bounded sample and prints one JSON line with the
product arm's metric, unit and direction plus `impl`, `cpu_baseline` and an
`e2e` object without host<->device bytes; under torchrun only rank 0 prints.
Also the bench's clock sampler, against a fake nvidia-smi."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(extra_env=None):
    env = dict(os.environ)
    env.update(extra_env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "0"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_one_contract_line():
    p = _run()
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["unit"] == "frames/s" and line["higher_is_better"] is True
    assert line["metric"].startswith("frames/s integrate+raycast 640x480@4mm")
    assert line["value"] > 0 and line["steps"] == 1 and line["n_gpus"] == 1
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert line["config"]["workload"].startswith("tabletop 30x640x480")
    # the same config dict as the product arm's line (bench.headline_config)
    assert line["config"] == {"workload": line["config"]["workload"], "frames_per_step": 30,
                              "l2": "inputs larger than L2 (30 resident frames, 250 MB per step)",
                              "parallelism": "replicas1"}
    assert line["sampling"]["sample"] == cb["sample"]


def test_reference_arm_other_ranks_exit_quietly():
    p = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert not [ln for ln in p.stdout.splitlines() if ln.startswith("{")]


def test_clock_sampler_keeps_only_rows_of_the_timed_region(tmp_path, monkeypatch):
    """The clock sampler waits for nvidia-smi's first row (taken before the
    timed region, GPU idle) and reports only the rows after it; a fake
    nvidia-smi on PATH prints an idle first row, then loaded rows."""
    import importlib.util
    import time

    fake = tmp_path / "nvidia-smi"
    fake.write_text("#!" + sys.executable + "\n"
                    "import time\n"
                    "time.sleep(0.2)\n"
                    "i = 0\n"
                    "while True:\n"
                    "    print(('120' if i == 0 else '1965') + ', 1965, 500.0, Not Active, Not Active, Not Active, '\n"
                    "          + ('Active' if i == 2 else 'Not Active'), flush=True)\n"
                    "    i += 1\n"
                    "    time.sleep(0.05)\n")
    fake.chmod(0o755)
    monkeypatch.setenv("PATH", str(tmp_path) + os.pathsep + os.environ.get("PATH", ""))
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    with bench.ClockSampler(0) as clk:
        time.sleep(0.3)
    s = clk.summary()
    assert s["samples"] >= 2
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
