"""The benchmark's output contract, on CPU: the reference arm's JSON line
(the CPU restatement of the implicit step, timed on the host cores) and the
clock record that travels with every GPU line (sampled during the timed
region, here from a stand-in nvidia-smi that prints fixed samples)."""
import importlib.util
import json
import os
import stat
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench_module():
    spec = importlib.util.spec_from_file_location("dare_bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_reference_arm_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "24",
                          "--steps", "2", "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "steps/s" and line["higher_is_better"]
    assert line["steps"] == 2 and line["warmup"] == 1 and line["value"] > 0
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["kind"] == "port" and cb["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": "steps/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["iterations_per_step"] > 0
    # the workload description is the one the GPU arm prints
    assert set(line["config"]) == {"workload", "cells"} and line["config"]["cells"] == 24 ** 3


def _fake_smi(tmp_path, reasons):
    """An executable `nvidia-smi` printing one CSV sample every 10 ms."""
    script = tmp_path / "nvidia-smi"
    script.write_text(
        "#!" + sys.executable + "\n"
        "import sys, time\n"
        "while True:\n"
        f"    print('0, 1900, 1965, 900.5, 0x4, {reasons}', flush=True)\n"
        "    time.sleep(0.01)\n")
    script.chmod(script.stat().st_mode | stat.S_IEXEC)
    return str(tmp_path)


def test_clock_sampler_counts_the_timed_region(tmp_path, monkeypatch):
    bench = _bench_module()
    monkeypatch.setenv("PATH", _fake_smi(tmp_path, "Not Active, Not Active, Not Active, Active") + os.pathsep +
                       os.environ["PATH"])
    c = bench.ClockSampler(0)
    time.sleep(0.2)        # samples before the timed region ...
    c.mark()               # ... are not counted
    time.sleep(0.2)
    rec = c.stop()
    assert rec["sm_mhz"] == 1900.0 and rec["sm_max_mhz"] == 1965.0
    assert rec["reasons"] == ["sw_power_cap"]
    assert 3 <= rec["samples"] <= 40


def test_clock_sampler_flags_slowdowns(tmp_path, monkeypatch):
    bench = _bench_module()
    monkeypatch.setenv("PATH", _fake_smi(tmp_path, "Active, Not Active, Active, Not Active") + os.pathsep +
                       os.environ["PATH"])
    c = bench.ClockSampler(0)
    c.mark()
    time.sleep(0.1)
    rec = c.stop()
    assert rec["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]


def test_clock_sampler_without_nvidia_smi(tmp_path, monkeypatch):
    bench = _bench_module()
    monkeypatch.setenv("PATH", str(tmp_path))   # nothing to run
    c = bench.ClockSampler(0)
    c.mark()
    rec = c.stop()
    assert rec["sm_mhz"] is None and rec["reasons"] == ["nvidia-smi unavailable"]


def test_reference_arm_under_torchrun():
    """Launched as the multi-GPU runs are (torchrun, two ranks, the same
    flags), the reference arm prints one line from rank 0 and every rank
    exits 0."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                          "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
                          "--impl", "reference", "--gpus", "2", "--cells-per-side", "16", "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1 and lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2
    assert lines[0]["config"]["cells"] == 16 ** 3
