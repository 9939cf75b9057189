"""bench.py's reference arm (the CPU restatement timed on the host): one JSON line
with the metric, the cpu_baseline and e2e objects; under a multi-rank launch only
rank 0 prints it and the others exit 0 without work."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra, gpus=None):
    env = dict(os.environ, **env_extra)
    gpus = gpus if gpus is not None else int(env_extra.get("WORLD_SIZE", "1"))
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "0", "--gpus", str(gpus)], cwd=ROOT, env=env, capture_output=True, text=True,
                          timeout=600)


def test_reference_arm_line():
    r = _run({"RANK": "0"})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "1080p SIFT detect+describe images/s"
    assert d["unit"] == "images/s" and d["higher_is_better"] is True and d["value"] > 0
    assert d["steps"] == 1 and d["n_gpus"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_quietly():
    r = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]


def test_gpus_must_match_the_launch():
    """--gpus N without N ranks is refused: the bench runs one process per GPU."""
    r = _run({"WORLD_SIZE": "1"}, gpus=8)
    assert r.returncode != 0 and "WORLD_SIZE" in r.stderr
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]
