"""The drop-in programs end to end on the GPU (marked gpu): the reference's
command lines, JSON layout and, for the f64 program, its published rows."""
import json
import os
import subprocess

import numpy as np
import pytest

import cmfw

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")

F64_KEYS = ["variant", "cmf", "p", "q", "z", "rank", "naxes", "N", "h", "n_traj", "mode", "block_size",
            "gpu_time_ms", "throughput_traj_per_s", "mem_used_mb", "n_valid", "n_with_limits", "avg_delta",
            "results"]
ROW_KEYS = ["idx", "valid", "limit", "delta", "p", "q", "precision", "log_scale", "n_limits"]
SUMMARY_KEYS = ["variant", "cmf", "p", "q", "z", "rank", "naxes", "N", "h", "n_traj", "mode", "block_size",
                "gpu_time_ms", "throughput_traj_per_s", "mem_used_mb", "n_valid", "n_with_limits", "avg_delta"]


def run(variant, tmp_path, *args):
    out = tmp_path / f"{variant}.json"
    exe = os.path.join(cmfw.BIN_DIR, f"cmf_walk_{variant}")
    r = subprocess.run([exe, *args, "--output", str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    text = out.read_text()
    return json.loads(text), text, r.stderr


def test_f64_program_reproduces_published_rows(cuda, tmp_path):
    with open(os.path.join(GOLD, "published_f64_rows.json")) as f:
        cfgs = json.load(f)
    cfg = next(c for c in cfgs if c["cmf"] == "4F3" and c["mode"] == "limit" and c["zeta"])
    data, text, err = run("f64", tmp_path, "--cmf", "4F3", "--N", "1000", "--h", "50", "--n-traj", "10000",
                          "--mode", "limit", "--zeta")
    assert list(data.keys()) == F64_KEYS
    assert list(data["results"][0].keys()) == ROW_KEYS
    assert data["n_valid"] == 10000 and data["rank"] == 3 and data["z"] == 1
    assert "=== f64 Benchmark: 4F3 z=1.0000 N=1000 h=50 n_traj=10000 rank=3 [ZETA] ===" in err
    for mine, pub in zip(data["results"], cfg["results"]):
        assert mine["valid"] == pub["valid"] and mine["n_limits"] == pub["n_limits"]
        for k in ("limit", "p", "q", "log_scale", "precision"):
            assert mine[k] == pytest.approx(pub[k], rel=1e-10), k


def test_f64_program_random_limit_counts(cuda, tmp_path):
    with open(os.path.join(GOLD, "published_summaries.json")) as f:
        summ = json.load(f)
    want = next(s for s in summ if s["variant"] == "f64" and s["cmf"] == "3F2" and s["mode"] == "limit"
                and not s["zeta"])
    data, _, _ = run("f64", tmp_path, "--cmf", "3F2", "--z", "0.5", "--n-traj", "10000", "--mode", "limit")
    assert data["n_valid"] == want["n_valid"]
    assert data["n_with_limits"] == want["n_with_limits"]
    assert data["avg_delta"] is None  # inf average, JSON null like the reference


@pytest.mark.parametrize("variant", ["df64", "rns"])
def test_summary_programs(cuda, tmp_path, variant):
    args = ["--cmf", "5F4", "--zeta", "--N", "1000", "--h", "50", "--n-traj", "2000", "--mode", "limit"]
    if variant == "rns":
        args += ["--n-primes", "8"]
    data, text, err = run(variant, tmp_path, *args)
    keys = SUMMARY_KEYS[:12] + (["n_primes"] if variant == "rns" else []) + SUMMARY_KEYS[12:]
    assert list(data.keys()) == keys
    assert data["n_valid"] == 2000
    if variant == "rns":
        # published RNS 5F4 zeta limit avg_delta (10,000 identical walks)
        assert data["avg_delta"] == pytest.approx(-1.0024904519548445, rel=1e-12)
        assert '"block_size": 128, "n_primes": 8,' in text


def test_inputs_file_flag(cuda, tmp_path):
    recs = cmfw.reference_inputs(3, 2, 50, 0, False)
    path = tmp_path / "in.bin"
    path.write_bytes(recs.tobytes())
    data, _, _ = run("f64", tmp_path, "--cmf", "3F2", "--z", "0.5", "--inputs", str(path), "--N", "200",
                     "--h", "20")
    assert data["n_traj"] == 50
    ref = cmfw.walk("f64", cmfw.make_desc(3, 2, 0.5), recs, 200, 20)
    assert data["n_valid"] == int(ref["valid"].sum())
    lim = [r["limit"] for r in data["results"]]
    np.testing.assert_allclose([x if x is not None else np.nan for x in lim], ref["limit"], rtol=0,
                               equal_nan=True)
