"""Benchmark sweep over CMF families, variants and modes with the reference
runner's result layout (benchmarks/run_benchmark.py).

Each configuration runs the drop-in program cmf_walk_<variant> with the
reference's argv (run_benchmark.py:41-56), reads its JSON, adds cmf,
variant, mode and the wall time, and the sweep writes
<out>/individual/<cmf>_<variant>_<mode>.json, <out>/summary/all_results.json
and the CSV and Markdown tables of run_benchmark.py:138-171 with the same
columns and number formats, so the published tables can be regenerated on
this hardware.

    python -m cmfw.sweep --output-dir results/zeta --zeta
"""
import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

from ._lib import BIN_DIR

CMF_TYPES = ["3F2", "4F3", "5F4", "6F5", "8F7"]
VARIANTS = ["f64", "rns", "df64"]
MODES = ["limit", "delta"]


def run_one(binary, cmf, z, N, h, n_traj, mode, output_path, block_size=None, n_primes=None, use_zeta=False):
    """One drop-in program run; returns its JSON plus wall_time_s, or None."""
    cmd = [str(binary), "--cmf", cmf, "--z", str(z), "--N", str(N), "--h", str(h), "--n-traj", str(n_traj),
           "--mode", mode, "--output", str(output_path)]
    if block_size:
        cmd += ["--block-size", str(block_size)]
    if n_primes and "rns" in os.path.basename(str(binary)):
        cmd += ["--n-primes", str(n_primes)]
    if use_zeta:
        cmd.append("--zeta")
    t0 = time.time()
    r = subprocess.run(cmd, capture_output=True, text=True)
    elapsed = time.time() - t0
    if r.returncode != 0:
        sys.stderr.write(f"  ERROR ({' '.join(cmd)}): {r.stderr}\n")
        return None
    try:
        with open(output_path) as f:
            data = json.load(f)
    except (OSError, ValueError) as e:
        sys.stderr.write(f"  ERROR parsing {output_path}: {e}\n")
        return None
    data["wall_time_s"] = elapsed
    return data


def write_tables(results, out_dir):
    """benchmark_table.csv and benchmark_table.md (run_benchmark.py:138-171)."""
    out_dir = Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    with open(out_dir / "benchmark_table.csv", "w") as f:
        f.write("cmf,variant,mode,rank,N,h,n_traj,gpu_time_ms,throughput_traj_s,"
                "mem_mb,n_valid,n_with_limits,avg_delta,wall_time_s\n")
        for r in results:
            f.write(f"{r.get('cmf', '')},{r.get('variant', '')},{r.get('mode', '')},"
                    f"{r.get('rank', 0)},{r.get('N', 0)},{r.get('h', 0)},"
                    f"{r.get('n_traj', 0)},{r.get('gpu_time_ms', 0):.3f},"
                    f"{r.get('throughput_traj_per_s', 0):.1f},"
                    f"{r.get('mem_used_mb', 0):.2f},"
                    f"{r.get('n_valid', 0)},{r.get('n_with_limits', 0)},"
                    f"{r.get('avg_delta', 'nan')},{r.get('wall_time_s', 0):.3f}\n")
    with open(out_dir / "benchmark_table.md", "w") as f:
        f.write("# RamanujanDreams-CUDA Benchmark Results\n\n")
        f.write("| CMF | Variant | Mode | Rank | GPU Time (ms) | Throughput (traj/s) | Memory (MB) "
                "| Valid | Limits | Avg Delta |\n")
        f.write("|-----|---------|------|------|---------------|---------------------|-------------"
                "|-------|--------|-----------|\n")
        for r in results:
            f.write(f"| {r.get('cmf', '')} | {r.get('variant', '')} | {r.get('mode', '')} "
                    f"| {r.get('rank', 0)} | {r.get('gpu_time_ms', 0):.1f} "
                    f"| {r.get('throughput_traj_per_s', 0):.0f} "
                    f"| {r.get('mem_used_mb', 0):.1f} "
                    f"| {r.get('n_valid', 0)}/{r.get('n_traj', 0)} "
                    f"| {r.get('n_with_limits', 0)} "
                    f"| {r.get('avg_delta', 'nan')} |\n")


def sweep(out_dir, bin_dir=BIN_DIR, cmfs=CMF_TYPES, variants=VARIANTS, modes=MODES, N=1000, h=50,
          n_traj=10000, z=0.5, n_primes=8, use_zeta=False, block_size=None):
    out_dir = Path(out_dir)
    (out_dir / "individual").mkdir(parents=True, exist_ok=True)
    (out_dir / "summary").mkdir(parents=True, exist_ok=True)
    results = []
    for cmf in cmfs:
        for variant in variants:
            binary = Path(bin_dir) / f"cmf_walk_{variant}"
            if not binary.exists():
                raise FileNotFoundError(f"{binary} is missing: build it with make")
            for mode in modes:
                path = out_dir / "individual" / f"{cmf}_{variant}_{mode}.json"
                r = run_one(binary, cmf, z, N, h, n_traj, mode, path, block_size, n_primes, use_zeta)
                if r is None:
                    continue
                r["cmf"], r["variant"], r["mode"] = cmf, variant, mode
                results.append(r)
    with open(out_dir / "summary" / "all_results.json", "w") as f:
        json.dump(results, f, indent=2)
    write_tables(results, out_dir / "summary")
    return results


def main(argv=None):
    ap = argparse.ArgumentParser(description="CMF walk benchmark sweep (reference runner layout)")
    ap.add_argument("--bin-dir", type=Path, default=Path(BIN_DIR))
    ap.add_argument("--output-dir", type=Path, default=Path("results"))
    ap.add_argument("--N", type=int, default=1000)
    ap.add_argument("--h", type=int, default=50)
    ap.add_argument("--n-traj", type=int, default=10000)
    ap.add_argument("--z", type=float, default=0.5)
    ap.add_argument("--cmfs", nargs="+", default=CMF_TYPES)
    ap.add_argument("--variants", nargs="+", default=VARIANTS)
    ap.add_argument("--modes", nargs="+", default=MODES)
    ap.add_argument("--n-primes", type=int, default=8)
    ap.add_argument("--block-size", type=int, default=None)
    ap.add_argument("--zeta", action="store_true")
    a = ap.parse_args(argv)
    res = sweep(a.output_dir, a.bin_dir, a.cmfs, a.variants, a.modes, a.N, a.h, a.n_traj, a.z, a.n_primes,
                a.zeta, a.block_size)
    print(f"{len(res)} configurations run; tables in {a.output_dir / 'summary'}")


if __name__ == "__main__":
    main()
