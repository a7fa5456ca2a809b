"""Checkpointed chunking for long runs (1e6 - 1e8 trajectories).

The batch is cut into fixed-size chunks walked one after another; after each
chunk its result records are written into a results file and its byte in a
completion bitmap (done.bin, one byte per chunk) is set, both flushed to
disk. A run that stops (killed, preempted) resumes from the same state
directory and walks only the chunks whose byte is not set. meta.json pins
the run's parameters: resuming with different ones is an error.
"""
import json
import os

import numpy as np

from . import api
from ._lib import OUT_DTYPE


def _meta(variant, desc, n, N, h, chunk, n_primes, flags):
    return {"variant": variant, "p": desc.p, "q": desc.q, "z": desc.z, "n": int(n), "N": int(N), "h": int(h),
            "chunk": int(chunk), "n_primes": int(n_primes), "flags": int(flags)}


def run_checkpointed(variant, desc, records, N, h, chunk, state_dir, n_primes=8, flags=0, on_chunk=None):
    """Walk `records` in chunks of `chunk` with resume state in `state_dir`.

    Returns (results, walked): all result records, and how many chunks this
    call walked. on_chunk(i, n_chunks) runs after chunk i is on disk.
    """
    n = len(records)
    n_chunks = (n + chunk - 1) // chunk
    os.makedirs(state_dir, exist_ok=True)
    meta_path = os.path.join(state_dir, "meta.json")
    done_path = os.path.join(state_dir, "done.bin")
    res_path = os.path.join(state_dir, "results.bin")
    meta = _meta(variant, desc, n, N, h, chunk, n_primes, flags)
    if os.path.exists(meta_path):
        with open(meta_path) as f:
            old = json.load(f)
        if old != meta:
            raise ValueError(f"{state_dir} holds a different run: {old} != {meta}")
    else:
        with open(meta_path, "w") as f:
            json.dump(meta, f)
    if not os.path.exists(done_path):
        with open(done_path, "wb") as f:
            f.write(bytes(n_chunks))
    if not os.path.exists(res_path):
        with open(res_path, "wb") as f:
            f.truncate(max(n, 1) * OUT_DTYPE.itemsize)
    with open(done_path, "rb") as f:
        done = bytearray(f.read())
    walked = 0
    for i in range(n_chunks):
        if done[i]:
            continue
        lo, hi = i * chunk, min(n, (i + 1) * chunk)
        out = api.walk(variant, desc, records[lo:hi], N, h, n_primes=n_primes, flags=flags)
        with open(res_path, "r+b") as f:
            f.seek(lo * OUT_DTYPE.itemsize)
            f.write(np.ascontiguousarray(out, dtype=OUT_DTYPE).tobytes())
            f.flush()
            os.fsync(f.fileno())
        done[i] = 1
        with open(done_path, "r+b") as f:
            f.seek(i)
            f.write(b"\x01")
            f.flush()
            os.fsync(f.fileno())
        walked += 1
        if on_chunk is not None:
            on_chunk(i, n_chunks)
    results = np.fromfile(res_path, dtype=OUT_DTYPE, count=n)
    return results, walked
