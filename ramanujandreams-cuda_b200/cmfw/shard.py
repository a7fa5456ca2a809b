"""Multi-GPU plumbing: trajectories are independent, so a batch shards by
contiguous index ranges with no exchange on the data path; the only
collective is one small gather of per-rank counters and best deltas at the
end (torch.distributed over NCCL on GPUs, gloo on CPU).
"""
import numpy as np


def shard_bounds(n, rank, world):
    """[lo, hi) of rank's contiguous share of n items (sizes differ by <= 1)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError(f"rank {rank} outside world {world}")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def summarize(results, verified=None, top_k=8):
    """Per-rank counters and the top-k finite deltas (with global indices
    supplied by the caller through results['index'] when present)."""
    valid = np.asarray(results["valid"]) == 1
    delta = np.asarray(results["delta"], dtype=float)
    idx = np.asarray(results["index"]) if "index" in results.dtype.names else np.arange(len(delta))
    fin = valid & np.isfinite(delta)
    order = np.argsort(-delta[fin], kind="stable")[:top_k]
    return {
        "n": int(len(delta)),
        "n_valid": int(valid.sum()),
        "n_verified": int(np.asarray(verified).sum()) if verified is not None else None,
        "top": [(float(delta[fin][i]), int(idx[fin][i])) for i in order],
    }


def merge(summaries, top_k=8):
    """Combine per-rank summaries (the order of ranks does not matter)."""
    out = {"n": 0, "n_valid": 0, "n_verified": 0, "top": []}
    for s in summaries:
        out["n"] += s["n"]
        out["n_valid"] += s["n_valid"]
        if s["n_verified"] is None or out["n_verified"] is None:
            out["n_verified"] = None
        else:
            out["n_verified"] += s["n_verified"]
        out["top"].extend(s["top"])
    out["top"] = sorted(out["top"], key=lambda t: (-t[0], t[1]))[:top_k]
    return out


def gather_merge(summary, top_k=8):
    """All-gather one summary per rank and merge (every rank gets the result)."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return merge([summary], top_k)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, summary)
    return merge(parts, top_k)
