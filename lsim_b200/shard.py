"""Sharding across ranks (one process per GPU).

Faults are independent given the good machine, and so are pattern rounds.

Pattern sharding (weak scaling): rank r simulates every fault over its own
contiguous block of rounds, and the per-fault results combine with one
reduction -- count by SUM, first detecting pattern by MIN (after shifting by
the block's first pattern), detected by OR -- while the reference-compatible
last-round flag comes from the rank that holds the last round.

Fault sharding (strong scaling): rank r simulates its own part of the fault
list over all patterns.  The parts keep every group of faults that share a
sweep (one fanout-free region, fsimb_fault_costs) together and balance the
groups' estimated costs; results combine with the same reductions, each
fault being present on exactly one rank.

No data moves during simulation in either form.
"""
import numpy as np

INT64_MAX = np.iinfo(np.int64).max


def round_block(n_rounds, rank, world, align=32):
    """Contiguous rounds [r0, r1) of this rank, cut at multiples of `align`
    (one 2048-pattern tile) so that every block but the last is full."""
    tiles = (n_rounds + align - 1) // align
    per = (tiles + world - 1) // world
    r0 = min(n_rounds, rank * per * align)
    r1 = min(n_rounds, (rank + 1) * per * align)
    return r0, r1


def local_patterns(words, n_patterns, n_pi, rank, world):
    """This rank's slice of a [rounds][n_pi] pattern block: (words, P, first pattern)."""
    n_rounds = (n_patterns + 63) // 64
    r0, r1 = round_block(n_rounds, rank, world)
    w = np.asarray(words, dtype=np.uint64).reshape(n_rounds, n_pi)[r0:r1]
    P = min(n_patterns, r1 * 64) - r0 * 64 if r1 > r0 else 0
    return np.ascontiguousarray(w), P, r0 * 64


def merge_results(res, first_pattern, holds_last_round, total_rounds, group=None, device="cpu"):
    """All-reduce per-fault results of pattern shards into the full-block view.

    res: structured array with detected / first_pattern / count /
    ref_last_round_flag (lsim_b200.RESULT_DTYPE).  Returns the merged array
    (identical on every rank)."""
    import torch
    import torch.distributed as dist

    cnt = torch.from_numpy(res["count"].astype(np.int64)).to(device)
    fp = res["first_pattern"].astype(np.int64)
    fp = np.where(fp < 0, INT64_MAX, fp + int(first_pattern))
    first = torch.from_numpy(fp).to(device)
    flag = torch.from_numpy(res["ref_last_round_flag"].astype(np.int64) *
                            (1 if holds_last_round else 0)).to(device)
    dist.all_reduce(cnt, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(first, op=dist.ReduceOp.MIN, group=group)
    dist.all_reduce(flag, op=dist.ReduceOp.SUM, group=group)
    out = np.zeros(len(res), dtype=res.dtype)
    c = cnt.cpu().numpy()
    f = first.cpu().numpy()
    out["count"] = c.astype(np.uint64)
    out["detected"] = (c > 0).astype(np.uint8)
    out["first_pattern"] = np.where(f == INT64_MAX, -1, f)
    out["ref_last_round_flag"] = flag.cpu().numpy().astype(np.uint8)
    out["ref_last_rd"] = max(0, total_rounds - 1)
    return out


def split_faults(group, cost, world):
    """Fault indices of each rank: whole groups (faults sharing a sweep),
    largest estimated cost first, each to the rank with the least cost so
    far.  group / cost: per fault, from Simulator.fault_costs()."""
    group = np.asarray(group)
    cost = np.asarray(cost, dtype=np.float64)
    uniq, inv = np.unique(group, return_inverse=True)
    gcost = np.zeros(len(uniq))
    np.maximum.at(gcost, inv, cost)
    order = np.argsort(-gcost, kind="stable")
    load = np.zeros(world)
    owner = np.empty(len(uniq), dtype=np.int64)
    for gi in order:
        r = int(np.argmin(load))
        owner[gi] = r
        load[r] += gcost[gi]
    fault_owner = owner[inv]
    return [np.nonzero(fault_owner == r)[0] for r in range(world)]


def _fill(n_faults, idx, res):
    cnt = np.zeros(n_faults, dtype=np.int64)
    first = np.full(n_faults, INT64_MAX, dtype=np.int64)
    flag = np.zeros(n_faults, dtype=np.int64)
    fp = res["first_pattern"].astype(np.int64)
    cnt[idx] = res["count"].astype(np.int64)
    first[idx] = np.where(fp < 0, INT64_MAX, fp)
    flag[idx] = res["ref_last_round_flag"].astype(np.int64)
    return cnt, first, flag


def _assemble(cnt, first, flag, last_rd, dtype):
    out = np.zeros(len(cnt), dtype=dtype)
    out["count"] = cnt.astype(np.uint64)
    out["detected"] = (cnt > 0).astype(np.uint8)
    out["first_pattern"] = np.where(first == INT64_MAX, -1, first)
    out["ref_last_round_flag"] = flag.astype(np.uint8)
    out["ref_last_rd"] = last_rd
    return out


def combine_fault_shards(parts, n_faults):
    """Results of the whole fault list from (fault indices, results) of every
    part, on one process."""
    cnt = np.zeros(n_faults, dtype=np.int64)
    first = np.full(n_faults, INT64_MAX, dtype=np.int64)
    flag = np.zeros(n_faults, dtype=np.int64)
    last_rd, dtype = 0, None
    for idx, res in parts:
        c, f, g = _fill(n_faults, idx, res)
        cnt += c
        first = np.minimum(first, f)
        flag += g
        if len(res):
            last_rd = int(res["ref_last_rd"][0])
        dtype = res.dtype
    return _assemble(cnt, first, flag, last_rd, dtype)


def merge_fault_shards(res, idx, n_faults, total_rounds, group=None, device="cpu"):
    """All-reduce the results of this rank's faults (indices idx) into the
    results of the whole fault list (identical on every rank)."""
    import torch
    import torch.distributed as dist

    c, f, g = _fill(n_faults, idx, res)
    cnt, first, flag = (torch.from_numpy(x).to(device) for x in (c, f, g))
    dist.all_reduce(cnt, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(first, op=dist.ReduceOp.MIN, group=group)
    dist.all_reduce(flag, op=dist.ReduceOp.SUM, group=group)
    return _assemble(cnt.cpu().numpy(), first.cpu().numpy(), flag.cpu().numpy(),
                     max(0, total_rounds - 1), res.dtype)
