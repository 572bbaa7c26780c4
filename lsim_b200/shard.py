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
groups' estimated costs; each fault lives on exactly one rank, so the merge
gathers the parts (no reduction over the whole list).

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


def merge_results(res, first_pattern, holds_last_round, total_rounds, group=None, device="cpu",
                  dst=None):
    """Reduce per-fault results of pattern shards into the full-block view.

    res: structured array with detected / first_pattern / count /
    ref_last_round_flag (lsim_b200.RESULT_DTYPE).  Two reductions: count and
    last-round flag together by SUM, first pattern by MIN.  dst=None: every
    rank gets the merged array (all-reduce); dst=r: only rank r does (the
    others get None), which halves the bytes each rank sends."""
    import torch
    import torch.distributed as dist

    n = len(res)
    sums = np.empty(2 * n, dtype=np.int64)
    sums[:n] = res["count"].astype(np.int64)
    sums[n:] = res["ref_last_round_flag"].astype(np.int64) * (1 if holds_last_round else 0)
    fp = res["first_pattern"].astype(np.int64)
    fp = np.where(fp < 0, INT64_MAX, fp + int(first_pattern))
    st = torch.from_numpy(sums).to(device)
    first = torch.from_numpy(fp).to(device)
    if dst is None:
        dist.all_reduce(st, op=dist.ReduceOp.SUM, group=group)
        dist.all_reduce(first, op=dist.ReduceOp.MIN, group=group)
    else:
        dist.reduce(st, dst, op=dist.ReduceOp.SUM, group=group)
        dist.reduce(first, dst, op=dist.ReduceOp.MIN, group=group)
        if dist.get_rank() != dst:
            return None
    sm = st.cpu().numpy()
    f = first.cpu().numpy()
    out = np.zeros(n, dtype=res.dtype)
    out["count"] = sm[:n].astype(np.uint64)
    out["detected"] = (sm[:n] > 0).astype(np.uint8)
    out["first_pattern"] = np.where(f == INT64_MAX, -1, f)
    out["ref_last_round_flag"] = sm[n:].astype(np.uint8)
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


def merge_fault_shards(res, idx, n_faults, total_rounds, group=None, device="cpu", dst=None):
    """Gather the results of every rank's faults (this rank's: indices idx)
    into the results of the whole fault list.  Each fault lives on one rank,
    so only the parts move: every rank sends its own faults as rows of
    (index | flag << 40, count, first pattern), padded to the longest part.
    dst=None: every rank gets the merged array (all-gather); dst=r: only rank
    r does (gather; the others get None)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    n_local = torch.tensor([len(idx)], dtype=torch.int64, device=device)
    sizes = [torch.zeros_like(n_local) for _ in range(world)]
    dist.all_gather(sizes, n_local, group=group)
    width = max(int(x.item()) for x in sizes)
    rows = np.zeros((width, 3), dtype=np.int64)
    rows[:, 0] = -1
    fp = res["first_pattern"].astype(np.int64)
    rows[:len(idx), 0] = np.asarray(idx, dtype=np.int64) | (res["ref_last_round_flag"].astype(np.int64) << 40)
    rows[:len(idx), 1] = res["count"].astype(np.int64)
    rows[:len(idx), 2] = np.where(fp < 0, INT64_MAX, fp)
    mine = torch.from_numpy(rows).to(device)
    if dst is None:
        parts = [torch.empty_like(mine) for _ in range(world)]
        dist.all_gather(parts, mine, group=group)
    else:
        parts = [torch.empty_like(mine) for _ in range(world)] if dist.get_rank() == dst else None
        dist.gather(mine, parts, dst=dst, group=group)
        if dist.get_rank() != dst:
            return None
    allrows = torch.cat(parts).cpu().numpy()
    allrows = allrows[allrows[:, 0] >= 0]
    cnt = np.zeros(n_faults, dtype=np.int64)
    first = np.full(n_faults, INT64_MAX, dtype=np.int64)
    flag = np.zeros(n_faults, dtype=np.int64)
    fi = allrows[:, 0] & ((1 << 40) - 1)
    cnt[fi] = allrows[:, 1]
    first[fi] = allrows[:, 2]
    flag[fi] = allrows[:, 0] >> 40
    return _assemble(cnt, first, flag, max(0, total_rounds - 1), res.dtype)
