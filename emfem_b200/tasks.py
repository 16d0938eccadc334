"""Task distribution over replicas (the reference's distribute_tasks,
src/em_fwd.cc:1273-1318): the (frequency, source) pairs of the observations
are split into contiguous blocks, CSEM tasks first, then MT tasks, the first
(n % groups) groups taking one more task.  Each GPU replica owns one group;
there is no data-path exchange between replicas."""

from __future__ import annotations


def distribute_tasks(fidx, tidx, n_groups: int, group_id: int):
    """Tasks (fidx, tidx) of group `group_id` in the reference's order."""
    if not 0 <= group_id < n_groups:
        raise ValueError("group_id out of range")
    pairs = sorted(set(zip((int(f) for f in fidx), (int(t) for t in tidx))))
    mt = [p for p in pairs if p[1] < 0]
    cs = [p for p in pairs if p[1] >= 0]
    out = []
    for tasks in (cs, mt):
        n = len(tasks)
        beg = sum(n // n_groups + (1 if (n % n_groups) > i else 0) for i in range(group_id))
        end = beg + n // n_groups + (1 if (n % n_groups) > group_id else 0)
        out.extend(tasks[beg:end])
    return out
