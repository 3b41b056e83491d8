"""Multi-GPU plumbing: one process per GPU, roots striped over ranks.

The path shards without a data-path exchange: rank r counts the embeddings
whose root u has u % world == r (the reference's multi-node striping,
device_funcs.cu:267-279), every rank holding a replica of the data graph.
The only collective is the final reduction below: counts summed, device
times combined as the maximum over ranks.
"""
from typing import List, Sequence, Tuple


def reduce_counts(counts: Sequence[int], ms: float, group=None, device=None) -> Tuple[List[int], float]:
    """Sum per-query counts and take the max of per-rank times over the group."""
    import torch
    import torch.distributed as dist
    c = torch.tensor([int(x) for x in counts], dtype=torch.int64, device=device)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return [int(x) for x in c.cpu()], float(t.cpu()[0])
