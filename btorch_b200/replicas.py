"""Data parallelism over replicas of one network (one process per GPU).

Samples are independent in the recurrent step and the weights are read-only
during a forward pass, so inference and serving shard by sample or request
with no collective at all.  Training does need one exchange per optimizer
step: every rank runs its own share of the batch through the forward and the
hand-written backward, then the parameter gradients -- the sparse
connection's magnitude (one value per stored synapse), the input layer, the
readout -- are averaged over the ranks before the optimizer step, so that each
rank applies the gradient of the mean loss over the whole batch.

That exchange is one all-reduce of a single flat buffer holding every
gradient (NCCL over NVLink between GPUs; gloo between CPU processes),
instead of one collective per parameter: the recurrent magnitude alone is
nnz fp32 values (13 MB for a 3.3M-synapse network), and one large transfer
keeps the link at its bandwidth rather than at its per-call latency.  No
peer memory or multicast load is involved.

The reference trains on one device; this module has no counterpart there.
"""

from __future__ import annotations

from collections.abc import Iterable

import torch
import torch.distributed as dist


def _grads(params: Iterable[torch.nn.Parameter]) -> list[torch.Tensor]:
    return [p.grad for p in params if p.requires_grad and p.grad is not None]


def allreduce_gradients(params: Iterable[torch.nn.Parameter] | torch.nn.Module, group=None,
                        average: bool = True) -> int:
    """Sum (or average) the gradients of `params` over the ranks of `group`
    in one all-reduce of a flat buffer, in place.  Every rank must pass the
    same parameters in the same order, with gradients of the same shapes
    (they are concatenated in that order).  Returns the number of bytes
    exchanged per rank (0 without a process group or with one rank)."""
    if isinstance(params, torch.nn.Module):
        params = list(params.parameters())
    grads = _grads(params)
    if not grads or not dist.is_available() or not dist.is_initialized():
        return 0
    world = dist.get_world_size(group)
    if world == 1:
        return 0
    dtypes = {g.dtype for g in grads}
    devices = {g.device for g in grads}
    if len(dtypes) != 1 or len(devices) != 1:
        raise ValueError(f"gradients must share one dtype and device, got {dtypes} / {devices}")
    flat = torch.cat([g.reshape(-1) for g in grads])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    if average:
        flat.div_(world)
    off = 0
    for g in grads:
        k = g.numel()
        g.copy_(flat[off:off + k].view_as(g))
        off += k
    return flat.numel() * flat.element_size()


__all__ = ["allreduce_gradients"]
