"""Event-sharded evaluation over several processes, one GPU each.

Every rank holds one block of the events (``analysis(cfg, shard=(rank,
world))``, or its own sample files). One evaluation is: this rank's
per-sample sums on its GPU (``getShardSums``), one all-reduce (sum) of that
small float64 buffer over the process group (NCCL between GPUs), then the
loss and gradient of the union of the shards from the summed buffer
(``finalizeShardSums``), identical on every rank. The reference splits its
samples over devices the same way and gathers per-device results with peer
copies (src/Analysis.cu:4210-4238).
"""
from __future__ import annotations

import torch


def nll_grad(ana, params: torch.Tensor, group=None, precision=None):
    """(nll, grad) of the sharded likelihood; every rank must call it with the same params."""
    import torch.distributed as dist

    sums = ana.getShardSums(params, precision)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=group)
    return ana.finalizeShardSums(params, sums)


class _ShardedNLL(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params, ana, group, precision):
        nll, grad = nll_grad(ana, params.detach(), group, precision)
        ctx.save_for_backward(grad)
        return nll

    @staticmethod
    def backward(ctx, grad_out):
        (grad,) = ctx.saved_tensors
        return grad * grad_out, None, None, None


def getNLL(ana, params: torch.Tensor, group=None, precision=None) -> torch.Tensor:
    """Differentiable NLL of the union of all ranks' shards (0-d float64 CUDA tensor)."""
    return _ShardedNLL.apply(params, ana, group, precision)


def hessian(ana, params: torch.Tensor, group=None) -> torch.Tensor:
    """Exact FP64 Hessian of the union of all ranks' shards: the FP64 value
    sums and the tangent sums along every unit direction are each summed with
    one all-reduce, then every rank forms the same symmetrised matrix."""
    import torch.distributed as dist

    n = params.numel()
    dirs = torch.eye(n, dtype=torch.float64, device=params.device)
    sums = ana.getShardSums(params, "fp64")
    tsums = ana.getShardHvpSums(params, dirs)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=group)
        dist.all_reduce(tsums, op=dist.ReduceOp.SUM, group=group)
    H = ana.finalizeShardHvp(params, dirs, sums, tsums)
    return 0.5 * (H + H.T)
