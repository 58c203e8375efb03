"""Two-layer GCN over a CBM adjacency (the differentiation form's workload).

    logits = Ahat relu(Ahat X W1) W2,   Ahat = D^-1/2 A D^-1/2 (a cbm4dad)

Each layer aggregates in its narrower width: the first as (Ahat X) W1 (128
columns rather than 256), the second as Ahat (H W2) (40 columns).  Ahat's
products and, in backward, its adjoint run as CBM kernels through
torch.autograd (cbm.autograd.CBMProduct); the dense H W products run through
torch.matmul.

Two precisions: ``act_dtype=torch.bfloat16`` keeps X, the activations and the
CBM operands in BF16 (FP32 accumulation inside the kernels, FP32 logits and
FP32 master weights cast per use), ``torch.float32`` is the plain FP32 form.
"""
from __future__ import annotations

import math

import torch

from .autograd import cbm_apply

__all__ = ["GCN", "glorot", "cross_entropy"]


def cross_entropy(logits, labels):
    """Mean cross-entropy as log-softmax, gather and mean (the same value as
    torch.nn.functional.cross_entropy, without its slow single-block reduction)."""
    logp = torch.log_softmax(logits, dim=1)
    return -logp.gather(1, labels[:, None]).mean()


def glorot(fan_in, fan_out, generator=None, device=None):
    bound = math.sqrt(6.0 / (fan_in + fan_out))
    w = torch.rand(fan_in, fan_out, generator=generator, device=device) * (2 * bound) - bound
    return w


class GCN(torch.nn.Module):
    def __init__(self, adjacency, in_dim, hidden, out_dim, act_dtype=torch.bfloat16, seed=3):
        super().__init__()
        self.adj = adjacency
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.w1 = torch.nn.Parameter(glorot(in_dim, hidden, g).cuda())
        self.w2 = torch.nn.Parameter(glorot(hidden, out_dim, g).cuda())
        self.act_dtype = act_dtype

    def forward(self, x):
        act = self.act_dtype
        ax = cbm_apply(self.adj, x.to(act), out_dtype=act)          # Ahat X        [N, in]
        h = torch.relu(ax @ self.w1.to(act))                          # relu(. W1)    [N, hidden]
        hw = h @ self.w2.to(act)                                     # H W2          [N, out]
        return cbm_apply(self.adj, hw, out_dtype=torch.float32)      # Ahat (H W2)   [N, out], fp32
