"""ORACLE -- test infrastructure only.

The learned warm start's network restated in PyTorch float64 on the CPU (autograd for the gradients), from the same
parameters and inputs as the engine's BF16 kernels: the checker of their forward outputs and of every gradient.
"""
from __future__ import annotations

import numpy as np
import torch


def forward(params, x0, outage, src, dst, branch, es, nb, layers, h=64):
    """params: name -> float64 tensor; x0: [B * nb, 16]; outage: [B]; src/dst/branch: [E]; es: [E, 4]."""
    B = outage.shape[0]
    relu = torch.relu
    hcur = relu(x0 @ params["w_in"] + params["b_in"])
    for l in range(layers):
        c = es @ params[f"w_e{l}"]                                    # [E, h]
        pq = hcur @ params[f"w_pq{l}"]                                # [B * nb, 2h]
        p = pq[:, :h].reshape(B, nb, h)
        q = pq[:, h:].reshape(B, nb, h)
        pre = p[:, src, :] + q[:, dst, :] + c[None] + params[f"b_msg{l}"]
        keep = (branch[None, :] != outage[:, None]).to(pre.dtype)[..., None]
        msg = relu(pre) * keep                                        # [B, E, h]
        agg = torch.zeros((B, nb, h), dtype=pre.dtype).index_add(1, dst, msg).reshape(B * nb, h)
        hcur = hcur + relu(torch.cat([hcur, agg], dim=1) @ params[f"w_upd{l}"] + params[f"b_upd{l}"])
    return hcur @ params["w_out"] + params["b_out"]


def loss_and_grads(host_params, x0, outage, target, graph_np, nb, layers):
    """MSE over the first two output columns (mean over rows x 2) and its gradient per parameter (float64)."""
    params = {k: torch.tensor(np.asarray(v, dtype=np.float64), requires_grad=True) for k, v in host_params.items()}
    src, dst, branch, es = (torch.tensor(graph_np[k]) for k in ("src", "dst", "branch", "es"))
    out = forward(params, torch.tensor(np.asarray(x0, dtype=np.float64)), torch.tensor(outage), src.long(), dst.long(),
                  branch.long(), es.double(), nb, layers)
    t = torch.tensor(np.asarray(target, dtype=np.float64))
    loss = ((out[:, :2] - t) ** 2).mean()
    loss.backward()
    return float(loss), out.detach().numpy(), {k: v.grad.numpy() for k, v in params.items()}
