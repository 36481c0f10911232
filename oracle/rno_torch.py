"""torch (CPU, float32, autograd) restatement of the surrogate's training loop -- test and
baseline infrastructure only.

The reference trains its RVE-RNO with torch modules and autograd on the host
(src/concrete_impact/nn/training/rve_rno.py:113-197, 200-415); this is the same loop for the
network of this package (18 -> 128 -> 128 -> 128 GELU -> 12, latent forward-Euler step
z' = z + (dt / tau_ref) zdot as in src/concrete_impact/nn/models/rve_rno.py:383-387), batch
of paths, truncated backpropagation through time, Adam.  Used as the CPU baseline of the
training workload.
"""

from __future__ import annotations

import time

import torch


class TorchRNO(torch.nn.Module):
    def __init__(self, hidden: int = 128) -> None:
        super().__init__()
        self.net = torch.nn.Sequential(
            torch.nn.Linear(18, hidden), torch.nn.GELU(), torch.nn.Linear(hidden, hidden), torch.nn.GELU(),
            torch.nn.Linear(hidden, hidden), torch.nn.GELU(), torch.nn.Linear(hidden, 12))  # fmt: skip

    def step(self, strain, rate, z, coef):
        y = self.net(torch.cat([strain, rate, z], dim=1))
        return y[:, :6], z + coef[:, None] * y[:, 6:]


def train_windows(strain, rate, stress, coef, windows: int, batch: int = 512, tbptt: int = 50, lr: float = 1e-3,
                  threads: int | None = None) -> dict:  # fmt: skip
    """Run ``windows`` TBPTT windows over normalised (P, T, 6) float32 inputs; returns the
    seconds taken, the path-steps processed and the first and last window losses."""
    if threads:
        torch.set_num_threads(threads)
    torch.manual_seed(0)
    model = TorchRNO()
    opt = torch.optim.Adam(model.parameters(), lr=lr)
    P, T = strain.shape[0], strain.shape[1]
    done, t0 = 0, time.perf_counter()
    w = 0
    losses = []
    while w < windows:
        idx = torch.randperm(P)[:batch]
        z = torch.zeros(len(idx), 6)
        for t0w in range(0, T - tbptt + 1, tbptt):
            loss = 0.0
            for t in range(t0w, t0w + tbptt):
                s, z = model.step(strain[idx, t], rate[idx, t], z, coef[idx, t])
                loss = loss + ((s - stress[idx, t]) ** 2).mean()
            opt.zero_grad()
            (loss / tbptt).backward()
            opt.step()
            losses.append(float(loss.detach()) / tbptt)
            z = z.detach()
            done += len(idx) * tbptt
            w += 1
            if w >= windows:
                break
    return {"seconds": time.perf_counter() - t0, "path_steps": done, "threads": torch.get_num_threads(),
            "loss_first": losses[0], "loss_last": losses[-1]}
