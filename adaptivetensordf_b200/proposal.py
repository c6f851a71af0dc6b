"""Online training and gating of the learned proposal sampler.

ProposalSampler (C++ host layer over the atdf_proposal_* kernels) places a
budget of samples per ray by a small MLP's predicted density. This schedule
drives it inside a training loop:

* judge steps run the plain uniform per-node sampler (the reference's
  sampling) with per-segment bins of rho * w; that image trains the main
  model for the step, the bins train the proposal (cross-entropy on the bin
  distribution + log-mass regression, MLP backward by the proposal MLP
  kernel, Adam) and refresh the leaf occupancy, and the proposal's own
  projection of the same rays is compared with it: a relative L2 error <=
  gate (1%) opens the proposal for the following steps, above it closes it;
* other steps, while the gate is open, train the main model through the
  proposal's samples (a budget per ray instead of the uniform count).

Judge steps come every judge_every steps while the gate is open and on every
step while it is closed. Only the gate's error is read back to the host.
"""

from __future__ import annotations

import torch


class ProposalSchedule:
    def __init__(self, tree, geo, max_samples_per_node: int, budget: int = 64, judge_every: int = 10,
                 gate: float = 0.01, lr: float = 3e-3, warmup: int = 20, device: str = "cuda", seed: int = 1005,
                 jitter: bool = True):
        from . import ProposalSampler

        self.tree, self.geo = tree, geo
        self.M = max_samples_per_node
        self.ps = ProposalSampler(tree.NumNodes(), 64, 3, seed, device)
        self.ps.budget = budget
        self.adam = torch.optim.Adam(self.ps.parameters(), lr=lr)
        self.judge_every = judge_every
        self.gate = gate
        self.warmup = warmup
        self.open = False
        self.step = 0
        self.judge_steps = 0
        self.proposal_steps = 0
        self.last_error = None
        self.last_loss = None
        self.jitter = jitter  # False: proposal samples at stratum midpoints (seed 0)

    def project(self, rays, seed: int):
        """Image of this training step's rays (autograd over the field)."""
        judge = (not self.open) or (self.step % self.judge_every == 0)
        self.step += 1
        pseed = seed if self.jitter else 0
        if not judge:
            self.proposal_steps += 1
            return self.ps.Project(self.tree, self.geo, rays, pseed)
        self.judge_steps += 1
        img = self.ps.ProjectUniformBinned(self.tree, self.geo, rays, self.M, seed)
        if self.step > self.warmup:
            with torch.no_grad():
                ip = self.ps.Project(self.tree, self.geo, rays, (seed ^ 0x5BD1E995) if self.jitter else 0)
                ref = img.detach()
                self.last_error = float((ip - ref).norm() / ref.norm().clamp_min(1e-30))
            self.open = self.last_error <= self.gate
        self.adam.zero_grad(set_to_none=True)
        self.last_loss = self.ps.ComputeGradients(self.tree)
        self.adam.step()
        return img

    def stats(self):
        return {"proposal_open": self.open, "proposal_error": self.last_error,
                "judge_steps": self.judge_steps, "proposal_steps": self.proposal_steps,
                "proposal_loss": None if self.last_loss is None else float(self.last_loss)}
