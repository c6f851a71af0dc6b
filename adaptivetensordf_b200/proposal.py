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
* between judge steps the main model trains through the proposal's samples
  (a budget per ray instead of the uniform count) while the gate is open,
  and through the plain uniform sampler while it is closed.

Judge steps come every judge_every_open steps while the gate is open and
every judge_every_closed steps while it is closed (every step during the
first `warmup` steps, to train the proposal). Only the gate's error is read
back to the host, once per judge step after the warm-up.

With the default Voronoi-cell weights the proposal's samples follow a
quadrature rule, not an unbiased estimator, so its error is a bias that the
field learns to fit. With ``importance=True`` the samples carry importance
weights 1 / (n q) and the proposal density follows the predicted density
(bin power 1): each projection is an unbiased estimate of the uniform one,
and its error is noise of zero mean. With ``residual_gate``
> 0 (and the batch's targets passed to ``project``) the gate also requires
that error to stay small beside the current fit: ||proposal - judge|| <=
residual_gate * ||judge - target||. Early in training the residual is large
and the proposal runs; once the fit's residual approaches the proposal's
error the uniform sampler takes over, and while the residual condition
fails the gate is checked only every judge_every_retired steps (the residual
keeps falling, so it rarely reopens).
"""

from __future__ import annotations

import torch


class ProposalSchedule:
    def __init__(self, tree, geo, max_samples_per_node: int, budget: int = 64, judge_every: int = 10,
                 gate: float = 0.01, lr: float = 3e-3, warmup: int = 20, device: str = "cuda", seed: int = 1005,
                 jitter: bool = True, judge_every_closed: int = 4, sampler=None, residual_gate: float = 0.0,
                 judge_every_retired: int = 100, importance: bool = False):
        self.tree, self.geo = tree, geo
        self.M = max_samples_per_node
        if sampler is None:
            from . import ProposalSampler

            sampler = ProposalSampler(tree.NumNodes(), 64, 3, seed, device)
        self.ps = sampler
        self.ps.budget = budget
        if importance:
            self.ps.importance_weights = True
            self.ps.bin_power = 1.0
        # the BF16 form runs the proposal MLP on the tensor cores too (3 hidden layers)
        if getattr(geo, "precision", "fp32") == "bf16" and len(getattr(sampler, "weight", [])) == 4:
            self.ps.precision = "bf16"
        self.adam = torch.optim.Adam(self.ps.parameters(), lr=lr)
        self.judge_every = judge_every
        self.judge_every_closed = judge_every_closed
        self.gate = gate
        self.warmup = warmup
        self.jitter = jitter  # False: proposal samples at stratum midpoints (seed 0)
        self.open = False
        self.step = 0
        self.judge_steps = 0
        self.proposal_steps = 0
        self.uniform_steps = 0
        self.last_error = None
        self.last_loss = None
        self.residual_gate = residual_gate
        self.judge_every_retired = judge_every_retired
        self.retired = False        # closed by the residual condition
        self.last_residual_ratio = None

    def is_judge_step(self, step: int) -> bool:
        if step < self.warmup:
            return True
        if self.open:
            every = self.judge_every
        else:
            every = self.judge_every_retired if self.retired else self.judge_every_closed
        return step % every == 0

    def project(self, rays, seed: int, target=None):
        """Image of this training step's rays (autograd over the field);
        target: the rays' measured projections (for the residual gate)."""
        step = self.step
        self.step += 1
        pseed = seed if self.jitter else 0
        if not self.is_judge_step(step):
            if self.open:
                self.proposal_steps += 1
                return self.ps.Project(self.tree, self.geo, rays, pseed)
            self.uniform_steps += 1
            return self.geo.ProjectRays(self.tree, rays, self.M, seed)
        self.judge_steps += 1
        img = self.ps.ProjectUniformBinned(self.tree, self.geo, rays, self.M, seed)
        self.adam.zero_grad(set_to_none=True)
        self.last_loss = self.ps.ComputeGradients(self.tree)
        self.adam.step()
        if step + 1 >= self.warmup:
            with torch.no_grad():
                ip = self.ps.Project(self.tree, self.geo, rays, (seed ^ 0x5BD1E995) if self.jitter else 0)
                ref = img.detach()
                norms = [(ip - ref).norm(), ref.norm()]
                use_res = self.residual_gate > 0 and target is not None
                if use_res:
                    norms.append((ref.reshape(-1) - target.reshape(-1)).norm())
                vals = torch.stack(norms).tolist()  # one read-back
            self.last_error = vals[0] / max(vals[1], 1e-30)
            rel_ok = self.last_error <= self.gate
            res_ok = True
            if use_res:
                self.last_residual_ratio = vals[0] / max(vals[2], 1e-30)
                res_ok = self.last_residual_ratio <= self.residual_gate
            self.open = rel_ok and res_ok
            self.retired = not res_ok
        return img

    def stats(self):
        return {"proposal_open": self.open, "proposal_error": self.last_error,
                "judge_steps": self.judge_steps, "proposal_steps": self.proposal_steps,
                "uniform_steps": self.uniform_steps, "proposal_residual_ratio": self.last_residual_ratio,
                "proposal_loss": None if self.last_loss is None else float(self.last_loss)}
