"""CPU test of the proposal schedule's gate logic with a stand-in sampler:
judge every step during warm-up, open when the proposal's error against
the judge is within the gate, close when it is not, and which sampler
serves each step."""

import torch

from adaptivetensordf_b200.proposal import ProposalSchedule


class FakeSampler:
    def __init__(self, errors):
        self.errors = list(errors)  # relative error of the next gate checks
        self.calls = []
        self.w = torch.zeros(3, requires_grad=True)
        self.budget = 0

    def parameters(self):
        return [self.w]

    def ProjectUniformBinned(self, tree, geo, rays, M, seed):
        self.calls.append("judge")
        return torch.ones(1, 4)

    def ComputeGradients(self, tree):
        self.calls.append("train")
        self.w.grad = torch.zeros(3)
        return torch.tensor(0.5, dtype=torch.float64)

    def Project(self, tree, geo, rays, seed):
        self.calls.append("proposal")
        e = 0.0
        if not torch.is_grad_enabled():  # the gate check runs without autograd
            e = self.errors.pop(0) if self.errors else 0.0
        return torch.ones(1, 4) * (1 + e)


class FakeGeo:
    def __init__(self, log):
        self.log = log

    def ProjectRays(self, tree, rays, M, seed):
        self.log.append("uniform")
        return torch.ones(1, 4)


def test_gate_opens_and_closes():
    fs = FakeSampler([0.05, 0.005, 0.002, 0.03])
    sched = ProposalSchedule(None, FakeGeo(fs.calls), 24, budget=64, judge_every=3, judge_every_closed=2, gate=0.01,
                             warmup=2, sampler=fs)
    kinds = []
    for step in range(10):
        fs.calls.clear()
        sched.project(None, step + 1)
        kinds.append(tuple(fs.calls))
    J = ("judge", "train", "proposal")
    assert kinds == [("judge", "train"),   # warm-up, no gate check yet
                     J,                    # error 0.05: closed
                     J,                    # closed: judge every 2 steps; 0.005 opens
                     J,                    # open: judge every 3 steps; 0.002 keeps it open
                     ("proposal",), ("proposal",),
                     J,                    # 0.03 closes
                     ("uniform",),         # closed, between judges: the uniform sampler
                     J, J]
    st = sched.stats()
    assert (st["judge_steps"], st["proposal_steps"], st["uniform_steps"]) == (7, 2, 1)
    assert st["proposal_open"] is True


def test_residual_gate_retires_the_proposal():
    """With residual_gate, the proposal also needs its error within that
    share of the fit residual ||judge - target||: open while the residual is
    large, closed ("retired", judged only every judge_every_retired steps)
    once the residual has fallen to its error."""
    fs = FakeSampler([0.005] * 5)
    sched = ProposalSchedule(None, FakeGeo(fs.calls), 24, budget=64, judge_every=2, judge_every_closed=2, gate=0.01,
                             warmup=1, sampler=fs, residual_gate=0.5, judge_every_retired=5)
    residual = [0.1, 0.1, 0.1, 0.1, 0.004, 0.004, 0.004, 0.004, 0.004, 0.004, 0.004]
    kinds = []
    for step, r in enumerate(residual):
        fs.calls.clear()
        sched.project(None, step + 1, target=torch.ones(4) * (1 + r))
        kinds.append(tuple(fs.calls))
    J = ("judge", "train", "proposal")
    assert kinds == [J,                    # ratio 0.05: open
                     ("proposal",), J,     # open, judged every 2 steps
                     ("proposal",), J,     # residual 0.004: ratio 1.25 > 0.5, retired
                     J,                    # retired: judged on multiples of 5 (still 1.25)
                     ("uniform",), ("uniform",), ("uniform",), ("uniform",),
                     J]
    st = sched.stats()
    assert st["proposal_open"] is False and abs(st["proposal_residual_ratio"] - 1.25) < 1e-4  # float32 norms


def test_residual_gate_retires_whatever_the_relative_error():
    """A failed residual condition retires the proposal even when the
    relative error is also above the gate (the slower closed-gate judging
    is for a proposal that may still catch up with the field)."""
    fs = FakeSampler([0.05] * 3)
    sched = ProposalSchedule(None, FakeGeo(fs.calls), 24, budget=64, judge_every=2, judge_every_closed=2, gate=0.01,
                             warmup=1, sampler=fs, residual_gate=0.5, judge_every_retired=5)
    kinds = []
    for step in range(6):
        fs.calls.clear()
        sched.project(None, step + 1, target=torch.ones(4) * 1.01)
        kinds.append(tuple(fs.calls))
    J = ("judge", "train", "proposal")
    assert kinds == [J, ("uniform",), ("uniform",), ("uniform",), ("uniform",), J]
