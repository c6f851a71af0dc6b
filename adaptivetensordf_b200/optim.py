"""Adam whose step also refreshes the BF16 working copies of the factors.

The BF16 form projects from BF16 copies of the FP32 factor planes and lines
(``GeometryTensorQO.RefreshLowPrecision``). With ``torch.optim.Adam`` a
training step updates the FP32 masters and then casts them again, a second
pass over 227 MB of planes on the C2 workload. ``Adam`` here performs the same
update (torch.optim.Adam's, no amsgrad) through ``atdf_adam_step_multi``:
every parameter in one launch (a block range per parameter), which also
writes each parameter's BF16 copy, so no ``RefreshLowPrecision`` is needed
after ``step()``.

The reference trains the grid and decoder with ``torch::optim::Adam``
(hyperacorn/csrc/geometry/geometry_tensor_qo.cpp:79-81, 209-220).
"""

from __future__ import annotations

import ctypes as ct

import torch

from . import capi


def _dense(t):
    """Dense storage in row-major or channels-last order (what the parameters use)."""
    return t.is_contiguous() or (t.dim() == 4 and t.is_contiguous(memory_format=torch.channels_last))


class Adam(torch.optim.Optimizer):
    """torch.optim.Adam's update on CUDA FP32 parameters, every parameter in
    one launch. ``geometry``: a GeometryTensorQO whose BF16 working copies
    (planes_bf16 / lines_bf16, precision "bf16") are written in the same pass
    for its planes and lines; other parameters are updated alone.

    ``stream``: run the update on this stream instead of the current one. The
    step waits for the current stream (the gradients), and an event recorded
    after it becomes ``geometry.params_ready``. The geometry's projections
    wait for that event only after their segment pass, which reads only the
    rays and the tree, so the next step's segment pass overlaps the update.
    Any other reader of the parameters must call ``wait()`` first."""

    def __init__(self, params, lr=1e-3, betas=(0.9, 0.999), eps=1e-8, weight_decay=0.0, geometry=None,
                 stream=None):
        if not 0.0 <= betas[0] < 1.0 or not 0.0 <= betas[1] < 1.0 or eps < 0.0:
            raise ValueError("invalid Adam hyper-parameters")
        super().__init__(params, dict(lr=lr, betas=betas, eps=eps, weight_decay=weight_decay))
        self.geometry = geometry
        self.stream = stream
        self._done = None  # event recorded after the last update on `stream`
        self._inputs = None  # the last update's gradients, held until the current stream has waited for it

    def wait(self):
        """Make the current stream wait for the last update."""
        if self._done is not None:
            torch.cuda.current_stream().wait_event(self._done)

    def __del__(self):
        # the geometry must not keep the handle of an event destroyed with us
        try:
            if self._done is not None and self.geometry is not None and \
                    self.geometry.params_ready == self._done.cuda_event:
                self.geometry.params_ready = 0
        except Exception:
            pass

    def _twins(self):
        g = self.geometry
        if g is None or g.precision != "bf16":
            return {}
        pb, lb = g.planes_bf16, g.lines_bf16
        if len(pb) != 3 or len(lb) != 3:
            raise RuntimeError("Adam: the geometry's BF16 copies are missing; call RefreshLowPrecision() once")
        out = {}
        for m in range(3):
            out[g.planes[m].data_ptr()] = pb[m]
            out[g.lines[m].data_ptr()] = lb[m]
        return out

    @torch.no_grad()
    def step(self, closure=None):
        loss = None
        if closure is not None:
            with torch.enable_grad():
                loss = closure()
        L = capi.lib()
        side = self.stream
        if side is not None and self._inputs is not None:
            # the previous update's gradients may be freed now: the current
            # stream waits for that update (a projection has usually done so)
            self.wait()
            self._inputs = None
        stream = ct.c_void_p((side or torch.cuda.current_stream()).cuda_stream)
        twins = self._twins()
        batch, keep, copies = [], [], []  # one atdf_adam_step_multi call for every parameter
        for group in self.param_groups:
            b1, b2 = group["betas"]
            for p in group["params"]:
                if p.grad is None:
                    continue
                if not (p.is_cuda and p.dtype == torch.float32 and p.grad.dtype == torch.float32):
                    raise TypeError("Adam: CUDA FP32 parameters and gradients only")
                st = self.state[p]
                if not st:
                    st["step"] = 0
                    st["exp_avg"] = torch.zeros_like(p, memory_format=torch.preserve_format)
                    st["exp_avg_sq"] = torch.zeros_like(p, memory_format=torch.preserve_format)
                st["step"] += 1
                g = p.grad
                twin = twins.get(p.data_ptr())
                dense = _dense(p)
                same = dense and all(t.stride() == p.stride() for t in (g, st["exp_avg"], st["exp_avg_sq"]))
                fused_twin = twin is not None and same and twin.stride() == p.stride() and twin.shape == p.shape
                if not same:  # one element order for every array
                    g = g.contiguous(memory_format=torch.preserve_format)
                    if g.stride() != p.stride():
                        raise RuntimeError("Adam: gradient and parameter layouts differ")
                t = capi.AdamTensor()
                t.n = p.numel()
                t.param, t.grad = p.data_ptr(), g.data_ptr()
                t.exp_avg, t.exp_avg_sq = st["exp_avg"].data_ptr(), st["exp_avg_sq"].data_ptr()
                t.param_bf16 = twin.data_ptr() if fused_twin else None
                t.lr, t.beta1, t.beta2 = float(group["lr"]), float(b1), float(b2)
                t.eps, t.weight_decay, t.step = float(group["eps"]), float(group["weight_decay"]), int(st["step"])
                batch.append(t)
                keep.append(g)
                if twin is not None and not fused_twin:
                    copies.append((twin, p))
        if side is not None:  # the gradients, new optimizer state and layout copies come from the current stream
            side.wait_stream(torch.cuda.current_stream())
        if batch:
            arr = (capi.AdamTensor * len(batch))(*batch)
            status = L.atdf_adam_step_multi(len(batch), arr, stream)
            if status != 0:
                raise RuntimeError(f"atdf_adam_step_multi: {L.atdf_status_string(status).decode()}")
        if side is not None:
            with torch.cuda.stream(side):
                for twin, p in copies:
                    twin.copy_(p)
            # the gradients stay referenced until the next step, after the
            # current stream has waited for this update, so their memory is
            # reused in stream order (no cross-stream frees, no pool growth
            # when the host runs ahead of the device)
            self._inputs = keep
            self._done = torch.cuda.Event()
            self._done.record(side)
            if self.geometry is not None:
                self.geometry.params_ready = self._done.cuda_event
        else:
            for twin, p in copies:
                twin.copy_(p)
        return loss
