"""Tomographic reconstruction driver: trains the tensorial density field on a
synthetic tilt series with the fused projection and its hand-written
adjoint, and scores it against the phantom.

It follows the reference trainer's loop for the projection path
(hyperacorn/src/samples/hyper_train.cpp: TrainStep :920-944 -- rays of a
shuffled batch, ComputeImage, MSE against the measured pixels, backward,
optimizer step; the Adam learning rates of Settings.h:161,537 and the per-epoch
decay of Settings.h:545) and its volume evaluation (Eval_cell_density /
UniformSampledVolume, hyper_train.cpp:1780-1831, geometry.cpp:478-495:
the field sampled at voxel centres through the tree's node lookup).

PSNR (stated, since the reference's Saiga PSNR is not available): the
reconstruction and the phantom are both divided by max(phantom), and
PSNR = 10 log10(1 / MSE) over all N^3 voxel centres.

Forms:
  fp32       plain method: FP32 factors, FP32 SIMT fused kernels;
  bf16       BF16 factor copies, tcgen05 decoder GEMMs with FP32 accumulation;
  bf16+prop  the bf16 form with the learned proposal sampler
             (adaptivetensordf_b200.proposal), judged periodically by the
             uniform sampler; fp32+prop likewise on the FP32 kernels.

    python -m adaptivetensordf_b200.recon --config C1 --form fp32 --epochs 20
"""

from __future__ import annotations

import argparse
import dataclasses
import json
import math
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import synthetic as syn


# ----------------------------------------------------------------------------
# data
# ----------------------------------------------------------------------------
def voxelize_boxes(ph, N: int, speckle: float = 0.0, seed: int = 1001):
    """Same volume as synthetic.voxelize (z, y, x order, summed and clamped
    to 1), evaluated only inside each ellipsoid's bounding box."""
    c = (np.arange(N) + 0.5) / N * 2 - 1
    vol = np.zeros((N, N, N), np.float64)
    for cen, ax, d in zip(ph["centres"], ph["axes"], ph["density"]):
        lo = np.clip(np.floor((cen - ax + 1) / 2 * N - 0.5).astype(int), 0, N - 1)
        hi = np.clip(np.ceil((cen + ax + 1) / 2 * N - 0.5).astype(int) + 1, 0, N)
        if np.any(hi <= lo):
            continue
        x = c[lo[0]:hi[0]]
        y = c[lo[1]:hi[1]]
        z = c[lo[2]:hi[2]]
        q = (((z[:, None, None] - cen[2]) / ax[2]) ** 2 + ((y[None, :, None] - cen[1]) / ax[1]) ** 2 +
             ((x[None, None, :] - cen[0]) / ax[0]) ** 2)
        vol[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] += d * (q <= 1.0)
    if speckle > 0:
        rng = np.random.default_rng(seed + 7)
        m = rng.random(vol.shape) < speckle
        vol[m] += rng.uniform(0, 0.2, int(m.sum()))
    return np.minimum(vol, 1.0)


@dataclass
class TiltSeries:
    origin: torch.Tensor     # [A * P, 3] float32, device
    direction: torch.Tensor  # [A * P, 3] float32, device
    target: torch.Tensor     # [A * P] float32, device (noisy measurement)
    clean: torch.Tensor      # [A * P] float64, device (noise-free Siddon integrals)
    volume: torch.Tensor     # [N, N, N] float32 phantom (z, y, x), device
    angles: np.ndarray
    image_id: torch.Tensor = None  # [A * P] long: the tilt of each ray
    uv: torch.Tensor = None        # [A * P, 2] float32: the ray's pixel centre in [0, 1] (u along the width)
    height: int = 0                # detector size in pixels
    width: int = 0
    # the cameras, for the visibility mask of the max-density grid:
    # rotation [A, 4] unit quaternions (x, y, z, w) and translation [A, 3]
    # (or None) float64, intrinsics fx fy cx cy s, model (0 pinhole, 1
    # orthographic) and the ROI box
    cam_rotation: np.ndarray = None
    cam_translation: np.ndarray = None
    cam_intrinsics: tuple = None
    cam_model: int = 1
    roi_min: tuple = (-1.0, -1.0, -1.0)
    roi_max: tuple = (1.0, 1.0, 1.0)

    @property
    def num_rays(self):
        return self.origin.shape[0]


def tilt_quaternions(angles_deg, off_axis_deg: float = 0.0):
    """Unit quaternions (x, y, z, w) of the parallel-beam tilts: a rotation by
    the tilt angle about y, after the specimen's off-axis rotation about x
    (synthetic.parallel_beam_rays: d = R (0, 0, 1), origin = R (u, v, 0) -
    sqrt(2) d)."""
    out = []
    ax = math.radians(off_axis_deg) / 2
    qx = np.array([math.sin(ax), 0.0, 0.0, math.cos(ax)])
    for a in np.asarray(angles_deg, np.float64):
        h = math.radians(a) / 2
        qy = np.array([0.0, math.sin(h), 0.0, math.cos(h)])
        # q = qx * qy (Hamilton product, x y z w)
        x1, y1, z1, w1 = qx
        x2, y2, z2, w2 = qy
        out.append([w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2, w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2,
                    w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2, w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2])
    return np.asarray(out)


def make_tilt_series(cfg, device="cuda", noise_seed: int = 1002) -> TiltSeries:
    """Parallel-beam tilt series of the voxelised phantom: FP64 Siddon line
    integrals, then (when cfg.noise > 0) a per-tilt multiplicative jitter
    U[1 - cfg.jitter, 1 + cfg.jitter] and additive N(0, (noise * max y)^2)."""
    from . import SiddonProject

    ph = syn.ellipsoid_phantom(cfg.ellipsoids, 1001)
    vol = voxelize_boxes(ph, cfg.volume, cfg.speckle)
    vol_t = torch.from_numpy(vol.astype(np.float32)).to(device)
    angles = syn.tilt_angles(cfg)
    A, P = cfg.angles, cfg.detector * cfg.detector
    img = np.repeat(np.arange(A), P)
    pix = np.tile(np.arange(P), A)
    o, d = syn.parallel_beam_rays(angles, cfg.detector, img, pix)
    o_t = torch.from_numpy(o).to(device)
    d_t = torch.from_numpy(d).to(device)
    clean = SiddonProject(vol_t, o_t, d_t)
    y = clean.clone()
    if cfg.noise > 0 or cfg.jitter > 0:
        rng = np.random.default_rng(noise_seed)
        mult = rng.uniform(1 - cfg.jitter, 1 + cfg.jitter, A)
        y = y * torch.from_numpy(mult).to(device).repeat_interleave(P)
        if cfg.noise > 0:
            sigma = cfg.noise * float(y.max())
            y = y + torch.from_numpy(rng.normal(0.0, sigma, A * P)).to(device)
    n = cfg.detector
    uv = np.stack([(pix % n + 0.5) / n, (pix // n + 0.5) / n], 1).astype(np.float32)
    # the parallel beam as orthographic cameras: pixel centre i maps to
    # (i - (n - 1) / 2) / (n / 2), the detector coordinate of the rays
    return TiltSeries(o_t, d_t, y.float(), clean, vol_t, angles, torch.from_numpy(img).to(device),
                      torch.from_numpy(uv).to(device), n, n, cam_rotation=tilt_quaternions(angles),
                      cam_intrinsics=(n / 2, n / 2, (n - 1) / 2, (n - 1) / 2, 0.0), cam_model=1)


def point_in_any_image(points: torch.Tensor, data: TiltSeries) -> torch.Tensor:
    """SceneBase::PointInAnyImage (SceneBase.cu:13-97) of points [P, 3] on the
    series' cameras: 1 where a point lies in the ROI and projects into some
    image, else 0 (float32, on the points' device). Without cameras every
    point counts as seen."""
    import ctypes as ct

    from . import capi

    pts = points.contiguous().float()
    if data.cam_rotation is None:
        return torch.ones(pts.shape[0], device=pts.device)
    dev = pts.device
    rot = torch.from_numpy(np.ascontiguousarray(data.cam_rotation, np.float64)).to(dev)
    tr = None if data.cam_translation is None else \
        torch.from_numpy(np.ascontiguousarray(data.cam_translation, np.float64)).to(dev)
    K = torch.tensor(data.cam_intrinsics, dtype=torch.float64, device=dev)
    mask = torch.empty(pts.shape[0], device=dev)
    lo = (ct.c_float * 3)(*data.roi_min)
    hi = (ct.c_float * 3)(*data.roi_max)
    st = capi.lib().atdf_point_in_any_image(pts.shape[0], capi.ptr(pts), capi.ptr(rot), capi.ptr(tr),
                                            rot.shape[0], capi.ptr(K), data.width, data.height, data.cam_model,
                                            lo, hi, capi.ptr(mask),
                                            ct.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    if st != 0:
        raise RuntimeError(f"atdf_point_in_any_image: {capi.lib().atdf_status_string(st).decode()}")
    return mask


# ----------------------------------------------------------------------------
# evaluation
# ----------------------------------------------------------------------------
def voxel_centres(N: int, z0: int, z1: int, device="cuda"):
    c = (torch.arange(N, device=device, dtype=torch.float64) + 0.5) / N * 2 - 1
    zz, yy, xx = torch.meshgrid(c[z0:z1], c, c, indexing="ij")
    return torch.stack([xx, yy, zz], -1).reshape(-1, 3).float().contiguous()


@torch.no_grad()
def density_volume(tree, geo, N: int, chunk_points: int = 1 << 21, device="cuda"):
    """The field's density at the N^3 voxel centres, [N, N, N] (z, y, x)."""
    out = torch.empty((N, N, N), device=device, dtype=torch.float32)
    zc = max(1, chunk_points // (N * N))
    for z0 in range(0, N, zc):
        z1 = min(N, z0 + zc)
        pts = voxel_centres(N, z0, z1, device)
        nid, _ = tree.NodeIdForPositionGPU(pts)
        dens = geo.SampleVolumeIndirect(tree, pts, nid)
        out[z0:z1] = dens.reshape(z1 - z0, N, N)
    return out


@torch.no_grad()
def psnr(tree, geo, phantom: torch.Tensor):
    N = phantom.shape[0]
    rec = density_volume(tree, geo, N, device=phantom.device)
    m = float(phantom.max())
    mse = float(((rec.double() - phantom.double()) / m).pow(2).mean())
    return 10.0 * math.log10(1.0 / max(mse, 1e-30))


# ----------------------------------------------------------------------------
# adaptive tree refinement
# ----------------------------------------------------------------------------
_PLANE_AXES = ((1, 2, 0), (0, 2, 1), (0, 1, 2))  # plane m: (u axis, v axis, third axis)


def uniform_global_samples(tree, node_ids: torch.Tensor, g: int = 20) -> torch.Tensor:
    """HyperTreeBase::UniformGlobalSamples (HyperTree.cu:1618-1653): per node
    a g^3 grid spanning its box corner to corner, local = index / (g - 1) and
    position = local * size + min in FP32; [N, g^3, 3] with x fastest."""
    dev = node_ids.device
    local = torch.arange(g, device=dev, dtype=torch.float32) / float(g - 1)
    zz, yy, xx = torch.meshgrid(local, local, local, indexing="ij")
    unit = torch.stack([xx, yy, zz], -1).reshape(-1, 3)
    mn = tree.node_position_min[node_ids]
    sz = tree.node_position_max[node_ids] - mn
    return unit[None] * sz[:, None, :] + mn[:, None, :]


@torch.no_grad()
def compute_max_density(tree, geo, data: TiltSeries = None, g: int = 20):
    """Per active leaf, the maximum decoded density over its g^3 corner-to-
    corner grid, each point masked by the series' visibility
    (hyper_train.cpp:662-707 ComputeMaxDensity: grid 20 for the VM geometry,
    PointInAnyImage); written into tree.node_max_density."""
    ids = tree.active_node_ids
    mx = torch.empty(ids.numel(), device=ids.device)
    chunk = max(1, (1 << 21) // (g * g * g))
    for i in range(0, ids.numel(), chunk):
        nid = ids[i:i + chunk]
        pts = uniform_global_samples(tree, nid, g).reshape(-1, 3).contiguous()
        node = nid[:, None].expand(-1, g * g * g).reshape(-1).contiguous()
        dens = geo.SampleVolumeIndirect(tree, pts, node).reshape(-1)
        if data is not None:
            dens = dens * point_in_any_image(pts, data)
        mx[i:i + chunk] = dens.reshape(nid.numel(), -1).max(1).values
    md = tree.node_max_density.clone()
    md[ids] = mx.to(md.device)
    tree.node_max_density = md


@torch.no_grad()
def node_errors(tree, geo, data: TiltSeries, max_samples_per_node: int, rays: int = 1 << 18, batch: int = 16384,
                seed: int = 1006):
    """Per-node error for the structure optimisation: the FP64 per-node sums of
    AccumulateSampleLossPerNode (geometry.cpp:33-53; hyper_train.cpp:1472-1523)
    over a random subset of the tilt series, loss sum / weight sum, set with
    SetErrorForActiveNodes("override")."""
    from . import RayList

    g = torch.Generator(device=data.origin.device).manual_seed(seed)
    idx = torch.randint(0, data.num_rays, (rays,), device=data.origin.device, generator=g)
    ls = ws = None
    for i in range(0, rays, batch):
        j = idx[i:i + batch]
        _, l, w = geo.ProjectNodeError(tree, RayList(data.origin[j], data.direction[j]), max_samples_per_node, 0,
                                       data.target[j][None])
        ls = l if ls is None else ls + l
        ws = w if ws is None else ws + w
    err = torch.where(ws > 0, ls / ws.clamp_min(1e-30), torch.zeros_like(ls)).float()
    tree.SetErrorForActiveNodes(err, "override")


def _tree_like(tree, node_active):
    from . import HyperTreeBase

    t = HyperTreeBase(3, tree.max_depth)
    t.settree(tree.use_quad_tree, -1.0, 1.0)
    t.node_active = node_active.cpu().clone()
    t.UpdateActive()
    t.to(str(tree.node_position_min.device))
    return t


@torch.no_grad()
def transfer_planes(old_tree, tree, geo, old_planes):
    """New factor planes for the active leaves of `tree` from `old_planes` of
    `old_tree`'s active leaves: each texel of a new leaf's plane takes the old
    field's plane value at the texel's position (two positions along the
    plane's third axis, averaged): a copy for unchanged leaves, the parent's
    plane resampled for split children, the children's planes averaged and
    placed for merged parents. Split children reproduce the parent's planes
    exactly (the parent's bilinear cells are unions of the child's)."""
    from . import IndirectGridSample2D

    ids = tree.active_node_ids
    dev = ids.device
    K = ids.numel()
    mn = tree.node_position_min[ids]
    mxp = tree.node_position_max[ids]
    ctr = 0.5 * (mn + mxp)
    out = []
    for m, P in enumerate(old_planes):
        C, H, W = P.shape[1], P.shape[2], P.shape[3]
        a, b, e = _PLANE_AXES[m]
        u = torch.arange(W, device=dev, dtype=torch.float32) / (W - 1)
        v = torch.arange(H, device=dev, dtype=torch.float32) / (H - 1)
        vv, uu = torch.meshgrid(v, u, indexing="ij")  # [H, W]
        vals = torch.zeros(K, H, W, C, device=dev)
        for s in (0.25, 0.75):
            pos = torch.empty(K, H, W, 3, device=dev)
            pos[..., a] = mn[:, None, None, a] + uu[None] * (mxp - mn)[:, None, None, a]
            pos[..., b] = mn[:, None, None, b] + vv[None] * (mxp - mn)[:, None, None, b]
            pos[..., e] = (mn[:, e] + s * (mxp - mn)[:, e])[:, None, None]
            # a hair inside the new leaf, so boundary texels find the old leaf that covers it
            pos = ctr[:, None, None, :] + (pos - ctr[:, None, None, :]) * (1.0 - 1e-6)
            pts = pos.reshape(-1, 3).contiguous()
            old_id, _ = old_tree.NodeIdForPositionGPU(pts)
            omn = old_tree.node_position_min[old_id]
            osz = old_tree.node_position_max[old_id] - omn
            loc = (pts - omn) / osz * 2 - 1
            uv = torch.stack([loc[:, a], loc[:, b]], 1).contiguous()
            slot = old_tree.node_active_prefix_sum[old_id].contiguous()
            vals += 0.5 * IndirectGridSample2D(P.detach(), slot, uv).reshape(K, H, W, C)
        out.append(vals.permute(0, 3, 1, 2).contiguous(memory_format=torch.channels_last))
    return out


def refine(tree, geo, data: TiltSeries, max_active_nodes: int, max_samples_per_node: int,
           error_merge_factor: float = 1.1, error_split_factor: float = 0.75):
    """One structure-refinement round (hyper_train.cpp:1886-1912): node errors,
    max densities, the structure optimisation, and the planes moved to the new
    leaves. Returns whether the tree changed; the caller resets the optimizer
    (reset_optimizer_after_structure_change)."""
    node_errors(tree, geo, data, max_samples_per_node)
    compute_max_density(tree, geo, data)
    old_tree = _tree_like(tree, tree.node_active)
    old_planes = [p.detach() for p in geo.planes]
    if not tree.OptimizeStructure(max_active_nodes, error_merge_factor, error_split_factor):
        return False
    new = transfer_planes(old_tree, tree, geo, old_planes)
    geo.planes = [p.requires_grad_(True) for p in new]
    geo.leaf_slot = tree.node_active_prefix_sum
    if geo.precision == "bf16":
        geo.RefreshLowPrecision()
    return True


# ----------------------------------------------------------------------------
# training
# ----------------------------------------------------------------------------
@dataclass
class TrainOptions:
    epochs: int = 10
    batch: int = 4096
    max_samples_per_node: int = 32
    lr_grid: float = 0.01       # Settings.h:537 lr_exex_grid_adam
    lr_decoder: float = 5e-4    # Settings.h:161 decoder_lr
    lr_decay: float = 0.95      # Settings.h:545, per epoch
    loss_tv: float = 0.0        # plane TV weight (Settings.h:565 loss_tv)
    init_scale: float = 0.5     # factor init uniform(-s, s) (vm_init_scale)
    budget: int = 64            # proposal: samples per ray
    gate: float = 0.01          # proposal: relative L2 projection error allowed vs the uniform judge
    judge_every: int = 10       # proposal: steps between judge passes while open
    residual_gate: float = 0.5   # proposal: its error must stay within this share of the fit residual (0: off)
    proposal_jitter: bool = True  # proposal: jittered (True) or midpoint stratum samples
    proposal_importance: bool = False  # proposal: importance weights 1 / (n q) instead of Voronoi cells
    start_depth: int = 0        # active depth of the initial tree (0: the config's depth)
    refine_every: int = 0       # epochs between structure refinements (0: none)
    max_active_nodes: int = 0   # leaf budget of the refinement
    tone_mapper: bool = False   # photometric calibration of the projections (ToneMapper.cpp:141-227)
    tone_params: object = None  # tonemap.PhotometricCalibrationParams (None: the reference's defaults)
    tone_after_epochs: int = 1  # Settings.h:530 optimize_tone_mapper_after_epochs
    eval_every: int = 0         # steps between evaluations (0: once per epoch)
    target_psnr: float = 30.0
    time_limit: float = 0.0     # seconds of training; 0 = no limit
    stop_at_target: bool = True
    order_seed: int = 1004


def plane_tv(planes):
    """TV loss of the plane factors (geometry.h:31-75 TVLoss on the
    [N, C, H, W] planes, geometry_tensor_qo.cpp:580-582): per spatial axis the
    mean absolute difference of neighbouring texels, summed over axes and
    planes."""
    tv = 0.0
    for p in planes:
        tv = tv + (p[:, :, 1:, :] - p[:, :, :-1, :]).abs().mean() + (p[:, :, :, 1:] - p[:, :, :, :-1]).abs().mean()
    return tv


def build_model(cfg, form: str, device="cuda", param_seed: int = 1003, init_scale: float = 0.5,
                start_depth: int = 0):
    tree = syn.make_tree(cfg.tree_depth, active_depth=start_depth or cfg.tree_depth, device=device)
    geo = syn.make_geometry(tree, cfg.channels, cfg.grid, cfg.lines(), cfg.hidden, seed=param_seed, device=device,
                            init_scale=init_scale)
    geo.precision = "fp32" if form.startswith("fp32") else "bf16"
    if geo.precision == "bf16":
        geo.RefreshLowPrecision()
    return tree, geo


def fit(tree, geo, data: TiltSeries, opt: TrainOptions, device="cuda"):
    """opt.epochs epochs of uniform-sampling training of an existing model
    (no evaluation)."""
    from . import RayList

    adam = torch.optim.Adam([{"params": list(geo.planes) + list(geo.lines), "lr": opt.lr_grid},
                             {"params": list(geo.decoder_weight) + list(geo.decoder_bias), "lr": opt.lr_decoder}])
    gen = torch.Generator(device=device).manual_seed(opt.order_seed)
    n = data.num_rays
    step = 0
    for epoch in range(opt.epochs):
        perm = torch.randperm(n, device=device, generator=gen)
        for s in range(n // opt.batch):
            idx = perm[s * opt.batch:(s + 1) * opt.batch]
            img = geo.ProjectRays(tree, RayList(data.origin[idx], data.direction[idx]), opt.max_samples_per_node,
                                  (step + 1) * 0x9E3779B1)
            loss = (img.view(-1) - data.target[idx]).pow(2).mean()
            adam.zero_grad(set_to_none=True)
            loss.backward()
            adam.step()
            if geo.precision == "bf16":
                geo.RefreshLowPrecision()
            step += 1
    torch.cuda.synchronize()


def train(cfg, form: str, data: TiltSeries, opt: TrainOptions, log=None, device="cuda"):
    """Train one form; returns (evaluation records, seconds to the target
    PSNR or None). A record is {t, step, epoch, psnr, loss}, t the training
    wall time (seconds, GPU-synchronised, evaluations excluded)."""
    from . import RayList

    tree, geo = build_model(cfg, form, device, init_scale=opt.init_scale, start_depth=opt.start_depth)

    def make_optimizer(lr_grid, lr_decoder):
        groups = [{"params": list(geo.planes) + list(geo.lines), "lr": lr_grid},
                  {"params": list(geo.decoder_weight) + list(geo.decoder_bias), "lr": lr_decoder}]
        if geo.precision == "bf16":  # the step also writes the BF16 working copies
            from .optim import Adam

            # on a side stream: the next step's segment pass overlaps the update
            a = Adam(groups, geometry=geo, stream=adam_stream)
        else:
            a = torch.optim.Adam(groups, fused=True)
        return a, torch.optim.lr_scheduler.ExponentialLR(a, opt.lr_decay)

    adam_stream = torch.cuda.Stream(device=device)
    adam, sched = make_optimizer(opt.lr_grid, opt.lr_decoder)
    tm = None
    if opt.tone_mapper:
        # the scene's PhotometricCalibration between the projection and the
        # loss, with its own SGD / Adam groups (SceneBase.cpp:135-227, 679-694)
        from .tonemap import PhotometricCalibration

        if data.uv is None:
            raise ValueError("the tone mapper needs the rays' pixel coordinates (TiltSeries.uv)")
        tm = PhotometricCalibration(len(data.angles), 1, data.height, data.width, opt.tone_params, device)
        tm_sgd, tm_adam = tm.make_optimizers()
    prop = None
    if form.endswith("+prop"):
        from .proposal import ProposalSchedule

        prop = ProposalSchedule(tree, geo, opt.max_samples_per_node, budget=opt.budget, gate=opt.gate,
                                residual_gate=opt.residual_gate,
                                judge_every=opt.judge_every, device=device, jitter=opt.proposal_jitter,
                                importance=opt.proposal_importance)

    n = data.num_rays
    steps_per_epoch = n // opt.batch
    gen = torch.Generator(device=device).manual_seed(opt.order_seed)
    records = []
    t_train = 0.0
    step = 0
    loss_acc = torch.zeros((), device=device, dtype=torch.float64)
    reached = None

    def evaluate(epoch):
        nonlocal reached
        geo.CheckErrors()  # device error bits of the steps since the last evaluation
        p = psnr(tree, geo, data.volume) if data.volume is not None else None  # no ground truth: loss only
        rec = {"form": form, "t": t_train, "step": step, "epoch": epoch, "psnr": p,
               "loss": float(loss_acc) / max(1, step)}
        if tm is not None:
            rec["exposure_bias"] = tm.exposure_bias.tolist()
        if prop is not None:
            rec.update(prop.stats())
        records.append(rec)
        if log:
            log(rec)
        if reached is None and p is not None and p >= opt.target_psnr:
            reached = t_train
        return p

    # The training clock runs from one synchronisation point to the next
    # (evaluations, the time limit, refinement logs): steps are enqueued back
    # to back, as in a plain training loop, and evaluation time is excluded.
    clock = [0.0]

    def pause():
        nonlocal t_train
        torch.cuda.synchronize()
        t_train += time.perf_counter() - clock[0]

    def resume():
        torch.cuda.synchronize()
        clock[0] = time.perf_counter()

    if tm is not None:
        tm.check_errors = False  # image ids come from the series: no per-step read-back
    resume()
    for epoch in range(opt.epochs):
        perm = torch.randperm(n, device=device, generator=gen)
        for s in range(steps_per_epoch):
            idx = perm[s * opt.batch:(s + 1) * opt.batch]
            rays = RayList(data.origin[idx], data.direction[idx])
            target = data.target[idx]
            seed = (step + 1) * 0x9E3779B1
            if prop is not None:
                img = prop.project(rays, seed, target)
            else:
                img = geo.ProjectRays(tree, rays, opt.max_samples_per_node, seed)
            pred = img.view(-1)
            if tm is not None:
                pred = tm(pred.view(1, -1), data.uv[idx], data.image_id[idx]).view(-1)
            loss = (pred - target).pow(2).mean()
            if tm is not None:
                loss = loss + tm.ParameterLoss().sum()
            if opt.loss_tv > 0:
                loss = loss + opt.loss_tv * plane_tv(geo.planes)
            adam.zero_grad(set_to_none=True)
            loss.backward()
            adam.step()
            if tm is not None:
                for o in (tm_sgd, tm_adam):
                    if o is not None:
                        if epoch >= opt.tone_after_epochs:
                            o.step()
                        o.zero_grad(set_to_none=True)
                tm.ApplyConstraints()
            loss_acc += loss.detach().double()
            step += 1
            if opt.eval_every and step % opt.eval_every == 0:
                pause()
                evaluate(epoch)
                if reached is not None and opt.stop_at_target:
                    return records, reached
                resume()
            if opt.time_limit and t_train + (time.perf_counter() - clock[0]) >= opt.time_limit:
                pause()
                evaluate(epoch)
                return records, reached
        sched.step()
        if opt.refine_every and (epoch + 1) % opt.refine_every == 0 and epoch + 1 < opt.epochs:
            if hasattr(adam, "wait"):
                adam.wait()
            if refine(tree, geo, data, opt.max_active_nodes or tree.NumActiveNodes(), opt.max_samples_per_node):
                # reset_optimizer_after_structure_change: fresh Adam state at the current rates
                adam, sched = make_optimizer(*[g["lr"] for g in adam.param_groups])
            if log:
                pause()
                log({"form": form, "refined_epoch": epoch, "leaves": int(tree.NumActiveNodes()), "t": t_train})
                resume()
        if not opt.eval_every:
            pause()
            evaluate(epoch)
            if reached is not None and opt.stop_at_target:
                return records, reached
            resume()
    pause()
    return records, reached


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="C1")
    ap.add_argument("--form", default="fp32", choices=["fp32", "bf16", "bf16+prop", "fp32+prop"])
    ap.add_argument("--epochs", type=int, default=10)
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--samples", type=int, default=0, help="max samples per node (0: config value)")
    ap.add_argument("--eval-every", type=int, default=0)
    ap.add_argument("--target", type=float, default=30.0)
    ap.add_argument("--time-limit", type=float, default=0.0)
    ap.add_argument("--lr-grid", type=float, default=0.01)
    ap.add_argument("--lr-decoder", type=float, default=5e-4)
    ap.add_argument("--lr-decay", type=float, default=0.95, help="learning-rate factor per epoch")
    ap.add_argument("--no-stop", action="store_true")
    ap.add_argument("--tv", type=float, default=0.0)
    ap.add_argument("--init-scale", type=float, default=0.5)
    ap.add_argument("--noise", type=float, default=-1.0, help="override the config's noise level")
    ap.add_argument("--angles", type=int, default=0, help="override the number of tilts")
    ap.add_argument("--angle-step", type=float, default=0.0, help="override the tilt step (degrees)")
    ap.add_argument("--budget", type=int, default=64)
    ap.add_argument("--gate", type=float, default=0.01)
    ap.add_argument("--judge-every", type=int, default=10)
    ap.add_argument("--residual-gate", type=float, default=0.5)
    ap.add_argument("--no-prop-jitter", action="store_true")
    ap.add_argument("--prop-importance", action="store_true", help="proposal samples with importance weights")
    ap.add_argument("--start-depth", type=int, default=0)
    ap.add_argument("--refine-every", type=int, default=0)
    ap.add_argument("--max-leaves", type=int, default=0)
    ap.add_argument("--tone-mapper", action="store_true")
    ap.add_argument("--scene", default="", help="train on a scene directory (dataset.ini, camera.ini, poses.txt, "
                                                 "images.txt, numpy projections) instead of the synthetic series")
    a = ap.parse_args()
    cfg = syn.CONFIGS[a.config]
    if a.noise >= 0:
        cfg = dataclasses.replace(cfg, noise=a.noise, jitter=0.0 if a.noise == 0 else cfg.jitter)
    if a.angles:
        cfg = dataclasses.replace(cfg, angles=a.angles)
    if a.angle_step:
        cfg = dataclasses.replace(cfg, angle_step=a.angle_step)
    t0 = time.perf_counter()
    if a.scene:
        from .scene import load_scene

        data = load_scene(a.scene).tilt_series()
    else:
        data = make_tilt_series(cfg)
    torch.cuda.synchronize()
    print(json.dumps({"data_s": time.perf_counter() - t0, "rays": data.num_rays}), flush=True)
    opt = TrainOptions(epochs=a.epochs, batch=a.batch or cfg.rays_per_batch,
                       max_samples_per_node=a.samples or cfg.max_samples_per_node, eval_every=a.eval_every,
                       target_psnr=a.target, time_limit=a.time_limit, stop_at_target=not a.no_stop,
                       lr_grid=a.lr_grid, lr_decoder=a.lr_decoder, lr_decay=a.lr_decay, loss_tv=a.tv,
                       init_scale=a.init_scale,
                       budget=a.budget, gate=a.gate, judge_every=a.judge_every, residual_gate=a.residual_gate,
                       proposal_jitter=not a.no_prop_jitter, proposal_importance=a.prop_importance,
                       start_depth=a.start_depth,
                       refine_every=a.refine_every, max_active_nodes=a.max_leaves, tone_mapper=a.tone_mapper)
    recs, reached = train(cfg, a.form, data, opt, log=lambda r: print(json.dumps(r), flush=True))
    print(json.dumps({"form": a.form, "config": a.config, "seconds_to_target": reached, "target": a.target,
                      "final_psnr": recs[-1]["psnr"] if recs else None}), flush=True)


if __name__ == "__main__":
    main()
