"""ctypes view of the C ABI in include/atdf.h (libatdf_b200.so).

This is the binding a caller outside PyTorch would write; the tests use it
to drive the kernels through the C ABI with raw device pointers. Structures
mirror the header field by field.
"""

from __future__ import annotations

import ctypes as ct
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libatdf_b200.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "atdf.h")

MAX_LAYERS = 8
MAX_HITS = 256

ATDF_OK = 0
DEVERR = {"hit_overflow": 0x1, "seg_capacity": 0x2, "sample_capacity": 0x4, "index": 0x8, "tree": 0x10}


class Tree(ct.Structure):
    _fields_ = [
        ("node_position_min", ct.c_void_p),
        ("node_position_max", ct.c_void_p),
        ("node_children", ct.c_void_p),
        ("node_active", ct.c_void_p),
        ("node_flags", ct.c_void_p),
        ("num_nodes", ct.c_int64),
        ("ns", ct.c_int32),
        ("max_depth", ct.c_int32),
    ]


class Segments(ct.Structure):
    _fields_ = [
        ("ray_seg_offset", ct.c_void_p),
        ("ray_sample_offset", ct.c_void_p),
        ("node", ct.c_void_p),
        ("tmin", ct.c_void_p),
        ("tmax", ct.c_void_p),
        ("nsamp", ct.c_void_p),
        ("ray", ct.c_void_p),
        ("first", ct.c_void_p),
        ("capacity", ct.c_int64),
        ("totals", ct.c_void_p),
    ]


class Field(ct.Structure):
    _fields_ = [
        ("channels", ct.c_int32),
        ("mode", ct.c_int32),
        ("dtype", ct.c_int32),
        ("plane", ct.c_void_p * 3),
        ("plane_h", ct.c_int32 * 3),
        ("plane_w", ct.c_int32 * 3),
        ("line", ct.c_void_p * 3),
        ("line_len", ct.c_int32 * 3),
        ("leaf_slot", ct.c_void_p),
        ("num_slots", ct.c_int64),
        ("roi_min", ct.c_float * 3),
        ("roi_max", ct.c_float * 3),
    ]


class FieldGrad(ct.Structure):
    _fields_ = [("plane", ct.c_void_p * 3), ("line", ct.c_void_p * 3)]


class Mlp(ct.Structure):
    _fields_ = [
        ("num_layers", ct.c_int32),
        ("dims", ct.c_int32 * (MAX_LAYERS + 1)),
        ("weight", ct.c_void_p * MAX_LAYERS),
        ("bias", ct.c_void_p * MAX_LAYERS),
        ("hidden_activation", ct.c_int32),
        ("last_activation", ct.c_int32),
        ("softplus_beta", ct.c_float),
    ]


class MlpGrad(ct.Structure):
    _fields_ = [("weight", ct.c_void_p * MAX_LAYERS), ("bias", ct.c_void_p * MAX_LAYERS)]


class AdamTensor(ct.Structure):
    _fields_ = [
        ("n", ct.c_int64),
        ("param", ct.c_void_p),
        ("grad", ct.c_void_p),
        ("exp_avg", ct.c_void_p),
        ("exp_avg_sq", ct.c_void_p),
        ("param_bf16", ct.c_void_p),
        ("lr", ct.c_float),
        ("beta1", ct.c_float),
        ("beta2", ct.c_float),
        ("eps", ct.c_float),
        ("weight_decay", ct.c_float),
        ("step", ct.c_int64),
    ]


class ToneMapper(ct.Structure):
    _fields_ = [
        ("num_images", ct.c_int32),
        ("exposure_mode", ct.c_int32),
        ("exposure", ct.c_void_p),
        ("sensor_w", ct.c_int32),
        ("sensor_h", ct.c_int32),
        ("sensor_bias", ct.c_void_p),
        ("response_params", ct.c_int32),
        ("response", ct.c_void_p),
        ("response_range", ct.c_float),
        ("leak", ct.c_int32),
    ]


def declared_symbols(header: str = HEADER):
    """Names of the functions include/atdf.h declares."""
    src = open(header).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(atdf_\w+)\s*\(", src, flags=re.M)))


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ct.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


P, I64, I32, F32, U64, SZ = ct.c_void_p, ct.c_int64, ct.c_int32, ct.c_float, ct.c_uint64, ct.c_size_t


def _declare(L):
    sig = {
        "atdf_status_string": (ct.c_char_p, [I32]),
        "atdf_version": (I32, []),
        "atdf_tree_flags": (I32, [P, P, I32, I64, P, P, P]),
        "atdf_ray_segments": (I32, [ct.POINTER(Tree), P, P, I64, I32, ct.POINTER(Segments), P, P]),
        "atdf_emit_samples": (I32, [ct.POINTER(Segments), I64, P, P, P, U64, P, P, P, P, P, P, I64, P, P]),
        "atdf_local_samples": (I32, [P, P, I64, I64, P, P, I64, P, P, P]),
        "atdf_node_id_for_position": (I32, [ct.POINTER(Tree), P, P, I64, P, P, P, P]),
        "atdf_grid_sample2d_forward": (I32, [P, I64, I64, I64, I64, P, P, P, I64, P, P, P]),
        "atdf_grid_sample2d_backward": (I32, [P, I64, I64, I64, I64, P, P, P, I64, P, P, P, P, P]),
        "atdf_grid_sample1d_forward": (I32, [P, I64, I64, I64, P, P, P, I64, P, P, P]),
        "atdf_grid_sample1d_backward": (I32, [P, I64, I64, I64, P, P, P, I64, P, P, P, P, P]),
        "atdf_gradient_correction_backward": (I32, [P, P, I64, P, I64, P, P, P]),
        "atdf_vm_features_forward": (I32, [ct.POINTER(Field), P, P, I64, P, P, I64, P, P, P]),
        "atdf_vm_features_backward": (I32, [ct.POINTER(Field), P, P, I64, P, P, I64, P, ct.POINTER(FieldGrad), P,
                                            P]),
        "atdf_mlp_forward": (I32, [ct.POINTER(Mlp), P, I64, P, P]),
        "atdf_mlp_backward": (I32, [ct.POINTER(Mlp), P, I64, P, P, ct.POINTER(MlpGrad), P]),
        "atdf_integrate_xray": (I32, [P, P, P, I64, I32, I64, P, P, P]),
        "atdf_accumulate_loss_per_node": (I32, [P, I32, I64, P, P, P, I64, I64, P, P, P, P]),
        "atdf_project_workspace_size": (I32, [I64, I32, I32, I64, I32, ct.POINTER(SZ)]),
        "atdf_project_forward": (I32, [ct.POINTER(Tree), ct.POINTER(Field), ct.POINTER(Mlp), P, P, I64, I32, U64, P,
                                       P, SZ, P, P]),
        "atdf_project_backward": (I32, [ct.POINTER(Tree), ct.POINTER(Field), ct.POINTER(Mlp), P, P, I64, I32, U64,
                                        P, ct.POINTER(FieldGrad), ct.POINTER(MlpGrad), P, SZ, P, P]),
        "atdf_mse_loss": (I32, [P, P, I64, F32, P, P, P, P]),
        "atdf_project_node_error": (I32, [ct.POINTER(Tree), P, P, I64, I32, U64, P, I32, P, P, P, SZ, P, P]),
        "atdf_project_forward_noalloc": (I32, [ct.POINTER(Tree), ct.POINTER(Field), ct.POINTER(Mlp), P, P, I64, I32,
                                               U64, P, P, P]),
        "atdf_siddon_project": (I32, [P, I32, I32, I32, ct.POINTER(ct.c_double), ct.POINTER(ct.c_double), P, P,
                                      I64, P, P]),
        "atdf_project_forward_segmented": (I32, [ct.POINTER(Tree), ct.POINTER(Field), ct.POINTER(Mlp), P, P, I64, U64,
                                                 P, P, SZ, P, P]),
        "atdf_project_forward_binned": (I32, [ct.POINTER(Tree), ct.POINTER(Field), ct.POINTER(Mlp), P, P, I64, I32,
                                              U64, P, P, P, SZ, P, P]),
        "atdf_project_segments": (I32, [ct.POINTER(Tree), P, P, I64, I32, I64, P, SZ, ct.POINTER(Segments), P, P]),
        "atdf_project_segment_view": (I32, [I64, I32, I64, P, SZ, ct.POINTER(Segments)]),
        "atdf_project_forward_samples": (I32, [ct.POINTER(Tree), ct.POINTER(Field), ct.POINTER(Mlp), P, P, I64, P, P,
                                               P, P, SZ, P, P]),
        "atdf_project_backward_samples": (I32, [ct.POINTER(Tree), ct.POINTER(Field), ct.POINTER(Mlp), P, P, I64, P,
                                                P, P, ct.POINTER(FieldGrad), ct.POINTER(MlpGrad), P, SZ, P, P]),
        "atdf_proposal_features": (I32, [ct.POINTER(Tree), ct.POINTER(Segments), P, P, P, P, P, P]),
        "atdf_proposal_mlp_forward": (I32, [ct.POINTER(Mlp), ct.POINTER(Segments), P, P, P]),
        "atdf_proposal_mlp_backward": (I32, [ct.POINTER(Mlp), ct.POINTER(Segments), P, P, ct.POINTER(MlpGrad), P]),
        "atdf_proposal_mlp_forward_bf16": (I32, [ct.POINTER(Mlp), ct.POINTER(Segments), P, P, P, P]),
        "atdf_proposal_mlp_backward_bf16": (I32, [ct.POINTER(Mlp), ct.POINTER(Segments), P, P, ct.POINTER(MlpGrad), P,
                                                  P]),
        "atdf_proposal_allocate": (I32, [ct.POINTER(Segments), I64, P, I32, F32, F32, P]),
        "atdf_proposal_samples": (I32, [ct.POINTER(Segments), P, F32, F32, U64, I32, P, P, I64, P, P]),
        "atdf_proposal_loss": (I32, [ct.POINTER(Segments), P, P, P, F32, P, P, P, P, I64, P, P]),
        "atdf_proposal_occupancy": (I32, [P, P, I64, P, P]),
        "atdf_adam_step": (I32, [I64, P, P, P, P, P, F32, F32, F32, F32, F32, I64, P]),
        "atdf_adam_step_multi": (I32, [I32, P, P]),
        "atdf_camera_rays": (I32, [I64, P, P, P, P, P, I64, P, I64, I32, I32, I32, I32, P, P, P, P, P]),
        "atdf_point_in_any_image": (I32, [I64, P, P, P, I64, P, I32, I32, I32, ct.POINTER(F32),
                                          ct.POINTER(F32), P, P]),
        "atdf_tone_map_forward": (I32, [ct.POINTER(ToneMapper), I64, I64, P, P, P, P, P, P]),
        "atdf_tone_map_backward": (I32, [ct.POINTER(ToneMapper), I64, I64, P, P, P, P, P, P, P, P, P, P]),
        "atdf_tone_response_loss": (I32, [I32, P, F32, P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


# ----------------------------------------------------------------------------
# helpers building the structures from torch tensors
# ----------------------------------------------------------------------------
def ptr(t):
    return None if t is None else ct.c_void_p(t.data_ptr())


def tree_struct(tree):
    t = Tree()
    t.node_position_min = tree.node_position_min.data_ptr()
    t.node_position_max = tree.node_position_max.data_ptr()
    t.node_children = tree.node_children.data_ptr()
    t.node_active = tree.node_active.data_ptr()
    t.node_flags = tree.node_flags.data_ptr()
    t.num_nodes = tree.NumNodes()
    t.ns = tree.NS()
    t.max_depth = tree.max_depth
    return t


def field_struct(geo, planes=None, lines=None):
    import torch

    planes = planes or [p.contiguous(memory_format=torch.channels_last) for p in geo.planes]
    lines = lines or [ln.contiguous(memory_format=torch.channels_last) for ln in geo.lines]
    f = Field()
    f.channels = planes[0].shape[1]
    f.mode = 1 if geo.tensor_op == "cat" else 0
    f.dtype = 0
    for m in range(3):
        f.plane[m] = planes[m].data_ptr()
        f.plane_h[m] = planes[m].shape[2]
        f.plane_w[m] = planes[m].shape[3]
        f.line[m] = lines[m].data_ptr()
        f.line_len[m] = lines[m].shape[2]
        f.roi_min[m] = geo.roi_min[m]
        f.roi_max[m] = geo.roi_max[m]
    f.leaf_slot = geo.leaf_slot.data_ptr()
    f.num_slots = planes[0].shape[0]
    return f, (planes, lines)


def field_struct_bf16(geo):
    """The field over the geometry's BF16 working copies (RefreshLowPrecision)."""
    f = Field()
    planes, lines = list(geo.planes_bf16), list(geo.lines_bf16)
    f.channels = planes[0].shape[1]
    f.mode = 1 if geo.tensor_op == "cat" else 0
    f.dtype = 1
    for m in range(3):
        f.plane[m] = planes[m].data_ptr()
        f.plane_h[m] = planes[m].shape[2]
        f.plane_w[m] = planes[m].shape[3]
        f.line[m] = lines[m].data_ptr()
        f.line_len[m] = lines[m].shape[2]
        f.roi_min[m] = geo.roi_min[m]
        f.roi_max[m] = geo.roi_max[m]
    f.leaf_slot = geo.leaf_slot.data_ptr()
    f.num_slots = planes[0].shape[0]
    return f, (planes, lines)


def grad_structs(geo, device="cuda"):
    """Preallocated FP32 gradient buffers shaped like the parameters
    (channels-last planes / lines) and their C structures."""
    import torch

    gp = [torch.empty_like(p, memory_format=torch.channels_last) for p in geo.planes]
    gl = [torch.empty_like(ln, memory_format=torch.channels_last) for ln in geo.lines]
    gw = [torch.empty_like(w) for w in geo.decoder_weight]
    gb = [torch.empty_like(b) for b in geo.decoder_bias]
    fg = FieldGrad()
    for m in range(3):
        fg.plane[m] = gp[m].data_ptr()
        fg.line[m] = gl[m].data_ptr()
    mg = MlpGrad()
    for i in range(len(gw)):
        mg.weight[i] = gw[i].data_ptr()
        mg.bias[i] = gb[i].data_ptr()
    return fg, mg, (gp, gl, gw, gb)


ACT = {"id": 0, "none": 0, "relu": 1, "silu": 2, "sigmoid": 3, "softplus": 4, "leakyrelu": 5, "abs": 6, "tanh": 7}


def mlp_struct(geo):
    m = Mlp()
    ws = [w.detach().contiguous() for w in geo.decoder_weight]
    bs = [b.detach().contiguous() for b in geo.decoder_bias]
    m.num_layers = len(ws)
    m.dims[0] = ws[0].shape[1]
    for i, w in enumerate(ws):
        m.dims[i + 1] = w.shape[0]
        m.weight[i] = w.data_ptr()
        m.bias[i] = bs[i].data_ptr()
    m.hidden_activation = ACT[geo.activation]
    m.last_activation = ACT[geo.last_activation]
    m.softplus_beta = geo.softplus_beta
    return m, (ws, bs)
