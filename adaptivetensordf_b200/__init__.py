"""B200 (sm_100a) forward-projection path of the adaptive tensorial density
field reconstructor (HyperAcorn / adaptivetensordf).

The native pieces live next to this file:
  * libatdf_b200.so   hand-written sm_100a kernels behind the C ABI of
                      include/atdf.h;
  * _atdf_host*.so    the C++/libtorch host layer with the reference's
                      operator surface (HyperTreeBase, SampleList,
                      IndirectGridSample2D/1D, GeometryTensorQO, ...).
Both are built in place by ``adaptivetensordf_b200/build.py``. The first use
of a native name (``HyperTreeBase``, ``GeometryTensorQO``, ``ext``, ...) loads
them and fails loudly when they are missing: there is no CPU or pure-PyTorch
fallback for the path. The workload generators of ``synthetic`` (numpy
phantoms, rays, projections and tree refinement) load nothing native until
they build a tree or a geometry.
"""

from __future__ import annotations

import glob
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libatdf_b200.so")


def _load_ext():
    import torch  # noqa: F401  (libtorch must be loaded before the extension)

    cands = glob.glob(os.path.join(_HERE, "_atdf_host*.so"))
    if not cands or not os.path.exists(LIB_PATH):
        raise ImportError(
            "adaptivetensordf_b200: native libraries are not built; run "
            "`python adaptivetensordf_b200/build.py` (or __graft_entry__.build())"
        )
    from . import _atdf_host  # type: ignore

    return _atdf_host


_NATIVE = ("HyperTreeBase", "RayList", "SampleList", "GeometryTensorQO", "IndirectGridSample2D",
           "IndirectGridSample1D", "GradientCorrection", "IntegrateSamplesXRay", "AccumulateSampleLossPerNode",
           "MseLossAndGrad", "DecodeFeatures", "SiddonProject", "ProposalSampler")
_ext = None


def __getattr__(name):
    global _ext
    if name == "ext" or name in _NATIVE:
        if _ext is None:
            _ext = _load_ext()
        return _ext if name == "ext" else getattr(_ext, name)
    raise AttributeError(f"module 'adaptivetensordf_b200' has no attribute '{name}'")


__all__ = [
    "ext",
    "LIB_PATH",
    "HyperTreeBase",
    "RayList",
    "SampleList",
    "GeometryTensorQO",
    "IndirectGridSample2D",
    "IndirectGridSample1D",
    "GradientCorrection",
    "IntegrateSamplesXRay",
    "AccumulateSampleLossPerNode",
    "MseLossAndGrad",
    "DecodeFeatures",
    "SiddonProject",
    "ProposalSampler",
]
