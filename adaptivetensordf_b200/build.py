"""Builds the package's native code in place: libatdf_b200.so (the sm_100a
kernels behind the C ABI of include/atdf.h) and the C++/libtorch host
extension _atdf_host*.so. Runs make with the torch / Python paths of the
current interpreter."""

from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))


def make_vars():
    import torch
    from torch.utils import cpp_extension

    torch_inc = cpp_extension.include_paths()[0]
    torch_lib = os.path.join(os.path.dirname(torch.__file__), "lib")
    return {
        "TORCH_INC": torch_inc,
        "TORCH_LIB": torch_lib,
        "PY_INC": sysconfig.get_paths()["include"],
        "EXT_SUFFIX": sysconfig.get_config_var("EXT_SUFFIX"),
        "CXX11_ABI": str(int(torch._C._GLIBCXX_USE_CXX11_ABI)),
    }


def build(target: str = "all", jobs: int | None = None) -> None:
    jobs = jobs or max(1, os.cpu_count() or 1)
    args = ["make", "-C", HERE, f"-j{jobs}", target] + [f"{k}={v}" for k, v in make_vars().items()]
    subprocess.run(args, check=True)


if __name__ == "__main__":
    build(sys.argv[1] if len(sys.argv) > 1 else "all")
