"""Builds the `_cubvh` torch extension (cubvh/csrc/bindings.cpp) in place,
next to this file, linked against the in-tree libcubvh_b200.so (found at run
time through an $ORIGIN-relative rpath).  Run by __graft_entry__.build();
`python cubvh/_build.py` does the same.  A C++-only extension: the CUDA work
is in libcubvh_b200.so, so g++ with torch's include and library paths is
enough (no nvcc)."""

from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc", "bindings.cpp")
HEADER = os.path.join(ROOT, "include", "cubvh_b200.h")
LIB_DIR = os.path.join(ROOT, "cubvh_b200")


def ext_path() -> str:
    return os.path.join(HERE, "_cubvh" + sysconfig.get_config_var("EXT_SUFFIX"))


def build(force: bool = False) -> str:
    out = ext_path()
    if not force and os.path.exists(out) and \
            os.path.getmtime(out) >= max(os.path.getmtime(SRC), os.path.getmtime(HEADER)):
        return out
    import torch
    from torch.utils import cpp_extension as ce
    inc = ce.include_paths(device_type="cuda") + [sysconfig.get_paths()["include"]]
    libdirs = ce.library_paths(device_type="cuda")
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
           "-DTORCH_EXTENSION_NAME=_cubvh", "-DTORCH_API_INCLUDE_EXTENSION_H",
           f"-D_GLIBCXX_USE_CXX11_ABI={abi}", "-w"]
    cmd += [f"-I{p}" for p in inc] + [SRC, "-o", out]
    cmd += [f"-L{p}" for p in libdirs] + [f"-L{LIB_DIR}"]
    cmd += ["-lcubvh_b200", "-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu", "-ltorch_cuda", "-ltorch_python"]
    # libcubvh_b200.so beside ../cubvh_b200; torch's own libraries are
    # loaded by `import torch` before the extension
    cmd += ["-Wl,-rpath,$ORIGIN/../cubvh_b200", "-Wl,--no-as-needed"]
    subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
