"""Build the GPU library in-tree: C11 host objects (gcc) + sm_100a CUDA objects
(nvcc), linked with the static CUDA runtime into
topos_codec_b200/lib/libtopos_codec.so. Rebuilds only what changed."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(ROOT, "_build", "obj")
LIB = os.path.join(PKG, "lib", "libtopos_codec.so")

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
CUDA_HOME = os.path.dirname(os.path.dirname(os.path.realpath(NVCC)))
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-std=c11", "-O2", "-fPIC", "-Wall", "-Wextra", "-fvisibility=hidden", "-ffp-contract=off"]
CXXFLAGS = ["-std=c++17", "-O2", "-fPIC", "-Wall", "-Wextra", "-fvisibility=hidden", f"-I{os.path.join(CUDA_HOME, 'include')}"]
NVFLAGS = GENCODE + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden"]


def _sources():
    host = sorted(os.path.join(CSRC, "host", f) for f in os.listdir(os.path.join(CSRC, "host"))
                  if f.endswith((".c", ".cpp")))
    cuda = sorted(os.path.join(CSRC, "cuda", f) for f in os.listdir(os.path.join(CSRC, "cuda")) if f.endswith(".cu"))
    return host, cuda


def _headers():
    out = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]
    out.append(os.path.join(CSRC, "tcg_device.h"))
    for sub in ("host", "cuda"):
        d = os.path.join(CSRC, sub)
        out += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".h", ".cuh"))]
    return out


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    return r.stdout


def build_library(verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    host, cuda = _sources()
    hdrs = _headers()
    objs = []
    for src in host:
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        if _stale(obj, [src] + hdrs):
            if src.endswith(".cpp"):
                _run(["g++"] + CXXFLAGS + ["-c", src, "-o", obj])
            else:
                _run(["gcc"] + CFLAGS + ["-c", src, "-o", obj])
        objs.append(obj)
    for src in cuda:
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        if _stale(obj, [src] + hdrs):
            out = _run([NVCC] + NVFLAGS + ["-c", src, "-o", obj])
            if verbose and out:
                print(out)
        objs.append(obj)
    if _stale(LIB, objs):
        _run(["g++", "-shared", "-o", LIB] + objs +
             ["-Wl,-Bsymbolic", f"-L{CUDA_HOME}/lib64", "-lcudart_static", "-lpthread", "-ldl", "-lrt"])
    return LIB


def build_oracle() -> None:
    """The CPU checker (test infrastructure): oracle restatement, and - where the
    reference sources are present - the reference library and golden driver."""
    _run(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    ref = os.environ.get("TOPOS_REFERENCE_DIR", "/root/reference")
    if os.path.isdir(os.path.join(ref, "native")):
        _run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "oracle"), "ref", f"TOPOS_REFERENCE_DIR={ref}"])


if __name__ == "__main__":
    print(build_library(verbose=True))
    build_oracle()
