"""Build recipe for the checker libraries (test infrastructure only).

* ``oracle/liboracle.so``      -- the CPU restatement (siddon_oracle.c).
* ``oracle/_ref/libref_cpu.so`` -- the reference's own kernel sources built with
  the host compiler (ref_cpu_harness.cpp + shims), OpenMP.
* ``oracle/_ref/libref_gpu.so`` -- the reference's own CUDA sources built with
  nvcc for sm_100a (ref_gpu_harness.cu + shims).

The reference sources are compiled where they lie (``REFERENCE_SRC``: the
environment variable RECON_REFERENCE_SRC, else ``CT_Recon`` of a checkout of
the reference named ``reference`` beside this repository); nothing is copied.  The two reference builds only run where that directory exists
(the development container); elsewhere the prebuilt ``.so`` files are used.
Outputs go to ``oracle/`` and ``oracle/_ref/`` only.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")
REFERENCE_SRC = os.environ.get("RECON_REFERENCE_SRC",
                               os.path.normpath(os.path.join(HERE, "..", "..", "reference", "CT_Recon")))
NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout)
        raise RuntimeError("command failed: " + " ".join(cmd))


def _stale(out: str, inputs: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(p) > t for p in inputs if os.path.exists(p))


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "siddon_oracle.c")
    out = os.path.join(HERE, "liboracle.so")
    if force or _stale(out, [src, os.path.join(HERE, "siddon_oracle.h")]):
        _run(["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
              "-fPIC", "-shared", src, "-o", out, "-lm"])
    return out


def reference_available() -> bool:
    return os.path.isfile(os.path.join(REFERENCE_SRC, "siddon_kernelsMLEM.cuh"))


def build_ref_cpu(force: bool = False) -> str | None:
    out = os.path.join(REF_OUT, "libref_cpu.so")
    if not reference_available():
        return out if os.path.exists(out) else None
    os.makedirs(REF_OUT, exist_ok=True)
    shim = os.path.join(HERE, "ref_shim")
    harness = os.path.join(HERE, "ref_cpu_harness.cpp")
    deps = [harness, os.path.join(shim, "host_cuda", "ref_prelude_cpu.h"),
            os.path.join(HERE, "siddon_oracle.c")]
    if not (force or _stale(out, deps)):
        return out
    objdir = os.path.join(REF_OUT, "obj_cpu")
    os.makedirs(objdir, exist_ok=True)
    common = ["-O2", "-fPIC", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-w"]
    inc = ["-I", os.path.join(shim, "host_cuda"), "-I", os.path.join(shim, "common"),
           "-I", REFERENCE_SRC, "-I", HERE]
    o1 = os.path.join(objdir, "ref_cpu_harness.o")
    o2 = os.path.join(objdir, "ConfigFile.o")
    o3 = os.path.join(objdir, "siddon_oracle.o")
    _run(["g++", "-std=c++17", *common, "-include", os.path.join(shim, "host_cuda", "ref_prelude_cpu.h"),
          *inc, "-c", harness, "-o", o1])
    _run(["g++", "-std=c++17", *common, "-I", REFERENCE_SRC, "-c",
          os.path.join(REFERENCE_SRC, "ConfigFile.cpp"), "-o", o2])
    _run(["gcc", "-std=c11", *common, "-c", os.path.join(HERE, "siddon_oracle.c"), "-o", o3])
    _run(["g++", "-shared", "-fopenmp", o1, o2, o3, "-o", out, "-lm"])
    return out


def build_ref_gpu(force: bool = False) -> str | None:
    out = os.path.join(REF_OUT, "libref_gpu.so")
    if not reference_available():
        return out if os.path.exists(out) else None
    os.makedirs(REF_OUT, exist_ok=True)
    shim = os.path.join(HERE, "ref_shim", "common")
    harness = os.path.join(HERE, "ref_gpu_harness.cu")
    deps = [harness, os.path.join(shim, "ref_prelude_gpu.h"), os.path.join(shim, "Windows.h")]
    if not (force or _stale(out, deps)):
        return out
    _run([NVCC, "-O3", *ARCH, "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-w",
          "-include", os.path.join(shim, "ref_prelude_gpu.h"), "-I", shim, "-I", REFERENCE_SRC,
          "-I", HERE, harness, os.path.join(REFERENCE_SRC, "ConfigFile.cpp"), "-o", out])
    return out


def build_all(force: bool = False) -> dict:
    return {
        "oracle": build_oracle(force),
        "ref_cpu": build_ref_cpu(force),
        "ref_gpu": build_ref_gpu(force),
    }


if __name__ == "__main__":
    print(build_all(force="--force" in sys.argv))
