"""Build recipe for libcuot.so (sm_100a) and the CPU oracle.

`python -m cuot_b200.build` compiles every CUDA source under cuot_b200/csrc
into cuot_b200/libcuot.so with nvcc for sm_100a, and the oracle (test
infrastructure) into oracle/liboracle.so.  Builds are in-tree so the shared
objects travel with the repository snapshot.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libcuot.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_lib(force: bool = False, verbose: bool = False) -> str:
    srcs = sources()
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hdrs += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    if not force and not _stale(LIB, srcs + hdrs + [__file__]):
        return LIB
    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    nvcc = _nvcc()
    objs = []
    procs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        cmd = [nvcc, *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-c", s, "-o", o]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for s, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode:
            sys.stdout.write(out.decode(errors="replace"))
        if p.returncode:
            failed.append(s)
    if failed:
        raise RuntimeError(f"nvcc failed for: {failed}")
    tmp = LIB + ".tmp"
    subprocess.check_call([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a",
                           *objs, "-o", tmp, "-cudart", "static"])
    os.replace(tmp, LIB)
    return LIB


def build_oracle() -> str:
    """Test infrastructure: the CPU oracle and, when the reference tree is
    present, its pins built from the reference's own sources (oracle/_ref:
    cryptoTools AES/PRNG, emp-ot's GGM/SPCOT/LPN headers, the program that
    drives emp-ot's MpcotReg/LpnF2 callers through libcuot.so, and the
    reference's own GPU path for speed context and the transpose pin)."""
    odir = os.path.join(ROOT, "oracle")
    subprocess.check_call(["make", "-s", "-C", odir])
    ref_script = os.path.join(odir, "build_ref.sh")
    shim = os.path.join(odir, "emp_shim")
    deps = [os.path.join(odir, "ref_driver.cpp"), os.path.join(odir, "emp_ref.cpp"), ref_script, LIB,
            os.path.join(odir, "ref_gpu_driver.cu"), os.path.join(odir, "refgpu.map"),
            os.path.join(ROOT, "tests", "cpp", "test_emp_callers.cpp"),
            os.path.join(ROOT, "include", "cuot_dev_layer.h")]
    for d, _, files in os.walk(shim):
        deps += [os.path.join(d, f) for f in files]
    outs = [os.path.join(odir, "_ref", f) for f in ("libctref.so", "libempref.so", "test_emp_callers",
                                                      "librefgpu.so")]
    if any(_stale(o, [d for d in deps if os.path.exists(d)]) for o in outs):
        subprocess.check_call(["sh", ref_script])  # skips itself without the reference tree
    return os.path.join(odir, "liboracle.so")


if __name__ == "__main__":
    v = "-v" in sys.argv
    print(build_lib(force="-f" in sys.argv, verbose=v))
    print(build_oracle())
