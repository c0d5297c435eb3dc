"""Build libscfd_b200.so in-tree with nvcc for sm_100a.

    python -m shared_cfd_b200.build
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libscfd_b200.so")
HEADERS = sorted(f for f in os.listdir(CSRC) if f.endswith((".h", ".cuh")))  # every header: a change rebuilds
SOURCES = ["scfd_api.cu", "k_thermo.cu", "k_bc.cu", "k_residual.cu", "k_lusgs.cu", "k_chem.cu", "k_misc.cu", "k_sweep2.cu", "k_wave.cu", "k_residual2.cu", "k_residual2_f32.cu", "k_residual2_f64.cu", "noalloc.cu", "k_reactors.cu", "k_shard.cu", "k_adjoint.cu", "k_cea.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-fopenmp", "-shared",
    "-cudart", "shared",
]


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, s) for s in SOURCES] + [os.path.join(CSRC, h) for h in HEADERS] + \
        [os.path.join(HERE, "..", "include", "scfd_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build():
        return OUT
    objs = []
    bdir = os.path.join(HERE, "_build")
    os.makedirs(bdir, exist_ok=True)
    procs = []
    for s in SOURCES:
        o = os.path.join(bdir, s.replace(".cu", ".o"))
        cmd = [NVCC, "-c", os.path.join(CSRC, s), "-o", o] + [f for f in FLAGS if f != "-shared"] + list(extra)
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(o)
    for cmd, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode:
            sys.stdout.write(out.decode())
        if p.returncode:
            raise RuntimeError("nvcc failed: " + " ".join(cmd))
    cmd = [NVCC] + FLAGS + objs + ["-o", OUT]
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, extra=[a for a in sys.argv[1:] if a != "--force"])
    print(OUT)
