"""Build the B200 extension: nvcc for sm_100a + g++ for the host C ABI.

Produces ch4-project_b200/ch4b200/libch4b200.so in-tree (it travels with the
repository snapshot; nothing is installed).  The FP64 kernels are compiled with
FMA contraction off (-fmad=false) so they round like the reference CPU build.
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "ch4b200", "libch4b200.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_INC = "/usr/local/cuda/include"


def run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: %s" % cmd[-1])
    return r


def newer(src_list, dst):
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(s) > t for s in src_list)


def build(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h", ".inc"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "ch4.h"))
    objs = []
    units = [
        ("lb_f64.cu", ["-fmad=false"]),
        ("lb_f32.cu", []),
        ("noalloc.cu", ["-fmad=false"]),
    ]
    jobs = []  # (command, object, keep the ptxas report)
    for src, extra in units:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if newer([s] + headers, o):
            jobs.append(([NVCC] + ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v"]
                         + extra + ["-c", s, "-o", o], o, True))
        objs.append(o)
    for src in ["ch4_host.cpp", "h5file.cpp"]:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if newer([s] + headers, o):
            jobs.append((["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I", CUDA_INC, "-c", s, "-o", o],
                         o, False))
        objs.append(o)
    # the translation units are independent: compile them side by side
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda j: (j, run(j[0])), jobs))
    for (cmd, o, keep), r in results:
        if keep:
            with open(o + ".ptxas.txt", "w") as f:  # registers, spills and shared memory per kernel
                f.write(r.stdout + r.stderr)
    if newer(objs, OUT):
        run([NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", OUT] + objs)
    return OUT


if __name__ == "__main__":
    print(build())
