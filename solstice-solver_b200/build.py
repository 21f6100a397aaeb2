"""In-tree build of libssol_b200.so (sm_100a CUDA + C++ host code).

Compiles every source of csrc/ with nvcc (device code for
``-gencode arch=compute_100a,code=sm_100a``) or g++ (host code), and links one
shared library next to this file with the CUDA runtime linked statically, so
that the library loads on any machine with the driver. Object files go to
``_build/`` beside this file. Rebuilds only what changed.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libssol_b200.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-fvisibility=hidden", "-Xptxas", "-v"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-Wall",
             "-Wextra", "-Wno-unused-parameter", "-Wno-missing-field-initializers",
             "-I" + os.path.join(CUDA, "include")]


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))] + [
        os.path.join(HERE, "..", "include", f)
        for f in os.listdir(os.path.join(HERE, "..", "include"))
    ]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, log):
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if log is not None:
        log.append(proc.stdout)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return proc.stdout


def build(verbose=False):
    """Build the library if needed; return its path. The translation units
    compile in parallel (the device code is split so that its template
    instances spread over several nvcc runs)."""
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    objs = []
    log = []
    jobs = []
    for name in sorted(os.listdir(CSRC)):
        src = os.path.join(CSRC, name)
        if not name.endswith((".cu", ".cpp")):
            continue
        obj = os.path.join(BUILD, name + ".o")
        objs.append(obj)
        if _stale(obj, [src] + headers):
            jobs.append((name, src, obj))

    def compile_one(job):
        name, src, obj = job
        if name.endswith(".cu"):
            out = _run([NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj], None)
            with open(os.path.join(BUILD, name + ".ptxas.txt"), "w") as f:
                f.write(out)
            return out
        return _run(["g++"] + CXX_FLAGS + ["-c", src, "-o", obj], None)

    if jobs:
        workers = max(1, min(len(jobs), os.cpu_count() or 1))
        with ThreadPoolExecutor(max_workers=workers) as ex:
            log.extend(ex.map(compile_one, jobs))
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs +
             ["-Xcompiler", "-fPIC", "-lpthread", "-ldl", "-lrt"], log)
    if verbose:
        sys.stdout.write("".join(log))
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
