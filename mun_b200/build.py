"""Build the in-tree CUDA library ``mun_b200/_sem.so`` for sm_100a with nvcc."""
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SO = os.path.join(HERE, "_sem.so")
SOURCES = [os.path.join(HERE, "csrc", "sem_kernels.cu"), os.path.join(HERE, "csrc", "sem_velocity.cu")]
HEADERS = [os.path.join(ROOT, "include", "mun_sem.h")]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-shared", "-Xcompiler", "-fPIC", "-Xptxas", "-v"]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def needs_build():
    if not os.path.exists(SO):
        return True
    t = os.path.getmtime(SO)
    return any(os.path.getmtime(p) > t for p in SOURCES + HEADERS)


def build(force=False, verbose=False, out=None, defines=()):
    """Compile the library if a source is newer than the .so (or ``force``).  ``out`` and
    ``defines`` build a variant elsewhere (kernel tuning experiments)."""
    target = out or SO
    if out is None and not force and not needs_build():
        return SO
    cmd = [nvcc_path()] + NVCC_FLAGS + [f"-D{d}" for d in defines] + ["-o", target + ".tmp"] + SOURCES
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stderr)
    if verbose:
        print(res.stderr)
    os.replace(target + ".tmp", target)
    return target


if __name__ == "__main__":
    build(force=True, verbose=True)
