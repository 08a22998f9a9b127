"""Build recipe for the native parts of gct_b200.

``build_library()`` compiles ``csrc/`` into ``gct_b200/libgct_fdk.so`` for sm_100a with nvcc.
The library is built in-tree so that it ships with the source snapshot; it is rebuilt only when a
source file is newer than the library (or ``force=True``).
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
REPO_DIR = PKG_DIR.parent
CSRC = PKG_DIR / "csrc"
LIB_PATH = PKG_DIR / "libgct_fdk.so"

NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build gct_b200")
    return cand


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _deps() -> list[Path]:
    return _sources() + sorted(CSRC.glob("*.hpp")) + sorted(CSRC.glob("*.cuh")) + sorted(
        (REPO_DIR / "include").glob("*.h"))


def _source_hash(deps: list[Path]) -> str:
    h = hashlib.sha256()
    for d in deps:
        h.update(d.name.encode())
        h.update(d.read_bytes())
    h.update(" ".join(NVCC_ARCH).encode())
    return h.hexdigest()


def _stale(target: Path, deps: list[Path]) -> bool:
    """A build is stale when the library is missing or was built from different sources.

    The check hashes file contents (recorded beside the library), not mtimes, so a copy of the
    tree with fresh timestamps does not trigger a rebuild."""
    stamp = target.with_name(target.name + ".srchash")
    if not target.exists() or not stamp.exists():
        return True
    return stamp.read_text().strip() != _source_hash(deps)


def build_library(force: bool = False, verbose: bool = False) -> Path:
    """Compile every CUDA/C++ source of the engine into one shared library."""
    if not force and not _stale(LIB_PATH, _deps()):
        return LIB_PATH
    obj_dir = PKG_DIR / "_build"
    obj_dir.mkdir(exist_ok=True)
    nvcc = _nvcc()
    cuda_home = Path(nvcc).resolve().parent.parent
    common = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "-I", str(REPO_DIR / "include"), "--expt-relaxed-constexpr"] + NVCC_ARCH
    objs = []
    procs = []
    for src in _sources():
        obj = obj_dir / (src.name + ".o")
        objs.append(obj)
        cmd = [nvcc, *common, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    errors = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            errors.append(f"{src.name}:\n{out}")
        elif verbose and out.strip():
            print(out)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    tmp = LIB_PATH.with_suffix(".so.tmp")
    link = [nvcc, *NVCC_ARCH, "-shared", "-o", str(tmp), *map(str, objs),
            "-L", str(cuda_home / "lib64"), "-lcudart"]
    if verbose:
        print(" ".join(link))
    res = subprocess.run(link, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if res.returncode != 0:
        raise RuntimeError("link failed:\n" + res.stdout)
    os.replace(tmp, LIB_PATH)
    LIB_PATH.with_name(LIB_PATH.name + ".srchash").write_text(_source_hash(_deps()))
    return LIB_PATH


if __name__ == "__main__":
    print(build_library(force=True, verbose=True))
