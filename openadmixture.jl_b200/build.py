"""Build the in-tree native libraries for sm_100a.

    lib/libadmix.so        the C-ABI engine (include/admix.h): csrc/{admix_capi,sweeps_f64,qp_batch,qn,loglik_noalloc}.cu
    lib/libadmix_synth.so  seeded synthetic-cohort generator (csrc/synth.cu), host + device

Each translation unit is compiled separately (in parallel) with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` and linked as a shared object.  Objects are
rebuilt only when a source or header is newer than the object.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "lib"
OBJ = PKG / "_build"
REPO = PKG.parent
INCLUDE = REPO / "include"

ENGINE_SOURCES = ["admix_capi.cu", "sweeps_f64.cu", "qp_batch.cu", "qn.cu", "loglik_noalloc.cu", "sweeps_mixed.cu", "mlp.cu",
                  "tc_probe.cu", "skfr.cu"]
SYNTH_SOURCES = ["synth.cu"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-fopenmp,-O3",
    f"-I{INCLUDE}", f"-I{CSRC}",
]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found (expected /usr/local/cuda/bin/nvcc)")
    return cand


def _headers() -> list[Path]:
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, obj: Path, extra: list[str]) -> None:
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def _build_so(name: str, sources: list[str], jobs: int, extra: list[str]) -> Path:
    OBJ.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    hdrs = _headers()
    objs, todo = [], []
    for s in sources:
        src = CSRC / s
        obj = OBJ / (Path(s).stem + ".o")
        objs.append(obj)
        if _stale(obj, [src, *hdrs]):
            todo.append((src, obj))
    with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        for f in [ex.submit(_compile, s, o, extra) for s, o in todo]:
            f.result()
    out = LIB / name
    if todo or _stale(out, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fopenmp", "-o", str(out), *map(str, objs),
               "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link of {name} failed:\n{r.stdout}\n{r.stderr}")
    return out


def build(jobs: int | None = None, extra: list[str] | None = None) -> dict[str, Path]:
    """Compile libadmix.so and libadmix_synth.so in place; returns their paths."""
    jobs = jobs or min(8, os.cpu_count() or 1)
    extra = extra or []
    return {
        "admix": _build_so("libadmix.so", ENGINE_SOURCES, jobs, extra),
        "synth": _build_so("libadmix_synth.so", SYNTH_SOURCES, jobs, extra),
    }


if __name__ == "__main__":
    for k, v in build().items():
        print(k, v)
