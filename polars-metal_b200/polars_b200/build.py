"""Builds libpmb.so (sm_100a) in-tree with nvcc.

The library is compiled for `sm_100a` only (`-gencode arch=compute_100a,code=sm_100a`); nvcc
cross-compiles it on a machine without a GPU. The output lands next to this file so that it
travels with the source tree.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
CSRC = PKG_DIR.parent / "csrc"
INCLUDE = PKG_DIR.parent.parent / "include"
LIB_PATH = PKG_DIR / "libpmb.so"

SOURCES = [
    "pmb_runtime.cu",
    "pmb_plan.cu",
    "pmb_groupby.cu",
    "pmb_filter.cu",
    "pmb_sort.cu",
    "pmb_batched.cu",
    "pmb_learned.cu",
    "pmb_jit.cu",
    "pmb_noalloc.cu",
    "pmb_exprcol.cu",
    "pmb_order.cu",
    "pmb_arrow.cu",
]

# device sources compiled at run time by NVRTC, embedded into the library as string literals
JIT_EMBED = [("kDeviceHeader", "pmb_device.cuh"), ("kSkeleton", "pmb_jit_skeleton.cuh"),
             ("kBatchSkeleton", "pmb_jit_batch.cuh"), ("kPartSkeleton", "pmb_jit_part.cuh"),
             ("kCompactSkeleton", "pmb_jit_compact.cuh")]


def write_jit_sources() -> Path:
    out = CSRC / "pmb_jit_sources.inc"
    parts = ["// generated by polars_b200/build.py from the .cuh files it names; do not edit\n"]
    for name, fname in JIT_EMBED:
        text = (CSRC / fname).read_text()
        assert ")PMBSRC" not in text
        parts.append(f'static const char {name}[] = R"PMBSRC({text})PMBSRC";\n')
    content = "".join(parts)
    if not out.exists() or out.read_text() != content:
        out.write_text(content)
    return out

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    """Compiles every CUDA source into libpmb.so; a no-op when it is up to date."""
    write_jit_sources()
    srcs = [CSRC / s for s in SOURCES if (CSRC / s).exists()]
    deps = srcs + sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [INCLUDE / "pmb.h", Path(__file__)]
    if not force and not _stale(LIB_PATH, deps):
        return LIB_PATH
    obj_dir = PKG_DIR.parent / "_build"
    obj_dir.mkdir(exist_ok=True)
    nvcc = nvcc_path()
    common = [
        "-O3",
        "-std=c++17",
        "-lineinfo",
        *ARCH_FLAGS,
        "-Xcompiler",
        "-fPIC",
        "-I",
        str(INCLUDE),
        "--expt-relaxed-constexpr",
        "-DPMB_BUILDING",
    ]
    if extra:
        common += extra
    objs = [obj_dir / (s.stem + ".o") for s in srcs]
    cmds = [[nvcc, *common, "-c", str(s), "-o", str(o)] for s, o in zip(srcs, objs)]
    if verbose:
        for cmd in cmds:
            print(" ".join(cmd), file=sys.stderr)
    # one nvcc per source, in parallel (each is single-threaded)
    workers = max(1, min(len(cmds), len(os.sched_getaffinity(0))))
    with ThreadPoolExecutor(max_workers=workers) as ex:
        for f in [ex.submit(subprocess.run, cmd, check=True) for cmd in cmds]:
            f.result()
    tmp = LIB_PATH.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH_FLAGS, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart", "-ldl"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB_PATH)
