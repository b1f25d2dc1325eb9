"""Builds libyrcuda.so (the CUDA backend and its C ABI) in-tree for sm_100a.

Every CUDA translation unit is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo``; host C++ units are
compiled with ``-ffp-contract=off`` so that host-side geometry preprocessing
rounds exactly like the reference build. The library links the CUDA runtime
statically, so loading it needs nothing but the driver.

Usage: ``python -m yaoray_b200.build [--verbose-ptxas]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "libyrcuda.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NO_FMA_UNITS = {"render_kernels.cu": ["-fmad=false"], "sample_eval.cu": ["-fmad=false"], "measured.cu": ["-fmad=false"],
                "shading_eval.cu": ["-fmad=false"]}


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libyrcuda")
    return cand


def _common_flags() -> list[str]:
    return [
        "-O3",
        "-std=c++17",
        "-lineinfo",
        f"-I{ROOT / 'include'}",
        f"-I{CSRC}",
        "-Xcompiler",
        "-fPIC,-ffp-contract=off,-Wall",
    ]


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: Path, ptxas_verbose: bool) -> tuple[Path, str]:
    obj = OBJ / (src.name + ".o")
    cmd = [_nvcc(), *ARCH, *_common_flags(), "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cu":
        cmd += ["-Xptxas", "-v"] if ptxas_verbose else []
        cmd += ["--expt-relaxed-constexpr"]
        # Shading follows the reference's rounding: no fused multiply-add.
        cmd += NO_FMA_UNITS.get(src.name, [])
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    return obj, res.stderr


def build(force: bool = False, ptxas_verbose: bool = False, jobs: int | None = None) -> Path:
    """Compiles and links libyrcuda.so if any source is newer than it."""
    OBJ.mkdir(exist_ok=True)
    srcs = _sources()
    newest = max([s.stat().st_mtime for s in srcs] + [_headers_mtime(), Path(__file__).stat().st_mtime])
    if not force and LIB.exists() and LIB.stat().st_mtime >= newest:
        return LIB
    logs = []
    # An object is reused when it is newer than its source, every header and
    # this script (a header change rebuilds every unit).
    common = max(_headers_mtime(), Path(__file__).stat().st_mtime)

    def fresh(src: Path) -> bool:
        obj = OBJ / (src.name + ".o")
        return (not force and not ptxas_verbose and obj.exists()
                and obj.stat().st_mtime >= max(src.stat().st_mtime, common))

    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        futs = [None if fresh(s) else ex.submit(_compile, s, ptxas_verbose) for s in srcs]
        objs = []
        for src, f in zip(srcs, futs):
            if f is None:
                objs.append(OBJ / (src.name + ".o"))
                continue
            obj, log = f.result()
            objs.append(obj)
            if log.strip():
                logs.append(log)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [_nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs), "-lpthread"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, LIB)
    if ptxas_verbose:
        sys.stderr.write("\n".join(logs))
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    args = ap.parse_args()
    path = build(force=args.force, ptxas_verbose=args.verbose_ptxas)
    print(path)


if __name__ == "__main__":
    main()
