"""Builds libpct_b200.so and the drop-in CLI in-tree for sm_100a with nvcc.

    python pseudoctimaging_b200/build.py [--force] [--verbose] [--ptxas-info]

(run it as a script: importing the package loads the library this builds)

Objects go to pseudoctimaging_b200/_build/, the library to pseudoctimaging_b200/lib/ and the CLI
to pseudoctimaging_b200/bin/. Built files are git-ignored but stay inside the repository so they
travel with it. Rebuilds only what changed (sources, the private header or include/*.h).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "lib" / "libpct_b200.so"
CLI = PKG / "bin" / "PatchBasedPseudoCT_b200"  # the drop-in command line
INCLUDE = REPO / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_CXX = shutil.which("g++", path="/usr/bin") or "g++"
COMMON = ["-O3", "-std=c++17", "-lineinfo", f"-ccbin={HOST_CXX}", "-Xcompiler", "-fPIC",
          f"-I{INCLUDE}", f"-I{CSRC}", f"-I{OBJ}"]
# Sources that make up the shared library; the CLI main is linked separately against it.
LIB_SOURCES = ["pct_api.cu", "pct_fuse_tma.cu", "pct_pointwise.cu", "pct_regularize.cu",
               "pct_noalloc.cu", "pct_synth.cpp", "pct_io.cpp", "pct_learned_train.cu",
               "pct_learned_api.cu", "pct_learned_infer.cu", "pct_tc_fuse.cu", "pct_jit.cpp",
               "pct_mat.cpp"]
# Device sources that are also compiled at run time (NVRTC): each is embedded as a string in
# _build/<stem>_src.inc, which the library sources include.
EMBEDDED = ["pct_rescore.cuh"]
CLI_SOURCES = ["pct_cli.cpp"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build pct_b200")


def _headers() -> list[pathlib.Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _embed(name: str) -> pathlib.Path:
    """Writes _build/<stem>_src.inc: the file's text as a C++ raw string constant."""
    src = CSRC / name
    stem = src.name.split(".")[0]
    out = OBJ / f"{stem}_src.inc"
    text = src.read_text()
    if ")pct_src\"" in text:
        raise RuntimeError(f"{src} contains the raw-string delimiter")
    body = (f"// Generated from csrc/{src.name} by build.py; do not edit.\n"
            f"static const char k_{stem}_source[] = R\"pct_src({text})pct_src\";\n")
    if not out.exists() or out.read_text() != body:
        out.write_text(body)
    return out


def _stale(target: pathlib.Path, deps: list[pathlib.Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> str:
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"command failed ({res.returncode}): {' '.join(cmd)}\n{res.stdout}{res.stderr}")
    return res.stdout + res.stderr


def _compile(src: pathlib.Path, force: bool, verbose: bool, ptxas_info: bool) -> tuple[pathlib.Path, str]:
    obj = OBJ / (src.name + ".o")
    if not force and not _stale(obj, [src] + _headers()):
        return obj, ""
    cmd = [nvcc(), *ARCH, *COMMON, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cu" and ptxas_info:
        cmd += ["-Xptxas", "-v"]
    return obj, _run(cmd, verbose)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> pathlib.Path:
    """Compiles every CUDA/C++ source for sm_100a and links the library and the CLI."""
    OBJ.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    CLI.parent.mkdir(parents=True, exist_ok=True)
    for name in EMBEDDED:
        _embed(name)
    srcs = [CSRC / s for s in LIB_SOURCES]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, force, verbose, ptxas_info), srcs))
    objs = [o for o, _ in results]
    if ptxas_info:
        for _, log in results:
            if log:
                sys.stdout.write(log)
    if force or _stale(LIB, objs):
        _run([nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lpthread", "-ldl", "-lz"], verbose)
    cli_src = [CSRC / s for s in CLI_SOURCES if (CSRC / s).exists()]
    if cli_src:
        cli_objs = [_compile(s, force, verbose, False)[0] for s in cli_src]
        if force or _stale(CLI, cli_objs + [LIB]):
            _run([nvcc(), *ARCH, "-o", str(CLI), *map(str, cli_objs), f"-L{LIB.parent}",
                  "-lpct_b200", f"-Xlinker=-rpath,$ORIGIN/../lib", "-lpthread"], verbose)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers/spills per kernel")
    args = ap.parse_args()
    print(build(force=args.force, verbose=args.verbose, ptxas_info=args.ptxas_info))


if __name__ == "__main__":
    main()
