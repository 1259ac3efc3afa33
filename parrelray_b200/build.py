"""Builds libprr_b200.so (CUDA for sm_100a + host C++) in-tree.

    python -m parrelray_b200.build            # library
    python -m parrelray_b200.build --oracle   # + CPU oracle (tests only)

nvcc cross-compiles for sm_100a without a GPU.  Objects go to
parrelray_b200/_build/, the library to parrelray_b200/_lib/.  Sources whose
FP32 operation order must match the reference's (the REFERENCE-mode tracer and
the SSAA/FXAA pass) are built with -fmad=false.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIBDIR = PKG / "_lib"
LIB = LIBDIR / "libprr_b200.so"
INCLUDE = REPO / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NO_FMAD = {"k_reference.cu", "post.cu"}
CU_SOURCES = ["capi.cu", "render.cu", "k_reference.cu", "post.cu", "k_persistent.cu", "k_plain.cu", "fma_peak.cu",
              "noalloc.cu", "k_adjoint.cu", "graph.cu", "frame_loop.cu", "k_pair.cu", "k_ham.cu"]
CPP_SOURCES = ["textures.cpp", "deck.cpp", "image_io.cpp"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _newer(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return False
    t = target.stat().st_mtime
    return all(d.stat().st_mtime <= t for d in deps if d.exists())


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_library(verbose: bool = False, ptxas_verbose: bool = False, defines: list[str] | None = None,
                  build_dir: Path | None = None, lib_path: Path | None = None) -> Path:
    """Compiles every source and links the library.  `defines` (-D values)
    with `build_dir`/`lib_path` build a variant elsewhere (tuning studies)."""
    bdir = Path(build_dir) if build_dir else BUILD
    lib = Path(lib_path) if lib_path else LIB
    bdir.mkdir(parents=True, exist_ok=True)
    lib.parent.mkdir(parents=True, exist_ok=True)
    dflags = [f"-D{d}" for d in (defines or [])]
    hdrs = _headers()
    objs: list[Path] = []
    for src in CU_SOURCES:
        s = CSRC / src
        o = bdir / (src + ".o")
        objs.append(o)
        if _newer(o, [s] + hdrs) and not ptxas_verbose:
            continue
        cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
               *dflags, "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(s), "-o", str(o)]
        if src in NO_FMAD:
            cmd.insert(1, "-fmad=false")
        if ptxas_verbose:
            cmd += ["-Xptxas", "-v"]
        _run(cmd, verbose)
    for src in CPP_SOURCES:
        s = CSRC / src
        o = bdir / (src + ".o")
        objs.append(o)
        if _newer(o, [s] + hdrs):
            continue
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-I", str(INCLUDE), "-c", str(s), "-o", str(o)], verbose)
    if not _newer(lib, objs):
        _run([nvcc(), *ARCH, "-shared", "-o", str(lib), *map(str, objs), "-lz", "-ldl"], verbose)
    # the `prr` command (the reference's executable, prr.cpp:345-404)
    exe = lib.parent / "prr"
    main_src = CSRC / "prr_main.cpp"
    if not _newer(exe, [main_src, lib, INCLUDE / "prr.h"]):
        _run(["g++", "-O2", "-std=c++17", "-I", str(INCLUDE), str(main_src), "-L", str(lib.parent),
              "-l:" + lib.name, "-Wl,-rpath,$ORIGIN", "-o", str(exe)], verbose)
    return lib


COMPAT = PKG / "compat"


def reference_tree() -> Path | None:
    """The reference source tree the oracle recipe reads ($PRR_REFERENCE, or
    the location oracle/ref/build_ref.sh knows), or None where it is absent
    (e.g. on a machine that only runs prebuilt libraries)."""
    env = os.environ.get("PRR_REFERENCE")
    if env:
        p = Path(env)
        return p if (p / "kernels" / "solver.cuh").exists() else None
    script = REPO / "oracle" / "ref" / "build_ref.sh"
    if not script.exists():
        return None
    r = subprocess.run(["bash", str(script), "--locate"], capture_output=True, text=True)
    loc = r.stdout.strip()
    return Path(loc) if r.returncode == 0 and loc else None


def build_metric_plugin(header: Path, name: str | None = None, verbose: bool = False,
                        lib_dir: Path | None = None, spherical: bool = False) -> Path:
    """Compiles an unchanged ParRelRay metric plug-in header (the files the
    reference's main/metric.h selects, e.g. metrics/schwarzschild.cuh) into
    libprr_metric_<name>.so for prr_load_metric_plugin.  The header is copied
    into a staging tree whose main/, cudamaths/ and scene/ are this package's
    compatibility headers, so its "../main/base.h"-style includes resolve to
    them; the staging copy is deleted after the build.  `spherical` defines
    SPHERICAL, the reference's compile-time switch for headers whose states
    are (r, theta, phi, t) (e.g. metrics/"schwarzschild - sph.cuh")."""
    header = Path(header)
    name = name or header.stem.replace(" ", "").replace("-", "")
    out = Path(lib_dir or LIBDIR) / f"libprr_metric_{name}.so"
    deps = [header, COMPAT / "prr_plugin.cuh"] + sorted(COMPAT.rglob("*.h")) + sorted(COMPAT.rglob("*.cuh")) + _headers()
    if _newer(out, deps):
        return out
    stage = BUILD / "plugins" / name
    if stage.exists():
        shutil.rmtree(stage)
    for sub in ("main", "cudamaths", "scene"):
        shutil.copytree(COMPAT / sub, stage / sub)
    (stage / "metrics").mkdir(parents=True)
    shutil.copy(header, stage / "metrics" / header.name)
    # two translation units: the REFERENCE renderer and the colouring with -fmad=false (the reference's
    # FP32 operation order), the PHYSICAL renderer with contraction on; the header's rayToRGB kernel is
    # renamed in the second, which does not launch it
    tu_ref = stage / f"plugin_{name}_reference.cu"
    tu_ref.write_text(f'#define PRR_PLUGIN_PART 1\n#include "metrics/{header.name}"\n#include "prr_plugin.cuh"\n')
    tu_phys = stage / f"plugin_{name}_physical.cu"
    tu_phys.write_text(f'#define PRR_PLUGIN_PART 2\n#define rayToRGB prr_plugin_header_rayToRGB_unused\n'
                       f'#include "metrics/{header.name}"\n#undef rayToRGB\n#include "prr_plugin.cuh"\n')
    out.parent.mkdir(parents=True, exist_ok=True)
    common = [*ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-w",
              f'-DPRR_PLUGIN_NAME="{name}"', *(["-DSPHERICAL"] if spherical else []),
              "-I", str(stage), "-I", str(COMPAT), "-I", str(CSRC), "-I", str(INCLUDE)]
    try:
        _run([nvcc(), "-fmad=false", *common, "-c", str(tu_ref), "-o", str(stage / "reference.o")], verbose)
        _run([nvcc(), *common, "-c", str(tu_phys), "-o", str(stage / "physical.o")], verbose)
        # the header's functions are defined in both units (their host-side stubs would collide): every
        # symbol of the second but its entry point becomes local to it
        _run(["objcopy", "--keep-global-symbol=prr_plugin_trace_physical", str(stage / "physical.o")], verbose)
        _run([nvcc(), *ARCH, "-shared", str(stage / "reference.o"), str(stage / "physical.o"), "-o", str(out)], verbose)
    finally:
        shutil.rmtree(stage, ignore_errors=True)
    return out


def build_plugins(verbose: bool = False) -> list[Path]:
    """The Kerr plug-in shipped in compat/metrics, and - where the reference
    tree is mounted - the reference's own Schwarzschild and flat headers, its
    alternative Cartesian Schwarzschild header and its spherical-coordinate
    Schwarzschild header (with SPHERICAL), compiled unchanged."""
    outs = [build_metric_plugin(COMPAT / "metrics" / "kerr.cuh", "kerr", verbose)]
    ref = reference_tree()
    if ref is None:
        return outs
    for stem, name, sph in (("schwarzschild", "schwarzschild", False), ("flat", "flat", False),
                            ("schwarzschild - cart", "schwarzschildcart", False),
                            ("schwarzschild - sph", "schwarzschildsph", True)):
        h = ref / "metrics" / f"{stem}.cuh"
        if h.exists():
            outs.append(build_metric_plugin(h, name, verbose, spherical=sph))
    return outs


ORACLE_DIR = REPO / "oracle"
ORACLE_BUILD = ORACLE_DIR / "_build"
ORACLE_LIB = ORACLE_BUILD / "libprr_oracle.so"


def build_oracle(verbose: bool = False) -> Path:
    """CPU restatement (test infrastructure).  System g++ (has libgomp).  The
    seeded texture generator (csrc/textures.cpp, integer arithmetic) is
    compiled in as prr_oracle_make_texture, so CPU-only users of the oracle
    (the bench's reference arm) make the workload's textures without loading
    the product library."""
    ORACLE_BUILD.mkdir(parents=True, exist_ok=True)
    src = ORACLE_DIR / "prr_oracle.cpp"
    tex = CSRC / "textures.cpp"
    if not _newer(ORACLE_LIB, [src, tex, INCLUDE / "prr.h"]):
        _run(["g++", "-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
              "-Dprr_make_texture=prr_oracle_make_texture",
              "-I", str(INCLUDE), str(src), str(tex), "-o", str(ORACLE_LIB)], verbose)
    return ORACLE_LIB


def build_reference(verbose: bool = False) -> bool:
    """Reference sources compiled for the host (oracle/_ref); needs the
    reference tree, so only where it is mounted."""
    ref = reference_tree()
    if ref is None:
        return False
    out = ORACLE_DIR / "_ref"
    libs = [out / f"libprr_ref_{t}.so" for t in ("schw", "flat", "kerr", "cart", "sph")] + [out / "libprr_refcu_kerr.so"]
    deps = [ORACLE_DIR / "ref" / "build_ref.sh", ORACLE_DIR / "ref" / "ref_driver.cpp", ORACLE_DIR / "ref" / "ref_cuda_driver.cu",
            PKG / "compat" / "metrics" / "kerr.cuh"] + sorted((ORACLE_DIR / "ref" / "shim").glob("*.h"))
    if all(_newer(l, deps) for l in libs):
        return True
    _run(["bash", str(ORACLE_DIR / "ref" / "build_ref.sh")], verbose)
    return True


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--oracle", action="store_true", help="also build the CPU oracle and the reference host build")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="rebuild with -Xptxas -v (register/spill report)")
    a = ap.parse_args(argv)
    build_library(a.verbose, a.ptxas)
    build_plugins(a.verbose)
    if a.oracle:
        build_oracle(a.verbose)
        build_reference(a.verbose)
    return 0


if __name__ == "__main__":
    sys.exit(main())
