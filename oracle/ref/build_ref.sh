#!/usr/bin/env bash
# Builds the reference ParRelRay solver as a host C++/OpenMP shared library
# (the CPU oracle, test infrastructure only).  Reads the reference sources
# from $PRR_REFERENCE (default /root/reference), writes ONLY into
# oracle/_ref/ (git-ignored).  The reference's own build (compile.bat) is not
# used: its sources are compiled directly with g++.
#
# The shipped reference does not compile as-is.  Three of its defects are
# supplied by oracle/ref/ref_driver.cpp without touching the sources (the
# lowercase ray/tracer names, the undefined fx(), the undeclared `frames`).
# The recipe applies exactly three mechanical edits to its private copy:
#   1. cudamaths/tex2d.cuh:121-128 - delete the non-const operator[](f2),
#      which returns a reference to a temporary (a hard error); the const
#      overload at tex2d.cuh:112-119 with the same body stays and is the one
#      every caller uses.
#   2. prr.cpp - rewrite each `k<<<grid, block>>>(args);` launch as
#      `prr_ref_launch(grid, block, [&]{ k(args); });` (host emulation).
#   3. main/metric.h - the reference's compile-time metric selection point;
#      replaced by a switch over PRR_REF_METRIC_{SCHW,FLAT,CART,SPH,KERR}.
#      SCHW, FLAT, CART and SPH select the reference's own headers (CART: its
#      alternative "schwarzschild - cart.cuh"; SPH: its spherical-coordinate
#      "schwarzschild - sph.cuh", built with SPHERICAL defined); KERR selects
#      the Kerr-Schild plug-in header shipped by this repository in the
#      reference's plug-in shape (parrelray_b200/compat/metrics/kerr.cuh),
#      since the reference's metrics/kerr.cuh is a stub whose hooks do not
#      match the solver.
#   4. kernels/solver.cuh:35 - the SPHERICAL branch of initRays assigns `u`
#      without declaring it (declared only in the #else branch); the
#      assignment becomes a declaration.  Without SPHERICAL nothing changes.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REPO="$(cd "$HERE/../.." && pwd)"
REF="${PRR_REFERENCE:-/root/reference}"
OUT="$REPO/oracle/_ref"
# `build_ref.sh --locate` prints the reference tree it would read (nothing when
# absent) and builds nothing: the one place that knows where the tree lives.
if [ "${1:-}" = "--locate" ]; then
    if [ -f "$REF/kernels/solver.cuh" ]; then echo "$REF"; fi
    exit 0
fi
if [ ! -f "$REF/kernels/solver.cuh" ]; then
    echo "build_ref.sh: reference sources not found at $REF" >&2
    exit 2
fi
rm -rf "$OUT/src"
mkdir -p "$OUT/src"
for d in main kernels metrics scene cudamaths stb; do
    cp -r "$REF/$d" "$OUT/src/$d"
done
cp "$REF/prr.cpp" "$OUT/src/prr.cpp"

# 1. drop the non-const bilinear operator[](f2) (reference-to-temporary)
python3 - "$OUT/src/cudamaths/tex2d.cuh" <<'PY'
import sys, re
p = sys.argv[1]
s = open(p, encoding="utf-8-sig").read()
pat = re.compile(r"\t__device__ inline f3 &operator\[\]\(f2 uv\) \{.*?\n\t\}\n", re.S)
s2, n = pat.subn("", s, count=1)
assert n == 1, "tex2d.cuh: non-const operator[](f2) not found"
open(p, "w", encoding="utf-8").write(s2)
PY

# 4. declare `u` in the SPHERICAL branch of initRays
python3 - "$OUT/src/kernels/solver.cuh" <<'PY'
import sys
p = sys.argv[1]
s = open(p, encoding="utf-8-sig").read()
old = "#ifdef SPHERICAL\n\tu = f4(vel_cartTOspher("
assert s.count(old) == 1, "solver.cuh: SPHERICAL initRays branch not found"
open(p, "w", encoding="utf-8").write(s.replace(old, "#ifdef SPHERICAL\n\tf4 u = f4(vel_cartTOspher("))
PY

# 3. metric selection
mkdir -p "$OUT/src/compat"
cp "$REPO/parrelray_b200/compat/metrics/kerr.cuh" "$OUT/src/compat/kerr_plugin.cuh"
cat > "$OUT/src/main/metric.h" <<'EOF'
#pragma once
#if defined(PRR_REF_METRIC_FLAT)
#include "../metrics/flat.cuh"
#elif defined(PRR_REF_METRIC_CART)
#include "../metrics/schwarzschild - cart.cuh"
#elif defined(PRR_REF_METRIC_SPH)
#include "../metrics/schwarzschild - sph.cuh"
#elif defined(PRR_REF_METRIC_KERR)
#include "../compat/kerr_plugin.cuh"
#else
#include "../metrics/schwarzschild.cuh"
#endif
EOF

# The reference's own CUDA build starts from the tree as patched so far (its
# <<<>>> launches kept), with one edit for device compilation:
#   5. cudamaths/tex2d.cuh - checkCuda (fprintf/exit/cudaDeviceReset) and the
#      allocating constructor tex2d(i2) are declared __device__ __host__ but are
#      host-only code; nvcc rejects them in device code, so they become __host__.
rm -rf "$OUT/src_cuda"
cp -r "$OUT/src" "$OUT/src_cuda"
python3 - "$OUT/src_cuda/cudamaths/tex2d.cuh" <<'PY'
import sys
p = sys.argv[1]
s = open(p, encoding="utf-8-sig").read()
for old, new in (("__device__ __host__ void checkCuda(", "__host__ void checkCuda("),
                 ("__device__ __host__ tex2d(i2 resolution)", "__host__ tex2d(i2 resolution)")):
    assert s.count(old) == 1, f"tex2d.cuh: {old} not found"
    s = s.replace(old, new)
open(p, "w", encoding="utf-8").write(s)
PY

# 2. host emulation of kernel launches
python3 - "$OUT/src/prr.cpp" <<'PY'
import sys, re
p = sys.argv[1]
s = open(p, encoding="utf-8-sig").read()
pat = re.compile(r"(\w+)<<<\s*([^,>]+?)\s*,\s*([^>]+?)\s*>>>\((.*?)\);")
s2, n = pat.subn(lambda m: f"prr_ref_launch({m.group(2)}, {m.group(3)}, [&] {{ {m.group(1)}({m.group(4)}); }});", s)
assert n == 7, f"prr.cpp: expected 7 kernel launches, rewrote {n}"
open(p, "w", encoding="utf-8").write(s2)
PY

# $CXX may point at a toolchain without libgomp; the system g++ has it.
CXX="${PRR_ORACLE_CXX:-g++}"
CXXFLAGS=(-O2 -std=c++17 -fopenmp -fPIC -ffp-contract=off -w -I "$HERE/shim" -I "$OUT/src")
build_one() {
    local tag="$1" def="$2" extra="${3:-}"
    "$CXX" "${CXXFLAGS[@]}" -D"$def" ${extra} -shared -o "$OUT/libprr_ref_${tag}.so" \
        -x c++ "$HERE/ref_driver.cpp" \
        -x c++ "$OUT/src/main/Spacetime.cpp" \
        -x c++ "$OUT/src/main/Camera.cpp" \
        -x c++ "$OUT/src/main/Parameters.cpp" \
        -x c++ "$OUT/src/cudamaths/image.cu"
}
build_one schw PRR_REF_METRIC_SCHW
build_one flat PRR_REF_METRIC_FLAT
build_one kerr PRR_REF_METRIC_KERR
# the reference's alternative Cartesian Schwarzschild header (Christoffel tables;
# not selected by the shipped main/metric.h)
build_one cart PRR_REF_METRIC_CART
# the reference's spherical-coordinate Schwarzschild header, with the
# reference's SPHERICAL switch (kernels/solver.cuh:34-41, prr.cpp:250-252,
# main/base.h:71-83,121-124)
build_one sph PRR_REF_METRIC_SPH -DSPHERICAL
# the reference's CUDA build for sm_100a with the Kerr plug-in header (the bench
# workload's metric): nvcc's defaults otherwise, as the reference's compile.bat
# (`nvcc -x cu -w -O3`) has them
NVCC="${NVCC:-nvcc}"
if command -v "$NVCC" > /dev/null; then
    "$NVCC" -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -w -shared -Xcompiler -fPIC \
        -DPRR_REF_METRIC_KERR -I "$OUT/src_cuda" -o "$OUT/libprr_refcu_kerr.so" \
        -x cu "$HERE/ref_cuda_driver.cu" \
        -x cu "$OUT/src_cuda/main/Spacetime.cpp" \
        -x cu "$OUT/src_cuda/main/Camera.cpp" \
        -x cu "$OUT/src_cuda/main/Parameters.cpp" \
        -x cu "$OUT/src_cuda/cudamaths/image.cu"
fi
echo "built: $(ls "$OUT"/libprr_ref*.so | tr '\n' ' ')"
# the patched source copies are only build intermediates: keep just the libraries
rm -rf "$OUT/src" "$OUT/src_cuda"
