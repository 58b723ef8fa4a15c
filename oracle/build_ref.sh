#!/bin/sh
# Builds the reference's own BVH sources, read in place from the reference tree, into
# oracle/_ref/<variant>/libref.so (test oracle only; nothing here is shipped), together with
# the reference's path loop, src/main.cpp, reached through oracle/ref_main_harness.cpp.
#
# The reference fixes its build parameters as constexpr values in
# src/bvh/bvh_defines.hpp, included with quotes from the same directory. Each variant
# gets a sed-patched copy of that one header in oracle/_ref/<variant>/, and GCC's
# '-I-' switch stops the compiler from searching the including file's own directory
# first, so the reference sources pick up the patched header without being copied.
#
# usage: oracle/build_ref.sh [reference-root]
# The reference tree is the first argument, else $RT_REFERENCE_ROOT, else the read-only
# checkout this build environment mounts; without its sources the script builds nothing.
set -e
REF=${1:-${RT_REFERENCE_ROOT:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
if [ ! -f "$REF/src/bvh/bvh_defines.hpp" ]; then
    echo "reference sources not found under $REF; oracle/_ref not built" >&2
    exit 0
fi
SRCS=""
for f in bvh_bake.cpp bvh_bfs.cpp bvh_IO.cpp bvh_morton.cpp bvh_sah.cpp bvh_geo.cpp AABB.cpp bvh_traverse.cpp; do
    SRCS="$SRCS $REF/src/bvh/$f"
done
DEFS="$REF/src/bvh/bvh_defines.hpp"
# '-I-' also applies to quoted includes inside the C++ library headers (the parallel
# algorithms headers include their siblings with quotes), so name their directory.
CXXINC=$(echo '#include <algorithm>' | g++ -std=c++2b -x c++ -M - | tr ' ' '\n' | grep '/algorithm$' | head -1 | xargs dirname)

build_variant() {
    name=$1; shift
    mkdir -p "$OUT/$name"
    sed "$@" "$DEFS" > "$OUT/$name/bvh_defines.hpp.new"
    if ! cmp -s "$OUT/$name/bvh_defines.hpp.new" "$OUT/$name/bvh_defines.hpp" 2>/dev/null || [ ! -f "$OUT/$name/libref.so" ] \
        || [ "$HERE/ref_harness.cpp" -nt "$OUT/$name/libref.so" ] || [ "$HERE/ref_main_harness.cpp" -nt "$OUT/$name/libref.so" ]; then
        mv "$OUT/$name/bvh_defines.hpp.new" "$OUT/$name/bvh_defines.hpp"
        # Same language level and optimisation as the reference Makefile (-std=c++2b -O2),
        # plain x86-64 (SSE, no FMA contraction), as the reference is built.
        g++ -std=c++2b -O2 -fPIC -shared -w -Wno-deprecated \
            -I"$OUT/$name" -I- -I"$HERE/stubs" -I"$REF/src/bvh" -I"$REF/src/math" -I"$REF/src" -I"$CXXINC/pstl" \
            -o "$OUT/$name/libref.so" $SRCS "$HERE/ref_harness.cpp" "$HERE/ref_main_harness.cpp" -lpthread
        echo "built oracle/_ref/$name/libref.so"
    else
        rm -f "$OUT/$name/bvh_defines.hpp.new"
    fi
}

# reference defaults: hybrid Morton split + binned SAH below 64 triangles, leaf 16, 63-bit codes
build_variant hybrid   -e 's/^//' &
# pure Morton split (the reference's LBVH), 63-bit and 30-bit codes
build_variant lbvh63   -e 's/BVH_LBVH_THRESHOLD   = 64/BVH_LBVH_THRESHOLD   = 0/' &
build_variant lbvh30   -e 's/BVH_LBVH_THRESHOLD   = 64/BVH_LBVH_THRESHOLD   = 0/' \
                       -e 's/MORTON_UNIT_BIT_SIZE    = 21/MORTON_UNIT_BIT_SIZE    = 10/' &
build_variant lbvh63l4 -e 's/BVH_LBVH_THRESHOLD   = 64/BVH_LBVH_THRESHOLD   = 0/' \
                       -e 's/BVH_MAX_LEAF_SIZE    = 16/BVH_MAX_LEAF_SIZE    = 4/' &
wait
# binned SAH with spatial splits from the root, leaf 4 and leaf 16
build_variant sah4     -e 's/BVH_LBVH_THRESHOLD   = 64/BVH_LBVH_THRESHOLD   = 2147483647/' \
                       -e 's/BVH_MAX_LEAF_SIZE    = 16/BVH_MAX_LEAF_SIZE    = 4/' &
build_variant sah16    -e 's/BVH_LBVH_THRESHOLD   = 64/BVH_LBVH_THRESHOLD   = 2147483647/' &
# binned SAH without spatial splits (spatial extent threshold raised above any box)
build_variant sah4ns   -e 's/BVH_LBVH_THRESHOLD   = 64/BVH_LBVH_THRESHOLD   = 2147483647/' \
                       -e 's/BVH_MAX_LEAF_SIZE    = 16/BVH_MAX_LEAF_SIZE    = 4/' \
                       -e 's/BVH_SPATIAL_EPS      = 1e-6f/BVH_SPATIAL_EPS      = 3.0e38f/' &
wait

# The reference's own mesh files (bunny.ply: extra vertex properties; letterX / letterY.ply:
# quads), copied for the mesh-ingestion tests, which also run where the reference tree is absent.
mkdir -p "$OUT/meshes"
for m in bunny.ply letterX.ply letterY.ply; do
    if [ -f "$REF/$m" ]; then cp -f "$REF/$m" "$OUT/meshes/$m"; fi
done

# The reference's own unit and integration tests, read in place and compiled unchanged against
# this repository's drop-in headers (include/bvh, include/math) and librt_b200.so: the proof that
# code written for the reference's bake/load/trace/AABB interface builds and links against the
# product. Outputs: oracle/_ref/tests/test_aabb, oracle/_ref/tests/test_traverse.
LIBDIR="$HERE/../ray-tracer_b200/lib"
if [ -f "$LIBDIR/librt_b200.so" ] && [ -f "$REF/tests/test_aabb.cpp" ]; then
    mkdir -p "$OUT/tests"
    for t in test_aabb test_traverse; do
        g++ -std=c++2b -O2 -w -I"$HERE/../include/bvh" -I"$HERE/../include" "$REF/tests/$t.cpp" \
            -L"$LIBDIR" -lrt_b200 -Wl,-rpath,'$ORIGIN/../../../ray-tracer_b200/lib' -o "$OUT/tests/$t"
        echo "built oracle/_ref/tests/$t against librt_b200.so"
    done
fi
