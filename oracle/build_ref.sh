#!/usr/bin/env bash
# Builds oracle/_ref/libfluidity_ref.so: the reference's own numerics functors
# (robclu/fluidity, header-only) driven by oracle/ref_driver.cpp.
#
# TEST INFRASTRUCTURE ONLY.  Usage: build_ref.sh REFERENCE_ROOT (or set
# FLUIDITY_REF).  The reference headers are read from REFERENCE_ROOT/include
# and copied to a temporary directory
# outside the repository, where two one-line fixes are applied without which
# the host build does not compile (the reference as shipped does not build):
#   1. flux_method/flux_hllc.hpp: Hllc::get sits in the private section while
#      FaceFlux calls it (flux_solver.hpp:95,152) -> make it public.
#   2. flux_method/flux_hllc.hpp:155: star_state is declared to return
#      Array<T, State::dimensions> but builds a State::elements vector ->
#      return State::elements.
# Nothing else is changed; no reference source is written into the repository.
set -euo pipefail
here="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
root="${1:-${FLUIDITY_REF:-}}"
if [ -z "$root" ]; then
  echo "build_ref.sh: give the reference checkout as the argument or in FLUIDITY_REF" >&2
  exit 2
fi
src="$root/include"
if [ ! -d "$src/fluidity" ]; then
  echo "build_ref.sh: reference headers not found at $src" >&2
  exit 2
fi
tmp="$(mktemp -d /tmp/fluidity_ref.XXXXXX)"
trap 'rm -rf "$tmp"' EXIT
cp -r "$src" "$tmp/include"
find "$tmp/include" -name ".*.swp" -delete
hllc="$tmp/include/fluidity/flux_method/flux_hllc.hpp"
# (1) insert 'public:' before the static get() of Hllc (the first one in file)
python3 - "$hllc" <<'PY'
import sys
p = sys.argv[1]
s = open(p).read()
key = "  template <typename Mat, typename T, typename Dim>\n  fluidity_host_device static auto get(const Mat& mat, T dtdh, Dim) {"
assert key in s, "flux_hllc.hpp: get() not found"
s = s.replace(key, " public:\n" + key, 1)
old = ") const -> Array<typename State::value_t, State::dimensions> {"
assert old in s, "flux_hllc.hpp: star_state signature not found"
s = s.replace(old, ") const -> Array<typename State::value_t, State::elements> {", 1)
open(p, "w").write(s)
PY
mkdir -p "$here/_ref"
${FL_CXX:-g++} -O3 -march=x86-64-v2 -ffp-contract=off -fno-fast-math -std=c++17 \
  -fopenmp -fPIC -shared -w -fpermissive -DFLUIDITY_CUDA_AVAILABLE=1 \
  -include cstddef -include cmath -include limits -include algorithm \
  -include fluidity/container/array.hpp -include fluidity/traits/container_traits.hpp \
  -I"$tmp/include" -I"${CUDA_HOME:-/usr/local/cuda}/include" -o "$here/_ref/libfluidity_ref.so" "$here/ref_driver.cpp"
echo "built $here/_ref/libfluidity_ref.so"
