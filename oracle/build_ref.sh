#!/usr/bin/env bash
# Builds the reference-side checkers into oracle/_ref/ from the reference
# sources where they lie (REF, default /root/reference).  Nothing here is
# copied into the repository; outputs go to oracle/_ref/ only.
#
#   oracle/_ref/libref_kernels.so  GSAP/kernels.hpp compiled for the host
#                                  through oracle/ref_shim (dS pin tests)
#   oracle/_ref/ref_host           GSAP/load.hpp + GSAP/evaluate (goldens)
#   oracle/_ref/gsap_ref           the unmodified GSAP GPU path (sm_100a)
#                                  driven by oracle/gsap_ref_main.cu
#   oracle/_ref/gsap_csr           GSAP's blockmodel builder (calculate_new_csr)
#                                  on given partitions, oracle/gsap_csr_main.cu
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${REF:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -d "$REF/GSAP" ]; then
  echo "reference tree not found at $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
# where the checkers came from, for the tests that read the reference's
# bundled graphs (tests/test_host.py); the file stays out of the repository
printf '%s\n' "$REF" > "$OUT/ref_root"
CXX="${CXX:-g++}"
NVCC="${NVCC:-nvcc}"

build_if_stale() {  # target, sources...
  local tgt="$1"; shift
  if [ -f "$tgt" ]; then
    local stale=0
    for s in "$@"; do [ "$s" -nt "$tgt" ] && stale=1; done
    [ $stale -eq 0 ] && return 1
  fi
  return 0
}

if build_if_stale "$OUT/libref_kernels.so" "$HERE/ref_kernels_harness.cpp" "$HERE/ref_shim/cuda_emul.h"; then
  "$CXX" -std=c++17 -O2 -fPIC -shared -w \
    -I"$HERE/ref_shim" -I"$REF/GSAP" \
    "$HERE/ref_kernels_harness.cpp" -o "$OUT/libref_kernels.so"
fi

if build_if_stale "$OUT/ref_host" "$HERE/ref_host_harness.cpp"; then
  "$CXX" -std=c++17 -O2 -w -I"$REF/GSAP" "$HERE/ref_host_harness.cpp" -o "$OUT/ref_host"
fi

if [ "${SKIP_GSAP_GPU:-0}" != "1" ] && command -v "$NVCC" >/dev/null 2>&1; then
  if build_if_stale "$OUT/gsap_ref" "$HERE/gsap_ref_main.cu"; then
    # the flags of the reference's CMakeLists.txt:22-27, for sm_100a
    "$NVCC" -std=c++17 -O3 -use_fast_math --expt-relaxed-constexpr --extended-lambda -w \
      -gencode arch=compute_100a,code=sm_100a \
      -I"$REF/GSAP" -I"$REF" "$HERE/gsap_ref_main.cu" -o "$OUT/gsap_ref"
  fi
fi
if [ "${SKIP_GSAP_GPU:-0}" != "1" ] && command -v "$NVCC" >/dev/null 2>&1; then
  if build_if_stale "$OUT/gsap_csr" "$HERE/gsap_csr_main.cu"; then
    "$NVCC" -std=c++17 -O3 -use_fast_math --expt-relaxed-constexpr --extended-lambda -w \
      -gencode arch=compute_100a,code=sm_100a \
      -I"$REF/GSAP" -I"$REF" "$HERE/gsap_csr_main.cu" -o "$OUT/gsap_csr"
  fi
fi
echo "oracle/_ref ready"
