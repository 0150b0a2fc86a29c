#!/usr/bin/env bash
# Compiles the reference's own index helpers (quax/integrals/utils.h, read in
# place from the reference tree) with oracle/ref_utils_shim.cpp into
# oracle/_ref/libquax_ref_utils.so.  Test infrastructure only.
# Usage: build_ref.sh [REFERENCE_ROOT]
#   REFERENCE_ROOT: the argument, else $QUAX_REFERENCE, else the checkout this
#   oracle was pinned against (/root/reference); without one, nothing is built.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${QUAX_REFERENCE:-/root/reference}}"
HDR="$REF/quax/integrals/utils.h"
if [ ! -f "$HDR" ]; then
  echo "reference header $HDR not found; nothing built" >&2
  exit 0
fi
mkdir -p "$HERE/_ref"
/usr/bin/g++ -O2 -std=c++17 -fPIC -shared -DREF_UTILS_H="\"$HDR\"" \
  "$HERE/ref_utils_shim.cpp" -o "$HERE/_ref/libquax_ref_utils.so"
echo "built $HERE/_ref/libquax_ref_utils.so"
