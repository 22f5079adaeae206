#!/usr/bin/env bash
# Builds the CPU oracle: the unmodified reference sources + oracle/ref_harness.cpp,
# one binary per lattice size and level count (the reference fixes both at compile
# time, include/config.h.in:3-5).  TEST INFRASTRUCTURE ONLY.
#
#   oracle/build_ref.sh NS NT LEVELS [REFDIR]
#
# Reads the sources where they lie (REFDIR; default $AMG_REFERENCE_DIR, else a directory
# named `reference` beside the repository root); writes only under
# oracle/_ref/.  The reference's include/config.h is bypassed by force-including a
# generated header that defines its include guard (CONFIG_H) first.
set -euo pipefail
NS=${1:?NS}; NT=${2:?NT}; LEVELS=${3:?LEVELS}
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${4:-${AMG_REFERENCE_DIR:-$(cd "$HERE/../.." && pwd)/reference}}
OUT="$HERE/_ref"
TAG="${NS}x${NT}_l${LEVELS}"
OBJ="$OUT/obj_$TAG"
mkdir -p "$OBJ"
CFG="$OBJ/oracle_config.h"
printf '#ifndef CONFIG_H\n#define CONFIG_H\n#define NS %s\n#define NT %s\n#define LEVELS %s\n#endif\n' "$NS" "$NT" "$LEVELS" > "$CFG"
CXX=${CXX:-g++}
FLAGS=(-std=c++20 -O3 -include "$CFG" -I "$HERE/mpi_shim" -I "$REF/include" -w)
SRCS=(variables gauge_conf dirac_operator bi_cgstab conjugate_gradient sap amg level fgmres tests)
pids=()
for s in "${SRCS[@]}"; do
  "$CXX" "${FLAGS[@]}" -c "$REF/src/$s.cpp" -o "$OBJ/$s.o" & pids+=($!)
done
"$CXX" "${FLAGS[@]}" -c "$HERE/ref_harness.cpp" -o "$OBJ/ref_harness.o" & pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done
"$CXX" -o "$OUT/ref_$TAG" "$OBJ"/*.o
echo "$OUT/ref_$TAG"
