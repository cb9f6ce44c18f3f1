#!/usr/bin/env bash
# Build the reference's Cholesky drivers on the B200 runtime plugin, into
# oracle/_ref/libchamb200rt.so (test infrastructure).
#
# A Chameleon build chooses one runtime for the INSERT_TASK_* / RUNTIME_*
# interface its algorithms submit through.  This recipe compiles the
# reference's control code and its d-precision dposv / dpotrf / dpotrs drivers
# and algorithms (generated by oracle/build_ref.sh, whose generated tree it
# reuses) with chameleon_b200/runtime/runtime_b200.c as that runtime, plus the
# test driver oracle/plugin_harness.c, and links libchameleon_b200.so (the
# executor the plugin records into).  Kernels of other algorithms that the
# generic control code references get aborting stubs (never reached here).
set -euo pipefail

HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
ROOT="$(dirname "$HERE")"
REF="${CHAMREF_SRC:-/root/reference}"
OUT="$HERE/_ref"
GEN="$OUT/gen"
PLUG="$OUT/plugin"
CUDA="${CUDA_HOME:-/usr/local/cuda}"

[ -d "$REF/compute" ] || { echo "build_plugin.sh: reference sources not found at $REF" >&2; exit 2; }
[ -f "$GEN/generated.txt" ] || bash "$HERE/build_ref.sh"
[ -f "$ROOT/chameleon_b200/libchameleon_b200.so" ] || { echo "build_plugin.sh: build libchameleon_b200.so first" >&2; exit 2; }
OPENBLAS="$(awk '/libscipy_openblas/ {print; exit}' "$GEN/openblas.txt" 2>/dev/null || true)"
if [ -z "$OPENBLAS" ]; then
  OPENBLAS="$(python3 - <<'PY'
import glob, os, scipy
d = os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs")
c = sorted(glob.glob(os.path.join(d, "libscipy_openblas*.so")))
print(os.path.realpath(c[0]) if c else "")
PY
)"
fi

rm -rf "$PLUG"
mkdir -p "$PLUG/include/chameleon" "$PLUG/obj"
# the same configuration as the reference build, without the OpenMP runtime
sed -e 's/#define CHAMELEON_SCHED_OPENMP/#define CHAMELEON_SCHED_B200/' "$GEN/include/chameleon/config.h" \
  > "$PLUG/include/chameleon/config.h"

CFLAGS="-O2 -fPIC -std=gnu11 -w -DPRECISION_d -DNDEBUG -include $GEN/include/blasmap.h
  -I$PLUG/include -I$GEN/include -I$GEN -I$REF/include -I$REF -I$REF/coreblas/include -I$REF/control
  -I$CUDA/include"

OBJS=""
fail=0
compile() {
  local src="$1" obj="$PLUG/obj/$(echo "$1" | tr '/' '_').o"
  if gcc $CFLAGS -c "$src" -o "$obj" 2> "$obj.log"; then OBJS="$OBJS $obj"; else echo "FAILED: $src" >&2; head -20 "$obj.log" >&2; fail=1; fi
}
for f in control/async.c control/auxiliary.c control/context.c control/control.c control/descriptor.c \
         control/descriptor_helpers.c control/lamch.c control/tile.c control/workspace.c; do
  compile "$REF/$f"
done
for f in compute/dposv.c compute/dpotrf.c compute/dpotrs.c compute/pdpotrf.c compute/pdtrsm.c; do
  compile "$GEN/src/$f"
done
compile "$ROOT/chameleon_b200/runtime/runtime_b200.c"
compile "$HERE/plugin_harness.c"
[ "$fail" = 0 ] || { echo "build_plugin.sh: compile failures" >&2; exit 1; }

link() {
  gcc -shared -Wl,-Bsymbolic -o "$OUT/libchamb200rt.so" $OBJS "$@" \
      -L"$ROOT/chameleon_b200" -lchameleon_b200 -Wl,-rpath,'$ORIGIN/../../chameleon_b200' \
      -L"$CUDA/lib64" -lcudart -Wl,-rpath,"$CUDA/lib64" \
      "$OPENBLAS" -Wl,-rpath,"$(dirname "$OPENBLAS")" -lm
}
link
nm -D "$OUT/libchamb200rt.so" | awk '$1 == "U" && $2 !~ /@|^scipy_|^_|^cuda|^CHAM_B200_/ {print $2}' > "$PLUG/undef.txt"
{
  echo '#include <stdlib.h>'
  while read -r sym; do echo "void $sym(void) { abort(); }"; done < "$PLUG/undef.txt"
} > "$PLUG/stubs.c"
gcc -O2 -fPIC -c "$PLUG/stubs.c" -o "$PLUG/obj/stubs.o"
link "$PLUG/obj/stubs.o" -Wl,--no-undefined
echo "built $OUT/libchamb200rt.so ($(wc -l < "$PLUG/undef.txt") off-path stubs)"
