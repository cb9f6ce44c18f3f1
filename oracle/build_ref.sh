#!/usr/bin/env bash
# Build the reference's own CPU path (Chameleon d-precision dposv / dpotrf /
# dpotrs / dpotrf_batch / dtrsm_batch through the OpenMP runtime and coreblas)
# from its sources, into oracle/_ref/libchamref.so.
#
# Test infrastructure only: the parity tests use this library as the checker
# and bench.py's reference arm times it.  The reference's CMake build cannot run
# as shipped (its precision generator and find-modules live in an empty
# submodule), so this recipe:
#   1. writes a config.h for the OpenMP runtime, d precision, no MPI/CUDA;
#   2. stubs libhqr.h (empty submodule, only a type name is used);
#   3. generates d-precision files from the z sources with oracle/z2d.py;
#   4. maps cblas_* / LAPACKE_* onto the scipy-bundled OpenBLAS exports
#      (scipy_cblas_* / scipy_LAPACKE_*) with a forced-include header;
#   5. compiles everything with gcc -fopenmp -DPRECISION_d and links it.
# Generated sources and all outputs stay under oracle/_ref/.
set -euo pipefail

HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${CHAMREF_SRC:-/root/reference}"
OUT="$HERE/_ref"
GEN="$OUT/gen"
PY="${PYTHON:-python3}"

if [ ! -d "$REF/compute" ]; then
  echo "build_ref.sh: reference sources not found at $REF" >&2
  exit 2
fi

OPENBLAS="${CHAMREF_OPENBLAS:-$($PY - <<'EOF'
import glob, os, scipy
d = os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs")
c = sorted(glob.glob(os.path.join(d, "libscipy_openblas*.so")))
print(os.path.realpath(c[0]) if c else "")
EOF
)}"
if [ -z "$OPENBLAS" ] || [ ! -f "$OPENBLAS" ]; then
  echo "build_ref.sh: no scipy OpenBLAS found" >&2
  exit 2
fi

rm -rf "$GEN"
mkdir -p "$GEN/include/chameleon" "$GEN/include/coreblas" "$GEN/control" "$GEN/obj"

# 1. config.h
cat > "$GEN/include/chameleon/config.h" <<'EOF'
#ifndef CHAMELEON_CONFIG_H_HAS_BEEN_INCLUDED
#define CHAMELEON_CONFIG_H_HAS_BEEN_INCLUDED
#define CHAMELEON_VERSION_MAJOR 1
#define CHAMELEON_VERSION_MINOR 4
#define CHAMELEON_VERSION_MICRO 0
#define CHAMELEON_SCHED_OPENMP
#define CHAMELEON_PREC_D
#define CHAMELEON_BATCH_SIZE 256
#define chameleon_attr_fallthrough __attribute__((fallthrough))
#ifdef BEGIN_C_DECLS
#undef BEGIN_C_DECLS
#endif
#ifdef END_C_DECLS
#undef END_C_DECLS
#endif
#if defined(c_plusplus) || defined(__cplusplus)
#define BEGIN_C_DECLS extern "C" {
#define END_C_DECLS }
#else
#define BEGIN_C_DECLS
#define END_C_DECLS
#endif
#define __chameleon_func__ __func__
#endif
EOF

# 2. libhqr stub
echo 'typedef struct { int dummy; } libhqr_tree_t;' > "$GEN/include/libhqr.h"

# 3a. empty headers for precisions that are not generated
for h in chameleon/chameleon_s.h chameleon/chameleon_c.h chameleon/chameleon_ds.h \
         chameleon/tasks_s.h chameleon/tasks_c.h chameleon/tasks_ds.h \
         coreblas/coreblas_s.h coreblas/coreblas_c.h coreblas/coreblas_ds.h \
         coreblas/coreblas_stile.h coreblas/coreblas_ctile.h coreblas/coreblas_dstile.h ; do
  : > "$GEN/include/$h"
done
for h in compute_s.h compute_c.h compute_ds.h ; do : > "$GEN/control/$h"; done

# 3b. generated d headers
$PY "$HERE/z2d.py" "$REF" "$GEN/hdr" \
  include/chameleon/chameleon_z.h include/chameleon/tasks_z.h \
  coreblas/include/coreblas/coreblas_z.h coreblas/include/coreblas/coreblas_ztile.h \
  control/compute_z.h > /dev/null
cp "$GEN/hdr/include/chameleon/chameleon_d.h" "$GEN/include/chameleon/"
cp "$GEN/hdr/include/chameleon/tasks_d.h" "$GEN/include/chameleon/"
cp "$GEN/hdr/coreblas/include/coreblas/coreblas_d.h" "$GEN/include/coreblas/"
cp "$GEN/hdr/coreblas/include/coreblas/coreblas_dtile.h" "$GEN/include/coreblas/"
cp "$GEN/hdr/control/compute_d.h" "$GEN/control/"

# 3c. generated d sources (the dposv path, its generators, norms used by the
# checks, batch drivers)
CORE_Z="core_zgemm core_zsyrk core_ztrsm core_zpotrf core_zplgsy core_zplrnt
        core_zlacpy core_zlaset core_zlansy core_zlange core_zgessq core_zsyssq core_zplssq
        core_zlascal core_zgeadd core_zsymm core_ztile core_zlatro core_ztradd core_ztrmm
        core_zlauum core_ztrtri"
COMPUTE_Z="zposv zpotrf zpotrs pzpotrf pztrsm zplgsy pzplgsy zplrnt pzplrnt pzlacpy zlacpy
           zlansy pzlansy zlange pzlange zlaset pzlaset zpotrf_batch ztrsm_batch ztile
           zpotri ztrtri zlauum pztrtri pzlauum zgemm_batch zherk_batch
           zpotrimm pzpotrimm"
CODELET_Z="codelet_zgemm codelet_zsyrk codelet_ztrsm codelet_zpotrf codelet_zplgsy
           codelet_zplrnt codelet_zlacpy codelet_zlaset codelet_zlansy codelet_zlange
           codelet_zgessq codelet_zsyssq codelet_zplssq codelet_zlascal codelet_zgeadd
           codelet_zsymm codelet_zlatro codelet_ztradd codelet_ztrmm codelet_zlauum codelet_ztrtri"
FILES=""
for f in $CORE_Z; do FILES="$FILES coreblas/compute/$f.c"; done
for f in $COMPUTE_Z; do [ -f "$REF/compute/$f.c" ] && FILES="$FILES compute/$f.c"; done
for f in $CODELET_Z; do [ -f "$REF/runtime/openmp/codelets/$f.c" ] && FILES="$FILES runtime/openmp/codelets/$f.c"; done
FILES="$FILES control/workspace_z.c runtime/openmp/control/runtime_zlocality.c runtime/openmp/control/runtime_zprofiling.c"
$PY "$HERE/z2d.py" "$REF" "$GEN/src" $FILES > "$GEN/generated.txt"

# precision-generic sources compiled as they are
GENERIC="control/async.c control/auxiliary.c control/context.c control/control.c
         control/descriptor.c control/descriptor_helpers.c control/lamch.c control/tile.c
         control/workspace.c control/descriptor_ipiv.c
         runtime/openmp/control/runtime_async.c runtime/openmp/control/runtime_context.c
         runtime/openmp/control/runtime_control.c runtime/openmp/control/runtime_descriptor.c
         runtime/openmp/control/runtime_options.c runtime/openmp/control/runtime_profiling.c
         runtime/openmp/codelets/codelet_map.c compute/pmap.c compute/map.c
         coreblas/compute/global.c"

# 4. BLAS / LAPACKE name map onto the OpenBLAS exports
nm -D --defined-only "$OPENBLAS" | awk '$3 ~ /^scipy_(cblas|LAPACKE)_/ {n=$3; sub(/^scipy_/, "", n); print "#define " n " " $3}' > "$GEN/include/blasmap.h"

CFLAGS="-O2 -fPIC -fopenmp -std=gnu11 -w -DPRECISION_d -DNDEBUG -include $GEN/include/blasmap.h
  -I$GEN/include -I$GEN -I$REF/include -I$REF -I$REF/coreblas/include -I$REF/runtime/openmp/include
  -I$REF/runtime/openmp -I$REF/control"

OBJS=""
fail=0
compile() {
  local src="$1" obj="$GEN/obj/$(echo "$1" | tr '/' '_' ).o"
  if gcc $CFLAGS -c "$src" -o "$obj" 2> "$obj.log"; then OBJS="$OBJS $obj"; else echo "FAILED: $src" >&2; cat "$obj.log" | head -20 >&2; fail=1; fi
}
for f in $(cat "$GEN/generated.txt"); do compile "$f"; done
for f in $GENERIC; do compile "$REF/$f"; done
compile "$HERE/ref_driver.c"
[ "$fail" = 0 ] || { echo "build_ref.sh: compile failures" >&2; exit 1; }

# complex-only helpers referenced from the generated tile wrappers but never
# called on the real-double path
cat > "$GEN/stubs.c" <<'EOF'
#include <stdlib.h>
int scipy_LAPACKE_dlacgv_work(int n, double *x, int incx) { (void)n; (void)x; (void)incx; abort(); return 0; }
EOF
gcc -O2 -fPIC -c "$GEN/stubs.c" -o "$GEN/obj/stubs.o"

OBLAS_DIR="$(dirname "$OPENBLAS")"
link() {
  gcc -shared -fopenmp -o "$OUT/libchamref.so" $OBJS "$GEN/obj/stubs.o" "$@" \
      "$OPENBLAS" -Wl,-rpath,"$OBLAS_DIR" -lm
}
link
# The generic tile wrappers (core_dtile.c, workspace, descriptor code) reference
# kernels of other algorithms (QR, LU, ...) that are not on this path and are not
# built.  Give each such symbol an aborting stub so that the library loads with
# immediate binding; none of them is reached by dposv/dpotrf/dpotrs/batch.
nm -D "$OUT/libchamref.so" | awk '$1 == "U" && $2 !~ /@|^scipy_|^omp_|^GOMP_|^_/ {print $2}' > "$GEN/undef.txt"
{
  echo '#include <stdlib.h>'
  while read -r sym; do echo "void $sym(void) { abort(); }"; done < "$GEN/undef.txt"
} > "$GEN/stubs_off_path.c"
gcc -O2 -fPIC -c "$GEN/stubs_off_path.c" -o "$GEN/obj/stubs_off_path.o"
link "$GEN/obj/stubs_off_path.o" -Wl,--no-undefined
echo "built $OUT/libchamref.so ($(wc -l < "$GEN/undef.txt") off-path stubs)"
