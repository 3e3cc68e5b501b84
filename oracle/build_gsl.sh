#!/usr/bin/env bash
# Build GSL 2.1 from the tarball bundled in the reference tree
# (PIGFEM4.6.1/gsl-2.1.tar.gz) into oracle/_ref/gsl.  The reference links
# gsl + gslcblas (PIGFEM4.6.1/Makefile:32-36); the reference build in
# oracle/Makefile.ref needs both.  Outputs go only under oracle/_ref/.
#
# Usage: oracle/build_gsl.sh <PIGFEM4.6.1 directory>
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:?usage: build_gsl.sh <PIGFEM4.6.1 directory>}"
OUT="$HERE/_ref"
TARBALL="$REF/gsl-2.1.tar.gz"
if [ -f "$OUT/gsl/lib/libgsl.a" ]; then
  echo "gsl already built in $OUT/gsl"; exit 0
fi
[ -f "$TARBALL" ] || { echo "missing $TARBALL" >&2; exit 1; }
mkdir -p "$OUT/gsl-src"
tar -xzf "$TARBALL" -C "$OUT/gsl-src"
cd "$OUT/gsl-src/gsl-2.1"
./configure --prefix="$OUT/gsl" --disable-shared --with-pic CFLAGS="-O2 -fPIC" > "$OUT/gsl-configure.log" 2>&1
make -j"$(nproc)" > "$OUT/gsl-make.log" 2>&1
make install > "$OUT/gsl-install.log" 2>&1
echo "gsl built in $OUT/gsl"
