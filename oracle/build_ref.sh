#!/bin/sh
# Build the reference's own CPU MTGP32 generator (mtgp32-fast.c and the
# mtgp32dc-param-11213.c table, straight from the Esthera tree) plus the
# ref_mtgp_shim.c C-ABI wrapper into oracle/_ref/libmtgp_ref.so.
# Needs the reference tree ($ESTHERA_REF, else ../reference beside the
# repository); outputs only into oracle/_ref/.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
# the Esthera tree: $ESTHERA_REF, else a checkout named "reference" beside the repository
REF=${ESTHERA_REF:-$HERE/../../reference}
SRC="$REF/src/partfilt/cuda/mtgp"
[ -f "$SRC/mtgp32-fast.c" ] || { echo "reference tree not found at $REF" >&2; exit 1; }
mkdir -p "$HERE/_ref"
${CC_REF:-$( [ -x /usr/bin/gcc ] && echo /usr/bin/gcc || echo gcc)} -O2 -fPIC -shared -std=gnu99 -I"$SRC" \
    "$SRC/mtgp32-fast.c" "$SRC/mtgp32dc-param-11213.c" "$HERE/ref_mtgp_shim.c" \
    -o "$HERE/_ref/libmtgp_ref.so"
echo "built $HERE/_ref/libmtgp_ref.so"
