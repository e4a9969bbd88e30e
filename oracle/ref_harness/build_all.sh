#!/bin/bash
# Builds the reference-side test binaries into oracle/_ref/ (test infrastructure): the module
# harness (Makefile) and the two MD driver builds (build_sponge.sh: stock modules and drop-ins).
# Does nothing when the reference tree is not present (the GPU box uses the binaries built here).
# The driver builds are redone only when a binary is missing or older than the drop-in sources.
# usage: oracle/ref_harness/build_all.sh
set -e
REF=${REF:-/root/reference/SPONGE}
HERE=$(cd "$(dirname "$0")" && pwd)
REPO=$(cd "$HERE/../.." && pwd)
if [ ! -d "$REF" ]; then
    echo "reference tree not present: oracle/_ref left as it is"
    exit 0
fi
make -s -C "$HERE" REF="$REF"
OUT=$REPO/oracle/_ref
stale=0
for b in "$OUT/sponge_stock" "$OUT/sponge_b200"; do
    if [ ! -x "$b" ]; then stale=1; fi
done
if [ $stale -eq 0 ] && [ -n "$(find "$REPO/sponge_b200/dropin" "$REPO/include" -newer "$OUT/sponge_b200" -type f)" ]; then
    stale=1
fi
if [ $stale -eq 1 ]; then
    REF="$REF" bash "$HERE/build_sponge.sh" both
fi
