#!/bin/bash
# Writes a B200 variant <name>_b200.conf of every KD-SLAM .conf in a directory that
# names a CUDA or CPU aligner type, by renaming the aligner and tree-generator types
# to the B200 ones (same parameters, same values).  The directory defaults to the
# one this script sits in.
#   ICPCUDA3D / ICPCPU3D      -> ICPB2003D
#   CTICPCUDA3D / CTICPCPU3D  -> CTICPB2003D
#   TreeGenerator3D           -> TreeGeneratorB2003D
set -euo pipefail

DIR=${1:-$(dirname "$0")}

for src in "$DIR"/*.conf; do
  [[ -e "$src" ]] || continue
  [[ "$src" == *_b200.conf ]] && continue
  [[ "$(basename "$src")" == dl.conf ]] && continue
  grep -qE '"(CT)?ICP(CUDA|CPU)3D"' "$src" || continue
  dst="${src%.conf}_b200.conf"
  sed -E \
    -e 's/"CTICP(CUDA|CPU)3D"/"CTICPB2003D"/g' \
    -e 's/"ICP(CUDA|CPU)3D"/"ICPB2003D"/g' \
    -e 's/"TreeGenerator3D"/"TreeGeneratorB2003D"/g' \
    "$src" > "$dst"
  echo "$(basename "$dst")"
done
