#!/usr/bin/env bash
# Stage the unmodified reference package under baseline/_ref/ so its own host
# code (binary_pursuit_parallel.binary_pursuit) can be imported in this
# container.  `pip install` of the reference fails here: its setup.py calls
# pkg_resources.require('pyopencl>=2019.1.2') at metadata time and pyopencl is
# not installable offline.  So the package tree is copied to /tmp, its one
# Cython extension (c_cython/sort_cython.pyx) is built there, and the result is
# copied to baseline/_ref/.  Nothing in the reference checkout is written.
set -euo pipefail
HERE=$(cd "$(dirname "$0")/.." && pwd)
# the reference checkout: $REF, else $FBP_REFERENCE_TREE, else `reference` beside this repository
REF=${REF:-${FBP_REFERENCE_TREE:-$HERE/../reference}}
DEST="$HERE/baseline/_ref"
[ -d "$REF/spikesorting_fullpursuit" ] || { echo "reference not found at $REF" >&2; exit 1; }
TMP=$(mktemp -d /tmp/sfp_ref.XXXXXX)
cp -r "$REF/spikesorting_fullpursuit" "$TMP/"
NPINC=$(python -c 'import numpy; print(numpy.get_include())')
( cd "$TMP/spikesorting_fullpursuit/c_cython" && \
  CFLAGS="-I$NPINC -O2" python -m cython -3 sort_cython.pyx -o sort_cython_build.c >/dev/null && \
  gcc -shared -fPIC -O2 -I"$NPINC" $(python -c 'import sysconfig;print("-I"+sysconfig.get_paths()["include"])') \
      sort_cython_build.c -o "sort_cython$(python -c 'import sysconfig;print(sysconfig.get_config_var("EXT_SUFFIX"))')" )
mkdir -p "$DEST"
rm -rf "$DEST/spikesorting_fullpursuit"
cp -r "$TMP/spikesorting_fullpursuit" "$DEST/"
rm -rf "$TMP"
echo "staged reference package at $DEST/spikesorting_fullpursuit"
