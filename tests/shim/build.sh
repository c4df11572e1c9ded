#!/bin/sh
# Builds the C driver against the library's header and shared object:
#   sh tests/shim/build.sh <output binary>
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT=$(cd "$HERE/../.." && pwd)
cc -O2 -std=c11 -Wall -I "$ROOT/include" -o "$1" "$HERE/gx_shim_driver.c" \
   -L "$ROOT/galaxy_b200" -lgalaxy_gpu -Wl,-rpath,"$ROOT/galaxy_b200"
