#!/bin/sh
# Compile the main.cpp-style driver (or another program of this directory)
# against the drop-in headers and the in-tree library:
#   build.sh <output binary> [source, default driver.cpp]
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT=$(cd "$HERE/../.." && pwd)
SRC=${2:-driver.cpp}
g++ -std=c++17 -O2 -Wall -I"$ROOT/include" "$HERE/$SRC" -o "$1" \
    -L"$ROOT/hsolver_b200" -lhsolver_b200 -Wl,-rpath,"$ROOT/hsolver_b200" \
    -L/usr/local/cuda/lib64 -lcudart -Wl,-rpath,/usr/local/cuda/lib64
