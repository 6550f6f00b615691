#!/bin/sh
# Builds the CPU restatement (oracle/dgsem_oracle.cpp) into oracle/liboracle.so.
# Test infrastructure only: the parity checker and the timed CPU baseline.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
g++ -O3 -march=native -fopenmp -ffp-contract=off -std=c++17 -shared -fPIC \
    "$HERE/dgsem_oracle.cpp" -o "$HERE/liboracle.so"
# the same source with fused multiply-adds: the spread between the two builds
# is the rounding floor of a state, which the parity tests measure
g++ -O3 -march=native -fopenmp -ffp-contract=fast -std=c++17 -shared -fPIC \
    "$HERE/dgsem_oracle.cpp" -o "$HERE/liboracle_fma.so"
echo "built $HERE/liboracle.so $HERE/liboracle_fma.so"
