#!/bin/sh
# Build the CPU oracle (test infrastructure) into oracle/liboracle.so.
# -ffp-contract=off keeps every product and sum rounded as written (reference FP32 semantics).
set -e
cd "$(dirname "$0")"
g++ -O2 -std=c++17 -ffp-contract=off -fopenmp -fPIC -shared -o liboracle.so.tmp oracle.cpp
mv liboracle.so.tmp liboracle.so
