#!/bin/sh
# Builds the CPU harness of the serving loop (test infrastructure only).
set -e
cd "$(dirname "$0")"
${LUTHE_CXX:-/usr/bin/g++} -std=c++17 -O1 -g -Wno-subobject-linkage ${HARNESS_FLAGS} -shared -fPIC -x c++ -I fake_cuda -I ../../include \
    -o libserve_harness.so harness.cpp
