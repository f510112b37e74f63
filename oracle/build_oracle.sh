#!/usr/bin/env bash
# Builds the oracle restatement (oracle/xnyz_oracle.cpp) into oracle/liboracle.so.
# Test infrastructure only.  Needs only g++; zstd is loaded at run time.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
"${XNYZ_CXX:-/usr/bin/g++}" -O2 -std=c++17 -fPIC -shared -Wall -Wno-sign-compare "$HERE/xnyz_oracle.cpp" -o "$HERE/liboracle.so" -ldl
echo "built $HERE/liboracle.so"
