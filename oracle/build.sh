#!/usr/bin/env bash
# Build the test oracle and, when the reference tree is present, the reference
# programs used to pin it.  Test infrastructure only; outputs:
#   oracle/liboracle.so        FP64 restatement (rte_oracle.cpp)
#   oracle/_ref/rte_cpu        CPU package built from its own sources (link order fixed)
#   oracle/_ref/fim_host       FisherInfo_IO forward path compiled as host C++ (fim_emu.h)
# The reference sources are compiled where they lie; nothing is copied into the repo.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${RTE_REFERENCE_DIR:-/root/reference}"
CXX="${RTE_CXX:-g++}"
CC="${RTE_CC:-gcc}"

"$CXX" -O2 -std=c++17 -fopenmp -fPIC -shared -o "$HERE/liboracle.so" "$HERE/rte_oracle.cpp"

if [ ! -d "$REF" ]; then
  echo "oracle/build.sh: reference tree not present; built liboracle.so only"
  exit 0
fi

OUT="$HERE/_ref"
mkdir -p "$OUT/cpu" "$OUT/fim"

# CPU package: its Makefile puts -lm before the objects, which modern ld rejects; build the
# same objects with the same flags and link with the libraries last.
CPU="$REF/CPU package/src"
for f in RTE_uniform Inits SphHarm Dist Kernels_selfsub iniparser dictionary; do
  "$CC" -O2 -fopenmp -m64 -w -c "$CPU/$f.c" -o "$OUT/cpu/$f.o"
done
"$CC" -O2 -fopenmp -m64 -o "$OUT/rte_cpu" "$OUT"/cpu/*.o -lpthread -lm

# FisherInfo_IO: host files as they are; kernels.cu only up to the end of the kernels
# (line 418), which leaves out the host launch wrapper prop_abs (re-enacted in fim_host.cpp).
FIM="$REF/FisherInfo_IO/src"
FLAGS=(-O2 -std=c++17 -fopenmp -w -x c++ -D__CUDACC__ -include "$HERE/ref/fim_emu.h"
       -I "$HERE/ref/include" -I "$FIM")
for f in dist sph_harm inits neumann iniparser dictionary; do
  "$CXX" "${FLAGS[@]}" -c "$FIM/$f.cu" -o "$OUT/fim/$f.o"
done
"$CXX" "${FLAGS[@]}" -Dmain=fim_rte_main -c "$FIM/rte.cu" -o "$OUT/fim/rte.o"
sed -n '1,418p' "$FIM/kernels.cu" | "$CXX" "${FLAGS[@]}" -c - -o "$OUT/fim/kernels.o"
"$CXX" -O2 -std=c++17 -fopenmp -w -D__CUDACC__ -include "$HERE/ref/fim_emu.h" -I "$HERE/ref/include" -I "$FIM" \
  -c "$HERE/ref/fim_host.cpp" -o "$OUT/fim/fim_host.o"
"$CXX" -fopenmp -o "$OUT/fim_host" "$OUT"/fim/*.o -lpthread -lm
echo "oracle/build.sh: built liboracle.so, _ref/rte_cpu, _ref/fim_host"
