#!/usr/bin/env bash
# Build the test oracle and, when the reference tree is present, the reference
# programs used to pin it.  Test infrastructure only; outputs:
#   oracle/liboracle.so        FP64 restatement (rte_oracle.cpp)
#   oracle/_ref/rte_cpu        CPU package built from its own sources (link order fixed)
#   oracle/_ref/fim_host       FisherInfo_IO forward path compiled as host C++ (fim_emu.h)
#   oracle/_ref/fim_fisher     the same with the Fisher main (rte_fim.cu) as its "program"
#   oracle/_ref/fim_snr        the same with the SNR main (rte_snr.cu) as its "program"
#   oracle/_ref/fim_grad       the same with the region-gradient main (compute_grad_rte.cu)
#   oracle/_ref/fim_shim       the forward main (rte.cu) as a program of its own, with the library's
#                              Neumann() shim (doi_b200/shim/neumann_b200.cu) in place of neumann.cu:
#                              the reference's host code around librte_b200 (needs doi_b200/lib built)
# The reference sources are compiled where they lie; nothing is copied into the repo.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
# the reference tree: $RTE_REFERENCE_DIR, else a "reference" directory beside the repository
REF="${RTE_REFERENCE_DIR:-$(cd "$HERE/../.." && pwd)/reference}"
CXX="${RTE_CXX:-g++}"
CC="${RTE_CC:-gcc}"

"$CXX" -O2 -std=c++17 -fopenmp -fPIC -shared -o "$HERE/liboracle.so" "$HERE/rte_oracle.cpp"

if [ ! -d "$REF" ]; then
  echo "oracle/build.sh: reference tree not present; built liboracle.so only"
  exit 0
fi

OUT="$HERE/_ref"
mkdir -p "$OUT/cpu" "$OUT/fim" "$OUT/main"

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
# the mains, each with main renamed to fim_prog_main (fim_host's "program" command runs it)
for f in rte rte_fim rte_snr compute_grad_rte; do
  "$CXX" "${FLAGS[@]}" -Dmain=fim_prog_main -c "$FIM/$f.cu" -o "$OUT/main/$f.o"
done
rm -f "$OUT/fim/rte.o"
sed -n '1,418p' "$FIM/kernels.cu" | "$CXX" "${FLAGS[@]}" -c - -o "$OUT/fim/kernels.o"
"$CXX" -O2 -std=c++17 -fopenmp -w -D__CUDACC__ -include "$HERE/ref/fim_emu.h" -I "$HERE/ref/include" -I "$FIM" \
  -c "$HERE/ref/fim_host.cpp" -o "$OUT/fim/fim_host.o"
"$CXX" -fopenmp -o "$OUT/fim_host" "$OUT"/fim/*.o "$OUT/main/rte.o" -lpthread -lm
"$CXX" -fopenmp -o "$OUT/fim_fisher" "$OUT"/fim/*.o "$OUT/main/rte_fim.o" -lpthread -lm
"$CXX" -fopenmp -o "$OUT/fim_snr" "$OUT"/fim/*.o "$OUT/main/rte_snr.o" -lpthread -lm
"$CXX" -fopenmp -o "$OUT/fim_grad" "$OUT"/fim/*.o "$OUT/main/compute_grad_rte.o" -lpthread -lm
built="liboracle.so, _ref/rte_cpu, _ref/fim_host, _ref/fim_fisher, _ref/fim_snr, _ref/fim_grad"
LIB="$HERE/../doi_b200/lib"
if [ -f "$LIB/librte_b200.so" ]; then
  mkdir -p "$OUT/shim"
  "$CXX" "${FLAGS[@]}" -I "$HERE/../include" -c "$HERE/../doi_b200/shim/neumann_b200.cu" -o "$OUT/shim/neumann_b200.o"
  "$CXX" "${FLAGS[@]}" -c "$FIM/rte.cu" -o "$OUT/shim/rte_main.o"
  "$CXX" -O2 -std=c++17 -w -D__CUDACC__ -include "$HERE/ref/fim_emu.h" -I "$HERE/ref/include" -I "$FIM" \
    -c "$HERE/ref/fim_shim_support.cpp" -o "$OUT/shim/support.o"
  "$CXX" -fopenmp -o "$OUT/fim_shim" "$OUT/shim/rte_main.o" "$OUT/shim/neumann_b200.o" "$OUT/shim/support.o" \
    "$OUT"/fim/{dist,sph_harm,inits,iniparser,dictionary,kernels}.o -L "$LIB" -lrte_b200 \
    -Wl,-rpath,'$ORIGIN/../../doi_b200/lib' -lpthread -lm
  built="$built, _ref/fim_shim"
fi
echo "oracle/build.sh: built $built"
