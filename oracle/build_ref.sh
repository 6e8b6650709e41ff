#!/usr/bin/env bash
# Builds the reference's own CPU implementation from its sources into
# oracle/_ref/ (git-ignored build output):
#   oracle/_ref/sc-nec-ncc.bin  the reference CLI, Makefile-nec recipe with g++
#   oracle/_ref/ref_oracle      oracle/ref_harness.cpp linked against the
#                               reference objects (full-precision dumps)
# The reference tree is read-only; sources are copied into oracle/_ref/src and
# the one harness-side fix is applied there: Graph::operator= has no
# `return *this;` (Graph.cpp:131-142), which GCC 13 turns into a trap.
# Usage: oracle/build_ref.sh [REFERENCE_DIR]
#   REFERENCE_DIR defaults to $SUBGRAPH_REFERENCE_DIR, else /root/reference.
#   Exit status 2: the reference sources are not there (nothing is built).
set -euo pipefail
REF="${1:-${SUBGRAPH_REFERENCE_DIR:-/root/reference}}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
SRC="$OUT/src"
if [ ! -f "$REF/CountMat.cpp" ]; then
    echo "build_ref.sh: reference sources not found at $REF" >&2
    exit 2
fi
mkdir -p "$SRC" "$OUT/obj"
for f in CountMat.cpp CountMat.hpp CSRGraph.cpp CSRGraph.hpp CSCGraph.hpp DataTableColMajor.cpp \
         DataTableColMajor.hpp DivideTemplates.cpp DivideTemplates.hpp EdgeList.cpp EdgeList.hpp \
         Graph.cpp Graph.hpp Helper.cpp Helper.hpp IndexSys.cpp IndexSys.hpp sc-main.cpp; do
    cp "$REF/$f" "$SRC/$f"
    chmod u+w "$SRC/$f"
done
# harness-side fix: add the missing return to Graph::operator=
python3 - "$SRC/Graph.cpp" <<'EOF'
import sys, re
p = sys.argv[1]
s = open(p).read()
pat = r"(std::memcpy\(deg_list, obj\.get_deg_list\(\), \(vert_num\+1\)\*sizeof\(unsigned\)\);\s*)\}"
s2, n = re.subn(pat, r"\1    return *this;\n}", s, count=1)
if n != 1:
    sys.exit("Graph.cpp patch point not found")
open(p, "w").write(s2)
EOF
CXX="${REF_CXX:-/usr/bin/g++}"
FLAGS="-std=c++11 -DNEC -fopenmp -O3 -I$SRC"
OBJS=""
for f in CountMat CSRGraph DataTableColMajor DivideTemplates EdgeList Graph Helper IndexSys sc-main; do
    "$CXX" -c -o "$OUT/obj/$f.o" "$SRC/$f.cpp" $FLAGS -w
    [ "$f" != "sc-main" ] && OBJS="$OBJS $OUT/obj/$f.o"
done
"$CXX" -o "$OUT/sc-nec-ncc.bin" $OBJS "$OUT/obj/sc-main.o" $FLAGS
"$CXX" -o "$OUT/ref_oracle" "$HERE/ref_harness.cpp" $OBJS $FLAGS -w
echo "built $OUT/sc-nec-ncc.bin and $OUT/ref_oracle"
