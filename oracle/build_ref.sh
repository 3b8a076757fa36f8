#!/bin/sh
# Builds the reference stereo library (ethan-li-coding/FasterStereoCuda) from its own sources
# for sm_100a, plus the dump harness oracle/ref_harness.cpp, into oracle/_ref/.
# TEST INFRASTRUCTURE ONLY: the result is used to pin the oracle and to time the reference;
# the product library never links it. Needs the reference sources (REF_ROOT, default
# /root/reference); nothing is written outside oracle/_ref/.
#
# The sources are Windows/MSVC code; compiling them with nvcc/g++ needs forced <cstdint>,
# <cstring>, <cmath> includes, an empty __declspec and a two-line corecrt_io.h stand-in.
set -e
R=${REF_ROOT:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
CUDA=${CUDA_HOME:-/usr/local/cuda}
if [ ! -d "$R/SgmStereoCuda" ]; then
  echo "reference sources not found at $R" >&2
  exit 1
fi
mkdir -p "$OUT/obj" "$OUT/shim"
printf '#include <unistd.h>\n#define _access access\n' > "$OUT/shim/corecrt_io.h"
ARCH="-gencode arch=compute_100a,code=sm_100a"
INC="-I$R/SgmStereoCuda -I$R/common -I$R/common/trial -I$R/FasterStereoCuda -I$OUT/shim -I$CUDA/include"
for f in cusgm_cc cusgm_ca cusgm_df cusgm_util; do
  nvcc -std=c++17 -O3 $ARCH -Xcompiler -fPIC -include cstdint -w -I$R/SgmStereoCuda -I$R/common \
       -c "$R/SgmStereoCuda/$f.cu" -o "$OUT/obj/$f.o" &
done
wait
for f in StereoCuda StereoCudaImpl; do
  g++ -std=c++17 -O2 -fPIC -w -include cstdint -include cstring $INC -c "$R/SgmStereoCuda/$f.cpp" -o "$OUT/obj/$f.o"
done
g++ -std=c++17 -O2 -fPIC -w -include cstdint -include cstring -include cmath "-D__declspec(x)=" \
    -DFASTERSTEREOCUDA_EXPORTS $INC -c "$R/FasterStereoCuda/FasterStereoCuda.cpp" -o "$OUT/obj/FasterStereoCuda.o"
g++ -std=c++17 -O2 -fPIC -w -include cstdint -include cstring -include cmath "-D__declspec(x)=" \
    -DFASTERSTEREOCUDA_EXPORTS -Dprivate=public $INC -c "$HERE/ref_harness.cpp" -o "$OUT/obj/ref_harness.o"
g++ -shared -o "$OUT/libsgmref.so" "$OUT"/obj/*.o -L"$CUDA/lib64" -lcudart -lpthread
rm -rf "$OUT/obj"
echo "$OUT/libsgmref.so"
