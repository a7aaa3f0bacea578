#!/bin/sh
# TEST INFRASTRUCTURE ONLY.  Compiles the reference's own GPU path for sm_100a from its
# sources where they lie (read-only) plus oracle/ref_harness.cu into
# oracle/_ref/libtgmm_ref.so.  Nothing is copied from the reference tree.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
# the reference project's src/ tree: TGMM_REFERENCE_SRC, else a checkout named "reference"
# beside this repository
REF=${TGMM_REFERENCE_SRC:-$HERE/../../reference/nmeth.3036-S2/src}
OUT="$HERE/_ref"
if [ ! -d "$REF/UtilsCUDA" ]; then
  echo "reference sources not found at $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
FLAGS="-std=c++17 -O2 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC -w"
$NVCC $FLAGS -c "$REF/UtilsCUDA/GMEMupdateCUDA.cu" -o "$OUT/GMEMupdateCUDA.o"
$NVCC $FLAGS -c "$REF/UtilsCUDA/knnCuda.cu" -o "$OUT/knnCuda.o"
g++ -O2 -fPIC -c "$REF/constants.cpp" -o "$OUT/constants.o"
$NVCC $FLAGS -I"$REF/UtilsCUDA" -I"$REF" -c "$HERE/ref_harness.cu" -o "$OUT/ref_harness.o"
$NVCC -gencode arch=compute_100a,code=sm_100a -shared -o "$OUT/libtgmm_ref.so" \
  "$OUT/GMEMupdateCUDA.o" "$OUT/knnCuda.o" "$OUT/constants.o" "$OUT/ref_harness.o" -lcusparse -lcuda
# the tracking graph's supervoxel kNN, in a library of its own (its symbols are distinct)
F3="$REF/temporalLogicalRules/knnCUDA"
$NVCC $FLAGS -c "$F3/knnCuda.cu" -o "$OUT/f3_knnCuda.o"
$NVCC $FLAGS -I"$F3" -c "$HERE/ref_f3_harness.cu" -o "$OUT/ref_f3_harness.o"
$NVCC -gencode arch=compute_100a,code=sm_100a -shared -o "$OUT/libtgmm_ref_f3.so" \
  "$OUT/f3_knnCuda.o" "$OUT/ref_f3_harness.o" -lcuda
# the frame preparation's supervoxel trimming and statistics (host C++ only: runs without a GPU)
TLR="$REF/temporalLogicalRules"
HSD="$REF/nucleiChSvWshedPBC"
CXXF="-std=c++14 -O2 -fPIC -w -I$REF -I$TLR -I$HSD"
g++ $CXXF -c "$TLR/supervoxel.cpp" -o "$OUT/f1_supervoxel.o"
g++ $CXXF -c "$TLR/localGeometricDescriptor.cpp" -o "$OUT/f1_lgd.o"
g++ $CXXF -c "$HSD/hierarchicalSegmentation.cpp" -o "$OUT/f1_hs.o"
g++ $CXXF -c "$HERE/ref_f1_harness.cpp" -o "$OUT/ref_f1_harness.o"
g++ -shared -Wl,--no-undefined -o "$OUT/libtgmm_ref_f1.so" "$OUT/f1_supervoxel.o" "$OUT/f1_lgd.o" "$OUT/f1_hs.o" \
  "$OUT/constants.o" "$OUT/ref_f1_harness.o"
# the split proposal of the Gaussian class (host C++ with the vendored Eigen; runs without a GPU)
g++ -std=gnu++11 $CXXF -c "$REF/GaussianMixtureModel.cpp" -o "$OUT/gmm_class.o"
g++ -std=gnu++11 $CXXF -c "$REF/external/xmlParser2/xmlParser.cpp" -o "$OUT/gmm_xml.o"
g++ -std=gnu++11 $CXXF -c "$HERE/ref_split_harness.cpp" -o "$OUT/ref_split_harness.o"
g++ -shared -Wl,--no-undefined -o "$OUT/libtgmm_ref_gmm.so" "$OUT/gmm_class.o" "$OUT/gmm_xml.o" "$OUT/constants.o" \
  "$OUT/ref_split_harness.o"
rm -f "$OUT"/*.o
echo "built $OUT/libtgmm_ref.so $OUT/libtgmm_ref_f3.so $OUT/libtgmm_ref_f1.so $OUT/libtgmm_ref_gmm.so"
