#!/usr/bin/env bash
# Builds the reference's own CPU reconstruction (TreeGather, reference
# src/reconstruction_lib) as a Linux shared library, oracle/_ref/libtlfr_ref.so,
# for parity checks and the CPU baseline.  Test infrastructure only.
#
# The reference sources are compiled where they lie under the reference tree
# (REF; by default the directory 'reference' beside the repository); nothing is
# copied into the repository.  Five
# headers need small portability edits for g++; the edited copies are generated
# into oracle/_ref/gen/ (git-ignored) by the sed lines below:
#   base/Array.hpp    explicit specialisations lack 'template<>' (Array.hpp:697-717)
#   base/Hash.hpp     Set<T>::findSlot uses hash<T> before its declaration (Hash.hpp:77)
#   common/Util.hpp   Sort<T> calls FW::sort without including base/Sort.hpp (Util.hpp:78-79)
#   common/SampleBuffer.hpp  MSVC-only opaque 'enum ReconstructionFilter;' (SampleBuffer.hpp:43)
#   common/ (all)     copied so that their relative includes see the edited SampleBuffer.hpp
# plus a variant of reconstruction/Reconstruction.hpp with NUM_OUTPUT_SAMPLES=64
# (Reconstruction.hpp:67) for the 64-output-sample configuration.
# Framework pieces the path links against but that are Win32/GL-bound are
# replaced by oracle/ref_shim (our own code).
#
# Flags: -O2 -ffp-contract=off -fno-fast-math (IEEE single precision, no FMA
# contraction); the reference shipped with /fp:fast (reconstruction_lib.vcproj:195),
# so "reference output" means this build.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${REF:-$(cd "$HERE/../.." && pwd)/reference}"
OUT="$HERE/_ref"
SRC="$REF/src"
if [ ! -d "$SRC/reconstruction_lib" ]; then
  echo "build_ref.sh: reference sources not found under $REF" >&2
  exit 2
fi
rm -rf "$OUT/gen" "$OUT/obj"
mkdir -p "$OUT/gen/base" "$OUT/obj/m128" "$OUT/obj/m64" "$OUT/gen_m64/reconstruction"

# --- generated, edited header copies (never committed) ---
sed -e 's/^inline void Array<\(.*\)>::copy/template<> inline void Array<\1>::copy/' \
    "$SRC/framework/base/Array.hpp" > "$OUT/gen/base/Array.hpp"
sed -e '37i template <class T> inline U32 hash(const T& value);' \
    "$SRC/framework/base/Hash.hpp" > "$OUT/gen/base/Hash.hpp"
cp -r "$SRC/reconstruction_lib/common" "$OUT/gen/common"
chmod -R u+w "$OUT/gen"
sed -i -e 's/^enum ReconstructionFilter;//' "$OUT/gen/common/SampleBuffer.hpp"
sed -i -e 's|#include "base/Random.hpp"|#include "base/Random.hpp"\n#include "base/Sort.hpp"|' "$OUT/gen/common/Util.hpp"
for f in Reconstruction.cpp ReconstructionOur.cpp ReconstructionTreeBuilder.cpp Reconstruction.hpp; do
  cp "$SRC/reconstruction_lib/reconstruction/$f" "$OUT/gen_m64/reconstruction/$f"
done
chmod -R u+w "$OUT/gen_m64"
sed -i -e 's/NUM_OUTPUT_SAMPLES\(\s*\)= 128/NUM_OUTPUT_SAMPLES\1= 64/' "$OUT/gen_m64/reconstruction/Reconstruction.hpp"
grep -q "NUM_OUTPUT_SAMPLES.*= 64" "$OUT/gen_m64/reconstruction/Reconstruction.hpp"

CXX="${CXX:-g++}"
CXXFLAGS="-std=c++14 -O2 -fPIC -ffp-contract=off -fno-fast-math -fpermissive -w -pthread"
DEFS=(-D__int64="long long" -D__w64= -D_M_X64)
INC=(-I"$HERE/ref_shim/include" -I"$OUT/gen" -I"$SRC/framework" -I"$SRC/reconstruction_lib")

compile() {  # compile <out.o> <src> [extra flags...]
  local o="$1" s="$2"; shift 2
  $CXX $CXXFLAGS "${DEFS[@]}" "$@" "${INC[@]}" -c "$s" -o "$o"
}

COMMON_SRCS=(
  "$OUT/gen/common/TimeBounds.cpp"
  "$OUT/gen/common/EdgeFunction.cpp"
  "$OUT/gen/common/Util.cpp"
  "$OUT/gen/common/SampleBuffer.cpp"
  "$SRC/framework/base/Sort.cpp"
  "$SRC/framework/base/Random.cpp"
  "$SRC/framework/base/String.cpp"
  "$SRC/framework/base/Math.cpp"
  "$SRC/framework/base/Hash.cpp"
  "$SRC/framework/io/Stream.cpp"
  "$HERE/ref_shim/fw_runtime.cpp"
)
RECON=(Reconstruction.cpp ReconstructionOur.cpp ReconstructionTreeBuilder.cpp)

pids=()
objs=()
for s in "${COMMON_SRCS[@]}"; do
  o="$OUT/obj/$(basename "${s%.cpp}").o"; objs+=("$o")
  compile "$o" "$s" & pids+=($!)
done
m128=(); m64=()
for f in "${RECON[@]}"; do
  o="$OUT/obj/m128/${f%.cpp}.o"; m128+=("$o")
  compile "$o" "$SRC/reconstruction_lib/reconstruction/$f" & pids+=($!)
  o="$OUT/obj/m64/${f%.cpp}.o"; m64+=("$o")
  compile "$o" "$OUT/gen_m64/reconstruction/$f" & pids+=($!)
done
# the driver sees private members (instrumentation only, see ref_driver.cpp)
compile "$OUT/obj/m128/ref_driver.o" "$HERE/ref_shim/ref_driver.cpp" -I"$SRC/reconstruction_lib/reconstruction" \
  -I"$HERE/ref_shim" & pids+=($!)
compile "$OUT/obj/m64/ref_driver.o" "$HERE/ref_shim/ref_driver.cpp" -I"$OUT/gen_m64/reconstruction" \
  -I"$HERE/ref_shim" -DTLFR_REF_NO_GPU_TOGGLE & pids+=($!)
# the reference's CPU restatement of its GPU-toggle algorithm (ReconstructionCuda.cpp),
# compiled where it lies (checker of the library's enable_cuda mode; 128 output samples)
compile "$OUT/obj/m128/ref_gpu_toggle.o" "$HERE/ref_shim/ref_gpu_toggle.cpp" -I"$SRC/reconstruction_lib/reconstruction" \
  -I"$HERE/ref_shim" & pids+=($!)
# the seeded scene generator (the package's own host code, renamed), so that the
# reference's CPU runs need no other library of this repository
$CXX -std=c++17 -O2 -fPIC -ffp-contract=off -fno-fast-math -pthread -Dtlfr_synth_scene=ref_synth_scene -DTLFR_SYNTH_HOST_ONLY \
  -I"$HERE/../include" -I"$HERE/../temporal-lightfield-reconstruction_b200/csrc" -c "$HERE/../temporal-lightfield-reconstruction_b200/csrc/synth_scene.cpp" \
  -o "$OUT/obj/ref_synth_scene.o" & pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done
objs+=("$OUT/obj/ref_synth_scene.o")

$CXX -shared -pthread -o "$OUT/libtlfr_ref.so"     "${objs[@]}" "${m128[@]}" "$OUT/obj/m128/ref_driver.o" \
  "$OUT/obj/m128/ref_gpu_toggle.o"
$CXX -shared -pthread -o "$OUT/libtlfr_ref_m64.so" "${objs[@]}" "${m64[@]}"  "$OUT/obj/m64/ref_driver.o"
echo "built $OUT/libtlfr_ref.so $OUT/libtlfr_ref_m64.so"
