#!/usr/bin/env bash
# Builds the reference's own spectral + BSDF code as a host shared library
# (oracle/_ref/libvlrref.so) for parity checks.  TEST INFRASTRUCTURE ONLY.
#
# Recipe:
#   1. mirror the reference tree under oracle/_ref/mirror with symlinks
#      (libVLR/shared/*, libVLR/include/vlr as both include/vlr and include/VLR
#      for the case-sensitive include in shared/basic_types_internal.h:4,
#      libVLR/GPU_kernels/materials.cu), plus our host stand-ins under
#      oracle/shim for the OptiX utility header and the empty ext/half;
#   2. write a patched copy of shared/spectrum_types.cpp into the mirror: its
#      four static-member definitions at :619-622 use MSVC-only syntax that
#      g++ rejects, so they get `template <>` and an empty initialiser;
#   3. compile with the reference's compile-time switch for spectral rendering
#      (common_internal.h:23) and link into one .so.
# The reference sources stay where they are; only build outputs land in
# oracle/_ref (git-ignored).
set -euo pipefail

HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${VLR_REFERENCE:-/root/reference}"
OUT="$HERE/_ref"
MIR="$OUT/mirror/libVLR"

if [ ! -d "$REF/libVLR/shared" ]; then
    echo "build_ref.sh: reference tree not found at $REF" >&2
    exit 2
fi

rm -rf "$OUT/mirror"
mkdir -p "$MIR/shared" "$MIR/include" "$MIR/GPU_kernels" "$MIR/utils" "$OUT/obj"

for f in "$REF"/libVLR/shared/*; do
    ln -s "$f" "$MIR/shared/$(basename "$f")"
done
rm "$MIR/shared/spectrum_types.cpp"
sed -E \
    -e 's/^([[:space:]]*)(DiscretizedSpectrumTemplate<float, NumStrataForStorage>::CMF DiscretizedSpectrumTemplate<float, NumStrataForStorage>::[xyz]bar);/\1template <> \2{};/' \
    -e 's/^([[:space:]]*)(float DiscretizedSpectrumTemplate<float, NumStrataForStorage>::integralCMF);/\1template <> \2 = 0.0f;/' \
    "$REF/libVLR/shared/spectrum_types.cpp" > "$MIR/shared/spectrum_types.cpp"

# FP64 oracle copy (ref_shim64.cpp): the patched file without the FP32
# Meng-Simon tables and the FP32 explicit instantiations, which clash with the
# FP64 ones once every float is compiled as double.
python3 - "$MIR/shared/spectrum_types.cpp" "$MIR/shared/spectrum_types64.cpp" <<'PYEOF'
import sys
lines = open(sys.argv[1]).read().split("\n")
def table_start(real):
    key = "UpsampledSpectrumTemplate<%s, NumSpectralSamples>::spectrum_grid_cell_t" % real
    i = next(k for k, l in enumerate(lines) if key in l)
    return i - 1 if lines[i - 1].strip() == "template <>" else i
a, b = table_start("float"), table_start("double")
assert a < b
out = [l for l in lines[:a] + lines[b:] if not (l.strip().startswith("template class") and "<float," in l)]
open(sys.argv[2], "w").write("\n".join(out))
PYEOF

ln -s "$REF/libVLR/include/vlr" "$MIR/include/vlr"
ln -s "$REF/libVLR/include/vlr" "$MIR/include/VLR"
ln -s "$REF/libVLR/GPU_kernels/materials.cu" "$MIR/GPU_kernels/materials.cu"
ln -s "$HERE/shim/utils/optixu_on_cudau.h" "$MIR/utils/optixu_on_cudau.h"

CXX="${VLR_HOST_CXX:-/usr/bin/g++}"
FLAGS=(-std=c++20 -O2 -fPIC -fopenmp -DVLR_USE_SPECTRAL_RENDERING -mlzcnt -mpopcnt -mbmi
       -w
       -I "$MIR/shared" -I "$MIR/include/vlr" -I "$MIR" -I "$HERE/shim"
       -I /usr/local/cuda/include)

"$CXX" "${FLAGS[@]}" -c "$MIR/shared/spectrum_base.cpp" -o "$OUT/obj/spectrum_base.o"
"$CXX" "${FLAGS[@]}" -c "$MIR/shared/spectrum_types.cpp" -o "$OUT/obj/spectrum_types.o"
"$CXX" "${FLAGS[@]}" -I "$HERE" -x c++ -c "$HERE/ref_shim.cpp" -o "$OUT/obj/ref_shim.o"
"$CXX" -shared -fopenmp -o "$OUT/libvlrref.so" \
    "$OUT/obj/ref_shim.o" "$OUT/obj/spectrum_base.o" "$OUT/obj/spectrum_types.o"
echo "built $OUT/libvlrref.so"

# The FP64 oracle: the same reference sources with every float compiled as
# double (ref_shim64.cpp), in a library of its own; -Bsymbolic keeps its
# classes bound to themselves when both libraries are loaded.
"$CXX" "${FLAGS[@]}" -I "$HERE" -x c++ -c "$HERE/ref_shim64.cpp" -o "$OUT/obj/ref_shim64.o"
"$CXX" -shared -fopenmp -Wl,-Bsymbolic -o "$OUT/libvlrref64.so" "$OUT/obj/ref_shim64.o"
echo "built $OUT/libvlrref64.so"
