#!/usr/bin/env bash
# Build zeknox's own code from its sources (test infrastructure only).
#
#   oracle/_ref/libzkref_cpu.so  zeknox's C++ CPU path (fill_digests_buf_linear_cpu,
#                                the Poseidon / Poseidon2 / Keccak CPU hashers) plus
#                                oracle/ref_shim.cpp; the CPU parity oracle and the
#                                timed CPU baseline.
#   oracle/_ref/libzkref_gpu.so  zeknox's CUDA sources compiled for sm_100a: the
#                                reference GPU build the -m gpu tests compare against.
#
# The sources are compiled where they lie; nothing is copied into this repo.
# Outputs go to oracle/_ref/ only.  Needs the zeknox tree, named by the
# ZEKNOX_SRC environment variable or the first argument; without it (or on a
# machine without the tree) this script does nothing.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
ROOT_SRC="${1:-${ZEKNOX_SRC:-}}"
if [ -z "$ROOT_SRC" ]; then
    echo "build_ref: set ZEKNOX_SRC (or pass the zeknox tree as the first argument); skipping" >&2
    exit 0
fi
SRC="$ROOT_SRC/native"
OUT="$HERE/_ref"
if [ ! -d "$SRC" ]; then
    echo "build_ref: zeknox sources not found at $SRC; skipping" >&2
    exit 0
fi
mkdir -p "$OUT/obj_cpu" "$OUT/obj_gpu"

# --- CPU path: the flags of native/CMakeLists.txt's release build ----------
CXXFLAGS="-std=c++17 -O3 -fPIC -fopenmp -DFEATURE_GOLDILOCKS -DEXPOSE_C_INTERFACE -DTAKE_RESPONSIBILITY_FOR_ERROR_MESSAGE -w -I$SRC"
for f in keccak/keccak.cu poseidon/element_bn128.cu poseidon/poseidon_bn128.cu poseidon2/poseidon2.cu monolith/monolith.cu; do
    g++ $CXXFLAGS -x c++ -c "$SRC/$f" -o "$OUT/obj_cpu/$(basename "$f").o"
done
for f in poseidon/poseidon.cpp merkle/merkle.cpp; do
    g++ $CXXFLAGS -c "$SRC/$f" -o "$OUT/obj_cpu/$(basename "$f").o"
done
g++ $CXXFLAGS -c "$HERE/ref_shim.cpp" -o "$OUT/obj_cpu/ref_shim.o"
g++ -shared -fopenmp -Wl,-Bsymbolic -o "$OUT/libzkref_cpu.so" "$OUT"/obj_cpu/*.o

# --- GPU path: zeknox's CUDA sources for sm_100a ---------------------------
if [ "${ZK_SKIP_REF_GPU:-0}" != "1" ]; then
    NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
    NVFLAGS="-std=c++17 -O3 -DNDEBUG -gencode arch=compute_100a,code=sm_100a -rdc=true -Xcompiler -fPIC,-fopenmp -w \
        -DUSE_CUDA -DFEATURE_GOLDILOCKS -DEXPOSE_C_INTERFACE -DTAKE_RESPONSIBILITY_FOR_ERROR_MESSAGE -I$SRC"
    objs=()
    for f in keccak/keccak.cu poseidon/poseidon.cu poseidon/element_bn128.cu poseidon/poseidon_bn128.cu \
             poseidon2/poseidon2.cu monolith/monolith.cu merkle/merkle.cu ntt/ntt.cu utils/all_gpus.cu lib.cu; do
        o="$OUT/obj_gpu/$(echo "$f" | tr '/' '_').o"
        "$NVCC" $NVFLAGS -c "$SRC/$f" -o "$o"
        objs+=("$o")
    done
    "$NVCC" -gencode arch=compute_100a,code=sm_100a -dlink -Xcompiler -fPIC "${objs[@]}" -o "$OUT/obj_gpu/dlink.o"
    g++ -shared -fopenmp -Wl,-Bsymbolic -o "$OUT/libzkref_gpu.so" "${objs[@]}" "$OUT/obj_gpu/dlink.o" \
        -L/usr/local/cuda/lib64 -lcudart_static -ldl -lrt -lpthread
fi
echo "build_ref: done ($OUT)"
