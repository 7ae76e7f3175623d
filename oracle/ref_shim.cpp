// Test-only shim compiled together with zeknox's own CPU sources (see
// build_ref.sh).  It exposes the C++ hasher entry points of zeknox
// (PoseidonHasher / Poseidon2Hasher / KeccakHasher / MonolithHasher /
// PoseidonBN128Hasher ::cpu_hash_one/two, native/poseidon/poseidon.cpp:453-461,
// native/poseidon2/poseidon2.cu:227-242, native/keccak/keccak.cu:139-156,
// native/monolith/monolith.cu:259-267, native/poseidon/poseidon_bn128.cu)
// under C names so the Python tests can call
// them through ctypes.  fill_digests_buf_linear_cpu is already extern "C".
#include "types/int_types.h"
#include "merkle/merkle.h"
#include "poseidon/poseidon.hpp"
#include "poseidon2/poseidon2.hpp"
#include "keccak/keccak.hpp"
#include "monolith/monolith.hpp"
#include "poseidon/poseidon_bn128.hpp"

extern "C" int zkref_hash_one(int ht, u64 *in, u64 n, u64 *out)
{
    switch (ht) {
    case HashPoseidon: PoseidonHasher::cpu_hash_one(in, n, out); return 0;
    case HashPoseidon2: Poseidon2Hasher::cpu_hash_one(in, n, out); return 0;
    case HashKeccak: KeccakHasher::cpu_hash_one(in, n, out); return 0;
    case HashMonolith: MonolithHasher::cpu_hash_one(in, n, out); return 0;
    case HashPoseidonBN128: PoseidonBN128Hasher::cpu_hash_one(in, n, out); return 0;
    default: return -1;
    }
}

extern "C" int zkref_hash_two(int ht, u64 *l, u64 *r, u64 *out)
{
    switch (ht) {
    case HashPoseidon: PoseidonHasher::cpu_hash_two(l, r, out); return 0;
    case HashPoseidon2: Poseidon2Hasher::cpu_hash_two(l, r, out); return 0;
    case HashKeccak: KeccakHasher::cpu_hash_two(l, r, out); return 0;
    case HashMonolith: MonolithHasher::cpu_hash_two(l, r, out); return 0;
    case HashPoseidonBN128: PoseidonBN128Hasher::cpu_hash_two(l, r, out); return 0;
    default: return -1;
    }
}
