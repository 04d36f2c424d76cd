// ref_shim.cpp -- C entry points onto the reference's own CPU hashers.
//
// TEST INFRASTRUCTURE ONLY: compiled together with the zeknox CPU sources
// (native/{keccak,poseidon,poseidon2,monolith,merkle}, the list of
// LIB_CXX_SRC in native/CMakeLists.txt:83-91) into oracle/_ref/, where the
// tests use it to pin the oracle restatement and bench.py's reference arm
// times fill_digests_buf_linear_cpu (native/merkle/merkle.cpp:126-161).
#include "types/int_types.h"
#include "poseidon/poseidon.hpp"
#include "poseidon2/poseidon2.hpp"
#include "keccak/keccak.hpp"
#include "monolith/monolith.hpp"
#include "poseidon/poseidon_bn128.hpp"

extern "C" int zkref_hash_one(int type, u64 *in, u64 n, u64 *out)
{
    switch (type) {
    case 0: PoseidonHasher::cpu_hash_one(in, n, out); return 0;
    case 1: KeccakHasher::cpu_hash_one(in, n, out); return 0;
    case 2: PoseidonBN128Hasher::cpu_hash_one(in, n, out); return 0;
    case 3: Poseidon2Hasher::cpu_hash_one(in, n, out); return 0;
    case 4: MonolithHasher::cpu_hash_one(in, n, out); return 0;
    default: return -1;
    }
}

extern "C" int zkref_hash_two(int type, u64 *l, u64 *r, u64 *out)
{
    switch (type) {
    case 0: PoseidonHasher::cpu_hash_two(l, r, out); return 0;
    case 1: KeccakHasher::cpu_hash_two(l, r, out); return 0;
    case 2: PoseidonBN128Hasher::cpu_hash_two(l, r, out); return 0;
    case 3: Poseidon2Hasher::cpu_hash_two(l, r, out); return 0;
    case 4: MonolithHasher::cpu_hash_two(l, r, out); return 0;
    default: return -1;
    }
}
