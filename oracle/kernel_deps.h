/* Helpers included by the oracle's generated C kernels -- test infrastructure.
 *
 * bh_random123(): BH_RANDOM's generator, Philox2x32 with 10 rounds, restated from the published
 * algorithm (Salmon, Moraes, Dror, Shaw: "Parallel Random Numbers: As Easy as 1, 2, 3", SC'11),
 * with the counter start+index split into two little-endian 32-bit words and the low 32 bits of
 * `key` as the key, returning the two output words as one little-endian uint64 -- the mapping of
 * include/bohrium/jitk/kernel_dependencies/random123_openmp.h:28-37 of the reference. It is pinned
 * against the reference's own Random123 header (oracle/_ref) and the known-answer vector
 * (counter 0, key 42) -> (624017136, 4231775638).
 */
#ifndef BH_ORACLE_KERNEL_DEPS_H
#define BH_ORACLE_KERNEL_DEPS_H
#include <stdint.h>

static inline uint64_t bh_random123(uint64_t start, uint64_t key, uint64_t index) {
    const uint64_t c = start + index;
    uint32_t x0 = (uint32_t)c, x1 = (uint32_t)(c >> 32), k = (uint32_t)key;
    for (int r = 0; r < 10; ++r) {
        const uint64_t prod = (uint64_t)0xD256D193u * (uint64_t)x0;
        const uint32_t hi = (uint32_t)(prod >> 32), lo = (uint32_t)prod;
        x0 = hi ^ k ^ x1;
        x1 = lo;
        k += 0x9E3779B9u;
    }
    return ((uint64_t)x1 << 32) | (uint64_t)x0;
}

#endif
