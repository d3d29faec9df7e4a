/* Thin C entry point around the reference's vendored Random123 header -- test infrastructure.
 * Built by oracle/Makefile into oracle/_ref/libref_random123.so straight from
 * thirdparty/Random123-1.09/include of the reference tree, so the oracle's and the engine's
 * restated Philox2x32-10 can be compared with the reference's own implementation. The mapping
 * (counter start+index as two little-endian 32-bit words, key = low 32 bits) is the one of
 * include/bohrium/jitk/kernel_dependencies/random123_openmp.h:28-37. */
#include <stdint.h>
#include <string.h>
#include <Random123/philox.h>

uint64_t ref_random123(uint64_t start, uint64_t key, uint64_t index) {
    uint64_t i = start + index;
    philox2x32_ctr_t ctr;
    philox2x32_key_t k;
    memcpy(&ctr, &i, sizeof(ctr));
    memcpy(&k, &key, sizeof(k));
    philox2x32_ctr_t r = philox2x32_R(philox2x32_rounds, ctr, k);
    uint64_t out;
    memcpy(&out, &r, sizeof(out));
    return out;
}

void ref_random123_fill(uint64_t start, uint64_t key, uint64_t n, uint64_t *out) {
    for (uint64_t i = 0; i < n; ++i) out[i] = ref_random123(start, key, i);
}
