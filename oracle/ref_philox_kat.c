/*
 * TEST INFRASTRUCTURE ONLY — known-answer vectors for Philox4x32 with 8 rounds (the
 * reference's generator, src/steps/rng/r123.hpp: Philox4x32_R<8>) and with 10 rounds
 * (Random123's default), produced by the reference's own vendored Random123
 * (src/third_party/Random123/philox.h), compiled from where it lies under the reference
 * tree by oracle/build_oracle.py into oracle/_ref/.  Prints a JSON list of
 * {rounds, ctr, key, out}; tests/golden/philox_kat.json is this program's output.
 */
#include <stdio.h>

#include <Random123/philox.h>

int main(void) {
    static const unsigned cases[][6] = {
        {0u, 0u, 0u, 0u, 0u, 0u},
        {0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu},
        {0x243f6a88u, 0x85a308d3u, 0x13198a2eu, 0x03707344u, 0xa4093822u, 0x299f31d0u},
        {0u, 7u, 3u, 0u, 1u, 0u},
        {5u, 123456u, 42u, 0x01000000u, 12345u, 0x9E3779B9u},
        {17u, 383999u, 337u, 0u, 2025u, 7u},
        {1u, 2u, 3u, 4u, 5u, 6u},
        {0x80000000u, 0x40000000u, 0x20000000u, 0x10000000u, 0x08000000u, 0x04000000u},
    };
    const int n = (int)(sizeof(cases) / sizeof(cases[0]));
    static const int rounds[2] = {8, 10};
    printf("[\n");
    for (int q = 0; q < 2; ++q)
        for (int i = 0; i < n; ++i) {
            philox4x32_ctr_t c = {{cases[i][0], cases[i][1], cases[i][2], cases[i][3]}};
            philox4x32_key_t k = {{cases[i][4], cases[i][5]}};
            philox4x32_ctr_t r = philox4x32_R(rounds[q], c, k);
            printf("  {\"rounds\": %d, \"ctr\": [%u, %u, %u, %u], \"key\": [%u, %u], "
                   "\"out\": [%u, %u, %u, %u]}%s\n",
                   rounds[q], c.v[0], c.v[1], c.v[2], c.v[3], k.v[0], k.v[1], r.v[0], r.v[1], r.v[2], r.v[3],
                   (q == 1 && i + 1 == n) ? "" : ",");
        }
    printf("]\n");
    return 0;
}
