/*
 * ref_mtgp_shim.c -- exports the REFERENCE's own CPU MTGP32 generator
 * (mtgp32-fast.c + mtgp32dc-param-11213.c, compiled from the Esthera tree by
 * build_ref.sh) through a plain C ABI so the tests can pin the oracle's
 * MTGP32 restatement against it.  Test infrastructure only.
 */
#include <stdint.h>
#include <string.h>
#include "mtgp32-fast.h"

extern mtgp32_params_fast_t mtgp32dc_params_fast_11213[];

/* kind 0: mtgp32_genrand_uint32; kind 1: bits of mtgp32_genrand_close1_open2 */
int ref_mtgp_generate(int set, uint32_t seed, int kind, int n, uint32_t* out)
{
    mtgp32_fast_t g;
    if (mtgp32_init(&g, &mtgp32dc_params_fast_11213[set], seed)) return -1;
    for (int i = 0; i < n; ++i) {
        if (kind) {
            float f = mtgp32_genrand_close1_open2(&g);
            memcpy(&out[i], &f, sizeof(f));
        } else {
            out[i] = mtgp32_genrand_uint32(&g);
        }
    }
    mtgp32_free(&g);
    return 0;
}

/* The reference's initial state words for (set, seed) (mtgp32_init_state). */
void ref_mtgp_init_state(int set, uint32_t seed, uint32_t* st)
{
    mtgp32_init_state(st, &mtgp32dc_params_fast_11213[set], seed);
}

uint32_t ref_mtgp_mask(int set) { return mtgp32dc_params_fast_11213[set].mask; }
