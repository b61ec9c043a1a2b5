/* Plain-C caller of libhoms: the header must compile as C99 and every call
 * below works without a GPU (argument checks, version, status strings,
 * ADC counting of a host sequence). */
#include <stdio.h>
#include <string.h>

#include "homs.h"

int main(void) {
    if (homs_abi_version() != HOMS_ABI_VERSION) return 1;
    if (strcmp(homs_status_string(HOMS_OK), "ok") != 0) return 2;
    if (homs_context_create(0, NULL, NULL) != HOMS_EINVAL) return 3;
    if (homs_simulate(NULL, NULL, NULL, NULL, NULL, NULL, HOMS_HOST) != HOMS_EINVAL) return 4;
    if (homs_count_adc(NULL, NULL) != HOMS_EINVAL) return 5;

    /* Two blocks over five nodes sharing node 2; ADC on nodes 1..4: the
     * boundary node's sample belongs to the first block, so 4 samples. */
    double t[5] = {0, 1e-5, 2e-5, 3e-5, 4e-5}, dt[4] = {1e-5, 1e-5, 1e-5, 1e-5}, zero[5] = {0};
    double b1[10] = {0};
    uint8_t adc[5] = {0, 1, 1, 1, 1};
    int64_t first[2] = {0, 2}, last[2] = {2, 4};
    uint8_t exc[2] = {0, 0};
    homs_sequence q;
    memset(&q, 0, sizeof(q));
    q.nnodes = 5;
    q.dtype = HOMS_F64;
    q.memory = HOMS_HOST;
    q.t = t;
    q.dt = dt;
    q.gx = q.gy = q.gz = zero;
    q.b1 = b1;
    q.df = q.psi = zero;
    q.adc = adc;
    for (int k = 0; k < 16; ++k) q.h[k] = zero;
    q.nblocks = 2;
    q.block_first = first;
    q.block_last = last;
    q.block_excitation = exc;
    q.gamma = 42.5774688e6;
    int64_t n = -1;
    if (homs_count_adc(&q, &n) != HOMS_OK || n != 4) return 6;
    printf("libhoms ABI %d from C: ok\n", homs_abi_version());
    return 0;
}
