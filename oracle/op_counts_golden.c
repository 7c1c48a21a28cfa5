/*
 * Golden vectors of the reference's flop model: includes hicma_parsec/op_counts.h
 * and hicma_parsec/flops.h from the reference tree unchanged (build recipe:
 * oracle/Makefile, output in oracle/_ref/) and prints op_counts(op, a, b, c, d)
 * for a fixed grid of arguments and FLOPS_DPOTRF(n) for a list of sizes, one
 * JSON object per line.  Test infrastructure only: the output is committed as
 * tests/golden/op_counts.json and nothing in the library runs this.
 */
#include <stdio.h>

#include "flops.h"
#include "op_counts.h"

static void emit(char op, unsigned long a, unsigned long b, unsigned long c, unsigned long d) {
    printf("{\"op\": \"%c\", \"a\": %lu, \"b\": %lu, \"c\": %lu, \"d\": %lu, \"r\": %lu}\n", op, a, b, c, d,
           op_counts(op, a, b, c, d));
}

int main(void) {
    /* sizes of the configs (NB, ranks, maxranks) plus edge and wrap-around values */
    static const unsigned long v[] = {0, 1, 2, 3, 5, 7, 17, 31, 54, 100, 130, 150, 270, 499, 1000, 1350,
                                      2700, 4096, 65535, 1UL << 21, 3000000UL};
    static const unsigned long w[] = {0, 1, 17, 130, 270, 1350, 2700, 1UL << 21};
    const int nv = (int)(sizeof v / sizeof v[0]), nw = (int)(sizeof w / sizeof w[0]);
    for (int i = 0; i < nv; ++i) {
        emit('c', v[i], 0, 0, 0);
        emit('s', v[i], 0, 0, 0);
        for (int j = 0; j < nv; ++j) {
            emit('q', v[i], v[j], 0, 0);
            for (unsigned long side = 1; side <= 2; ++side) {
                emit('t', v[i], v[j], side, 0);
                emit('r', v[i], v[j], side, 0);
            }
        }
    }
    for (int i = 0; i < nw; ++i)
        for (int j = 0; j < nw; ++j)
            for (int k = 0; k < nw; ++k) {
                emit('m', w[i], w[j], w[k], 0);
                for (unsigned long side = 1; side <= 2; ++side) emit('o', w[i], w[j], w[k], side);
            }
    /* dense-equivalent flops of the driver's GFLOP/s column (testing_dpotrf.c) */
    static const long sizes[] = {1, 2, 3, 54, 270, 2700, 27000, 108000, 216000, 270000, 1000000};
    for (int i = 0; i < (int)(sizeof sizes / sizeof sizes[0]); ++i)
        printf("{\"flops_dpotrf\": %ld, \"r\": %.17g}\n", sizes[i], (double)FLOPS_DPOTRF(sizes[i]));
    return 0;
}
