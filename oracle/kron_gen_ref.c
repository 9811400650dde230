/*
 * Oracle driver for the Graph500 Kronecker generator vendored in the
 * reference (graph500-generator/make_graph.c:41-60, graph_generator.c).
 * TEST INFRASTRUCTURE ONLY.  It calls the reference's make_graph() exactly
 * as the reference drivers do (generator_test_seq.c:265 uses seeds (1, 2))
 * and writes the packed_edge array {u32 v0; u32 v1} as raw binary, which is
 * the gedge_t input format of the reference converter (gstore.h:255-279).
 *
 * usage: kron_gen_ref <scale> <edgefactor> <out.bin> [seed1 seed2]
 */
#include <stdio.h>
#include <stdlib.h>
#include <stdint.h>
#include "make_graph.h"

int main(int argc, char** argv)
{
    if (argc < 4) {
        fprintf(stderr, "usage: %s scale edgefactor out.bin [seed1 seed2]\n", argv[0]);
        return 2;
    }
    int scale = atoi(argv[1]);
    int64_t ef = atoll(argv[2]);
    uint64_t s1 = argc > 5 ? strtoull(argv[4], 0, 10) : 1;
    uint64_t s2 = argc > 5 ? strtoull(argv[5], 0, 10) : 2;
    int64_t nedges = 0;
    packed_edge* edges = 0;
    make_graph(scale, ef << scale, s1, s2, &nedges, &edges);
    FILE* f = fopen(argv[3], "wb");
    if (!f) { perror("open"); return 2; }
    if ((int64_t)fwrite(edges, sizeof(packed_edge), nedges, f) != nedges) {
        perror("write");
        return 2;
    }
    fclose(f);
    free(edges);
    return 0;
}
