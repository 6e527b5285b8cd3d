/*
 * ORACLE — test infrastructure only. A plain-C restatement of the reference's
 * CPU algorithms for the all-pairs Needleman-Wunsch step and the
 * neighbor-joining step. Only tests/, the smoke check and bench.py's
 * CPU-baseline leg may load it, and only as the checker; the product never
 * links or calls it.
 *
 * Pinned against the compiled reference (oracle/_ref, built by
 * oracle/Makefile from the reference's own sources) and against the golden
 * fixtures under tests/golden/.
 */
#ifndef MSA_NW_ORACLE_H
#define MSA_NW_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Unit codes of the reference encoder (src/encoder.hpp:42-48). */
enum { ORACLE_UNIT_END = 0x18, ORACLE_UNIT_GAP = 0x19 };

/* encoder::encode(char) (src/encoder.cpp:46-57). */
uint8_t oracle_encode_char(char c);

/*
 * sequential::align_pair (src/pairwise/needleman/impl/sequential.cpp:29-68)
 * over unit strings. `rows`/`cols` hold `nrows`/`ncols` units; both are
 * treated as padded to a multiple of 3 with END units (sequence::length(),
 * src/sequence.hpp:101-104). `tables` is the reference's contiguous block of
 * scoring tables (table.cu:41-237), `ntables` of them, each 25x25; `table`
 * picks one. Entries are read by flat offset exactly as `(*m_contents)[x][y]`
 * addresses them, so a GAP unit (25) reads the following row/table the way the
 * reference's storage lays them out. Returns 0, or -1 when an index would fall
 * past the last table (undefined in the reference).
 */
int oracle_nw_pair(const uint8_t *rows, int64_t nrows, const uint8_t *cols, int64_t ncols,
                   const int32_t *tables, int ntables, int table, int32_t penalty,
                   int32_t *out_score);

/*
 * sequential::align (sequential.cpp:77-95) + algorithm::generate
 * (src/pairwise/pairwise.cpp:73-85): all pairs i > j of the n sequences
 * (units at units[offs[k] .. offs[k]+lens[k])), written to out[i(i-1)/2+j].
 * The row sequence is the one with more 3-unit blocks; on a tie it is the
 * pair's second element, j (sequential.cpp:87-91).
 */
int oracle_nw_all_pairs(int64_t n, const uint8_t *units, const uint64_t *offs,
                        const uint64_t *lens, const int32_t *tables, int ntables,
                        int table, int32_t penalty, int32_t *out);

/*
 * njoining::sequential<transform::symmetric>::run
 * (src/phylogeny/njoining/impl/sequential.cpp:80-346) restated over a logical
 * permutation instead of the packed shrinking matrix. `tri` is the packed
 * strict lower triangle (n(n-1)/2 floats, index i(i-1)/2+j). Writes 2n-1 tree
 * nodes (src/phylogeny/njoining/star.cuh:61-72) and, per join k (0..n-2),
 * the joined logical pair (join_x > join_y) and the two OTU ids.
 * Any output pointer may be NULL.
 */
int oracle_nj(int64_t n, const float *tri,
              uint32_t *parent, uint32_t *child0, uint32_t *child1,
              float *distance, uint32_t *level,
              uint32_t *join_x, uint32_t *join_y);

/*
 * The same with the removal order chosen: ORACLE_NJ_SYMMETRIC as above, or
 * ORACLE_NJ_LINEAR for njoining::sequential<transform::linear<2>>
 * (sequential.cpp:189-203, 356-358): the removed OTU y trades places with the
 * last logical OTU, which is then dropped, so no other index moves. Returns
 * -1 for an unknown order.
 */
#define ORACLE_NJ_SYMMETRIC 0
#define ORACLE_NJ_LINEAR 1
int oracle_nj_order(int64_t n, const float *tri, int order,
                    uint32_t *parent, uint32_t *child0, uint32_t *child1,
                    float *distance, uint32_t *level,
                    uint32_t *join_x, uint32_t *join_y);

#ifdef __cplusplus
}
#endif
#endif
