/*
 * ORACLE — test infrastructure only (see nw_oracle.h). Compiled with
 * -ffp-contract=off so that every float/double operation rounds exactly
 * where the reference's C++ does (x86-64 SSE, no FMA contraction).
 */
#include "nw_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* encode_table (src/encoder.cpp:27-30), restated. */
static const uint8_t letter_unit[26] = {
    0x00, 0x14, 0x01, 0x06, 0x08, 0x0E, 0x03, 0x09, 0x0A, 0x15, 0x0C, 0x0B, 0x0D,
    0x05, 0x17, 0x0F, 0x07, 0x04, 0x10, 0x02, 0x17, 0x13, 0x11, 0x17, 0x12, 0x16,
};

uint8_t oracle_encode_char(char c)
{
    /* toupper on the byte, then A..Z through the table; '-' is the gap unit;
     * everything else is the end/padding unit (encoder.cpp:46-57). */
    char u = (c >= 'a' && c <= 'z') ? (char) (c - 'a' + 'A') : c;
    if(u >= 'A' && u <= 'Z') return letter_unit[u - 'A'];
    if(c == '-') return ORACLE_UNIT_GAP;
    return ORACLE_UNIT_END;
}

static inline uint8_t unit_at(const uint8_t *s, int64_t n, int64_t k)
{
    return k < n ? s[k] : (uint8_t) ORACLE_UNIT_END;
}

static inline int64_t padded(int64_t n) { return ((n + 2) / 3) * 3; }

int oracle_nw_pair(const uint8_t *rows, int64_t nrows, const uint8_t *cols, int64_t ncols,
                   const int32_t *tables, int ntables, int table, int32_t penalty,
                   int32_t *out_score)
{
    const int64_t lr = padded(nrows), lc = padded(ncols);
    const int64_t limit = (int64_t) ntables * 625;
    const int64_t base = (int64_t) table * 625;
    int32_t *line = (int32_t *) malloc(sizeof(int32_t) * (size_t) (lc + 1));
    if(!line) return -2;

    /* 0-th line: j * -penalty (sequential.cpp:35-36). */
    for(int64_t j = 0; j <= lc; ++j) line[j] = (int32_t) (j * -penalty);

    for(int64_t i = 0; i < lr; ++i) {
        const uint8_t a = unit_at(rows, nrows, i);
        /* A padding row ends the matrix (sequential.cpp:42-43). */
        if(a == ORACLE_UNIT_END) break;

        int32_t done = line[0];
        line[0] = (int32_t) ((i + 1) * -penalty);

        for(int64_t j = 1; j <= lc; ++j) {
            int32_t value = line[j - 1];
            const uint8_t b = unit_at(cols, ncols, j - 1);

            /* A padding column copies its left neighbour (sequential.cpp:53-60). */
            if(b != ORACLE_UNIT_END) {
                const int64_t at = base + (int64_t) a * 25 + b;
                if(at >= limit) { free(line); return -1; }
                const int32_t insertd = value - penalty;
                const int32_t removed = line[j] - penalty;
                const int32_t matched = done + tables[at];
                const int32_t m = insertd > removed ? insertd : removed;
                value = matched > m ? matched : m;
            }

            done = line[j];
            line[j] = value;
        }
    }

    *out_score = line[lc];
    free(line);
    return 0;
}

int oracle_nw_all_pairs(int64_t n, const uint8_t *units, const uint64_t *offs,
                        const uint64_t *lens, const int32_t *tables, int ntables,
                        int table, int32_t penalty, int32_t *out)
{
    for(int64_t i = 1; i < n; ++i) {
        for(int64_t j = 0; j < i; ++j) {
            const int64_t bi = ((int64_t) lens[i] + 2) / 3, bj = ((int64_t) lens[j] + 2) / 3;
            /* one = db[i], two = db[j]; rows = one if it has more blocks, else two. */
            const int64_t r = bi > bj ? i : j, c = bi > bj ? j : i;
            int32_t s;
            const int rc = oracle_nw_pair(units + offs[r], (int64_t) lens[r],
                                          units + offs[c], (int64_t) lens[c],
                                          tables, ntables, table, penalty, &s);
            if(rc) return rc;
            out[i * (i - 1) / 2 + j] = s;
        }
    }
    return 0;
}

#define UNDEF 0xFFFFFFFFu

int oracle_nj(int64_t n, const float *tri,
              uint32_t *parent, uint32_t *child0, uint32_t *child1,
              float *distance, uint32_t *level,
              uint32_t *join_x, uint32_t *join_y)
{
    return oracle_nj_order(n, tri, ORACLE_NJ_SYMMETRIC, parent, child0, child1, distance, level, join_x, join_y);
}

int oracle_nj_order(int64_t n, const float *tri, int order,
                    uint32_t *parent, uint32_t *child0, uint32_t *child1,
                    float *distance, uint32_t *level,
                    uint32_t *join_x, uint32_t *join_y)
{
    if(order != ORACLE_NJ_SYMMETRIC && order != ORACLE_NJ_LINEAR) return -1;
    if(n < 2) return 0;
    const int64_t nodes = 2 * n - 1;

    float *D = (float *) calloc((size_t) (n * n), sizeof(float));
    float *S = (float *) calloc((size_t) n, sizeof(float));
    float *nd = (float *) calloc((size_t) n, sizeof(float));
    uint32_t *map = (uint32_t *) calloc((size_t) n, sizeof(uint32_t));
    int64_t *perm = (int64_t *) calloc((size_t) n, sizeof(int64_t));
    uint32_t *P = (uint32_t *) malloc(sizeof(uint32_t) * (size_t) nodes);
    uint32_t *C0 = (uint32_t *) malloc(sizeof(uint32_t) * (size_t) nodes);
    uint32_t *C1 = (uint32_t *) malloc(sizeof(uint32_t) * (size_t) nodes);
    float *DI = (float *) malloc(sizeof(float) * (size_t) nodes);
    uint32_t *LV = (uint32_t *) malloc(sizeof(uint32_t) * (size_t) nodes);
    if(!D || !S || !nd || !map || !perm || !P || !C0 || !C1 || !DI || !LV) return -2;

    /* Inflate the packed triangle (phylogeny/matrix.cuh:123-130); diagonal 0. */
    for(int64_t i = 1; i < n; ++i)
        for(int64_t j = 0; j < i; ++j)
            D[i * n + j] = D[j * n + i] = tri[i * (i - 1) / 2 + j];

    /* cache_init (sequential.cpp:80-94): per k, a float fold over j != k in
     * ascending j, starting from 0. */
    for(int64_t i = 0; i + 1 < n; ++i)
        for(int64_t j = i + 1; j < n; ++j) {
            const float cur = D[i * n + j];
            S[i] += cur;
            S[j] += cur;
        }

    for(int64_t i = 0; i < n; ++i) { map[i] = (uint32_t) i; perm[i] = i; }

    /* Tree nodes (phylogeny.cuh:171-180, hierarchy.hpp:46-47). */
    for(int64_t k = 0; k < nodes; ++k) {
        P[k] = C0[k] = C1[k] = UNDEF;
        DI[k] = FLT_MAX;
        LV[k] = 0;
    }

    uint32_t next_parent = (uint32_t) n;
    int64_t c = n;
    int64_t step = 0;

    while(c > 1) {
        /* pick_joinable (sequential.cpp:161-182): row-major scan of the
         * logical lower triangle, first strictly greater Q wins. */
        float best = -INFINITY;
        int64_t bx = -1, by = -1;
        const float cm2 = (float) (c - 2);
        for(int64_t i = 1; i < c; ++i) {
            const int64_t pi = perm[i];
            const float si = S[pi];
            for(int64_t j = 0; j < i; ++j) {
                const int64_t pj = perm[j];
                float q = cm2 * D[pi * n + pj];   /* q_transform, sequential.cpp:129-133 */
                q = q - si;
                q = q - S[pj];
                if(q > best) { best = q; bx = i; by = j; }
            }
        }
        if(bx < 0) goto fail;   /* every Q was NaN: the reference would index undefined */

        const int64_t px = perm[bx], py = perm[by];
        const float dxy = D[px * n + py];

        /* raise_candidate (sequential.cpp:142-152). */
        const float pairsum = S[px] - S[py];
        const float dx = (float) (0.5 * (double) dxy + (double) (pairsum / (float) (2 * (c - 2))));
        const float dy = dxy - dx;

        /* star::join (star.cuh:61-72): children ordered by OTU id. */
        {
            const uint32_t idx = map[px], idy = map[py];
            const uint32_t id1 = idx < idy ? idx : idy, id2 = idx < idy ? idy : idx;
            const float d1 = idx < idy ? dx : dy, d2 = idx < idy ? dy : dx;
            DI[id1] = d1; P[id1] = next_parent;
            DI[id2] = d2; P[id2] = next_parent;
            LV[next_parent] = (LV[id1] > LV[id2] ? LV[id1] : LV[id2]) + 1;
            C0[next_parent] = id1;
            C1[next_parent] = id2;
        }
        if(join_x) join_x[step] = (uint32_t) bx;
        if(join_y) join_y[step] = (uint32_t) by;

        /* join_pair (sequential.cpp:234-277). */
        float new_sum = 0.0f;
        for(int64_t i = 0; i < c; ++i) {
            const int64_t p = perm[i];
            const float previous = D[p * n + px] + D[p * n + py];
            const double updated = (double) (previous - dxy) * .5;
            nd[i] = (float) updated;
            S[p] = (float) ((double) S[p] + (updated - (double) previous));
            new_sum = (float) ((double) new_sum + updated);
        }
        for(int64_t i = 0; i < c; ++i) {
            const int64_t p = perm[i];
            D[p * n + px] = D[px * n + p] = nd[i];
        }
        S[px] = new_sum;
        map[px] = next_parent;

        if(order == ORACLE_NJ_SYMMETRIC) {
            /* update_cache, symmetric (sequential.cpp:210-224): swap logical 0
             * and y, then drop logical 0; every later index moves down by one. */
            const int64_t p0 = perm[0];
            for(int64_t k = 0; k + 1 < c; ++k) perm[k] = perm[k + 1];
            if(by > 0) perm[by - 1] = p0;
        } else {
            /* update_cache, linear (sequential.cpp:189-203): swap y and the
             * last logical index c-1 (matrix rows and columns, row sums and the
             * OTU map: matrix.cu:443-460 exchanges every off-diagonal pair, the
             * diagonal being zero), then drop the last; no index shifts. The
             * new node itself moves into y when x was the last. */
            const int64_t py2 = perm[by];
            perm[by] = perm[c - 1];
            perm[c - 1] = py2;
        }

        ++next_parent;
        --c;
        ++step;
    }

    if(parent) memcpy(parent, P, sizeof(uint32_t) * (size_t) nodes);
    if(child0) memcpy(child0, C0, sizeof(uint32_t) * (size_t) nodes);
    if(child1) memcpy(child1, C1, sizeof(uint32_t) * (size_t) nodes);
    if(distance) memcpy(distance, DI, sizeof(float) * (size_t) nodes);
    if(level) memcpy(level, LV, sizeof(uint32_t) * (size_t) nodes);

    free(D); free(S); free(nd); free(map); free(perm);
    free(P); free(C0); free(C1); free(DI); free(LV);
    return 0;

fail:
    free(D); free(S); free(nd); free(map); free(perm);
    free(P); free(C0); free(C1); free(DI); free(LV);
    return -3;
}
