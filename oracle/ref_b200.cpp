/*
 * Test infrastructure only: the reference-side binding of libmsa_b200.so,
 * compiled against the reference's own headers and types, so the drop-in
 * claim is checked with the classes a Museqa maintainer would register.
 *
 *   needleman_b200  : museqa::pairwise::algorithm   (src/pairwise/pairwise.cuh:205-222)
 *   njoining_b200   : museqa::phylogeny::algorithm  (src/phylogeny/phylogeny.cuh:94-110)
 *
 * Each implements `run(const context&)` through include/msa_b200.h only (no
 * torch, no Python). INTEGRATION.md shows the same classes with the two
 * dispatcher lines that register them (src/pairwise/pairwise.cpp:26-35,
 * src/phylogeny/phylogeny.cpp:26-41). The extern "C" functions at the end let
 * the tests build a reference database, call the algorithm objects directly
 * and compare them with the reference's own sequential algorithms.
 */
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "database.hpp"
#include "exception.hpp"
#include "sequence.hpp"
#include "pairwise.cuh"
#include "phylogeny.cuh"
#include "phylogeny/njoining/star.cuh"

#include "msa_b200.h"

namespace
{
    using namespace museqa;

    thread_local std::string last_error;

    /* A failed library call becomes the reference's exception type (its own
     * `enforce` is compiled out in production builds). */
    void check(bool ok, const std::string& what, const char *detail)
    {
        if(!ok) throw museqa::exception {what + ": " + (detail ? detail : "")};
    }

    /* One library context per process and device 0, created on first use. */
    msa_ctx *b200_context()
    {
        static msa_ctx *ctx = nullptr;
        if(!ctx) {
            const int rc = msa_create(0, &ctx);
            check(rc == MSA_OK, "no B200 device", msa_strerror(rc));
        }
        return ctx;
    }

    /* The scoring table by value. A table equal to one of the reference's
     * built-ins (entries and penalty) carries that table's index, so a GAP
     * unit reads the reference's contiguous table storage the same way
     * (src/pairwise/table.cu:41-262); any other table is the caller's own. */
    msa_table to_msa_table(const pairwise::scoring_table& table)
    {
        msa_table t {};
        for(size_t x = 0; x < 25; ++x)
            for(size_t y = 0; y < 25; ++y)
                t.score[x * 25 + y] = (int32_t) table[{x, y}];
        t.penalty = (int32_t) table.penalty();
        t.index = -1;
        for(const auto& name : pairwise::scoring_table::list()) {
            const auto builtin = pairwise::scoring_table::make(name);
            bool same = builtin.penalty() == table.penalty();
            for(size_t x = 0; same && x < 25; ++x)
                for(size_t y = 0; same && y < 25; ++y)
                    same = builtin[{x, y}] == table[{x, y}];
            if(same) {
                msa_table named {};
                if(msa_table_make(name.c_str(), &named) == MSA_OK) return named;
            }
        }
        return t;
    }

    /* pairwise::algorithm on the B200: the database's units (one byte each,
     * over the padded length, END padding included as the reference sweeps
     * it) go to a device store; msa_nw_all_pairs scores every pair i > j at
     * i(i-1)/2 + j; the exact integer scores become the float matrix. */
    struct needleman_b200 : public pairwise::algorithm
    {
        auto run(const pairwise::context& ctx) const -> pairwise::distance_matrix override
        {
            const size_t n = ctx.db.count();
            std::vector<uint8_t> units;
            std::vector<uint64_t> offs(n), lens(n);
            for(size_t k = 0; k < n; ++k) {
                const sequence& s = ctx.db[(ptrdiff_t) k].contents;
                offs[k] = units.size();
                lens[k] = s.length();
                for(size_t i = 0; i < s.length(); ++i) units.push_back((uint8_t) s[(ptrdiff_t) i]);
            }
            const msa_table t = to_msa_table(ctx.table);
            msa_ctx *c = b200_context();
            msa_seqs h = 0;
            int rc = msa_seqs_upload(c, units.data(), offs.data(), lens.data(), (uint32_t) n, &h);
            check(rc == MSA_OK, "sequence upload failed", msa_last_error(c));
            std::vector<int32_t> tri(n * (n ? n - 1 : 0) / 2);
            rc = msa_nw_all_pairs(c, h, &t, MSA_NW_PERSISTENT, tri.data(), 0);
            msa_seqs_release(c, h);
            check(rc == MSA_OK, "pairwise scoring failed", msa_last_error(c));
            return pairwise::distance_matrix {std::vector<pairwise::score>(tri.begin(), tri.end()), n};
        }
    };

    /* phylogeny::algorithm on the B200, in the symmetric or linear removal
     * order: the packed triangle goes to msa_nj_order; the joins come back as
     * the 2n-1 nodes, which are replayed into the reference's star tree in
     * join order (star::join, src/phylogeny/njoining/star.cuh:61-72). */
    struct njoining_b200 : public phylogeny::algorithm
    {
        int order;
        explicit njoining_b200(int o) : order(o) {}

        auto run(const phylogeny::context& ctx) const -> phylogeny::guidetree override
        {
            const uint32_t n = (uint32_t) ctx.count;
            if(n < 2) return phylogeny::guidetree {};
            std::vector<float> tri((size_t) n * (n - 1) / 2);
            for(size_t i = 1; i < n; ++i)
                for(size_t j = 0; j < i; ++j)
                    tri[i * (i - 1) / 2 + j] = ctx.matrix[{i, j}];
            std::vector<msa_otu> nodes(2 * (size_t) n - 1);
            msa_ctx *c = b200_context();
            const int rc = msa_nj_order(c, tri.data(), MSA_TRI_F32_HOST, n, order, nodes.data());
            check(rc == MSA_OK, "neighbor-joining failed", msa_last_error(c));
            auto tree = phylogeny::njoining::star::make(n);
            for(uint32_t p = n; p < 2 * n - 1; ++p) {
                const uint32_t a = nodes[p].child[0], b = nodes[p].child[1];
                tree.join(p, {a, nodes[a].distance}, {b, nodes[b].distance});
            }
            return tree;
        }
    };

    museqa::database make_db(int n, const char *const *seqs, const uint64_t *lens)
    {
        museqa::database db;
        for(int i = 0; i < n; ++i)
            db.add("s" + std::to_string(i), museqa::sequence {seqs[i], (size_t) lens[i]});
        return db;
    }

    void write_tree(const phylogeny::guidetree& tree, uint32_t nodes, uint32_t *out5)
    {
        for(uint32_t r = 0; r < nodes; ++r) {
            const auto& node = tree[r];
            float d = node.distance;
            out5[5 * r + 0] = node.parent;
            out5[5 * r + 1] = node.child[0];
            out5[5 * r + 2] = node.child[1];
            std::memcpy(&out5[5 * r + 3], &d, 4);
            out5[5 * r + 4] = node.level;
        }
    }
}

extern "C" {

const char *b200_ref_last_error(void) { return last_error.c_str(); }

/* Scores the n strings with the needleman_b200 algorithm object
 * (out_b200) and with pairwise::run(db, table, "sequential") (out_seq),
 * both at i(i-1)/2 + j. */
int b200_ref_nw_all_pairs(int n, const char *const *seqs, const uint64_t *lens, const char *table,
                          float *out_b200, float *out_seq)
try {
    auto db = make_db(n, seqs, lens);
    auto tbl = pairwise::scoring_table::make(table);
    const pairwise::algorithm *algo = new needleman_b200;
    auto dm = algo->run({db, tbl});
    delete algo;
    auto ref = pairwise::run(db, tbl, "sequential");
    for(size_t i = 1; i < (size_t) n; ++i)
        for(size_t j = 0; j < i; ++j) {
            out_b200[i * (i - 1) / 2 + j] = dm[{i, j}];
            out_seq[i * (i - 1) / 2 + j] = ref[{i, j}];
        }
    return 0;
} catch(const std::exception& e) {
    last_error = e.what();
    return -1;
}

/* Builds the guide tree of the packed triangle with the njoining_b200
 * algorithm object (linear != 0: the linear removal order) and with the
 * reference's phylogeny::run under `ref_name`; writes 2n-1 nodes of 5 words
 * (parent, child0, child1, distance bits, level) for each. */
int b200_ref_nj(int n, const float *tri, int linear, const char *ref_name, uint32_t *out_b200, uint32_t *out_ref)
try {
    std::vector<float> v(tri, tri + (size_t) n * (n - 1) / 2);
    pairwise::distance_matrix dm {v, (size_t) n};
    const phylogeny::algorithm *algo = new njoining_b200(linear ? MSA_NJ_LINEAR : MSA_NJ_SYMMETRIC);
    auto tree = algo->run({dm, (size_t) n});
    delete algo;
    auto ref = phylogeny::run(dm, (size_t) n, ref_name);
    if(n < 2) return 0;
    write_tree(tree, (uint32_t) (2 * n - 1), out_b200);
    write_tree(ref, (uint32_t) (2 * n - 1), out_ref);
    return 0;
} catch(const std::exception& e) {
    last_error = e.what();
    return -1;
}

}
