/*
 * Test infrastructure only: an extern "C" harness around the reference's own
 * CPU implementation (Museqa, compiled from its sources by oracle/Makefile).
 * Nothing in the product links or loads this file; only tests/, the smoke
 * check and bench.py's CPU-baseline leg call it, and only as the checker.
 *
 * Entry points drive the reference exactly the way its Python test harness
 * does (src/python/pairwise.pyx:88-98 -> museqa::pairwise::run), with the
 * "sequential" algorithms, i.e. needleman::sequential
 * (src/pairwise/needleman/impl/sequential.cpp:29-122) and
 * njoining::sequential_symmetric (src/phylogeny/njoining/impl/sequential.cpp:80-346).
 */
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "database.hpp"
#include "encoder.hpp"
#include "sequence.hpp"
#include "pairwise.cuh"
#include "phylogeny.cuh"
#include "io/loader/database.hpp"

/*
 * Array allocations are zero-filled. The reference's NJ row-sum cache is built
 * by `new float[n]` and only entries 0..n-2 are cleared before accumulation
 * (src/phylogeny/njoining/impl/sequential.cpp:83-85), so S[n-1] would start
 * from whatever the allocator returns. Zero-filling makes the harness
 * deterministic and equal to the evidently intended S[n-1] = 0 start.
 */
void *operator new[](std::size_t size)
{
    void *p = std::calloc(1, size ? size : 1);
    if(!p) throw std::bad_alloc {};
    return p;
}
void operator delete[](void *p) noexcept { std::free(p); }
void operator delete[](void *p, std::size_t) noexcept { std::free(p); }

namespace
{
    thread_local std::string last_error;

    museqa::database make_db(int n, const char *const *seqs, const uint64_t *lens)
    {
        museqa::database db;
        for(int i = 0; i < n; ++i)
            db.add("s" + std::to_string(i), museqa::sequence {seqs[i], (size_t) lens[i]});
        return db;
    }
}

extern "C" {

const char *ref_last_error(void) { return last_error.c_str(); }

/* Encodes `len` characters with encoder::encode (src/encoder.cpp:76-98) into
 * ceil(len/3) blocks; returns the number of blocks written. */
int64_t ref_encode(const char *str, uint64_t len, uint16_t *out_blocks)
{
    auto buf = museqa::encoder::encode(str, (size_t) len);
    for(size_t i = 0; i < buf.size(); ++i) out_blocks[i] = buf[i];
    return (int64_t) buf.size();
}

/* Unit at `offset` of the padded sequence built from `str` (sequence.hpp:82-85). */
int ref_unit_at(const char *str, uint64_t len, uint64_t offset)
{
    museqa::sequence s {str, (size_t) len};
    return (int) s[(ptrdiff_t) offset];
}

/* Scores all n(n-1)/2 pairs with pairwise::run(db, table, "sequential");
 * out[i(i-1)/2 + j] for i > j (pairwise/pairwise.cuh:99-107). */
int ref_nw_all_pairs(int n, const char *const *seqs, const uint64_t *lens,
                     const char *table, float *out)
try {
    auto db = make_db(n, seqs, lens);
    auto tbl = museqa::pairwise::scoring_table::make(table);
    auto dm = museqa::pairwise::run(db, tbl, "sequential");
    for(int i = 1; i < n; ++i)
        for(int j = 0; j < i; ++j)
            out[(int64_t) i * (i - 1) / 2 + j] = dm[{(size_t) i, (size_t) j}];
    return 0;
} catch(const std::exception& e) {
    last_error = e.what();
    return -1;
}

/* Scores an explicit list of pairs (first > second index into `seqs`), each
 * as a two-entry database {seqs[second], seqs[first]} so that the reference's
 * row/column role assignment (sequential.cpp:84-91) is the one it would use in
 * the full database. Runs on `threads` host threads, each owning a
 * contiguous slice of the list. */
int ref_nw_pairs(const char *const *seqs, const uint64_t *lens,
                 const int32_t *first, const int32_t *second, int64_t npairs,
                 const char *table, int threads, float *out)
try {
    auto tbl = museqa::pairwise::scoring_table::make(table);
    if(threads < 1) threads = 1;
    std::atomic<int> failed {0};
    std::vector<std::thread> pool;
    for(int t = 0; t < threads; ++t) {
        pool.emplace_back([&, t]() {
            const int64_t lo = npairs * t / threads, hi = npairs * (t + 1) / threads;
            try {
                for(int64_t k = lo; k < hi; ++k) {
                    museqa::database db;
                    const int32_t a = first[k], b = second[k];
                    db.add("b", museqa::sequence {seqs[b], (size_t) lens[b]});
                    db.add("a", museqa::sequence {seqs[a], (size_t) lens[a]});
                    auto dm = museqa::pairwise::run(db, tbl, "sequential");
                    out[k] = dm[{(size_t) 1, (size_t) 0}];
                }
            } catch(...) { failed = 1; }
        });
    }
    for(auto& th : pool) th.join();
    if(failed) { last_error = "reference pair scoring failed"; return -1; }
    return 0;
} catch(const std::exception& e) {
    last_error = e.what();
    return -1;
}

/* Builds the guide tree with phylogeny::run(dm, n, algorithm) over the packed
 * lower-triangle `tri` (n(n-1)/2 floats, index i(i-1)/2 + j). Writes the
 * 2n-1 nodes (star.cuh:61-72, phylogeny.cuh:171-180, hierarchy.hpp:46-47). */
int ref_nj(int n, const float *tri, const char *algorithm,
           uint32_t *parent, uint32_t *child0, uint32_t *child1,
           float *distance, uint32_t *level)
try {
    std::vector<float> v(tri, tri + (size_t) n * (n - 1) / 2);
    museqa::pairwise::distance_matrix dm {v, (size_t) n};
    auto tree = museqa::phylogeny::run(dm, (size_t) n, algorithm);
    if(n < 2) return 0;
    for(uint32_t r = 0; r < (uint32_t) (2 * n - 1); ++r) {
        const auto& node = tree[r];
        parent[r] = node.parent;
        child0[r] = node.child[0];
        child1[r] = node.child[1];
        distance[r] = node.distance;
        level[r] = node.level;
    }
    return 0;
} catch(const std::exception& e) {
    last_error = e.what();
    return -1;
}

/* Loads a FASTA file with the reference's parser (io/loader/parser/fasta.cpp:58-70).
 * Returns the sequence count; descriptions and decoded contents are written
 * NUL-separated into the caller's buffers (sizes checked). */
int64_t ref_fasta(const char *filename, char *descs, uint64_t descs_cap,
                  char *contents, uint64_t contents_cap)
try {
    auto db = museqa::io::parser::fasta(filename);
    uint64_t dpos = 0, cpos = 0;
    for(size_t i = 0; i < db.count(); ++i) {
        const auto& e = db[(ptrdiff_t) i];
        std::string c = e.contents.decode();
        if(dpos + e.description.size() + 1 > descs_cap) { last_error = "descs"; return -2; }
        if(cpos + c.size() + 1 > contents_cap) { last_error = "contents"; return -2; }
        std::memcpy(descs + dpos, e.description.c_str(), e.description.size() + 1);
        std::memcpy(contents + cpos, c.c_str(), c.size() + 1);
        dpos += e.description.size() + 1;
        cpos += c.size() + 1;
    }
    return (int64_t) db.count();
} catch(const std::exception& e) {
    last_error = e.what();
    return -1;
}

/* Scoring table entry and penalty as the reference holds them (table.cu:254-262). */
int ref_table(const char *name, float *out625, float *penalty)
try {
    auto t = museqa::pairwise::scoring_table::make(name);
    for(int x = 0; x < 25; ++x)
        for(int y = 0; y < 25; ++y)
            out625[x * 25 + y] = t[{(size_t) x, (size_t) y}];
    *penalty = t.penalty();
    return 0;
} catch(const std::exception& e) {
    last_error = e.what();
    return -1;
}

}

extern "C" {

/* scoring_table::list / pairwise::algorithm::list / phylogeny::algorithm::list
 * (table.cu:327-330, pairwise/pairwise.cpp:309-312, phylogeny/phylogeny.cpp:329-332),
 * written NUL-separated; returns the count. */
static int64_t join_names(const std::vector<std::string>& v, char *buf, uint64_t cap)
{
    uint64_t pos = 0;
    for(const auto& s : v) {
        if(pos + s.size() + 1 > cap) return -2;
        std::memcpy(buf + pos, s.c_str(), s.size() + 1);
        pos += s.size() + 1;
    }
    return (int64_t) v.size();
}

int64_t ref_table_list(char *buf, uint64_t cap)
{ return join_names(museqa::pairwise::scoring_table::list(), buf, cap); }

int64_t ref_pairwise_list(char *buf, uint64_t cap)
{ return join_names(museqa::pairwise::algorithm::list(), buf, cap); }

int64_t ref_phylogeny_list(char *buf, uint64_t cap)
{ return join_names(museqa::phylogeny::algorithm::list(), buf, cap); }

}
