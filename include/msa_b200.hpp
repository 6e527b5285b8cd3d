/*
 * C++ facade of libmsa_b200: the reference's C++ API for the pairwise and
 * phylogeny steps, over the C ABI of msa_b200.h. Class and function names
 * follow the reference so that code written against Museqa reads the same:
 *
 *   museqa::encoder            src/encoder.hpp:24-77
 *   museqa::sequence           src/sequence.hpp:24-129
 *   museqa::database           src/database.hpp:25-210
 *   museqa::io (FASTA loader)  src/io/loader/parser/fasta.cpp:26-70,
 *                              src/io/loader/database.cpp:31-52
 *   museqa::pairwise           src/pairwise/pairwise.cuh:53-244
 *   museqa::phylogeny          src/phylogeny/phylogeny.cuh:45-258
 *   museqa::watchdog           src/museqa.hpp:68-161
 *
 * Errors are thrown as msa_b200::exception (museqa::exception), with the
 * reference's messages where it has one. The distance matrix of a pairwise
 * run stays on the device that scored it, and phylogeny::run reads it there;
 * its host copy is made only when asked for.
 */
#pragma once

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "msa_b200.h"

namespace msa_b200 {

class exception : public std::runtime_error
{
  public:
    using std::runtime_error::runtime_error;
};

namespace encoder {
using unit = uint8_t;
constexpr unit end = MSA_UNIT_END;
constexpr unit gap = MSA_UNIT_GAP;
unit encode(char c);
char decode(unit u);
std::vector<unit> encode(const std::string &text);   // one unit per character, unpadded
std::string decode(const std::vector<unit> &units);
}  // namespace encoder

/* An encoded sequence, padded with `end` units to whole 3-unit blocks. */
class sequence
{
  public:
    sequence() = default;
    explicit sequence(const std::string &contents);
    explicit sequence(std::vector<encoder::unit> units);
    size_t length() const { return m_units.size(); }      // padded: 3 * blocks
    size_t size() const { return m_units.size() / 3; }    // blocks
    encoder::unit operator[](size_t offset) const;
    const std::vector<encoder::unit> &units() const { return m_units; }
    std::string str() const { return encoder::decode(m_units); }

  private:
    std::vector<encoder::unit> m_units;
};

class database
{
  public:
    struct entry {
        std::string description;
        msa_b200::sequence contents;
    };

    void add(const std::string &description, const std::string &contents);
    void add(const std::string &description, const sequence &contents);
    void merge(const database &other);
    size_t count() const { return m_entries.size(); }
    const entry &operator[](size_t offset) const;
    const entry &operator[](const std::string &description) const;
    std::vector<entry>::const_iterator begin() const { return m_entries.begin(); }
    std::vector<entry>::const_iterator end() const { return m_entries.end(); }

  private:
    std::vector<entry> m_entries;
    std::vector<std::pair<std::string, size_t>> m_index;
};

/* Sequences resident on the current device (a store of msa_seqs_load_fasta),
 * with their descriptions: the fast path from FASTA files to the pairwise
 * step, with no host database in between. */
class device_database
{
  public:
    device_database() = default;
    device_database(const device_database &) = delete;
    device_database &operator=(const device_database &) = delete;
    device_database(device_database &&o) noexcept { *this = std::move(o); }
    device_database &operator=(device_database &&o) noexcept;
    ~device_database();
    size_t count() const { return m_count; }
    int device() const { return m_device; }
    msa_seqs handle() const { return m_handle; }
    const std::vector<std::string> &descriptions() const { return m_names; }

  private:
    friend device_database load_to_device_impl(const std::vector<std::string> &);
    int m_device = -1;
    msa_seqs m_handle = 0;
    size_t m_count = 0;
    std::vector<std::string> m_names;
};

namespace io {
/* parser::fasta: records from '>' lines; a record's contents are the lines up
 * to the next '>' line or the first empty line. */
database fasta(const std::string &filename);
/* The loader by file extension ("fa", "fasta"); throws "unknown database
 * parser '<ext>'" otherwise. Files are merged in order. */
database load(const std::vector<std::string> &filenames);
/* The same files parsed, encoded and uploaded in one pass onto the current
 * device (msa_seqs_load_fasta). */
device_database load_to_device(const std::vector<std::string> &filenames);
}  // namespace io

/* The devices the facade runs on (cuda::device in the reference). */
namespace device {
int count();
void select(int id);   // device of the next runs in this thread
int current();
}  // namespace device

namespace pairwise {

class scoring_table
{
  public:
    static scoring_table make(const std::string &name);   // throws "unknown pairwise scoring table '<name>'"
    static bool has(const std::string &name);
    static std::vector<std::string> list();
    /* A caller table: 25 x 25 scores (unit row, unit column) and the penalty. */
    static scoring_table custom(const std::vector<int32_t> &scores, int32_t penalty);
    int32_t operator()(encoder::unit a, encoder::unit b) const { return m_t.score[a * 25 + b]; }
    int32_t penalty() const { return m_t.penalty; }
    const msa_table &raw() const { return m_t; }
    const std::string &name() const { return m_name; }

  private:
    msa_table m_t{};
    std::string m_name;
};

/* Packed strict lower triangle of n(n-1)/2 scores, entry i(i-1)/2+j for
 * i > j; (i, i) reads 0. Scores are exact integers. */
class distance_matrix
{
  public:
    distance_matrix() = default;
    distance_matrix(std::vector<int32_t> scores, size_t count);
    size_t count() const { return m_count; }
    float operator()(size_t a, size_t b) const;
    /* Host copy of the scores (downloaded once from the device if needed). */
    const std::vector<int32_t> &scores() const;
    /* The scores on the device that computed them, or nullptr. */
    const int32_t *device_scores() const;
    int device() const;

    struct storage;

  private:
    std::shared_ptr<storage> m_data;
    size_t m_count = 0;
    friend distance_matrix make_device_matrix(std::shared_ptr<storage>, size_t);
};

struct context {
    const database &db;
    const scoring_table &table;
};

struct algorithm {
    virtual ~algorithm() = default;
    virtual distance_matrix run(const context &ctx) const = 0;
    static bool has(const std::string &name);
    static std::unique_ptr<algorithm> make(const std::string &name);   // throws "unknown pairwise algorithm '<name>'"
    static std::vector<std::string> list();
};

/* pairwise::run. `devices` > 1 splits the job over devices 0..devices-1
 * (parts of equal DP cells, msa_nw_all_pairs_part) and assembles the matrix
 * on the current device. */
distance_matrix run(const database &db, const scoring_table &table, const std::string &algorithm = "default",
                    int devices = 1);
/* pairwise::run over sequences already resident on a device. */
distance_matrix run(const device_database &db, const scoring_table &table, const std::string &algorithm = "default");

}  // namespace pairwise

namespace phylogeny {

struct otu {
    uint32_t parent;
    uint32_t child[2];
    float distance;
    uint32_t level;
};

/* 2n-1 nodes: leaves 0..n-1, joins n..2n-2, the root last. */
class guidetree
{
  public:
    guidetree() = default;
    guidetree(std::vector<otu> nodes, size_t leaves) : m_nodes(std::move(nodes)), m_leaves(leaves) {}
    size_t count() const { return m_nodes.size(); }
    size_t leaves() const { return m_leaves; }
    const otu &operator[](size_t k) const { return m_nodes.at(k); }
    uint32_t root() const { return m_nodes.empty() ? 0xffffffffu : (uint32_t) (m_nodes.size() - 1); }
    /* Newick text; leaves named by `names` (their index when empty), branch
     * lengths as the shortest decimal that reads back as the same float. */
    std::string newick(const std::vector<std::string> &names = {}) const;

  private:
    std::vector<otu> m_nodes;
    size_t m_leaves = 0;
};

struct context {
    const pairwise::distance_matrix &matrix;
    size_t count;
};

struct algorithm {
    virtual ~algorithm() = default;
    virtual guidetree run(const context &ctx) const = 0;
    static bool has(const std::string &name);
    static std::unique_ptr<algorithm> make(const std::string &name);   // throws "unknown phylogeny algorithm '<name>'"
    static std::vector<std::string> list();
};

guidetree run(const pairwise::distance_matrix &matrix, size_t count, const std::string &algorithm = "default");

}  // namespace phylogeny

/* The reference's watchdog line protocol: "[watchdog|<event>|...]" lines. */
namespace watchdog {
extern bool report_only;
void info(const std::string &message);
void warning(const std::string &message);
void error(const std::string &message);
void init(const std::string &task, const std::string &message);
void finish(const std::string &task, const std::string &message);
void report(const std::string &task, double seconds);
}  // namespace watchdog

}  // namespace msa_b200
