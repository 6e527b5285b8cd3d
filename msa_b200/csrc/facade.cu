// The C++ facade (include/msa_b200.hpp) over the C ABI. Names, defaults and
// error messages follow the reference's C++ API; see the header for the map.
#include <cfloat>
#include <charconv>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <thread>

#include <cuda_runtime.h>

#include "msa_b200.hpp"

namespace msa_b200 {

namespace {

template <class... T>
std::string format(const char *fmt, T... args)
{
    const int n = std::snprintf(nullptr, 0, fmt, args...);
    std::string s((size_t) std::max(n, 0), '\0');
    std::snprintf(s.data(), s.size() + 1, fmt, args...);
    return s;
}

void check_status(int rc, msa_ctx *ctx = nullptr)
{
    if(rc == MSA_OK) return;
    std::string msg = msa_strerror(rc);
    if(ctx && msa_last_error(ctx) && *msa_last_error(ctx)) msg += std::string(": ") + msa_last_error(ctx);
    throw exception(msg);
}

void check_cuda(cudaError_t e, const char *what)
{
    if(e != cudaSuccess) throw exception(format("%s: %s", what, cudaGetErrorString(e)));
}

// One library context per device, created on first use and kept for the
// process (the OS reclaims it at exit).
msa_ctx *context_for(int dev)
{
    static std::mutex m;
    static std::vector<msa_ctx *> ctxs;
    std::lock_guard<std::mutex> lock(m);
    if(dev < 0) throw exception("invalid device");
    if((size_t) dev >= ctxs.size()) ctxs.resize(dev + 1, nullptr);
    if(!ctxs[dev]) {
        msa_ctx *c = nullptr;
        const int rc = msa_create(dev, &c);
        if(rc) throw exception(format("cannot use device %d: %s", dev, msa_strerror(rc)));
        ctxs[dev] = c;
    }
    return ctxs[dev];
}

thread_local int t_device = 0;

__global__ void accumulate_kernel(int32_t *out, const int32_t *part, uint64_t n)
{
    for(uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t) gridDim.x * blockDim.x)
        out[i] += part[i];
}

}  // namespace

// ------------------------------------------------------------------ encoder

namespace encoder {

unit encode(char c)
{
    uint8_t u = 0;
    check_status(msa_encode(&c, 1, &u));
    return u;
}

char decode(unit u)
{
    char c = 0;
    check_status(msa_decode(&u, 1, &c));
    return c;
}

std::vector<unit> encode(const std::string &text)
{
    std::vector<unit> out(text.size());
    if(!text.empty()) check_status(msa_encode(text.data(), text.size(), out.data()));
    return out;
}

std::string decode(const std::vector<unit> &units)
{
    std::string out(units.size(), '\0');
    if(!units.empty()) check_status(msa_decode(units.data(), units.size(), out.data()));
    return out;
}

}  // namespace encoder

// ------------------------------------------------------------------ sequence, database

sequence::sequence(const std::string &contents) : sequence(encoder::encode(contents)) {}

sequence::sequence(std::vector<encoder::unit> units) : m_units(std::move(units))
{
    while(m_units.size() % 3) m_units.push_back(encoder::end);
}

encoder::unit sequence::operator[](size_t offset) const
{
    if(offset >= m_units.size()) throw exception("sequence offset out of range");
    return m_units[offset];
}

void database::add(const std::string &description, const std::string &contents)
{
    add(description, sequence(contents));
}

void database::add(const std::string &description, const sequence &contents)
{
    m_index.emplace_back(description, m_entries.size());
    m_entries.push_back({description, contents});
}

void database::merge(const database &other)
{
    for(const entry &e : other.m_entries) add(e.description, e.contents);
}

const database::entry &database::operator[](size_t offset) const
{
    if(offset >= m_entries.size()) throw exception("database offset out of range");
    return m_entries[offset];
}

const database::entry &database::operator[](const std::string &description) const
{
    // The latest entry of that description wins, as with a key map.
    for(auto it = m_index.rbegin(); it != m_index.rend(); ++it)
        if(it->first == description) return m_entries[it->second];
    throw exception("cannot find key in database");
}

namespace io {

database fasta(const std::string &filename)
{
    std::ifstream file(filename);
    if(file.fail()) throw exception(format("file does not exist or cannot be read '%s'", filename.c_str()));
    database db;
    // One record per pass: skip to a '>' line (a record needs a description),
    // then gather the following lines until the next '>' or an empty line.
    while(!file.eof() && !file.fail()) {
        std::string line;
        bool found = true;
        while(line.empty() || line[0] != '>') {
            if(file.eof()) { found = false; break; }
            std::getline(file, line);
        }
        if(!found) break;
        const std::string description = line.substr(1);
        std::string contents;
        while(file.peek() != '>' && std::getline(file, line) && !line.empty()) contents += line;
        db.add(description, contents);
    }
    return db;
}

database load(const std::vector<std::string> &filenames)
{
    database all;
    for(const std::string &name : filenames) {
        const size_t dot = name.rfind('.');
        const std::string ext = dot == std::string::npos ? name : name.substr(dot + 1);
        if(ext != "fa" && ext != "fasta") throw exception(format("unknown database parser '%s'", ext.c_str()));
        all.merge(fasta(name));
    }
    return all;
}

}  // namespace io

// ------------------------------------------------------------------ devices

namespace device {

int count()
{
    int n = 0;
    if(cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

void select(int id)
{
    const int n = count();
    if(id < 0 || id >= n) throw exception(format("device %d is not available (%d found)", id, n));
    t_device = id;
}

int current() { return t_device; }

}  // namespace device

device_database &device_database::operator=(device_database &&o) noexcept
{
    if(this != &o) {
        std::swap(m_device, o.m_device);
        std::swap(m_handle, o.m_handle);
        std::swap(m_count, o.m_count);
        std::swap(m_names, o.m_names);
    }
    return *this;
}

device_database::~device_database()
{
    if(m_handle && m_device >= 0) {
        cudaSetDevice(m_device);
        msa_seqs_release(context_for(m_device), m_handle);
    }
}

device_database load_to_device_impl(const std::vector<std::string> &filenames)
{
    device_database db;
    const int dev = device::current();
    msa_ctx *c = context_for(dev);
    check_cuda(cudaSetDevice(dev), "select device");
    std::vector<const char *> names;
    for(const auto &f : filenames) names.push_back(f.c_str());
    uint32_t n = 0;
    msa_seqs h = 0;
    const int rc = msa_seqs_load_fasta(c, names.data(), (uint32_t) names.size(), &h, &n);
    if(rc) throw exception(msa_last_error(c) && *msa_last_error(c) ? msa_last_error(c) : msa_strerror(rc));
    db.m_device = dev;
    db.m_handle = h;
    db.m_count = n;
    for(uint32_t k = 0; k < n; ++k) {
        const char *d = msa_seqs_description(c, h, k);
        db.m_names.emplace_back(d ? d : "");
    }
    return db;
}

namespace io {
device_database load_to_device(const std::vector<std::string> &filenames) { return load_to_device_impl(filenames); }
}  // namespace io

// ------------------------------------------------------------------ pairwise

namespace pairwise {

scoring_table scoring_table::make(const std::string &name)
{
    scoring_table t;
    if(msa_table_make(name.c_str(), &t.m_t) != MSA_OK)
        throw exception(format("unknown pairwise scoring table '%s'", name.c_str()));
    t.m_name = name;
    return t;
}

bool scoring_table::has(const std::string &name) { return msa_table_has(name.c_str()) == 1; }

std::vector<std::string> scoring_table::list()
{
    const char *names[32];
    const int n = msa_table_list(names, 32);
    return std::vector<std::string>(names, names + std::min(n, 32));
}

scoring_table scoring_table::custom(const std::vector<int32_t> &scores, int32_t penalty)
{
    if(scores.size() != 625) throw exception("a scoring table has 25 x 25 entries");
    scoring_table t;
    std::memcpy(t.m_t.score, scores.data(), sizeof(t.m_t.score));
    t.m_t.penalty = penalty;
    t.m_t.index = -1;
    t.m_name = "custom";
    return t;
}

struct distance_matrix::storage {
    int device = -1;
    int32_t *dev = nullptr;
    std::mutex m;
    std::vector<int32_t> host;
    bool host_valid = false;
    ~storage()
    {
        if(dev) {
            cudaSetDevice(device);
            cudaFree(dev);
        }
    }
};

distance_matrix make_device_matrix(std::shared_ptr<distance_matrix::storage> s, size_t count)
{
    distance_matrix m;
    m.m_data = std::move(s);
    m.m_count = count;
    return m;
}

distance_matrix::distance_matrix(std::vector<int32_t> scores, size_t count) : m_count(count)
{
    if(scores.size() != count * (count ? count - 1 : 0) / 2) throw exception("distance matrix size mismatch");
    m_data = std::make_shared<storage>();
    m_data->host = std::move(scores);
    m_data->host_valid = true;
}

const std::vector<int32_t> &distance_matrix::scores() const
{
    static const std::vector<int32_t> empty;
    if(!m_data) return empty;
    std::lock_guard<std::mutex> lock(m_data->m);
    if(!m_data->host_valid) {
        const size_t np = m_count * (m_count ? m_count - 1 : 0) / 2;
        m_data->host.resize(np);
        check_cuda(cudaSetDevice(m_data->device), "select device");
        if(np) check_cuda(cudaMemcpy(m_data->host.data(), m_data->dev, np * 4, cudaMemcpyDeviceToHost), "download scores");
        m_data->host_valid = true;
    }
    return m_data->host;
}

float distance_matrix::operator()(size_t a, size_t b) const
{
    if(a == b) return 0.0f;
    const size_t hi = std::max(a, b), lo = std::min(a, b);
    if(hi >= m_count) throw exception("distance matrix offset out of range");
    return (float) scores()[hi * (hi - 1) / 2 + lo];
}

const int32_t *distance_matrix::device_scores() const { return m_data ? m_data->dev : nullptr; }

int distance_matrix::device() const { return m_data ? m_data->device : -1; }

namespace {

struct b200_needleman : algorithm {
    int mode;
    explicit b200_needleman(int m) : mode(m) {}
    distance_matrix run(const context &ctx) const override;
};

// The reference's pairwise names (src/pairwise/pairwise.cpp:26-35): the GPU
// names run the persistent batched kernel, the CPU/MPI names the plain one;
// both give the same scores.
const std::vector<std::pair<std::string, int>> &pairwise_names()
{
    static const std::vector<std::pair<std::string, int>> names = {
        {"default", MSA_NW_PERSISTENT},       {"distributed", MSA_NW_PLAIN},
        {"hybrid", MSA_NW_PERSISTENT},        {"needleman", MSA_NW_PERSISTENT},
        {"needleman-distributed", MSA_NW_PLAIN}, {"needleman-hybrid", MSA_NW_PERSISTENT},
        {"needleman-sequential", MSA_NW_PLAIN}, {"sequential", MSA_NW_PLAIN},
    };
    return names;
}

void flatten(const database &db, std::vector<uint8_t> &units, std::vector<uint64_t> &offs, std::vector<uint64_t> &lens)
{
    for(const auto &e : db) {
        offs.push_back(units.size());
        lens.push_back(e.contents.length());
        units.insert(units.end(), e.contents.units().begin(), e.contents.units().end());
    }
}

distance_matrix score(const database &db, const scoring_table &table, int mode, int devices)
{
    const size_t n = db.count();
    const uint64_t np = (uint64_t) n * (n ? n - 1 : 0) / 2;
    std::vector<uint8_t> units;
    std::vector<uint64_t> offs, lens;
    flatten(db, units, offs, lens);
    const int home = device::current();
    auto st = std::make_shared<distance_matrix::storage>();
    st->device = home;
    check_cuda(cudaSetDevice(home), "select device");
    check_cuda(cudaMalloc((void **) &st->dev, std::max<uint64_t>(np * 4, 16)), "allocate distance matrix");
    const int ndev = device::count();
    devices = std::max(1, std::min(devices, ndev));

    // Part p of `devices` on device p (home first); parts are zero-filled and
    // summed into the home device's matrix.
    auto run_part = [&](int dev, uint32_t part, int32_t *out) {
        msa_ctx *c = context_for(dev);
        check_cuda(cudaSetDevice(dev), "select device");
        msa_seqs h = 0;
        check_status(msa_seqs_upload(c, units.data(), offs.data(), lens.data(), (uint32_t) n, &h), c);
        const int rc = devices == 1 ? msa_nw_all_pairs(c, h, &table.raw(), mode, out, 1)
                                    : msa_nw_all_pairs_part(c, h, &table.raw(), mode, part, (uint32_t) devices, out, 1);
        msa_seqs_release(c, h);
        check_status(rc, c);
    };
    if(devices == 1) {
        run_part(home, 0, st->dev);
        return make_device_matrix(st, n);
    }
    check_cuda(cudaMemset(st->dev, 0, np * 4), "clear distance matrix");
    std::vector<int32_t *> bufs(devices, nullptr);
    std::vector<std::string> errors(devices);
    std::vector<std::thread> workers;
    for(int k = 0; k < devices; ++k) {
        const int dev = (home + k) % ndev;
        workers.emplace_back([&, k, dev] {
            try {
                check_cuda(cudaSetDevice(dev), "select device");
                check_cuda(cudaMalloc((void **) &bufs[k], np * 4), "allocate part");
                check_cuda(cudaMemset(bufs[k], 0, np * 4), "clear part");
                run_part(dev, (uint32_t) k, bufs[k]);
            } catch(const std::exception &e) {
                errors[k] = e.what();
            }
        });
    }
    for(auto &w : workers) w.join();
    std::string err;
    for(const auto &e : errors) if(!e.empty()) err = e;
    int32_t *staging = nullptr;
    if(err.empty()) {
        check_cuda(cudaSetDevice(home), "select device");
        check_cuda(cudaMalloc((void **) &staging, np * 4), "allocate staging");
        for(int k = 0; k < devices && err.empty(); ++k) {
            const int dev = (home + k) % ndev;
            const cudaError_t e = cudaMemcpyPeer(staging, home, bufs[k], dev, np * 4);
            if(e) { err = cudaGetErrorString(e); break; }
            accumulate_kernel<<<1024, 256>>>(st->dev, staging, np);
            if(cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) err = "accumulate parts";
        }
        cudaFree(staging);
    }
    for(int k = 0; k < devices; ++k) {
        if(bufs[k]) {
            cudaSetDevice((home + k) % ndev);
            cudaFree(bufs[k]);
        }
    }
    cudaSetDevice(home);
    if(!err.empty()) throw exception(err);
    return make_device_matrix(st, n);
}

distance_matrix b200_needleman::run(const context &ctx) const { return score(ctx.db, ctx.table, mode, 1); }

}  // namespace

bool algorithm::has(const std::string &name)
{
    for(const auto &p : pairwise_names()) if(p.first == name) return true;
    return false;
}

std::unique_ptr<algorithm> algorithm::make(const std::string &name)
{
    for(const auto &p : pairwise_names())
        if(p.first == name) return std::unique_ptr<algorithm>(new b200_needleman(p.second));
    throw exception(format("unknown pairwise algorithm '%s'", name.c_str()));
}

std::vector<std::string> algorithm::list()
{
    std::vector<std::string> out;
    for(const auto &p : pairwise_names()) out.push_back(p.first);
    return out;
}

distance_matrix run(const device_database &db, const scoring_table &table, const std::string &name)
{
    int mode = -1;
    for(const auto &p : pairwise_names())
        if(p.first == name) mode = p.second;
    if(mode < 0) throw exception(format("unknown pairwise algorithm '%s'", name.c_str()));
    const size_t n = db.count();
    const uint64_t np = (uint64_t) n * (n ? n - 1 : 0) / 2;
    auto st = std::make_shared<distance_matrix::storage>();
    st->device = db.device();
    check_cuda(cudaSetDevice(db.device()), "select device");
    check_cuda(cudaMalloc((void **) &st->dev, std::max<uint64_t>(np * 4, 16)), "allocate distance matrix");
    msa_ctx *c = context_for(db.device());
    check_status(msa_nw_all_pairs(c, db.handle(), &table.raw(), mode, st->dev, 1), c);
    return make_device_matrix(st, n);
}

distance_matrix run(const database &db, const scoring_table &table, const std::string &name, int devices)
{
    for(const auto &p : pairwise_names())
        if(p.first == name) return score(db, table, p.second, devices);
    throw exception(format("unknown pairwise algorithm '%s'", name.c_str()));
}

}  // namespace pairwise

// ------------------------------------------------------------------ phylogeny

namespace phylogeny {

namespace {

// The reference's phylogeny names (src/phylogeny/phylogeny.cpp:26-41). All
// run the device neighbor-joining; the four that select the linear matrix
// transform (lines 30, 33, 38, 40) in the linear removal order, which
// reproduces sequential_linear bit for bit, the others in the symmetric one
// (sequential_symmetric).
const std::vector<std::string> &phylogeny_names()
{
    static const std::vector<std::string> names = {
        "default", "distributed", "hybrid", "linear", "njoining", "njoining-distributed",
        "njoining-distributed-linear", "njoining-hybrid", "njoining-linear", "njoining-sequential",
        "njoining-sequential-linear", "njoining-symmetric", "sequential", "symmetric",
    };
    return names;
}

bool linear_name(const std::string &name)
{
    return name == "linear" || name == "njoining-linear" || name == "njoining-sequential-linear" ||
           name == "njoining-distributed-linear";
}

guidetree join(const pairwise::distance_matrix &matrix, size_t count, int order)
{
    if(count < 2) return guidetree({}, count);
    if(count != matrix.count()) throw exception("phylogeny count differs from the matrix's");
    std::vector<msa_otu> nodes(2 * count - 1);
    const int32_t *dev = matrix.device_scores();
    const int where = dev ? matrix.device() : device::current();
    msa_ctx *c = context_for(where);
    check_cuda(cudaSetDevice(where), "select device");
    const int rc = dev ? msa_nj_order(c, dev, MSA_TRI_I32_DEVICE, (uint32_t) count, order, nodes.data())
                       : msa_nj_order(c, matrix.scores().data(), MSA_TRI_I32_HOST, (uint32_t) count, order,
                                      nodes.data());
    check_status(rc, c);
    std::vector<otu> out(nodes.size());
    for(size_t k = 0; k < nodes.size(); ++k)
        out[k] = {nodes[k].parent, {nodes[k].child[0], nodes[k].child[1]}, nodes[k].distance, nodes[k].level};
    return guidetree(std::move(out), count);
}

struct b200_njoining : algorithm {
    int order;
    explicit b200_njoining(int o) : order(o) {}
    guidetree run(const context &ctx) const override { return join(ctx.matrix, ctx.count, order); }
};

}  // namespace

bool algorithm::has(const std::string &name)
{
    for(const auto &p : phylogeny_names()) if(p == name) return true;
    return false;
}

std::unique_ptr<algorithm> algorithm::make(const std::string &name)
{
    if(!has(name)) throw exception(format("unknown phylogeny algorithm '%s'", name.c_str()));
    return std::unique_ptr<algorithm>(new b200_njoining(linear_name(name) ? MSA_NJ_LINEAR : MSA_NJ_SYMMETRIC));
}

std::vector<std::string> algorithm::list() { return phylogeny_names(); }

guidetree run(const pairwise::distance_matrix &matrix, size_t count, const std::string &name)
{
    if(!algorithm::has(name)) throw exception(format("unknown phylogeny algorithm '%s'", name.c_str()));
    return join(matrix, count, linear_name(name) ? MSA_NJ_LINEAR : MSA_NJ_SYMMETRIC);
}

std::string guidetree::newick(const std::vector<std::string> &names) const
{
    if(m_nodes.empty()) return ";";
    std::string out;
    auto label = [&](uint32_t r) {
        if(r < m_leaves) out += r < names.size() ? names[r] : std::to_string(r);
    };
    auto length = [&](uint32_t r) {
        if(r == root()) return;
        char buf[64];
        const auto res = std::to_chars(buf, buf + sizeof(buf), m_nodes[r].distance);
        out += ':';
        out.append(buf, res.ptr);
    };
    // Iterative walk: (node, stage) with stage 0 = open, 1 = between, 2 = close.
    std::vector<std::pair<uint32_t, int>> stack{{root(), 0}};
    while(!stack.empty()) {
        auto &[r, stage] = stack.back();
        if(r < m_leaves) {
            label(r);
            length(r);
            stack.pop_back();
            continue;
        }
        if(stage == 0) {
            out += '(';
            stage = 1;
            stack.push_back({m_nodes[r].child[0], 0});
        } else if(stage == 1) {
            out += ',';
            stage = 2;
            stack.push_back({m_nodes[r].child[1], 0});
        } else {
            out += ')';
            const uint32_t done = r;
            stack.pop_back();
            length(done);
        }
    }
    return out + ";";
}

}  // namespace phylogeny

// ------------------------------------------------------------------ watchdog

namespace watchdog {

bool report_only = false;

static void notify(const char *event, const std::string &text)
{
    std::printf("[watchdog|%s|%s]\n", event, text.c_str());
    std::fflush(stdout);
}

void info(const std::string &message) { if(!report_only) notify("info", message); }
void warning(const std::string &message) { notify("warning", message); }
void error(const std::string &message) { notify("error", message); }
void init(const std::string &task, const std::string &message) { if(!report_only) notify("init", task + "|" + message); }
void finish(const std::string &task, const std::string &message) { if(!report_only) notify("finish", task + "|" + message); }
void report(const std::string &task, double seconds) { notify("report", format("%s|%lf", task.c_str(), seconds)); }

}  // namespace watchdog

}  // namespace msa_b200
