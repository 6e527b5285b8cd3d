// museqa: the command line of the reference (src/museqa.cpp:31-39, :210-272)
// over the B200 library: the same options, the same module order (loading,
// pairwise, phylogeny, pgalign) and the same "[watchdog|...]" lines, with the
// distance matrix kept on the device between pairwise and phylogeny.
//
// Options are matched exactly, as the reference's terminal::parse does
// (src/terminal.cpp:22-46): a known flag is an option, anything else an input
// file; an option that takes a value takes the next argument.
#include <chrono>
#include <cstdio>
#include <fstream>
#include <map>
#include <string>
#include <vector>

#include "msa_b200.hpp"

using namespace msa_b200;

namespace {

struct option {
    std::string name;
    std::vector<std::string> flags;
    std::string description;
    bool takes_value;
};

const std::vector<option> options = {
    {"multigpu", {"-m", "--multigpu"}, "Use multiple devices in a single host if possible.", false},
    {"report-only", {"-r", "--report-only"}, "Print only timing reports and nothing else.", false},
    {"gpu-id", {"-d", "--device"}, "Picks the GPU to be used on hosts with more than one.", true},
    {"scoring-table", {"-s", "--scoring-table"}, "The scoring table name or file to align sequences with.", true},
    {"pairwise", {"-1", "--pairwise"}, "Picks the algorithm to use within the pairwise module.", true},
    {"phylogeny", {"-2", "--phylogeny"}, "Picks the algorithm to use within the phylogeny module.", true},
    {"pgalign", {"-3", "--pgalign"}, "Picks the algorithm to use within the profile-aligner.", true},
    // Output options of this build (the reference registers no dumpers).
    {"newick", {"--newick"}, "Writes the guide tree, in Newick format, to the given file.", true},
    {"matrix", {"--matrix"}, "Writes the distance matrix (binary int32 triangle) to the given file.", true},
    {"help", {"-h", "--help"}, "Prints this help.", false},
};

struct command {
    std::vector<std::string> positional;
    std::map<std::string, std::vector<std::string>> parsed;
    bool has(const std::string &name) const
    {
        auto it = parsed.find(name);
        return it != parsed.end() && !it->second.empty();
    }
    std::string get(const std::string &name, const std::string &fallback) const
    {
        return has(name) ? parsed.at(name).front() : fallback;
    }
};

command parse(int argc, char **argv)
{
    std::map<std::string, const option *> by_flag;
    for(const option &o : options)
        for(const std::string &f : o.flags) by_flag[f] = &o;
    command cmd;
    for(int i = 1; i < argc; ++i) {
        auto it = by_flag.find(argv[i]);
        if(it == by_flag.end()) {
            cmd.positional.push_back(argv[i]);
            continue;
        }
        if(it->second->takes_value && ++i >= argc)
            throw exception("missing argument value for option '" + it->first + "'");
        cmd.parsed[it->second->name].push_back(argv[i]);
    }
    return cmd;
}

void usage()
{
    std::printf("usage: museqa [options] files...\n\noptions:\n");
    for(const option &o : options) {
        std::string flags;
        for(const auto &f : o.flags) flags += (flags.empty() ? "" : ", ") + f;
        std::printf("  %-24s %s\n", (flags + (o.takes_value ? " <value>" : "")).c_str(), o.description.c_str());
    }
}

double seconds_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Binary distance matrix: "MSAT", uint32 count, then count(count-1)/2 int32
// scores at i(i-1)/2+j (little endian).
void write_matrix(const std::string &path, const pairwise::distance_matrix &dm)
{
    std::ofstream f(path, std::ios::binary);
    if(!f) throw exception("cannot write '" + path + "'");
    const uint32_t n = (uint32_t) dm.count();
    f.write("MSAT", 4);
    f.write(reinterpret_cast<const char *>(&n), 4);
    const auto &s = dm.scores();
    f.write(reinterpret_cast<const char *>(s.data()), (std::streamsize) (s.size() * 4));
}

}  // namespace

int main(int argc, char **argv)
try {
    const auto t_total = std::chrono::steady_clock::now();
    const command cmd = parse(argc, argv);
    if(cmd.has("help")) {
        usage();
        return 0;
    }
    if(cmd.positional.empty()) throw exception("no input files given");
    watchdog::report_only = cmd.has("report-only");

    const std::string pw_algo = cmd.get("pairwise", "default");
    const std::string table_name = cmd.get("scoring-table", "default");
    const std::string pg_algo = cmd.get("phylogeny", "default");
    // The modules' option checks (src/pairwise.cpp:43-55, src/phylogeny.cpp:38-47).
    if(!pairwise::algorithm::has(pw_algo)) throw exception("unknown pairwise algorithm chosen: '" + pw_algo + "'");
    if(!pairwise::scoring_table::has(table_name)) throw exception("unknown scoring table chosen: '" + table_name + "'");
    if(!phylogeny::algorithm::has(pg_algo)) throw exception("unknown phylogeny algorithm chosen: '" + pg_algo + "'");

    const int ndev = device::count();
    if(ndev < 1) throw exception("no CUDA device found");
    device::select(cmd.has("gpu-id") ? std::stoi(cmd.get("gpu-id", "0")) % ndev : 0);
    const int devices = cmd.has("multigpu") ? ndev : 1;

    // loading: one device goes straight from the files to a device store;
    // several devices take the host database and split the job.
    auto t0 = std::chrono::steady_clock::now();
    database host_db;
    device_database dev_db;
    std::vector<std::string> names;
    if(devices > 1) {
        host_db = io::load(cmd.positional);
        for(const auto &e : host_db) names.push_back(e.description);
    } else {
        dev_db = io::load_to_device(cmd.positional);
        names = dev_db.descriptions();
    }
    const size_t count = names.size();
    if(count > 0) watchdog::info("loaded a total of <bold>" + std::to_string(count) + "</> sequences");
    watchdog::report("loading", seconds_since(t0));

    // pairwise
    t0 = std::chrono::steady_clock::now();
    watchdog::info("chosen pairwise algorithm <bold>" + pw_algo + "</>");
    watchdog::info("chosen pairwise scoring table <bold>" + table_name + "</>");
    const unsigned long long npairs = (unsigned long long) count * (count ? count - 1 : 0) / 2;
    watchdog::init("pairwise", "aligning <bold>" + std::to_string(npairs) + "</> pairs");
    const auto table = pairwise::scoring_table::make(table_name);
    const pairwise::distance_matrix dm =
        devices > 1 ? pairwise::run(host_db, table, pw_algo, devices) : pairwise::run(dev_db, table, pw_algo);
    watchdog::finish("pairwise", "aligned all sequence pairs");
    watchdog::report("pairwise", seconds_since(t0));

    // phylogeny
    t0 = std::chrono::steady_clock::now();
    watchdog::info("chosen phylogeny algorithm <bold>" + pg_algo + "</>");
    watchdog::init("phylogeny", "producing phylogenetic tree");
    const phylogeny::guidetree tree = phylogeny::run(dm, count, pg_algo);
    watchdog::finish("phylogeny", "phylogenetic tree produced");
    watchdog::report("phylogeny", seconds_since(t0));

    // pgalign: the profile aligner is outside this build.
    watchdog::warning("the profile-aligner module is not part of this build; the pipeline ends at the guide tree");

    if(cmd.has("newick")) {
        std::ofstream f(cmd.get("newick", ""));
        if(!f) throw exception("cannot write '" + cmd.get("newick", "") + "'");
        f << tree.newick(names) << "\n";
    }
    if(cmd.has("matrix")) write_matrix(cmd.get("matrix", ""), dm);

    watchdog::report("total", seconds_since(t_total));
    return 0;
} catch(const std::exception &e) {
    watchdog::error(e.what());
    return 1;
}
