// Prints the records the C++ facade's FASTA loader reads from the files given
// (one "description<TAB>decoded units" line each), for comparison with the
// Python loader. Touches no device.
#include <cstdio>
#include <vector>

#include "msa_b200.hpp"

int main(int argc, char **argv)
try {
    std::vector<std::string> files(argv + 1, argv + argc);
    const msa_b200::database db = msa_b200::io::load(files);
    for(const auto &e : db) std::printf("%s\t%s\n", e.description.c_str(), e.contents.str().c_str());
    return 0;
} catch(const std::exception &e) {
    std::printf("error\t%s\n", e.what());
    return 1;
}
