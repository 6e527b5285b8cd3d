// FASTA straight to the device store: one pass over each file that parses the
// records and encodes their letters into the flattened units, then one upload.
// The record rules are the reference's parser::fasta
// (src/io/loader/parser/fasta.cpp:26-70) run over an input stream:
//   * lines are split at '\n' only ('\r' stays in the line);
//   * a record starts at a line whose first character is '>' (its
//     description is the rest of that line); lines before it are skipped;
//   * its contents are the following lines, concatenated, up to the next
//     line that starts with '>' or the first empty line; lines after an
//     empty line up to the next '>' line are skipped;
//   * a file's extension picks the parser (src/io/loader/database.cpp:31-52):
//     "fa" and "fasta" only.
// Letters become encoder units as encoder::encode does (src/encoder.cpp:46-57).
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "msa_internal.hpp"

namespace msa {

namespace {

struct Parsed {
    std::vector<uint8_t> units;
    std::vector<uint64_t> offs, lens;
    std::vector<std::string> names;
    std::string error;
};

bool read_file(const char *path, std::string &out)
{
    FILE *f = std::fopen(path, "rb");
    if(!f) return false;
    char buf[1 << 16];
    size_t k;
    while((k = std::fread(buf, 1, sizeof(buf), f)) > 0) out.append(buf, k);
    std::fclose(f);
    return true;
}

std::string extension(const std::string &name)
{
    const size_t dot = name.rfind('.');
    return dot == std::string::npos ? name : name.substr(dot + 1);
}

int parse(const char *const *files, uint32_t nfiles, Parsed &p)
{
    for(uint32_t f = 0; f < nfiles; ++f) {
        if(!files[f]) return MSA_ERR_INVALID;
        const std::string name = files[f];
        const std::string ext = extension(name);
        if(ext != "fa" && ext != "fasta") {
            p.error = "unknown database parser '" + ext + "'";
            return MSA_ERR_INVALID;
        }
        std::string data;
        if(!read_file(files[f], data)) {
            p.error = "file does not exist or cannot be read '" + name + "'";
            return MSA_ERR_INVALID;
        }
        const char *s = data.data();
        const size_t n = data.size();
        size_t pos = 0;
        // Next line [b, e) and the position after its '\n'.
        auto line = [&](size_t at, size_t &b, size_t &e) {
            b = at;
            const void *nl = std::memchr(s + at, '\n', n - at);
            e = nl ? (size_t) ((const char *) nl - s) : n;
            return nl ? e + 1 : n;
        };
        while(pos < n) {
            size_t b, e;
            // Skip to a '>' line.
            size_t next = line(pos, b, e);
            while(!(e > b && s[b] == '>')) {
                pos = next;
                if(pos >= n) break;
                next = line(pos, b, e);
            }
            if(pos >= n && !(e > b && s[b] == '>')) break;
            p.names.emplace_back(s + b + 1, e - b - 1);
            pos = next;
            p.offs.push_back(p.units.size());
            uint64_t len = 0;
            while(pos < n && s[pos] != '>') {
                next = line(pos, b, e);
                if(e == b) {   // an empty line ends the record
                    pos = next;
                    break;
                }
                const size_t at = p.units.size();
                p.units.resize(at + (e - b));
                msa_encode(s + b, e - b, p.units.data() + at);
                len += e - b;
                pos = next;
            }
            p.lens.push_back(len);
        }
    }
    return MSA_OK;
}

}  // namespace

}  // namespace msa

extern "C" {

int msa_fasta_count(const char *const *files, uint32_t nfiles, uint32_t *nseqs, uint64_t *nunits)
{
    if((!files && nfiles) || !nseqs || !nunits) return MSA_ERR_INVALID;
    try {
        msa::Parsed p;
        const int rc = msa::parse(files, nfiles, p);
        if(rc) return rc;
        if(p.lens.size() > 0xffffffffu) return MSA_ERR_TOO_LARGE;
        *nseqs = (uint32_t) p.lens.size();
        *nunits = p.units.size();
        return MSA_OK;
    } catch(const std::bad_alloc &) {
        return MSA_ERR_NOMEM;
    }
}

int msa_fasta_encode(const char *const *files, uint32_t nfiles, uint8_t *units, uint64_t *offs, uint64_t *lens)
{
    if(!files && nfiles) return MSA_ERR_INVALID;
    try {
        msa::Parsed p;
        const int rc = msa::parse(files, nfiles, p);
        if(rc) return rc;
        if(!p.units.empty()) {
            if(!units) return MSA_ERR_INVALID;
            std::memcpy(units, p.units.data(), p.units.size());
        }
        if(!p.lens.empty()) {
            if(!offs || !lens) return MSA_ERR_INVALID;
            std::memcpy(offs, p.offs.data(), p.offs.size() * sizeof(uint64_t));
            std::memcpy(lens, p.lens.data(), p.lens.size() * sizeof(uint64_t));
        }
        return MSA_OK;
    } catch(const std::bad_alloc &) {
        return MSA_ERR_NOMEM;
    }
}

int msa_seqs_load_fasta(msa_ctx *ctx, const char *const *files, uint32_t nfiles, msa_seqs *out, uint32_t *count)
{
    if(!ctx || !out || (!files && nfiles)) return MSA_ERR_INVALID;
    try {
        msa::Parsed p;
        int rc = msa::parse(files, nfiles, p);
        if(rc) return msa::set_error(ctx, rc, p.error.empty() ? "cannot parse the FASTA input" : p.error);
        if(p.lens.size() > 0xffffffffu) return msa::set_error(ctx, MSA_ERR_TOO_LARGE, "too many sequences");
        const uint32_t n = (uint32_t) p.lens.size();
        rc = msa_seqs_upload(ctx, p.units.data(), p.offs.data(), p.lens.data(), n, out);
        if(rc) return rc;
        auto it = ctx->stores.find(*out);
        if(it != ctx->stores.end()) it->second->names = std::move(p.names);
        if(count) *count = n;
        return MSA_OK;
    } catch(const std::bad_alloc &) {
        return msa::set_error(ctx, MSA_ERR_NOMEM, "host allocation failed");
    }
}

const char *msa_seqs_description(msa_ctx *ctx, msa_seqs seqs, uint32_t index)
{
    if(!ctx) return nullptr;
    auto it = ctx->stores.find(seqs);
    if(it == ctx->stores.end() || index >= it->second->names.size()) return nullptr;
    return it->second->names[index].c_str();
}

}  // extern "C"
