// Scoring tables, names and the unit encoder.
//
// Tables: the seven named tables of the reference (src/pairwise/table.cu:41-262),
// same names, penalties and entries, kept in the same storage order because
// the reference's GAP-unit reads land in the next row/table of that storage.
// Encoder: the char -> unit map of src/encoder.cpp:27-57 and the 3-units-per-
// uint16 packing of src/encoder.cpp:76-98.
#include <algorithm>
#include <cstring>
#include <string>

#include "msa_internal.hpp"

namespace msa {

#define MSA_TABLE(idx, nm, pen, ...) {nm, pen, {__VA_ARGS__}},
static const BuiltinTable g_tables[] = {
#include "tables.inc"
};
#undef MSA_TABLE

static constexpr int kNumTables = (int) (sizeof(g_tables) / sizeof(g_tables[0]));

const BuiltinTable *builtin_tables(int *count)
{
    if(count) *count = kNumTables;
    return g_tables;
}

int make_ext_table(const msa_table *t, ExtTable *out, std::string *err)
{
    std::memset(out, 0, sizeof(*out));
    out->penalty = t->penalty;
    int32_t mx = 0, mpos = -128, mneg = 0, lpos = -128, lneg = 0;
    for(int x = 0; x < kAlpha; ++x) {
        for(int y = 0; y < kAlpha; ++y) {
            int32_t v = 0;
            bool ok;
            if(t->index >= 0 && t->index < kNumTables) {
                // Flat offset into the contiguous storage, as (*m_contents)[x][y] computes it.
                const int64_t flat = (int64_t) t->index * 625 + (int64_t) x * 25 + y;
                ok = flat < (int64_t) kNumTables * 625;
                if(ok) v = g_tables[flat / 625].score[flat % 625];
            } else {
                ok = x < 25 && y < 25;
                if(ok) v = t->score[x * 25 + y];
            }
            if(ok && (v < -128 || v > 127)) {
                if(err) *err = "table entries must lie in [-128, 127]";
                return MSA_ERR_INVALID;
            }
            out->valid[x * kAlpha + y] = ok ? 1 : 0;
            out->score[x * kAlpha + y] = (int8_t) v;
            if(ok && x != MSA_UNIT_END && y != MSA_UNIT_END) {
                mx = std::max(mx, v < 0 ? -v : v);
                mpos = std::max(mpos, v);
                if(v < 0) mneg = std::max(mneg, -v);
            }
            if(ok && x < MSA_UNIT_END && y < MSA_UNIT_END) {
                lpos = std::max(lpos, v);
                if(v < 0) lneg = std::max(lneg, -v);
            }
        }
    }
    if(t->penalty < 0 || t->penalty > (1 << 20)) {
        if(err) *err = "penalty must lie in [0, 2^20]";
        return MSA_ERR_INVALID;
    }
    out->max_abs = mx;
    out->max_pos = mpos;
    out->max_neg = mneg;
    out->letter_pos = lpos;
    out->letter_neg = lneg;
    return MSA_OK;
}

// encode_table (src/encoder.cpp:27-30).
static const uint8_t kLetterUnit[26] = {
    0x00, 0x14, 0x01, 0x06, 0x08, 0x0E, 0x03, 0x09, 0x0A, 0x15, 0x0C, 0x0B, 0x0D,
    0x05, 0x17, 0x0F, 0x07, 0x04, 0x10, 0x02, 0x17, 0x13, 0x11, 0x17, 0x12, 0x16,
};
// decode_table (src/encoder.cpp:36-39).
static const char kUnitChar[26] = {
    'A', 'C', 'T', 'G', 'R', 'N', 'D', 'Q', 'E', 'H', 'I', 'L', 'K',
    'M', 'F', 'P', 'S', 'W', 'Y', 'V', 'B', 'J', 'Z', 'X', '*', '-',
};

static inline uint8_t encode_char(char c)
{
    const char u = (c >= 'a' && c <= 'z') ? (char) (c - 'a' + 'A') : c;
    if(u >= 'A' && u <= 'Z') return kLetterUnit[u - 'A'];
    if(c == '-') return MSA_UNIT_GAP;
    return MSA_UNIT_END;
}

}  // namespace msa

extern "C" {

int msa_table_make(const char *name, msa_table *out)
{
    if(!name || !out) return MSA_ERR_INVALID;
    int n;
    const msa::BuiltinTable *t = msa::builtin_tables(&n);
    for(int k = 0; k < n; ++k) {
        if(std::strcmp(t[k].name, name) == 0) {
            for(int i = 0; i < 625; ++i) out->score[i] = t[k].score[i];
            out->penalty = t[k].penalty;
            out->index = k;
            return MSA_OK;
        }
    }
    return MSA_ERR_UNKNOWN_TABLE;
}

int msa_table_has(const char *name)
{
    msa_table t;
    return msa_table_make(name, &t) == MSA_OK ? 1 : 0;
}

int msa_table_list(const char **names, int cap)
{
    // The reference lists names in std::map (lexicographic) order (src/dispatcher.hpp:21-46).
    int n;
    const msa::BuiltinTable *t = msa::builtin_tables(&n);
    std::vector<const char *> v;
    for(int k = 0; k < n; ++k) v.push_back(t[k].name);
    std::sort(v.begin(), v.end(), [](const char *a, const char *b) { return std::strcmp(a, b) < 0; });
    for(int k = 0; k < n && names && k < cap; ++k) names[k] = v[k];
    return n;
}

int msa_encode(const char *chars, uint64_t len, uint8_t *out_units)
{
    if((!chars || !out_units) && len) return MSA_ERR_INVALID;
    for(uint64_t i = 0; i < len; ++i) out_units[i] = msa::encode_char(chars[i]);
    return MSA_OK;
}

int msa_decode(const uint8_t *units, uint64_t len, char *out_chars)
{
    if((!units || !out_chars) && len) return MSA_ERR_INVALID;
    for(uint64_t i = 0; i < len; ++i) {
        if(units[i] > MSA_UNIT_GAP) return MSA_ERR_INVALID;   // "cannot decode invalid unit"
        out_chars[i] = msa::kUnitChar[units[i]];
    }
    return MSA_OK;
}

int msa_encode_blocks(const char *chars, uint64_t len, uint16_t *out_blocks)
{
    if((!chars || !out_blocks) && len) return MSA_ERR_INVALID;
    // Units at bit offsets 1, 6, 11; bit 0 marks a block that reaches past the end.
    static const int shift[3] = {1, 6, 11};
    for(uint64_t i = 0, n = 0; n < len; ++i) {
        uint16_t block = (n + 3 > len) ? 1 : 0;
        for(int k = 0; k < 3; ++k, ++n) {
            const uint16_t u = n < len ? msa::encode_char(chars[n]) : (uint16_t) MSA_UNIT_END;
            block |= (uint16_t) (u << shift[k]);
        }
        out_blocks[i] = block;
    }
    return MSA_OK;
}

int msa_unpack_blocks(const uint16_t *blocks, uint64_t nblocks, uint8_t *out_units)
{
    if((!blocks || !out_units) && nblocks) return MSA_ERR_INVALID;
    static const int shift[3] = {1, 6, 11};
    for(uint64_t i = 0; i < nblocks; ++i)
        for(int k = 0; k < 3; ++k)
            out_units[3 * i + k] = (uint8_t) ((blocks[i] >> shift[k]) & 0x1F);
    return MSA_OK;
}

const char *msa_strerror(int status)
{
    switch(status) {
        case MSA_OK: return "success";
        case MSA_ERR_INVALID: return "invalid argument";
        case MSA_ERR_CUDA: return "CUDA runtime error";
        case MSA_ERR_NOMEM: return "out of memory";
        case MSA_ERR_UNKNOWN_TABLE: return "unknown pairwise scoring table";
        case MSA_ERR_UNKNOWN_ALGORITHM: return "unknown algorithm";
        case MSA_ERR_HANDLE: return "invalid sequence-store handle";
        case MSA_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
        case MSA_ERR_UNDEFINED: return "result undefined in the reference for this input";
        case MSA_ERR_NO_DEVICE: return "no usable CUDA device";
        case MSA_ERR_QUEUE: return "serving queue error";
        case MSA_ERR_TOO_LARGE: return "request exceeds a size limit";
        default: return "unknown status";
    }
}

}  // extern "C"
