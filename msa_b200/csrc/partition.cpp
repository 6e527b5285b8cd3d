// Splitting one all-pairs job into parts of about equal DP cells, for jobs
// spread over several devices (one part per device, the same split on all of
// them) and for the host-side query msa_nw_part_of_pairs.
//
// The reference splits the pair index evenly over MPI ranks
// (src/pairwise/needleman/needleman.cpp:31-52, utils::partition at
// src/utils.hpp:176-183); under uneven lengths that balances pairs, not work.
// Here the unit of work is the kernels' own: rows pairs (sorted 2k, 2k+1 of
// the clean sequences ordered by length, longest first) for the clean pairs,
// and single pairs of the generic list for the rest. Each part takes a
// contiguous run of each, cut where the running cell count crosses p/P of
// the total; integer arithmetic throughout, so every host computes the same
// split.
#include <algorithm>
#include <cstring>

#include "msa_internal.hpp"

namespace msa {

void scan_units(const uint8_t *src, uint64_t len, uint32_t plen, uint32_t *eff, uint8_t *dirty, uint8_t *gap)
{
    uint32_t first_end = plen;
    bool seen_end = false, d = false, g = false;
    for(uint64_t k = 0; k < len; ++k) {
        const uint8_t u = src[k];
        if(u == MSA_UNIT_END) {
            if(!seen_end) { first_end = (uint32_t) k; seen_end = true; }
        } else if(seen_end) {
            d = true;
        }
        if(u == MSA_UNIT_GAP) g = true;
    }
    if(!seen_end && len < plen) first_end = (uint32_t) len;
    *eff = first_end;
    *gap = g ? 1 : 0;
    *dirty = (d || first_end == 0 || g) ? 1 : 0;
}

void sort_clean(const std::vector<uint32_t> &eff, const std::vector<uint8_t> &dirty, std::vector<uint32_t> &out)
{
    out.clear();
    for(uint32_t i = 0; i < (uint32_t) eff.size(); ++i)
        if(!dirty[i]) out.push_back(i);
    std::stable_sort(out.begin(), out.end(), [&eff](uint32_t a, uint32_t b) { return eff[a] > eff[b]; });
}

void list_generic_pairs(const std::vector<uint8_t> &dirty, const std::vector<uint64_t> &len,
                        std::vector<uint32_t> &gpairs)
{
    gpairs.clear();
    const uint32_t n = (uint32_t) dirty.size();
    bool any = false;
    for(uint32_t i = 0; i < n; ++i) any = any || dirty[i];
    if(!any) return;
    // Row-major pair order; each pair in the reference's orientation (rows =
    // more 3-unit blocks, ties to the pair's second element).
    for(uint32_t i = 1; i < n; ++i) {
        for(uint32_t j = 0; j < i; ++j) {
            if(!dirty[i] && !dirty[j]) continue;
            const uint64_t bi = (len[i] + 2) / 3, bj = (len[j] + 2) / 3;
            gpairs.push_back(bi > bj ? i : j);
            gpairs.push_back(bi > bj ? j : i);
        }
    }
}

namespace {

using u128 = unsigned __int128;

// First index k of [0, m] with cum[k] * parts >= p * total, for p = 0..parts.
template <class T>
std::vector<T> cut(const std::vector<u128> &cum, uint32_t parts)
{
    const size_t m = cum.size() - 1;
    const u128 total = cum[m];
    std::vector<T> b(parts + 1, 0);
    size_t k = 0;
    for(uint32_t p = 1; p < parts; ++p) {
        while(k < m && cum[k] * parts < total * p) ++k;
        b[p] = (T) k;
    }
    b[parts] = (T) m;
    return b;
}

}  // namespace

JobSplit split_job(const std::vector<uint32_t> &eff, const std::vector<uint32_t> &plen,
                   const std::vector<uint32_t> &clean_sorted, const std::vector<uint32_t> &gpairs, uint32_t parts)
{
    JobSplit s;
    parts = std::max<uint32_t>(parts, 1);
    const uint32_t nclean = (uint32_t) clean_sorted.size();
    const uint32_t K = (nclean + 1) / 2;
    // Cells of rows pair k: its two rows against every later (shorter) sequence.
    std::vector<u128> suffix(nclean + 1, 0);
    for(uint32_t b = nclean; b-- > 0;) suffix[b] = suffix[b + 1] + eff[clean_sorted[b]];
    std::vector<u128> cum(K + 1, 0);
    for(uint32_t k = 0; k < K; ++k) {
        const uint32_t a1 = 2 * k, a2 = 2 * k + 1;
        u128 c = (u128) eff[clean_sorted[a1]] * suffix[a1 + 1];
        if(a2 < nclean) c += (u128) eff[clean_sorted[a2]] * suffix[a2 + 1];
        cum[k + 1] = cum[k] + c;
    }
    s.k = cut<uint32_t>(cum, parts);
    s.clean_cells = cum;
    const uint64_t ng = gpairs.size() / 2;
    std::vector<u128> gcum(ng + 1, 0);
    for(uint64_t q = 0; q < ng; ++q)
        gcum[q + 1] = gcum[q] + (u128) plen[gpairs[2 * q]] * plen[gpairs[2 * q + 1]];
    s.g = cut<uint64_t>(gcum, parts);
    return s;
}

}  // namespace msa

extern "C" int msa_nw_part_of_pairs(const uint8_t *units, const uint64_t *offs, const uint64_t *lens, uint32_t n,
                                    const msa_table *table, uint32_t nparts, uint32_t *out_part)
{
    using namespace msa;
    if(nparts == 0 || (n && (!offs || !lens)) || (n > 1 && !out_part) || !table) return MSA_ERR_INVALID;
    try {
        ExtTable ext;
        std::string err;
        const int rc = make_ext_table(table, &ext, &err);
        if(rc) return rc;
        std::vector<uint64_t> len(n);
        std::vector<uint32_t> eff(n), plen(n);
        std::vector<uint8_t> dirty(n), gap(n);
        for(uint32_t i = 0; i < n; ++i) {
            if(lens[i] && !units) return MSA_ERR_INVALID;
            len[i] = lens[i];
            plen[i] = (uint32_t) ((lens[i] + 2) / 3 * 3);
            scan_units(units + offs[i], lens[i], plen[i], &eff[i], &dirty[i], &gap[i]);
        }
        if(!table_is_symmetric(ext)) std::fill(dirty.begin(), dirty.end(), 1);
        std::vector<uint32_t> sorted, gpairs;
        sort_clean(eff, dirty, sorted);
        list_generic_pairs(dirty, len, gpairs);
        const JobSplit s = split_job(eff, plen, sorted, gpairs, nparts);
        auto tri = [](uint64_t i, uint64_t j) { return i > j ? i * (i - 1) / 2 + j : j * (j - 1) / 2 + i; };
        for(uint32_t p = 0; p < nparts; ++p) {
            for(uint32_t k = s.k[p]; k < s.k[p + 1]; ++k)
                for(uint32_t a = 2 * k; a < std::min<uint32_t>(2 * k + 2, (uint32_t) sorted.size()); ++a)
                    for(uint32_t b = a + 1; b < (uint32_t) sorted.size(); ++b) out_part[tri(sorted[a], sorted[b])] = p;
            for(uint64_t q = s.g[p]; q < s.g[p + 1]; ++q) out_part[tri(gpairs[2 * q], gpairs[2 * q + 1])] = p;
        }
        return MSA_OK;
    } catch(const std::bad_alloc &) {
        return MSA_ERR_NOMEM;
    }
}
