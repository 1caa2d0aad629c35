// Host planner arithmetic in the library: the cut rank over GF(2) of every prefix of a vertex
// order, the inner loop of the parity-slice choice (reference: prefix_ranks_matrix,
// source/dcs_rankwidth/parity_slicing.py:35-54, called once per trial removal by
// choose_parity_slices, :62-105).
//
// The reference row-reduces G = [e_0 | A_0 | e_1 | A_1 | ...] (the identity columns interleaved
// with the induced adjacency's columns) and reads the cut rank of prefix i as
// (number of pivot columns among the first 2i) - i.  A column is a pivot column exactly when it
// is independent of the columns before it, so the same numbers come out of an incremental
// column basis: each column, as an m-bit word vector, is reduced by the basis vectors whose
// lowest set bit (their pivot) it contains, and joins the basis when something is left.
#include <stdint.h>
#include <string.h>

#include <vector>

#include "common.cuh"

extern "C" int dcs_prefix_cut_ranks(const uint8_t* adj, int n, const int32_t* order, int m, int32_t* ranks) {
    if (!adj || !order || (m > 1 && !ranks) || n < 0 || m < 0 || m > n) {
        dcs_host::set_error("dcs_prefix_cut_ranks: invalid arguments");
        return DCS_E_ARG;
    }
    for (int i = 0; i < m; ++i)
        if (order[i] < 0 || order[i] >= n) {
            dcs_host::set_error("dcs_prefix_cut_ranks: order[%d] = %d out of range", i, order[i]);
            return DCS_E_ARG;
        }
    if (m < 2) return DCS_OK;
    const int W = (m + 63) / 64;
    std::vector<uint64_t> basis((size_t)m * W);  // basis vector with pivot p at row p
    std::vector<uint8_t> has(m, 0);
    std::vector<uint64_t> v(W);
    int pivots = 0;
    for (int c = 0; c < 2 * m; ++c) {
        const int j = c >> 1;
        memset(v.data(), 0, sizeof(uint64_t) * W);
        if (!(c & 1)) {
            v[j >> 6] = 1ull << (j & 63);  // e_j
        } else {
            const uint8_t* row = adj + (size_t)order[j] * n;  // A is symmetric: column j = row order[j]
            for (int i = 0; i < m; ++i)
                if (row[order[i]]) v[i >> 6] |= 1ull << (i & 63);
        }
        for (int w = 0; w < W;) {
            if (!v[w]) {
                ++w;
                continue;
            }
            const int p = w * 64 + __builtin_ctzll(v[w]);
            if (!has[p]) {
                memcpy(&basis[(size_t)p * W], v.data(), sizeof(uint64_t) * W);
                has[p] = 1;
                ++pivots;
                break;
            }
            const uint64_t* b = &basis[(size_t)p * W];
            for (int k = w; k < W; ++k) v[k] ^= b[k];  // b has no bits below p
        }
        if (c & 1 && j + 1 < m) ranks[j] = pivots - (j + 1);  // prefix {0..j}: first 2(j+1) columns
    }
    return DCS_OK;
}
