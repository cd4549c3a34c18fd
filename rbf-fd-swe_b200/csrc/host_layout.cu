// Host-side node ordering used by callers that prepare patches themselves.
//
// swe_host_rcm_mapping restates the reference's reverse Cuthill-McKee ordering
// (swe_code/rcm/rcm.c:9-62 with find_degree :107-120 and reorder_increasing
// :133-173) so that a host without the reference's rcm.c produces the same
// permutation: breadth-first from node 0; each visited node's stencil
// neighbours (slots 1..nnbr-1) are appended in increasing order of their count
// of still-unmapped stencil neighbours, ties by node id; finally the order is
// reversed with the reference's loop bound i < (n-1)/2, which leaves the middle
// pair of an even-length ordering in place.
#include <algorithm>
#include <vector>

#include "common.cuh"

extern "C" int swe_host_rcm_mapping(int n, int nnbr, const int* idx, int* mapping) {
    if (n <= 0 || nnbr <= 0 || !idx || !mapping) {
        swe::set_error("swe_host_rcm_mapping: bad arguments");
        return SWE_ERR_ARG;
    }
    for (long t = 0; t < (long)n * nnbr; ++t)
        if (idx[t] < 0 || idx[t] >= n) {
            swe::set_error("swe_host_rcm_mapping: idx[%ld] = %d outside [0, %d)", t, idx[t], n);
            return SWE_ERR_INDEX;
        }
    std::vector<char> mapped(n, 0);
    std::vector<int> x(nnbr), degree(nnbr), order(nnbr);
    mapping[0] = 0;
    mapped[0] = 1;
    int filled = 1;
    for (int i = 0; i < n && filled < n; ++i) {
        const int node = mapping[i];
        const int* row = idx + (long)nnbr * node;
        for (int j = 0; j < nnbr; ++j) {
            x[j] = row[j];
            degree[j] = 0;
        }
        for (int j = 1; j < nnbr; ++j) {
            const int* r2 = idx + (long)nnbr * x[j];
            for (int jj = 1; jj < nnbr; ++jj) degree[j] += mapped[r2[jj]] == 0;
        }
        for (int j = 0; j < nnbr; ++j) order[j] = j;
        std::sort(order.begin() + 1, order.end(), [&](int a, int b) {
            return degree[a] != degree[b] ? degree[a] < degree[b] : x[a] < x[b];
        });
        for (int t = 1; t < nnbr && filled < n; ++t) {
            const int nb = x[order[t]];
            if (!mapped[nb]) {
                mapping[filled++] = nb;
                mapped[nb] = 1;
            }
        }
    }
    if (filled != n) {
        swe::set_error("swe_host_rcm_mapping: stencil graph is not connected (%d of %d nodes reached)", filled, n);
        return SWE_ERR_ARG;
    }
    for (int i = 0; i < (n - 1) / 2; ++i) std::swap(mapping[i], mapping[n - 1 - i]);
    return SWE_OK;
}
