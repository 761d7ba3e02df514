// Element order of the column-wise directionally refined meshes (shared by the face-table
// builder, the refinement and the solution transfer): base column c = ix + nx iy holds
// 2^lx x 2^ly x 2^lz cells; columns are sorted by (lx, ly, lz, c), so elements come grouped by
// level tuple, and a column's cells are numbered sx + nxc (sy + nyc sz) from its offset.
#pragma once
#include <algorithm>
#include <cstdint>
#include <numeric>
#include <vector>

namespace drf {

// first element of each column (levels lv[3 c + d]); entry ncol is the element count
inline std::vector<int64_t> amr_column_offsets(int ncol, const int *lv) {
    std::vector<int> order(ncol);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        for (int d = 0; d < 3; ++d)
            if (lv[3 * a + d] != lv[3 * b + d]) return lv[3 * a + d] < lv[3 * b + d];
        return a < b;
    });
    std::vector<int64_t> off(ncol + 1, 0);
    int64_t acc = 0;
    for (int c : order) {
        off[c] = acc;
        acc += (int64_t)1 << (lv[3 * c] + lv[3 * c + 1] + lv[3 * c + 2]);
    }
    off[ncol] = acc;
    return off;
}

}  // namespace drf
