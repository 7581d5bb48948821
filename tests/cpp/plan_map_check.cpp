// The left-looking refactor's update map of a large AMD-LU plan (built on
// several host threads) equals the map recomputed here one column after
// another: for every U(r, j), the positions in column j of the rows of
// L(:, r).  A 5-point resistor-grid Laplacian of side 160 (about 1e8
// updates) takes the multi-threaded path.  The device pool holds the map
// packed as uint16 positions.  Prints "0 failure(s)" on success.
#include "host/amd_lu.hpp"
#include "host/plan.hpp"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

int main() {
    const int32_t side = 160, n = side * side;
    std::vector<int32_t> col_ptr(n + 1, 0), row_idx;
    std::vector<double> values;
    for (int32_t j = 0; j < n; ++j) {
        const int32_t x = j % side, y = j / side;
        // rows of column j in ascending order
        const int32_t nb[5] = {y > 0 ? j - side : -1, x > 0 ? j - 1 : -1, j,
                               x + 1 < side ? j + 1 : -1, y + 1 < side ? j + side : -1};
        for (int32_t r : nb) {
            if (r < 0) continue;
            row_idx.push_back(r);
            values.push_back(r == j ? 4.0 + 1e-3 * (j % 7) : -1.0);
        }
        col_ptr[j + 1] = static_cast<int32_t>(row_idx.size());
    }
    nsg::AmdLuFactor f(n, col_ptr, row_idx);
    if (!f.factor(values.data(), 0.0)) {
        std::printf("factor failed\n1 failure(s)\n");
        return 1;
    }
    const nsg::TopologyPlan p = nsg::build_plan_amd(f);
    int failures = 0;
    std::vector<int32_t> where(n, -1);
    int64_t at = 0;
    for (int32_t j = 0; j < n && failures < 10; ++j) {
        for (int32_t q = p.col_ptr[j]; q < p.col_ptr[j + 1]; ++q) where[p.row_idx[q]] = q;
        for (int32_t q = p.col_ptr[j]; q < p.diag_pos[j]; ++q) {
            if (p.upd_start[q] != at) {
                std::printf("upd_start mismatch at column %d entry %d\n", j, q);
                ++failures;
            }
            const int32_t r = p.row_idx[q];
            for (int32_t k = p.diag_pos[r] + 1; k < p.col_ptr[r + 1]; ++k, ++at) {
                const int32_t want = where[p.row_idx[k]] - p.col_ptr[j];
                if (p.upd_dst[at] != want) {
                    if (failures < 10)
                        std::printf("upd_dst mismatch at column %d update %lld\n", j,
                                    static_cast<long long>(at));
                    ++failures;
                }
            }
        }
        for (int32_t q = p.col_ptr[j]; q < p.col_ptr[j + 1]; ++q) where[p.row_idx[q]] = -1;
    }
    // The device copy: every column is short, so the map is packed as
    // uint16 positions; device_words() is the pool's exact size.
    if (!p.map16()) {
        std::printf("plan not packed (longest column %d)\n", p.max_col);
        ++failures;
    }
    std::vector<int32_t> pool;
    int64_t off[32] = {};
    p.append_to(pool, off);
    if (static_cast<int64_t>(pool.size()) > p.device_words()) {
        std::printf("pool %zu words, device_words %lld\n", pool.size(),
                    static_cast<long long>(p.device_words()));
        ++failures;
    }
    const int upd_dst_array = 7;  // position of upd_dst in the pool's array order
    std::vector<uint16_t> packed(p.upd_dst.size());
    std::memcpy(packed.data(), pool.data() + off[upd_dst_array], 2 * packed.size());
    for (size_t k = 0; k < packed.size() && failures < 10; ++k)
        if (packed[k] != p.upd_dst[k]) {
            std::printf("packed map mismatch at update %zu\n", k);
            ++failures;
        }
    if (off[upd_dst_array + 1] - off[upd_dst_array] != ((int64_t(packed.size()) + 1) / 2 + 3) / 4 * 4) {
        std::printf("packed map region %lld words for %zu positions\n",
                    static_cast<long long>(off[upd_dst_array + 1] - off[upd_dst_array]),
                    packed.size());
        ++failures;
    }
    if (at != p.updates) {
        std::printf("update count %lld, plan says %lld\n", static_cast<long long>(at),
                    static_cast<long long>(p.updates));
        ++failures;
    }
    std::printf("n %d, updates %lld\n%d failure(s)\n", n, static_cast<long long>(p.updates),
                failures);
    return failures == 0 ? 0 : 1;
}
