// Host check of sams::BoxShell: for each grid and inner cube, every box point
// outside the cube is produced exactly once and nothing else is.
#include <cstdio>
#include <vector>

#include "lare_device.cuh"

int main()
{
    const int grids[][3] = {{1, 1, 1}, {2, 9, 5}, {12, 10, 6}, {7, 3, 24}, {33, 17, 65}};
    const int cubes[][2] = {{1, 0}, {0, 0}};
    int bad = 0;
    for (const auto &n : grids)
        for (const auto &c : cubes) {
            const sams::BoxShell s{{n[0], n[1], n[2]}, c[0], c[1]};
            const int e0 = n[0] + 5, e1 = n[1] + 5, e2 = n[2] + 5;
            std::vector<int> hits((size_t)e0 * e1 * e2, 0);
            for (long long t = 0; t < s.count(); ++t) {
                int i, j, k;
                s.point(t, i, j, k);
                if (i < -2 || i > n[0] + 2 || j < -2 || j > n[1] + 2 || k < -2 || k > n[2] + 2) {
                    ++bad;
                    continue;
                }
                ++hits[((size_t)(i + 2) * e1 + (j + 2)) * e2 + (k + 2)];
            }
            for (int i = -2; i <= n[0] + 2; ++i)
                for (int j = -2; j <= n[1] + 2; ++j)
                    for (int k = -2; k <= n[2] + 2; ++k) {
                        const bool inside = i >= c[0] && i <= n[0] + c[1] && j >= c[0] && j <= n[1] + c[1] &&
                                            k >= c[0] && k <= n[2] + c[1];
                        const int h = hits[((size_t)(i + 2) * e1 + (j + 2)) * e2 + (k + 2)];
                        if (h != (inside ? 0 : 1)) ++bad;
                    }
        }
    std::printf("{\"bad\": %d}\n", bad);
    return bad ? 1 : 0;
}
