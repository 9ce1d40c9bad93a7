// Periodic folding, minimum image and cell indices, shared by the device kernels and the host
// test entry point vpbs_periodic_eval (so that the same code is checked on the CPU).
#pragma once

#include <cmath>
#include <cstdint>

namespace vpbs {

#if defined(__CUDACC__)
#define VPBS_HD __host__ __device__ __forceinline__
#else
#define VPBS_HD inline
#endif

// Fold into [0, L) (min_distance.jl:5-20).  Within four periods the reference's subtraction
// loops (at most five iterations, same rounding); beyond that, or for a non-finite coordinate,
// one exact fmod, so the cost never depends on the value (inf and NaN come out as NaN).
VPBS_HD double fold(double x, double L, int open) {
    if (open) return x;
    if (!(fabs(x) <= 4.0 * L)) {
        x = fmod(x, L);  // exact, |x| < L; NaN for inf / NaN
        if (x < 0.0) x += L;
        if (x >= L) x = 0.0;  // -tiny + L rounded to L
        return x;
    }
    while (x < 0.0) x += L;
    while (x >= L) x -= L;
    return x;
}

// Minimum image of a separation of two folded coordinates (min_distance.jl:61-67).
VPBS_HD double deper(double r, double L, double Lh, int open) {
    if (open) return r;
    r = (r >= Lh) ? r - L : r;
    r = (r < -Lh) ? r + L : r;
    return r;
}

// Cell of a finite folded coordinate: trunc(x / L * nc), clamped to [0, nc) (CellLists.jl:194-204,
// 0-based).
VPBS_HD int cell_coord(double x, double L, int nc) {
    int c = (int)((x / L) * nc);
    return c < 0 ? 0 : (c >= nc ? nc - 1 : c);
}

// Linear cell index of a point in an nc[0] x nc[1] x nc[2] grid (x fastest).  A point with a
// non-finite coordinate goes to the sentinel cell ncell = nc[0] nc[1] nc[2], which no
// neighbourhood contains: its pairs are skipped instead of piling up in cell 0 and making the
// pair search quadratic.
VPBS_HD int64_t cell_index(const int nc[3], const double L[3], double x, double y, double z) {
    if (!(std::isfinite(x) && std::isfinite(y) && std::isfinite(z))) return (int64_t)nc[0] * nc[1] * nc[2];
    const int cx = cell_coord(x, L[0], nc[0]);
    const int cy = cell_coord(y, L[1], nc[1]);
    const int cz = cell_coord(z, L[2], nc[2]);
    return ((int64_t)cz * nc[1] + cy) * nc[0] + cx;
}

}  // namespace vpbs
