// The reference's on-disk forward solution records and its element keys, on the host.
//
// TITAN2D keys every element by a 2-D Hilbert code of its centre (Element::gen_my_sons_key,
// src/datstr/element2.C:4360-4420, through fhsfc2d_ of src/main/hilbert.C, Zoltan's BSFC curve):
// the centre is normalised by the table's x and y ranges into the unit square, each coordinate
// scaled to 32 bits, and the 64-bit key built two bits per level from the most significant end.
// At each level the two coordinate bits are placed by the current axis order, combined with the
// current reflection and passed through the inverse Gray code into the level's digit; a digit 0
// swaps the axes, a digit 3 swaps them and flips the reflection.
//
// The dual solver's forward records (SolRec::wrtie_sol_to_disk / read_sol_from_disk,
// src/datstr/dualmesh.C:82-147, 234-297) are gz files solution_<rank>_<step>: int32 count of zero
// records, int32 count of non-zero records, the zero records' keys (2 x uint32 each), then per
// non-zero record its key and the three state values (double).  A cell is written as a zero record
// when its depth is not positive (dualmesh.C:53-61).
#include <zlib.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "da_mesh.h"
#include "discrete_adjoint.h"

namespace {

uint32_t unit_to_u32(double a) {
    const uint32_t imax = 0xffffffffu;
    if (a <= 0) return 0;
    const double s = double(imax) * a;
    return double(imax) < s ? imax : uint32_t(s);
}

void hilbert_key(double u, double v, uint32_t key[2]) {
    static const unsigned char inv_gray[4] = {0, 1, 3, 2};
    const uint32_t x = unit_to_u32(u), y = unit_to_u32(v);
    unsigned ax = 0, ay = 1, refl = 0;  // bit positions of the x and y bits in a quadrant code
    uint64_t k = 0;
    for (int lvl = 31; lvl >= 0; --lvl) {
        const unsigned q = (((x >> lvl) & 1u) << ax) | (((y >> lvl) & 1u) << ay);
        const unsigned d = inv_gray[(refl ^ q) & 3u];
        k = (k << 2) | d;
        if (d == 3) refl ^= 3u;
        if (d == 0 || d == 3) std::swap(ax, ay);
    }
    key[0] = uint32_t(k >> 32);
    key[1] = uint32_t(k);
}

uint64_t key64(const uint32_t *k) { return (uint64_t(k[0]) << 32) | k[1]; }

}  // namespace

extern "C" {

int da_cell_keys(int32_t n, const double *x, const double *y, const double xrange[2], const double yrange[2],
                 uint32_t *keys) {
    if (n < 0 || (n > 0 && (!x || !y || !keys)) || !xrange || !yrange || !(xrange[1] > xrange[0]) ||
        !(yrange[1] > yrange[0]))
        return DA_ERR_INVALID;
    for (int32_t i = 0; i < n; ++i) {
        const double u = (x[i] - xrange[0]) / (xrange[1] - xrange[0]);
        const double v = (y[i] - yrange[0]) / (yrange[1] - yrange[0]);
        hilbert_key(u, v, keys + 2 * (size_t)i);
    }
    return DA_OK;
}

int da_write_solution(const char *path, int32_t n, const uint32_t *keys, const double *h, const double *hu,
                      const double *hv) {
    if (!path || n < 0 || (n > 0 && (!keys || !h || !hu || !hv))) return DA_ERR_INVALID;
    gzFile f = gzopen(path, "wb");
    if (!f) return DA_ERR_INVALID;
    int32_t nz = 0;
    for (int32_t i = 0; i < n; ++i) nz += h[i] > 0. ? 0 : 1;
    const int32_t counts[2] = {nz, n - nz};
    bool ok = gzwrite(f, counts, sizeof(counts)) == (int)sizeof(counts);
    for (int32_t i = 0; i < n && ok; ++i)
        if (!(h[i] > 0.)) ok = gzwrite(f, keys + 2 * (size_t)i, 8) == 8;
    for (int32_t i = 0; i < n && ok; ++i)
        if (h[i] > 0.) {
            const double s[3] = {h[i], hu[i], hv[i]};
            ok = gzwrite(f, keys + 2 * (size_t)i, 8) == 8 && gzwrite(f, s, sizeof(s)) == (int)sizeof(s);
        }
    if (gzclose(f) != Z_OK) ok = false;
    return ok ? DA_OK : DA_ERR_INVALID;
}

int da_read_solution(const char *path, int32_t n, const uint32_t *keys, double *h, double *hu, double *hv,
                     int32_t *n_missing) {
    if (!path || n < 0 || (n > 0 && (!keys || !h || !hu || !hv))) return DA_ERR_INVALID;
    std::vector<int32_t> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(),
              [&](int32_t a, int32_t b) { return key64(keys + 2 * (size_t)a) < key64(keys + 2 * (size_t)b); });
    for (int32_t j = 1; j < n; ++j)
        if (key64(keys + 2 * (size_t)order[j]) == key64(keys + 2 * (size_t)order[j - 1])) return DA_ERR_INVALID;
    auto find = [&](const uint32_t k[2]) -> int32_t {
        const uint64_t q = key64(k);
        const auto it = std::lower_bound(order.begin(), order.end(), q,
                                         [&](int32_t a, uint64_t v) { return key64(keys + 2 * (size_t)a) < v; });
        return (it != order.end() && key64(keys + 2 * (size_t)*it) == q) ? *it : -1;
    };
    gzFile f = gzopen(path, "rb");
    if (!f) return DA_ERR_INVALID;
    std::vector<char> seen(n, 0);
    int32_t counts[2] = {0, 0};
    bool ok = gzread(f, counts, sizeof(counts)) == (int)sizeof(counts) && counts[0] >= 0 && counts[1] >= 0;
    for (int32_t r = 0; r < counts[0] && ok; ++r) {
        uint32_t k[2];
        ok = gzread(f, k, 8) == 8;
        const int32_t c = ok ? find(k) : -1;
        if (c < 0) ok = false;  // a record for an element this mesh does not have
        else {
            h[c] = hu[c] = hv[c] = 0.;
            seen[c] = 1;
        }
    }
    for (int32_t r = 0; r < counts[1] && ok; ++r) {
        uint32_t k[2];
        double s[3];
        ok = gzread(f, k, 8) == 8 && gzread(f, s, sizeof(s)) == (int)sizeof(s);
        const int32_t c = ok ? find(k) : -1;
        if (c < 0) ok = false;
        else {
            h[c] = s[0];
            hu[c] = s[1];
            hv[c] = s[2];
            seen[c] = 1;
        }
    }
    gzclose(f);
    if (!ok) return DA_ERR_INVALID;
    int32_t missing = 0;
    for (int32_t i = 0; i < n; ++i)
        if (!seen[i]) {
            h[i] = hu[i] = hv[i] = 0.;
            ++missing;
        }
    if (n_missing) *n_missing = missing;
    return DA_OK;
}

}  // extern "C"
