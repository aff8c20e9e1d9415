// Setup-side input generation: FCC lattices and distance-rule links. These make the
// synthetic workloads (the reference's own MeshBlock inputs are HDF5 point files that
// cannot be read here) and are host code, run once before the timestep loop.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "hidem_b200.h"

namespace {

// 64-bit Mersenne Twister (the std::mt19937_64 parameters), written out so the
// stream is fixed by the seed alone.
struct Mt64 {
    uint64_t mt[312];
    int idx = 313;
    explicit Mt64(uint64_t seed) {
        mt[0] = seed;
        for (int i = 1; i < 312; ++i)
            mt[i] = 6364136223846793005ULL * (mt[i - 1] ^ (mt[i - 1] >> 62)) + (uint64_t)i;
        idx = 312;
    }
    uint64_t next() {
        if (idx >= 312) {
            for (int i = 0; i < 312; ++i) {
                uint64_t x = (mt[i] & 0xFFFFFFFF80000000ULL) | (mt[(i + 1) % 312] & 0x7FFFFFFFULL);
                uint64_t xa = x >> 1;
                if (x & 1ULL) xa ^= 0xB5026F5AA96619E9ULL;
                mt[i] = mt[(i + 156) % 312] ^ xa;
            }
            idx = 0;
        }
        uint64_t x = mt[idx++];
        x ^= (x >> 29) & 0x5555555555555555ULL;
        x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
        x ^= (x << 37) & 0xFFF7EEE000000000ULL;
        x ^= (x >> 43);
        return x;
    }
    // uniform in [0, 1) with 53 random bits
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

template <class LP>
void put(void *arr, int64_t i, double v) {
    if (arr) static_cast<LP *>(arr)[i] = (LP)v;
}

}  // namespace

extern "C" {

hidem_status hidem_lattice_fcc(int32_t nx, int32_t ny, int32_t nz, double a, double radius,
                               const double origin[3], double jitter, uint64_t seed,
                               int32_t precision, hidem_particle_soa *out) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || !(a > 0) || !(radius > 0) || !out || !out->xCord ||
        !out->yCord || !out->zCord || !out->radius)
        return HIDEM_ERR_ARG;
    if (precision != HIDEM_PREC_FP64 && precision != HIDEM_PREC_MIXED) return HIDEM_ERR_ARG;
    const int64_t n = 4ll * nx * ny * nz;
    if (n >= (1ll << 31)) return HIDEM_ERR_CAPACITY;
    const double o[3] = {origin ? origin[0] : 0.0, origin ? origin[1] : 0.0, origin ? origin[2] : 0.0};
    // conventional FCC cell: corner + three face centres
    const double site[4][3] = {{0, 0, 0}, {0.5, 0.5, 0}, {0.5, 0, 0.5}, {0, 0.5, 0.5}};
    Mt64 rng(seed);
    int64_t i = 0;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int c = 0; c < nx; ++c)
                for (int s = 0; s < 4; ++s, ++i) {
                    double p[3] = {o[0] + (c + site[s][0]) * a, o[1] + (j + site[s][1]) * a,
                                   o[2] + (k + site[s][2]) * a};
                    if (jitter > 0)
                        for (int q = 0; q < 3; ++q) p[q] += -jitter + 2.0 * jitter * rng.uniform();
                    out->xCord[i] = p[0];
                    out->yCord[i] = p[1];
                    out->zCord[i] = p[2];
                    void *zero[9] = {out->xTheta, out->yTheta, out->zTheta, out->xDiff, out->yDiff,
                                     out->zDiff, out->uDiff, out->vDiff, out->wDiff};
                    for (void *z : zero) {
                        if (precision == HIDEM_PREC_MIXED) put<float>(z, i, 0.0);
                        else put<double>(z, i, 0.0);
                    }
                    if (precision == HIDEM_PREC_MIXED) put<float>(out->radius, i, radius);
                    else put<double>(out->radius, i, radius);
                    if (out->owners) out->owners[i] = 0;
                    if (out->type) out->type[i] = 0;
                    if (out->globalKeys) out->globalKeys[i] = i;
                }
    return HIDEM_OK;
}

// Link rule of LinkGenerator::genNewLinks (PLiB/Generators/LinkGenerator.h:60-110):
// pair (p, q) with globalKey[p] < globalKey[q] and |x_q - x_p| <= (r_p + r_q) * distScale,
// distance in double, radius sum in lp, distScale in lp; initialLen = |x_q - x_p|.
// Candidates come from a uniform grid of cell size max(2 r) * scale.
hidem_status hidem_links_by_distance(const hidem_particle_soa *p, int64_t n, int32_t precision,
                                     double scale, hidem_link_soa *out, int64_t cap,
                                     int64_t *count) {
    if (!p || n <= 0 || !count || !p->xCord || !p->yCord || !p->zCord || !p->radius)
        return HIDEM_ERR_ARG;
    if (precision != HIDEM_PREC_FP64 && precision != HIDEM_PREC_MIXED) return HIDEM_ERR_ARG;
    const bool mixed = precision == HIDEM_PREC_MIXED;
    auto rad = [&](int64_t i) -> double {
        return mixed ? (double)static_cast<const float *>(p->radius)[i]
                     : static_cast<const double *>(p->radius)[i];
    };
    auto key = [&](int64_t i) -> int64_t { return p->globalKeys ? p->globalKeys[i] : i; };
    const double distScale = mixed ? (double)(float)scale : scale;
    double rmax = 0, mn[3] = {p->xCord[0], p->yCord[0], p->zCord[0]}, mx[3] = {mn[0], mn[1], mn[2]};
    for (int64_t i = 0; i < n; ++i) {
        rmax = std::max(rmax, rad(i));
        const double v[3] = {p->xCord[i], p->yCord[i], p->zCord[i]};
        for (int q = 0; q < 3; ++q) {
            mn[q] = std::min(mn[q], v[q]);
            mx[q] = std::max(mx[q], v[q]);
        }
    }
    const double h = std::max(2.0 * rmax * distScale, 1e-12);
    int64_t dim[3];
    for (int q = 0; q < 3; ++q) dim[q] = 1 + (int64_t)std::floor((mx[q] - mn[q]) / h);
    const int64_t cells = dim[0] * dim[1] * dim[2];
    if (cells > (1ll << 33)) return HIDEM_ERR_CAPACITY;
    std::vector<int64_t> cellOf((size_t)n), start((size_t)cells + 1, 0);
    for (int64_t i = 0; i < n; ++i) {
        int64_t c[3];
        const double v[3] = {p->xCord[i], p->yCord[i], p->zCord[i]};
        for (int q = 0; q < 3; ++q) c[q] = std::min<int64_t>(dim[q] - 1, (int64_t)std::floor((v[q] - mn[q]) / h));
        cellOf[i] = c[0] + dim[0] * (c[1] + dim[1] * c[2]);
        start[cellOf[i] + 1]++;
    }
    for (int64_t c = 0; c < cells; ++c) start[c + 1] += start[c];
    std::vector<int32_t> members((size_t)n);
    {
        std::vector<int64_t> cur(start.begin(), start.end() - 1);
        for (int64_t i = 0; i < n; ++i) members[cur[cellOf[i]]++] = (int32_t)i;
    }
    // per particle: partners with a larger key, ascending by index
    std::vector<int32_t> nlinks((size_t)n, 0);
    std::vector<std::vector<std::pair<int32_t, double>>> rows((size_t)n);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < n; ++i) {
        const int64_t c = cellOf[i];
        const int64_t cx = c % dim[0], cy = (c / dim[0]) % dim[1], cz = c / (dim[0] * dim[1]);
        auto &row = rows[i];
        for (int64_t dz = -1; dz <= 1; ++dz)
            for (int64_t dy = -1; dy <= 1; ++dy)
                for (int64_t dx = -1; dx <= 1; ++dx) {
                    const int64_t x = cx + dx, y = cy + dy, z = cz + dz;
                    if (x < 0 || y < 0 || z < 0 || x >= dim[0] || y >= dim[1] || z >= dim[2]) continue;
                    const int64_t t = x + dim[0] * (y + dim[1] * z);
                    for (int64_t m = start[t]; m < start[t + 1]; ++m) {
                        const int32_t q = members[m];
                        if (q == i || key(i) >= key(q)) continue;
                        const double xd = p->xCord[q] - p->xCord[i];
                        const double yd = p->yCord[q] - p->yCord[i];
                        const double zd = p->zCord[q] - p->zCord[i];
                        const double dist = std::sqrt((xd * xd) + (yd * yd) + (zd * zd));
                        double radiusSum;
                        if (mixed) {
                            float rs = static_cast<const float *>(p->radius)[q] +
                                       static_cast<const float *>(p->radius)[i];
                            radiusSum = rs;
                        } else {
                            radiusSum = static_cast<const double *>(p->radius)[q] +
                                        static_cast<const double *>(p->radius)[i];
                        }
                        if (dist > radiusSum * distScale) continue;
                        row.push_back({q, dist});
                    }
                }
        std::sort(row.begin(), row.end());
        nlinks[i] = (int32_t)row.size();
    }
    int64_t total = 0;
    for (int64_t i = 0; i < n; ++i) total += nlinks[i];
    *count = total;
    if (!out) return HIDEM_OK;
    if (total > cap) return HIDEM_ERR_CAPACITY;
    int64_t w = 0;
    for (int64_t i = 0; i < n; ++i) {
        const auto &row = rows[i];
        for (size_t k = 0; k < row.size(); ++k, ++w) {
            const int64_t q = row[k].first;
            if (out->globalKeyEndA) out->globalKeyEndA[w] = key(i);
            if (out->globalKeyEndB) out->globalKeyEndB[w] = key(q);
            if (out->particleLinkNum) out->particleLinkNum[w] = (int32_t)k;
            if (out->globalKeys) out->globalKeys[w] = key(i) * 256 + (int64_t)k;  // LKeyOffset
            if (out->owners) out->owners[w] = p->owners ? p->owners[i] : 0;
            if (out->state) out->state[w] = 1;
            if (out->initialLen) {
                if (mixed) static_cast<float *>(out->initialLen)[w] = (float)row[k].second;
                else static_cast<double *>(out->initialLen)[w] = row[k].second;
            }
        }
    }
    return HIDEM_OK;
}

}  // extern "C"
