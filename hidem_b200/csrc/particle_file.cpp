// Particle point files of the reference's File lattice (HiDEM/Benchmark/*/particles.h5, read
// by PLiB/Generators/FileParticleGenerator.h:23-105): four 1-D datasets of coordinates and
// radii, written by libhdf5 (superblock 0, symbol-table root group, deflate-compressed
// chunks). Host code, run once before the timestep loop.
#include <cstring>
#include <string>
#include <vector>

#include "h5lite.h"
#include "hidem_b200.h"

namespace hidem {
extern thread_local std::string g_nocontext_error;
}

namespace {

hidem_status pf_fail(hidem_status s, const std::string &m) {
    hidem::g_nocontext_error = "hidem_read_particle_file: " + m;
    return s;
}

// the dataset's values as float, as the reference reads them (readVectorSpann<float>: the
// library converts each stored value to the memory type, double -> float rounding to nearest)
bool read_as_float(const std::string &path, const h5lite::Dataset &d, std::vector<float> &out,
                   std::string &err) {
    out.resize(d.count);
    if (d.type == h5lite::Type::F32) return h5lite::read_dataset(path, d, out.data(), err);
    if (d.type != h5lite::Type::F64) {
        err = "dataset '" + d.name + "' is not a floating-point dataset";
        return false;
    }
    std::vector<double> tmp(d.count);
    if (!h5lite::read_dataset(path, d, tmp.data(), err)) return false;
    for (size_t i = 0; i < tmp.size(); ++i) out[i] = (float)tmp[i];
    return true;
}

template <class LP>
void put(void *arr, int64_t i, double v) {
    if (arr) static_cast<LP *>(arr)[i] = (LP)v;
}

}  // namespace

extern "C" hidem_status hidem_read_particle_file(const char *path, const char *x_name, const char *y_name,
                                                 const char *z_name, const char *radius_name,
                                                 int32_t precision, hidem_particle_soa *out, int64_t cap,
                                                 int64_t *count) {
    hidem::g_nocontext_error.clear();
    if (!path || !count) return pf_fail(HIDEM_ERR_ARG, "path and count are required");
    if (precision != HIDEM_PREC_FP64 && precision != HIDEM_PREC_MIXED)
        return pf_fail(HIDEM_ERR_ARG, "unknown precision");
    const std::string names[4] = {x_name ? x_name : "xCord", y_name ? y_name : "yCord",
                                  z_name ? z_name : "zCord", radius_name ? radius_name : "radius"};
    h5lite::Group root;
    std::string err;
    if (!h5lite::read_file(path, root, err)) return pf_fail(HIDEM_ERR_IO, err);
    const h5lite::Dataset *ds[4];
    for (int k = 0; k < 4; ++k) {
        ds[k] = root.dataset(names[k]);
        if (!ds[k]) return pf_fail(HIDEM_ERR_IO, std::string(path) + ": no dataset '" + names[k] + "' in the root group");
        if (ds[k]->count != ds[0]->count)
            return pf_fail(HIDEM_ERR_IO, "datasets '" + names[0] + "' and '" + names[k] + "' differ in length");
    }
    const int64_t n = (int64_t)ds[0]->count;
    *count = n;
    if (!out) return HIDEM_OK;
    if (n > cap) return pf_fail(HIDEM_ERR_CAPACITY, "the file holds " + std::to_string(n) + " particles, more than cap");
    if (!out->xCord || !out->yCord || !out->zCord || !out->radius)
        return pf_fail(HIDEM_ERR_ARG, "xCord/yCord/zCord/radius output arrays are required");
    std::vector<float> v[4];
    for (int k = 0; k < 4; ++k)
        if (!read_as_float(path, *ds[k], v[k], err)) return pf_fail(HIDEM_ERR_IO, err);
    const bool mixed = precision == HIDEM_PREC_MIXED;
    for (int64_t i = 0; i < n; ++i) {
        out->xCord[i] = v[0][i];
        out->yCord[i] = v[1][i];
        out->zCord[i] = v[2][i];
        void *zero[9] = {out->xTheta, out->yTheta, out->zTheta, out->xDiff, out->yDiff,
                         out->zDiff,  out->uDiff,  out->vDiff,  out->wDiff};
        for (void *z : zero) mixed ? put<float>(z, i, 0.0) : put<double>(z, i, 0.0);
        mixed ? put<float>(out->radius, i, v[3][i]) : put<double>(out->radius, i, v[3][i]);
        if (out->owners) out->owners[i] = 0;
        if (out->type) out->type[i] = 0;
        if (out->globalKeys) out->globalKeys[i] = i;  // ParticleGenerator::setParticleKeys, one rank
    }
    return HIDEM_OK;
}
