// Checkpoint write / read in the reference's HDF5 layout (HiDEMLib/HiDEMH5Checkpoint.h:24-50,
// PLiB/H5IO/H5Checkpoint.h:42-111, PLiB/ParticleDataHandler.h:215-267,
// PLiB/LinkDataHandler.h:356-451) for one rank:
//   /                 attribute timeStep (int32)
//   /Domains          attributes domain{Upper,Lower}{X,Y,Z}, domain{Upper,Lower}Halo{X,Y,Z}
//                     (f64[1]) and domainOwner (int32[1])
//   /Particles        field_0..field_15 = xCord yCord zCord xTheta yTheta zTheta xDiff yDiff
//                     zDiff uDiff vDiff wDiff radius owners type globalKeys;
//                     attributes spann_sizes / spann_offsets (int64[1])
//   /Links            field_0..field_6 = owners state globalKeys globalKeyEndA globalKeyEndB
//                     initialLen particleLinkNum; spann attributes
//   /LinkSideData     side_field_7..side_field_12 = CT0..CT5 as [sideA(l0), sideB(l0), ...]
//                     (the field counter is not reset between the two groups,
//                     LinkDataHandler.h:384-392); spann attributes
// lp / ct fields are float in mixed precision and double in FP64; datasets are contiguous
// (the reference's HDF5.compression = false layout).
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "h5lite.h"
#include "hidem_b200.h"

using h5lite::Type;

namespace hidem {
// defined with the context (api.cu)
hidem_status ctx_fail(hidem_ctx *ctx, hidem_status s, const std::string &msg);
int ctx_precision(const hidem_ctx *ctx);
}  // namespace hidem

namespace {

hidem_status io_fail(hidem_ctx *ctx, const std::string &msg) { return hidem::ctx_fail(ctx, HIDEM_ERR_IO, msg); }

h5lite::Dataset ds(const std::string &name, Type t, uint64_t n, const void *data) {
    h5lite::Dataset d;
    d.name = name;
    d.type = t;
    d.count = n;
    d.data = data;
    return d;
}

void spans(h5lite::Group &g, int64_t count) {
    g.attrs.push_back(h5lite::array_attr<int64_t>("spann_sizes", Type::I64, {count}));
    g.attrs.push_back(h5lite::array_attr<int64_t>("spann_offsets", Type::I64, {0}));
}

}  // namespace


extern "C" hidem_status hidem_checkpoint_write(hidem_ctx *ctx, const char *path) {
    if (!ctx || !path) return HIDEM_ERR_ARG;
    hidem_stats st;
    hidem_status s = hidem_get_stats(ctx, &st);
    if (s != HIDEM_OK) return s;
    const int64_t n = st.num_particles, L = st.num_links;
    if (n <= 0) return io_fail(ctx, "checkpoint: no particles set");
    const bool mixed = hidem::ctx_precision(ctx) == HIDEM_PREC_MIXED;
    const size_t lp = mixed ? 4 : 8;
    const Type lpt = mixed ? Type::F32 : Type::F64;

    std::vector<double> xyz(3 * (size_t)n);
    std::vector<unsigned char> lpf(10 * lp * (size_t)n);
    std::vector<int32_t> owners((size_t)n);
    std::vector<uint8_t> type((size_t)n);
    std::vector<int64_t> keys((size_t)n);
    hidem_particle_soa p{};
    p.xCord = xyz.data();
    p.yCord = xyz.data() + n;
    p.zCord = xyz.data() + 2 * n;
    void **lps[10] = {&p.xTheta, &p.yTheta, &p.zTheta, &p.xDiff, &p.yDiff, &p.zDiff,
                      &p.uDiff, &p.vDiff, &p.wDiff, &p.radius};
    for (int k = 0; k < 10; ++k) *lps[k] = lpf.data() + lp * (size_t)n * k;
    p.owners = owners.data();
    p.type = type.data();
    p.globalKeys = keys.data();
    s = hidem_get_particles(ctx, &p);
    if (s != HIDEM_OK) return s;

    std::vector<int32_t> lowners((size_t)L), lnum((size_t)L);
    std::vector<uint8_t> lstate((size_t)L);
    std::vector<int64_t> lkeys((size_t)L), lA((size_t)L), lB((size_t)L);
    std::vector<unsigned char> l0(lp * (size_t)L), ct(6 * lp * 2 * (size_t)L);
    if (L > 0) {
        hidem_link_soa l{};
        l.owners = lowners.data();
        l.state = lstate.data();
        l.globalKeys = lkeys.data();
        l.globalKeyEndA = lA.data();
        l.globalKeyEndB = lB.data();
        l.initialLen = l0.data();
        l.particleLinkNum = lnum.data();
        for (int k = 0; k < 6; ++k) l.CT[k] = ct.data() + lp * 2 * (size_t)L * k;
        s = hidem_get_links(ctx, &l);
        if (s != HIDEM_OK) return s;
    }

    h5lite::Group root;
    root.name = "/";
    root.attrs.push_back(h5lite::scalar_attr<int32_t>("timeStep", Type::I32, (int32_t)st.step));

    // one rank: the domain is the particles' bounding box, the halo one search distance wider
    double mn[3], mx[3];
    for (int k = 0; k < 3; ++k) {
        const double *c = xyz.data() + (size_t)n * k;
        mn[k] = *std::min_element(c, c + n);
        mx[k] = *std::max_element(c, c + n);
    }
    const double h = st.search_distance;
    h5lite::Group dom;
    dom.name = "Domains";
    const char *ax = "XYZ";
    for (int k = 0; k < 3; ++k) dom.attrs.push_back(h5lite::array_attr<double>(std::string("domainUpper") + ax[k], Type::F64, {mx[k]}));
    for (int k = 0; k < 3; ++k) dom.attrs.push_back(h5lite::array_attr<double>(std::string("domainLower") + ax[k], Type::F64, {mn[k]}));
    for (int k = 0; k < 3; ++k) dom.attrs.push_back(h5lite::array_attr<double>(std::string("domainUpperHalo") + ax[k], Type::F64, {mx[k] + h}));
    for (int k = 0; k < 3; ++k) dom.attrs.push_back(h5lite::array_attr<double>(std::string("domainLowerHalo") + ax[k], Type::F64, {mn[k] - h}));
    dom.attrs.push_back(h5lite::array_attr<int32_t>("domainOwner", Type::I32, {0}));

    h5lite::Group part;
    part.name = "Particles";
    part.datasets.push_back(ds("field_0", Type::F64, n, p.xCord));
    part.datasets.push_back(ds("field_1", Type::F64, n, p.yCord));
    part.datasets.push_back(ds("field_2", Type::F64, n, p.zCord));
    for (int k = 0; k < 10; ++k) part.datasets.push_back(ds("field_" + std::to_string(3 + k), lpt, n, *lps[k]));
    part.datasets.push_back(ds("field_13", Type::I32, n, owners.data()));
    part.datasets.push_back(ds("field_14", Type::U8, n, type.data()));
    part.datasets.push_back(ds("field_15", Type::I64, n, keys.data()));
    spans(part, n);

    h5lite::Group links;
    links.name = "Links";
    links.datasets.push_back(ds("field_0", Type::I32, L, lowners.data()));
    links.datasets.push_back(ds("field_1", Type::U8, L, lstate.data()));
    links.datasets.push_back(ds("field_2", Type::I64, L, lkeys.data()));
    links.datasets.push_back(ds("field_3", Type::I64, L, lA.data()));
    links.datasets.push_back(ds("field_4", Type::I64, L, lB.data()));
    links.datasets.push_back(ds("field_5", lpt, L, l0.data()));
    links.datasets.push_back(ds("field_6", Type::I32, L, lnum.data()));
    spans(links, L);

    h5lite::Group side;
    side.name = "LinkSideData";
    for (int k = 0; k < 6; ++k)
        side.datasets.push_back(ds("side_field_" + std::to_string(7 + k), lpt, 2 * L, ct.data() + lp * 2 * (size_t)L * k));
    spans(side, 2 * L);

    root.groups = {dom, part, links, side};
    std::string err;
    if (!h5lite::write_file(path, root, err)) return io_fail(ctx, "checkpoint: " + err);
    return HIDEM_OK;
}

extern "C" hidem_status hidem_checkpoint_read(hidem_ctx *ctx, const char *path) {
    if (!ctx || !path) return HIDEM_ERR_ARG;
    hidem_status s = HIDEM_OK;
    const bool mixed = hidem::ctx_precision(ctx) == HIDEM_PREC_MIXED;
    const size_t lp = mixed ? 4 : 8;
    const Type lpt = mixed ? Type::F32 : Type::F64;
    h5lite::Group root;
    std::string err;
    if (!h5lite::read_file(path, root, err)) return io_fail(ctx, "checkpoint: " + err);
    const h5lite::Attr *ts = root.attr("timeStep");
    const h5lite::Group *part = root.group("Particles"), *links = root.group("Links"),
                        *side = root.group("LinkSideData");
    if (!ts || !part || !links || !side) return io_fail(ctx, "checkpoint: missing timeStep or a group");
    for (const h5lite::Group *g : {part, links, side}) {
        const h5lite::Attr *sz = g->attr("spann_sizes");
        if (sz && sz->data.size() != 8)
            return io_fail(ctx, "checkpoint: written by " + std::to_string(sz->data.size() / 8) +
                                    " ranks; restarting with a different rank count is not supported");
    }
    auto need = [&](const h5lite::Group *g, const std::string &name, Type t, uint64_t count,
                    uint64_t &outCount, std::vector<unsigned char> &buf) -> bool {
        const h5lite::Dataset *d = g->dataset(name);
        if (!d) { err = g->name + "/" + name + " missing"; return false; }
        if (d->type != t) {
            err = g->name + "/" + name + ": element type does not match this context's precision";
            return false;
        }
        if (count != ~0ull && d->count != count) { err = g->name + "/" + name + ": wrong length"; return false; }
        outCount = d->count;
        buf.resize(d->count * h5lite::type_size(t));
        return h5lite::read_dataset(path, *d, buf.data(), err);
    };
    uint64_t n = 0, L = 0, S = 0, tmp = 0;
    std::vector<unsigned char> pf[16];
    const Type ptypes[16] = {Type::F64, Type::F64, Type::F64, lpt, lpt, lpt, lpt, lpt, lpt,
                             lpt, lpt, lpt, lpt, Type::I32, Type::U8, Type::I64};
    if (!need(part, "field_0", Type::F64, ~0ull, n, pf[0])) return io_fail(ctx, "checkpoint: " + err);
    for (int k = 1; k < 16; ++k)
        if (!need(part, "field_" + std::to_string(k), ptypes[k], n, tmp, pf[k])) return io_fail(ctx, "checkpoint: " + err);
    std::vector<unsigned char> lf[7];
    const Type ltypes[7] = {Type::I32, Type::U8, Type::I64, Type::I64, Type::I64, lpt, Type::I32};
    if (!need(links, "field_0", Type::I32, ~0ull, L, lf[0])) return io_fail(ctx, "checkpoint: " + err);
    for (int k = 1; k < 7; ++k)
        if (!need(links, "field_" + std::to_string(k), ltypes[k], L, tmp, lf[k])) return io_fail(ctx, "checkpoint: " + err);
    std::vector<unsigned char> sf[6];
    for (int k = 0; k < 6; ++k)
        if (!need(side, "side_field_" + std::to_string(7 + k), lpt, 2 * L, S, sf[k])) return io_fail(ctx, "checkpoint: " + err);
    (void)lp;

    hidem_particle_soa p{};
    p.xCord = reinterpret_cast<double *>(pf[0].data());
    p.yCord = reinterpret_cast<double *>(pf[1].data());
    p.zCord = reinterpret_cast<double *>(pf[2].data());
    p.xTheta = pf[3].data();
    p.yTheta = pf[4].data();
    p.zTheta = pf[5].data();
    p.xDiff = pf[6].data();
    p.yDiff = pf[7].data();
    p.zDiff = pf[8].data();
    p.uDiff = pf[9].data();
    p.vDiff = pf[10].data();
    p.wDiff = pf[11].data();
    p.radius = pf[12].data();
    p.owners = reinterpret_cast<int32_t *>(pf[13].data());
    p.type = pf[14].data();
    p.globalKeys = reinterpret_cast<int64_t *>(pf[15].data());
    int32_t step = 0;
    if (ts->data.size() == 4) std::memcpy(&step, ts->data.data(), 4);
    else if (ts->data.size() == 8) { int64_t v; std::memcpy(&v, ts->data.data(), 8); step = (int32_t)v; }
    s = hidem_set_timestep(ctx, step);
    if (s != HIDEM_OK) return s;
    s = hidem_set_particles(ctx, &p, (int64_t)n);
    if (s != HIDEM_OK) return s;
    hidem_link_soa l{};
    l.owners = reinterpret_cast<int32_t *>(lf[0].data());
    l.state = lf[1].data();
    l.globalKeys = reinterpret_cast<int64_t *>(lf[2].data());
    l.globalKeyEndA = reinterpret_cast<int64_t *>(lf[3].data());
    l.globalKeyEndB = reinterpret_cast<int64_t *>(lf[4].data());
    l.initialLen = lf[5].data();
    l.particleLinkNum = reinterpret_cast<int32_t *>(lf[6].data());
    for (int k = 0; k < 6; ++k) l.CT[k] = sf[k].data();
    return hidem_set_links(ctx, &l, (int64_t)L);
}
