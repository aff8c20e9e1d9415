// Minimal HDF5 writer / reader; see h5lite.h for the supported subset. Field layouts
// follow the HDF5 file-format specification (superblock v2, object header v2, messages
// 0x0001 dataspace, 0x0002 link info, 0x0003 datatype, 0x0005 fill value, 0x0006 link,
// 0x0008 data layout, 0x000A group info, 0x000C attribute).
#include "h5lite.h"

#include <algorithm>
#include <cstring>
#include <fstream>
#include <functional>

namespace h5lite {

namespace {

constexpr uint64_t kUndef = ~0ull;
const uint8_t kSignature[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

struct Buf {
    std::vector<uint8_t> b;
    void u8(uint32_t v) { b.push_back((uint8_t)v); }
    void u16(uint32_t v) { for (int i = 0; i < 2; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
    void u32(uint32_t v) { for (int i = 0; i < 4; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
    void u64(uint64_t v) { for (int i = 0; i < 8; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
    void bytes(const void *p, size_t n) {
        const uint8_t *c = static_cast<const uint8_t *>(p);
        b.insert(b.end(), c, c + n);
    }
    void str(const std::string &s) { bytes(s.data(), s.size()); }
};

uint32_t rd16(const uint8_t *p) { return p[0] | (p[1] << 8); }
uint32_t rd32(const uint8_t *p) { return p[0] | (p[1] << 8) | (p[2] << 16) | ((uint32_t)p[3] << 24); }
uint64_t rd64(const uint8_t *p) {
    uint64_t v = 0;
    for (int i = 7; i >= 0; --i) v = (v << 8) | p[i];
    return v;
}

// ---------------------------------------------------------------- messages

void enc_datatype(Buf &m, Type t) {
    const size_t sz = type_size(t);
    if (t == Type::F32 || t == Type::F64) {
        const bool d = t == Type::F64;
        m.u8((1 << 4) | 1);         // version 1, class 1 (floating point)
        m.u8(0x20);                 // little endian, no padding, implied msb normalisation
        m.u8(d ? 63 : 31);          // sign bit location
        m.u8(0);
        m.u32((uint32_t)sz);
        m.u16(0);                   // bit offset
        m.u16((uint32_t)(8 * sz));  // bit precision
        m.u8(d ? 52 : 23);          // exponent location
        m.u8(d ? 11 : 8);           // exponent size
        m.u8(0);                    // mantissa location
        m.u8(d ? 52 : 23);          // mantissa size
        m.u32(d ? 1023 : 127);      // exponent bias
    } else {
        const bool sgn = t == Type::I8 || t == Type::I32 || t == Type::I64;
        m.u8((1 << 4) | 0);         // version 1, class 0 (fixed point)
        m.u8(sgn ? 0x08 : 0x00);    // little endian, no padding, signed bit
        m.u8(0);
        m.u8(0);
        m.u32((uint32_t)sz);
        m.u16(0);
        m.u16((uint32_t)(8 * sz));
    }
}

void enc_dataspace(Buf &m, bool scalar, uint64_t n) {
    m.u8(2);                 // version 2
    m.u8(scalar ? 0 : 1);    // rank
    m.u8(0);                 // no maximum dimensions
    m.u8(scalar ? 0 : 1);    // scalar / simple
    if (!scalar) m.u64(n);
}

void add_msg(Buf &oh, uint32_t type, const Buf &data, uint32_t flags = 0) {
    oh.u8(type);
    oh.u16((uint32_t)data.b.size());
    oh.u8(flags);
    oh.bytes(data.b.data(), data.b.size());
}

void add_attr(Buf &oh, const Attr &a) {
    Buf dt, ds, m;
    enc_datatype(dt, a.type);
    const size_t ts = type_size(a.type);
    enc_dataspace(ds, a.scalar, a.scalar ? 1 : a.data.size() / ts);
    m.u8(3);                                   // version 3
    m.u8(0);                                   // flags
    m.u16((uint32_t)a.name.size() + 1);        // name size with terminator
    m.u16((uint32_t)dt.b.size());
    m.u16((uint32_t)ds.b.size());
    m.u8(0);                                   // ASCII name
    m.str(a.name);
    m.u8(0);
    m.bytes(dt.b.data(), dt.b.size());
    m.bytes(ds.b.data(), ds.b.size());
    m.bytes(a.data.data(), a.data.size());
    add_msg(oh, 0x000C, m);
}

// object header version 2 around `msgs`
std::vector<uint8_t> make_oh(const Buf &msgs) {
    Buf h;
    h.str("OHDR");
    h.u8(2);                                   // version
    h.u8(0x02);                                // chunk #0 size stored in 4 bytes
    h.u32((uint32_t)msgs.b.size());
    h.bytes(msgs.b.data(), msgs.b.size());
    h.u32(lookup3(h.b.data(), h.b.size()));
    return h.b;
}

std::vector<uint8_t> dataset_oh(const Dataset &d, uint64_t dataAddr) {
    Buf msgs, m;
    enc_dataspace(m, false, d.count);
    add_msg(msgs, 0x0001, m);
    m.b.clear();
    enc_datatype(m, d.type);
    add_msg(msgs, 0x0003, m, 0x01);
    m.b.clear();
    m.u8(3);                                   // fill value message version 3
    m.u8(0x02 | (0x02 << 2));                  // allocation late, write fill value if set
    add_msg(msgs, 0x0005, m, 0x01);
    m.b.clear();
    m.u8(3);                                   // layout version 3
    m.u8(1);                                   // contiguous
    m.u64(d.count ? dataAddr : kUndef);
    m.u64(d.count * type_size(d.type));
    add_msg(msgs, 0x0008, m);
    for (const Attr &a : d.attrs) add_attr(msgs, a);
    return make_oh(msgs);
}

std::vector<uint8_t> group_oh(const Group &g, const std::vector<std::pair<std::string, uint64_t>> &links) {
    Buf msgs, m;
    m.u8(0);                                   // link info version 0
    m.u8(0);                                   // no creation order
    m.u64(kUndef);                             // no fractal heap: links are compact
    m.u64(kUndef);                             // no name index
    add_msg(msgs, 0x0002, m);
    m.b.clear();
    m.u8(0);                                   // group info version 0
    m.u8(0);
    add_msg(msgs, 0x000A, m);
    for (const auto &l : links) {
        m.b.clear();
        m.u8(1);                               // link message version 1
        m.u8(0);                               // hard link, 1-byte name length
        m.u8((uint32_t)l.first.size());
        m.str(l.first);
        m.u64(l.second);
        add_msg(msgs, 0x0006, m);
    }
    for (const Attr &a : g.attrs) add_attr(msgs, a);
    return make_oh(msgs);
}

// ---------------------------------------------------------------- reading

struct Reader {
    std::ifstream f;
    uint64_t eof = 0;
    std::string err;

    bool read_at(uint64_t addr, void *dst, size_t n) {
        f.seekg((std::streamoff)addr);
        f.read(static_cast<char *>(dst), (std::streamsize)n);
        return (size_t)f.gcount() == n;
    }

    bool parse_type(const uint8_t *p, size_t n, Type &t, size_t &used) {
        if (n < 8) return false;
        const int cls = p[0] & 0x0f;
        const uint32_t size = rd32(p + 4);
        if (p[1] & 0x01) {
            err = "big-endian data types are not supported";
            return false;
        }
        if (cls == 0) {
            const bool sgn = (p[1] & 0x08) != 0;
            if (size == 1) t = sgn ? Type::I8 : Type::U8;
            else if (size == 4) t = sgn ? Type::I32 : Type::U32;
            else if (size == 8) t = sgn ? Type::I64 : Type::U64;
            else { err = "unsupported integer size"; return false; }
            used = 12;
        } else if (cls == 1) {
            if (size == 4) t = Type::F32;
            else if (size == 8) t = Type::F64;
            else { err = "unsupported float size"; return false; }
            used = 20;
        } else {
            err = "unsupported datatype class " + std::to_string(cls);
            return false;
        }
        return used <= n;
    }

    bool parse_space(const uint8_t *p, size_t n, bool &scalar, uint64_t &count, size_t &used) {
        if (n < 4) return false;
        const int ver = p[0], rank = p[1], flags = p[2];
        size_t off;
        if (ver == 1) off = 8;
        else if (ver == 2) off = 4;
        else { err = "unsupported dataspace version"; return false; }
        if (ver == 2 && p[3] == 2) { scalar = false; count = 0; used = off; return true; }  // null
        count = 1;
        for (int r = 0; r < rank; ++r) {
            if (off + 8 > n) return false;
            count *= rd64(p + off);
            off += 8;
        }
        if (flags & 1) off += 8 * rank;
        scalar = rank == 0;
        used = off;
        return true;
    }

    bool parse_attr(const uint8_t *p, size_t n, Attr &a) {
        const int ver = p[0];
        size_t nameSize = rd16(p + 2), dtSize = rd16(p + 4), dsSize = rd16(p + 6);
        size_t off;
        auto pad8 = [](size_t v) { return (v + 7) & ~size_t(7); };
        if (ver == 3) {
            off = 9;
            a.name.assign(reinterpret_cast<const char *>(p + off), nameSize ? nameSize - 1 : 0);
            off += nameSize;
        } else if (ver == 1) {
            off = 8;
            a.name.assign(reinterpret_cast<const char *>(p + off), nameSize ? nameSize - 1 : 0);
            off += pad8(nameSize);
        } else {
            err = "unsupported attribute version";
            return false;
        }
        size_t used = 0;
        if (!parse_type(p + off, dtSize, a.type, used)) return false;
        off += ver == 1 ? pad8(dtSize) : dtSize;
        uint64_t count = 0;
        if (!parse_space(p + off, dsSize, a.scalar, count, used)) return false;
        off += ver == 1 ? pad8(dsSize) : dsSize;
        const size_t bytes = count * type_size(a.type);
        if (off + bytes > n) { err = "attribute data truncated"; return false; }
        a.data.assign(p + off, p + off + bytes);
        return true;
    }

    // parses the object header at addr into a group or a dataset
    bool parse_object(uint64_t addr, const std::string &name, Group *g, Dataset *d, bool &isGroup,
                      int depth) {
        if (depth > 16) { err = "group nesting too deep"; return false; }
        uint8_t pre[16];
        if (!read_at(addr, pre, 6) || std::memcmp(pre, "OHDR", 4) != 0) {
            err = "object header at " + std::to_string(addr) + ": not a version-2 header (only the "
                  "superblock-v2 / object-header-v2 layout is supported)";
            return false;
        }
        const int flags = pre[5];
        size_t off = 6;
        if (flags & 0x20) off += 16;
        if (flags & 0x10) off += 4;
        const int w = 1 << (flags & 3);
        uint8_t sz[8] = {0};
        if (!read_at(addr + off, sz, w)) return false;
        uint64_t chunk = 0;
        for (int i = w - 1; i >= 0; --i) chunk = (chunk << 8) | sz[i];
        off += w;
        std::vector<uint8_t> all(off + chunk + 4);
        if (!read_at(addr, all.data(), all.size())) { err = "truncated object header"; return false; }
        if (lookup3(all.data(), off + chunk) != rd32(all.data() + off + chunk)) {
            err = "object header checksum mismatch at " + std::to_string(addr);
            return false;
        }
        const uint8_t *p = all.data() + off;
        const uint8_t *end = p + chunk;
        bool haveLayout = false, haveLinks = false;
        Type dtype = Type::U8;
        uint64_t count = 0, dataAddr = kUndef, dataSize = 0;
        std::vector<Attr> attrs;
        std::vector<std::pair<std::string, uint64_t>> links;
        while (p + 4 <= end) {
            const int type = p[0];
            const size_t msize = rd16(p + 1);
            const int mflags = p[3];
            p += 4;
            if (flags & 0x04) p += 2;  // creation order
            if (p + msize > end) { err = "message overruns its header"; return false; }
            (void)mflags;
            size_t used = 0;
            bool scalar = false;
            switch (type) {
            case 0x0001:
                if (!parse_space(p, msize, scalar, count, used)) return false;
                break;
            case 0x0002:
                haveLinks = true;
                if (rd64(p + 2 + ((p[1] & 1) ? 8 : 0)) != kUndef) {
                    err = "dense link storage is not supported";
                    return false;
                }
                break;
            case 0x0003:
                if (!parse_type(p, msize, dtype, used)) return false;
                break;
            case 0x0006: {
                haveLinks = true;
                const int lf = p[1];
                size_t o = 2;
                int ltype = 0;
                if (lf & 0x08) ltype = p[o++];
                if (lf & 0x04) o += 8;
                if (lf & 0x10) o += 1;
                const int lw = 1 << (lf & 3);
                uint64_t len = 0;
                for (int i = lw - 1; i >= 0; --i) len = (len << 8) | p[o + i];
                o += lw;
                std::string lname(reinterpret_cast<const char *>(p + o), len);
                o += len;
                if (ltype != 0) break;  // soft / external links are not followed
                links.push_back({lname, rd64(p + o)});
                break;
            }
            case 0x0008:
                if (p[0] != 3) { err = "unsupported layout message version"; return false; }
                if (p[1] != 1) { err = "dataset '" + name + "' is not contiguous (chunked or compact)"; return false; }
                haveLayout = true;
                dataAddr = rd64(p + 2);
                dataSize = rd64(p + 10);
                break;
            case 0x000B:
                err = "filtered datasets are not supported";
                return false;
            case 0x000C: {
                Attr a;
                if (!parse_attr(p, msize, a)) return false;
                attrs.push_back(a);
                break;
            }
            case 0x0010:
                err = "object header continuation blocks are not supported";
                return false;
            default:
                break;  // NIL, fill value, modification time, ...
            }
            p += msize;
        }
        if (haveLayout) {
            isGroup = false;
            if (!d) return true;
            d->name = name;
            d->type = dtype;
            d->count = count;
            d->fileOffset = dataAddr;
            d->attrs = attrs;
            if (dataSize != count * type_size(dtype)) { err = "dataset '" + name + "' size mismatch"; return false; }
            return true;
        }
        isGroup = true;
        (void)haveLinks;
        if (!g) return true;
        g->name = name;
        g->attrs = attrs;
        for (const auto &l : links) {
            Group cg;
            Dataset cd;
            bool childIsGroup = false;
            if (!parse_object(l.second, l.first, &cg, &cd, childIsGroup, depth + 1)) return false;
            if (childIsGroup) g->groups.push_back(cg);
            else g->datasets.push_back(cd);
        }
        return true;
    }
};

}  // namespace

size_t type_size(Type t) {
    switch (t) {
    case Type::I8:
    case Type::U8: return 1;
    case Type::I32:
    case Type::U32:
    case Type::F32: return 4;
    default: return 8;
    }
}

const Group *Group::group(const std::string &n) const {
    for (const Group &g : groups) if (g.name == n) return &g;
    return nullptr;
}
const Dataset *Group::dataset(const std::string &n) const {
    for (const Dataset &d : datasets) if (d.name == n) return &d;
    return nullptr;
}
const Attr *Group::attr(const std::string &n) const {
    for (const Attr &a : attrs) if (a.name == n) return &a;
    return nullptr;
}

uint32_t lookup3(const uint8_t *k, size_t length, uint32_t initval) {
    auto rot = [](uint32_t x, int r) { return (x << r) | (x >> (32 - r)); };
    uint32_t a, b, c;
    a = b = c = 0xdeadbeefu + (uint32_t)length + initval;
    while (length > 12) {
        a += k[0] + ((uint32_t)k[1] << 8) + ((uint32_t)k[2] << 16) + ((uint32_t)k[3] << 24);
        b += k[4] + ((uint32_t)k[5] << 8) + ((uint32_t)k[6] << 16) + ((uint32_t)k[7] << 24);
        c += k[8] + ((uint32_t)k[9] << 8) + ((uint32_t)k[10] << 16) + ((uint32_t)k[11] << 24);
        a -= c; a ^= rot(c, 4);  c += b;
        b -= a; b ^= rot(a, 6);  a += c;
        c -= b; c ^= rot(b, 8);  b += a;
        a -= c; a ^= rot(c, 16); c += b;
        b -= a; b ^= rot(a, 19); a += c;
        c -= b; c ^= rot(b, 4);  b += a;
        length -= 12;
        k += 12;
    }
    switch (length) {
    case 12: c += (uint32_t)k[11] << 24; [[fallthrough]];
    case 11: c += (uint32_t)k[10] << 16; [[fallthrough]];
    case 10: c += (uint32_t)k[9] << 8; [[fallthrough]];
    case 9: c += k[8]; [[fallthrough]];
    case 8: b += (uint32_t)k[7] << 24; [[fallthrough]];
    case 7: b += (uint32_t)k[6] << 16; [[fallthrough]];
    case 6: b += (uint32_t)k[5] << 8; [[fallthrough]];
    case 5: b += k[4]; [[fallthrough]];
    case 4: a += (uint32_t)k[3] << 24; [[fallthrough]];
    case 3: a += (uint32_t)k[2] << 16; [[fallthrough]];
    case 2: a += (uint32_t)k[1] << 8; [[fallthrough]];
    case 1: a += k[0]; break;
    case 0: return c;
    }
    c ^= b; c -= rot(b, 14);
    a ^= c; a -= rot(c, 11);
    b ^= a; b -= rot(a, 25);
    c ^= b; c -= rot(b, 16);
    a ^= c; a -= rot(c, 4);
    b ^= a; b -= rot(a, 14);
    c ^= b; c -= rot(b, 24);
    return c;
}

bool write_file(const std::string &path, const Group &root, std::string &err) {
    // 1. object-header sizes do not depend on address values: lay out headers, then data
    struct Node {
        const Group *g = nullptr;
        const Dataset *d = nullptr;
        uint64_t addr = 0, size = 0, dataAddr = 0;
        std::vector<size_t> children;
    };
    std::vector<Node> nodes;
    std::function<size_t(const Group &)> add_group = [&](const Group &g) -> size_t {
        const size_t id = nodes.size();
        nodes.push_back(Node{&g});
        std::vector<size_t> ch;
        for (const Group &c : g.groups) ch.push_back(add_group(c));
        for (const Dataset &d : g.datasets) {
            nodes.push_back(Node{nullptr, &d});
            ch.push_back(nodes.size() - 1);
        }
        nodes[id].children = ch;
        return id;
    };
    add_group(root);
    auto encode = [&](const Node &nd) {
        if (nd.d) return dataset_oh(*nd.d, nd.dataAddr);
        std::vector<std::pair<std::string, uint64_t>> links;
        for (size_t c : nd.children)
            links.push_back({nodes[c].g ? nodes[c].g->name : nodes[c].d->name, nodes[c].addr});
        return group_oh(*nd.g, links);
    };
    uint64_t off = 48;
    for (Node &nd : nodes) {
        nd.size = encode(nd).size();
        nd.addr = off;
        off += nd.size;
    }
    for (Node &nd : nodes) {
        if (!nd.d) continue;
        off = (off + 7) & ~uint64_t(7);
        nd.dataAddr = off;
        off += nd.d->count * type_size(nd.d->type);
    }
    const uint64_t eof = off;

    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f) {
        err = "cannot create " + path;
        return false;
    }
    Buf sb;
    sb.bytes(kSignature, 8);
    sb.u8(2);        // superblock version 2
    sb.u8(8);        // size of offsets
    sb.u8(8);        // size of lengths
    sb.u8(0);        // file consistency flags
    sb.u64(0);       // base address
    sb.u64(kUndef);  // superblock extension
    sb.u64(eof);
    sb.u64(nodes[0].addr);
    sb.u32(lookup3(sb.b.data(), sb.b.size()));
    f.write(reinterpret_cast<const char *>(sb.b.data()), (std::streamsize)sb.b.size());
    for (Node &nd : nodes) {
        std::vector<uint8_t> h = encode(nd);
        f.seekp((std::streamoff)nd.addr);
        f.write(reinterpret_cast<const char *>(h.data()), (std::streamsize)h.size());
    }
    uint64_t written = nodes.back().addr + nodes.back().size;
    for (Node &nd : nodes) {
        if (!nd.d || nd.d->count == 0) continue;
        f.seekp((std::streamoff)nd.dataAddr);
        const uint64_t bytes = nd.d->count * type_size(nd.d->type);
        f.write(static_cast<const char *>(nd.d->data), (std::streamsize)bytes);
        written = std::max<uint64_t>(written, nd.dataAddr + bytes);
    }
    // the file must reach the end-of-file address stored in the superblock
    if (written < eof) {
        f.seekp((std::streamoff)(eof - 1));
        f.put('\0');
    }
    f.flush();
    if (!f) {
        err = "write failed: " + path;
        return false;
    }
    return true;
}

bool read_file(const std::string &path, Group &root, std::string &err) {
    Reader r;
    r.f.open(path, std::ios::binary);
    if (!r.f) {
        err = "cannot open " + path;
        return false;
    }
    uint8_t sb[48];
    if (!r.read_at(0, sb, 48) || std::memcmp(sb, kSignature, 8) != 0) {
        err = path + ": not an HDF5 file (signature at offset 0)";
        return false;
    }
    if (sb[8] != 2 && sb[8] != 3) {
        err = path + ": superblock version " + std::to_string(sb[8]) + " is not supported (2 or 3)";
        return false;
    }
    if (sb[9] != 8 || sb[10] != 8) {
        err = path + ": only 8-byte offsets and lengths are supported";
        return false;
    }
    if (lookup3(sb, 44) != rd32(sb + 44)) {
        err = path + ": superblock checksum mismatch";
        return false;
    }
    if (rd64(sb + 12) != 0) {
        err = path + ": non-zero base address is not supported";
        return false;
    }
    r.eof = rd64(sb + 28);
    bool isGroup = false;
    Dataset unused;
    if (!r.parse_object(rd64(sb + 36), "/", &root, &unused, isGroup, 0) || !isGroup) {
        err = r.err.empty() ? "root object is not a group" : r.err;
        return false;
    }
    return true;
}

bool read_dataset(const std::string &path, const Dataset &d, void *out, std::string &err) {
    const size_t bytes = d.count * type_size(d.type);
    if (bytes == 0) return true;
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        err = "cannot open " + path;
        return false;
    }
    f.seekg((std::streamoff)d.fileOffset);
    f.read(static_cast<char *>(out), (std::streamsize)bytes);
    if ((size_t)f.gcount() != bytes) {
        err = "dataset '" + d.name + "' truncated";
        return false;
    }
    return true;
}

}  // namespace h5lite
