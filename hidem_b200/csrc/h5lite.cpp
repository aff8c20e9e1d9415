// Minimal HDF5 writer / reader; see h5lite.h for the supported subset. Field layouts
// follow the HDF5 file-format specification (superblocks 0-3, object headers 1 and 2,
// messages 0x0001 dataspace, 0x0002 link info, 0x0003 datatype, 0x0005 fill value,
// 0x0006 link, 0x0008 data layout, 0x000A group info, 0x000B filter pipeline, 0x000C
// attribute, 0x0010 continuation, 0x0011 symbol table; version-1 B-trees of group and
// chunk nodes, local heaps, symbol nodes). Deflate-filtered chunks are inflated with zlib.
#include "h5lite.h"

#include <algorithm>
#include <cstring>
#include <fstream>
#include <functional>

#include <zlib.h>

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
//
// Two generations of the on-disk format are read:
//  * what libhdf5 writes by default (the reference's files): superblock version 0 or 1,
//    version-1 object headers (messages padded to 8 bytes, continuation blocks), groups
//    as symbol tables (a version-1 B-tree of symbol nodes over a local heap of names),
//    datasets contiguous, compact or chunked (a version-1 B-tree of chunks) with the
//    deflate and shuffle filters, attributes of message versions 1 to 3;
//  * what this library writes: superblock version 2 or 3, version-2 object headers with
//    lookup3 checksums, compact link storage.

struct Message {
    int type = 0;
    std::vector<uint8_t> body;
};

struct Reader {
    std::ifstream f;
    uint64_t eof = 0;
    std::string err;

    bool read_at(uint64_t addr, void *dst, size_t n) {
        f.clear();
        f.seekg((std::streamoff)addr);
        f.read(static_cast<char *>(dst), (std::streamsize)n);
        return (size_t)f.gcount() == n;
    }

    bool fail(const std::string &m) {
        if (err.empty()) err = m;
        return false;
    }

    bool parse_type(const uint8_t *p, size_t n, Type &t, size_t &used) {
        if (n < 8) return fail("datatype message truncated");
        const int cls = p[0] & 0x0f;
        const uint32_t size = rd32(p + 4);
        if (p[1] & 0x01) return fail("big-endian data types are not supported");
        if (cls == 0) {
            const bool sgn = (p[1] & 0x08) != 0;
            if (size == 1) t = sgn ? Type::I8 : Type::U8;
            else if (size == 4) t = sgn ? Type::I32 : Type::U32;
            else if (size == 8) t = sgn ? Type::I64 : Type::U64;
            else return fail("unsupported integer size " + std::to_string(size));
            used = 12;
        } else if (cls == 1) {
            if (size == 4) t = Type::F32;
            else if (size == 8) t = Type::F64;
            else return fail("unsupported float size " + std::to_string(size));
            used = 20;
        } else {
            return fail("unsupported datatype class " + std::to_string(cls));
        }
        return used <= n || fail("datatype message truncated");
    }

    // dataspace message versions 1 and 2; dims receives the current extent
    bool parse_space(const uint8_t *p, size_t n, bool &scalar, uint64_t &count, size_t &used,
                     std::vector<uint64_t> *dims = nullptr) {
        if (n < 4) return fail("dataspace message truncated");
        const int ver = p[0], rank = p[1], flags = p[2];
        size_t off;
        if (ver == 1) off = 8;
        else if (ver == 2) off = 4;
        else return fail("unsupported dataspace version " + std::to_string(ver));
        if (dims) dims->clear();
        if (ver == 2 && p[3] == 2) { scalar = false; count = 0; used = off; return true; }  // null
        count = 1;
        for (int r = 0; r < rank; ++r) {
            if (off + 8 > n) return fail("dataspace message truncated");
            const uint64_t d = rd64(p + off);
            count *= d;
            if (dims) dims->push_back(d);
            off += 8;
        }
        if (flags & 1) off += 8 * rank;
        scalar = rank == 0;
        used = off;
        return true;
    }

    // attribute message versions 1 (fields padded to 8 bytes), 2 and 3
    bool parse_attr(const uint8_t *p, size_t n, Attr &a) {
        if (n < 8) return fail("attribute message truncated");
        const int ver = p[0];
        size_t nameSize = rd16(p + 2), dtSize = rd16(p + 4), dsSize = rd16(p + 6);
        size_t off;
        auto pad8 = [](size_t v) { return (v + 7) & ~size_t(7); };
        if (ver == 1 && p[1] != 0) return fail("unsupported attribute flags");
        if (ver == 2 && (p[1] & 3)) return fail("shared attribute datatypes are not supported");
        if (ver == 3 && (p[1] & 3)) return fail("shared attribute datatypes are not supported");
        if (ver == 3) off = 9;
        else if (ver == 1 || ver == 2) off = 8;
        else return fail("unsupported attribute version " + std::to_string(ver));
        if (off + nameSize > n) return fail("attribute message truncated");
        a.name.assign(reinterpret_cast<const char *>(p + off), nameSize ? nameSize - 1 : 0);
        off += ver == 1 ? pad8(nameSize) : nameSize;
        size_t used = 0;
        if (off + dtSize > n || !parse_type(p + off, dtSize, a.type, used)) return fail("attribute datatype");
        off += ver == 1 ? pad8(dtSize) : dtSize;
        uint64_t count = 0;
        if (off + dsSize > n || !parse_space(p + off, dsSize, a.scalar, count, used)) return fail("attribute dataspace");
        off += ver == 1 ? pad8(dsSize) : dsSize;
        const size_t bytes = count * type_size(a.type);
        if (off + bytes > n) return fail("attribute data truncated");
        a.data.assign(p + off, p + off + bytes);
        return true;
    }

    // all messages of the object header at addr (version 1 or 2), continuation blocks followed
    bool collect_messages(uint64_t addr, std::vector<Message> &out) {
        uint8_t pre[16];
        if (!read_at(addr, pre, 16)) return fail("object header at " + std::to_string(addr) + " truncated");
        struct Block { uint64_t addr, size; };
        std::vector<Block> pending;
        int hflags = 0;
        bool v2 = std::memcmp(pre, "OHDR", 4) == 0;
        if (v2) {
            if (pre[4] != 2) return fail("unsupported object header version");
            hflags = pre[5];
            size_t off = 6;
            if (hflags & 0x20) off += 16;
            if (hflags & 0x10) off += 4;
            const int w = 1 << (hflags & 3);
            uint64_t chunk = 0;
            for (int i = w - 1; i >= 0; --i) chunk = (chunk << 8) | pre[off + i];
            off += w;
            std::vector<uint8_t> all(off + chunk + 4);
            if (!read_at(addr, all.data(), all.size())) return fail("truncated object header");
            if (lookup3(all.data(), off + chunk) != rd32(all.data() + off + chunk))
                return fail("object header checksum mismatch at " + std::to_string(addr));
            if (!v2_messages(all.data() + off, chunk, hflags, out, pending)) return false;
        } else {
            if (pre[0] != 1) return fail("object header at " + std::to_string(addr) + ": unknown version");
            const uint32_t size = rd32(pre + 8);
            if (!v1_block(addr + 16, size, out, pending)) return false;
        }
        int guard = 0;
        while (!pending.empty()) {
            if (++guard > 4096) return fail("too many object header continuation blocks");
            const Block b = pending.front();
            pending.erase(pending.begin());
            if (b.size > (1u << 26)) return fail("object header continuation block too large");
            if (v2) {
                std::vector<uint8_t> blk(b.size);
                if (!read_at(b.addr, blk.data(), blk.size()) || b.size < 8 || std::memcmp(blk.data(), "OCHK", 4) != 0)
                    return fail("bad object header continuation block");
                if (lookup3(blk.data(), b.size - 4) != rd32(blk.data() + b.size - 4))
                    return fail("continuation block checksum mismatch");
                if (!v2_messages(blk.data() + 4, b.size - 8, hflags, out, pending)) return false;
            } else if (!v1_block(b.addr, b.size, out, pending)) {
                return false;
            }
        }
        return true;
    }

    template <class Pending>
    bool v2_messages(const uint8_t *p, size_t n, int hflags, std::vector<Message> &out, Pending &pending) {
        const uint8_t *end = p + n;
        const size_t hdr = (hflags & 0x04) ? 6 : 4;
        while (p + hdr <= end) {
            const int type = p[0];
            const size_t msize = rd16(p + 1);
            if (p[3] & 0x02) return fail("shared object header messages are not supported");
            p += hdr;
            if (p + msize > end) return fail("message overruns its header");
            if (type == 0x0010) {
                if (msize < 16) return fail("continuation message truncated");
                pending.push_back({rd64(p), rd64(p + 8)});
            } else {
                out.push_back(Message{type, std::vector<uint8_t>(p, p + msize)});
            }
            p += msize;
        }
        return true;
    }

    template <class Pending>
    bool v1_block(uint64_t addr, uint64_t size, std::vector<Message> &out, Pending &pending) {
        if (size > (1u << 26)) return fail("object header block too large");
        std::vector<uint8_t> blk(size);
        if (!read_at(addr, blk.data(), blk.size())) return fail("truncated object header block");
        size_t o = 0;
        while (o + 8 <= size) {
            const int type = (int)rd16(blk.data() + o);
            const size_t msize = rd16(blk.data() + o + 2);
            const int mflags = blk[o + 4];
            o += 8;
            if (o + msize > size) return fail("message overruns its header block");
            if ((mflags & 0x02) && type != 0) return fail("shared object header messages are not supported");
            if (type == 0x0010) {
                if (msize < 16) return fail("continuation message truncated");
                pending.push_back({rd64(blk.data() + o), rd64(blk.data() + o + 8)});
            } else if (type != 0) {
                out.push_back(Message{type, std::vector<uint8_t>(blk.data() + o, blk.data() + o + msize)});
            }
            o += msize;
        }
        return true;
    }

    // names and object addresses of a symbol-table group: its version-1 B-tree (node type 0)
    // over symbol nodes, names in the local heap
    bool symbol_table(uint64_t btree, uint64_t heap, std::vector<std::pair<std::string, uint64_t>> &links) {
        uint8_t h[32];
        if (!read_at(heap, h, 32) || std::memcmp(h, "HEAP", 4) != 0) return fail("bad local heap");
        const uint64_t heapSize = rd64(h + 8), heapData = rd64(h + 24);
        if (heapSize > (1u << 28)) return fail("local heap too large");
        std::vector<uint8_t> names(heapSize);
        if (!read_at(heapData, names.data(), names.size())) return fail("truncated local heap");
        return group_node(btree, names, links, 0);
    }

    bool group_node(uint64_t addr, const std::vector<uint8_t> &names,
                    std::vector<std::pair<std::string, uint64_t>> &links, int depth) {
        if (depth > 32) return fail("group B-tree too deep");
        uint8_t h[24];
        if (!read_at(addr, h, 24) || std::memcmp(h, "TREE", 4) != 0 || h[4] != 0)
            return fail("bad group B-tree node");
        const int level = h[5];
        const uint32_t used = rd16(h + 6);
        std::vector<uint8_t> kc(8 + 16 * (size_t)used);
        if (!read_at(addr + 24, kc.data(), kc.size())) return fail("truncated group B-tree node");
        for (uint32_t i = 0; i < used; ++i) {
            const uint64_t child = rd64(kc.data() + 8 + 16 * i);
            if (level > 0) {
                if (!group_node(child, names, links, depth + 1)) return false;
                continue;
            }
            uint8_t sh[8];
            if (!read_at(child, sh, 8) || std::memcmp(sh, "SNOD", 4) != 0) return fail("bad symbol node");
            const uint32_t nsym = rd16(sh + 6);
            std::vector<uint8_t> ent(40 * (size_t)nsym);
            if (!read_at(child + 8, ent.data(), ent.size())) return fail("truncated symbol node");
            for (uint32_t k = 0; k < nsym; ++k) {
                const uint64_t nameOff = rd64(ent.data() + 40 * k);
                const uint64_t oh = rd64(ent.data() + 40 * k + 8);
                if (nameOff >= names.size()) return fail("symbol name outside the local heap");
                const char *nm = reinterpret_cast<const char *>(names.data() + nameOff);
                links.push_back({std::string(nm, strnlen(nm, names.size() - nameOff)), oh});
            }
        }
        return true;
    }

    // parses the object header at addr into a group or a dataset
    bool parse_object(uint64_t addr, const std::string &name, Group *g, Dataset *d, bool &isGroup,
                      int depth) {
        if (depth > 16) return fail("group nesting too deep");
        std::vector<Message> msgs;
        if (!collect_messages(addr, msgs)) return false;
        bool haveLayout = false;
        Type dtype = Type::U8;
        uint64_t count = 0;
        std::vector<uint64_t> dims;
        Dataset ds;
        std::vector<Attr> attrs;
        std::vector<std::pair<std::string, uint64_t>> links;
        for (const Message &m : msgs) {
            const uint8_t *p = m.body.data();
            const size_t msize = m.body.size();
            size_t used = 0;
            bool scalar = false;
            switch (m.type) {
            case 0x0001:
                if (!parse_space(p, msize, scalar, count, used, &dims)) return false;
                break;
            case 0x0002:
                if (msize < 18 || rd64(p + 2 + ((p[1] & 1) ? 8 : 0)) != kUndef)
                    return fail("dense link storage is not supported");
                break;
            case 0x0003:
                if (!parse_type(p, msize, dtype, used)) return false;
                break;
            case 0x0006: {
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
                if (o + len + 8 > msize && ltype == 0) return fail("link message truncated");
                std::string lname(reinterpret_cast<const char *>(p + o), len);
                o += len;
                if (ltype != 0) break;  // soft / external links are not followed
                links.push_back({lname, rd64(p + o)});
                break;
            }
            case 0x0008:
                if (!parse_layout(p, msize, ds, name)) return false;
                haveLayout = true;
                break;
            case 0x000B:
                if (!parse_filters(p, msize, ds)) return false;
                break;
            case 0x000C: {
                Attr a;
                if (!parse_attr(p, msize, a)) return false;
                attrs.push_back(a);
                break;
            }
            case 0x0011:
                if (msize < 16 || !symbol_table(rd64(p), rd64(p + 8), links)) return false;
                break;
            default:
                break;  // NIL, fill value, modification time, group info, ...
            }
        }
        if (haveLayout) {
            isGroup = false;
            if (!d) return true;
            ds.name = name;
            ds.type = dtype;
            ds.count = count;
            ds.dims = dims;
            ds.attrs = attrs;
            const size_t es = type_size(dtype);
            if (ds.layout == 1 && ds.storedBytes != kUndef && ds.storedBytes != count * es && count != 0)
                return fail("dataset '" + name + "' size mismatch");
            if (ds.layout == 0 && ds.compact.size() != count * es) return fail("dataset '" + name + "' compact size mismatch");
            if (ds.layout == 2) {
                if (ds.chunk.size() != dims.size() + 1 || ds.chunk.back() != es)
                    return fail("dataset '" + name + "' chunk shape does not match its dataspace");
                ds.chunk.pop_back();
                for (uint64_t c : ds.chunk)
                    if (c == 0) return fail("dataset '" + name + "' has a zero chunk extent");
            }
            *d = ds;
            return true;
        }
        isGroup = true;
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

    // data layout message versions 1 to 3: compact, contiguous or chunked (v1 B-tree index)
    bool parse_layout(const uint8_t *p, size_t n, Dataset &ds, const std::string &name) {
        if (n < 2) return fail("layout message truncated");
        const int ver = p[0];
        if (ver == 3) {
            const int cls = p[1];
            if (cls == 0) {
                if (n < 4) return fail("layout message truncated");
                const size_t sz = rd16(p + 2);
                if (4 + sz > n) return fail("compact data truncated");
                ds.layout = 0;
                ds.compact.assign(p + 4, p + 4 + sz);
            } else if (cls == 1) {
                if (n < 18) return fail("layout message truncated");
                ds.layout = 1;
                ds.fileOffset = rd64(p + 2);
                ds.storedBytes = rd64(p + 10);
            } else if (cls == 2) {
                const int dim = p[2];
                if (n < 11 + 4 * (size_t)dim) return fail("layout message truncated");
                ds.layout = 2;
                ds.chunkIndex = rd64(p + 3);
                ds.chunk.clear();
                for (int k = 0; k < dim; ++k) ds.chunk.push_back(rd32(p + 11 + 4 * k));
            } else {
                return fail("dataset '" + name + "': unsupported layout class " + std::to_string(cls));
            }
            return true;
        }
        if (ver == 1 || ver == 2) {
            const int dim = p[1], cls = p[2];
            size_t o = 8;
            uint64_t a = kUndef;
            if (cls != 0) {
                if (o + 8 > n) return fail("layout message truncated");
                a = rd64(p + o);
                o += 8;
            }
            std::vector<uint64_t> dd;
            for (int k = 0; k < dim; ++k) {
                if (o + 4 > n) return fail("layout message truncated");
                dd.push_back(rd32(p + o));
                o += 4;
            }
            if (cls == 0) {
                if (o + 4 > n) return fail("layout message truncated");
                const size_t sz = rd32(p + o);
                o += 4;
                if (o + sz > n) return fail("compact data truncated");
                ds.layout = 0;
                ds.compact.assign(p + o, p + o + sz);
            } else if (cls == 1) {
                ds.layout = 1;
                ds.fileOffset = a;
                ds.storedBytes = kUndef;
            } else if (cls == 2) {
                ds.layout = 2;
                ds.chunkIndex = a;
                ds.chunk = dd;
            } else {
                return fail("dataset '" + name + "': unsupported layout class");
            }
            return true;
        }
        return fail("dataset '" + name + "': layout message version " + std::to_string(ver) +
                    " (chunk indices of files written with the newest format) is not supported");
    }

    // filter pipeline message versions 1 and 2
    bool parse_filters(const uint8_t *p, size_t n, Dataset &ds) {
        if (n < 2) return fail("filter pipeline message truncated");
        const int ver = p[0], nf = p[1];
        size_t o = ver == 1 ? 8 : 2;
        if (ver != 1 && ver != 2) return fail("unsupported filter pipeline version");
        ds.filters.clear();
        for (int k = 0; k < nf; ++k) {
            if (o + 4 > n) return fail("filter pipeline message truncated");
            Filter f;
            f.id = (uint16_t)rd16(p + o);
            o += 2;
            size_t nameLen = 0;
            if (ver == 1 || f.id >= 256) {
                nameLen = rd16(p + o);
                o += 2;
            }
            if (o + 4 > n) return fail("filter pipeline message truncated");
            f.optional = (rd16(p + o) & 1) != 0;
            const size_t nv = rd16(p + o + 2);
            o += 4;
            o += ver == 1 ? ((nameLen + 7) & ~size_t(7)) : nameLen;
            for (size_t v = 0; v < nv; ++v) {
                if (o + 4 > n) return fail("filter pipeline message truncated");
                f.values.push_back(rd32(p + o));
                o += 4;
            }
            if (ver == 1 && (nv & 1)) o += 4;
            if (f.id != 1 && f.id != 2)
                return fail("filter " + std::to_string(f.id) + " is not supported (deflate and shuffle are)");
            ds.filters.push_back(f);
        }
        return true;
    }

    // the chunks of a dataset: (chunk offsets in elements, filter mask, file address, stored size)
    struct Chunk {
        std::vector<uint64_t> offset;
        uint32_t mask = 0;
        uint64_t addr = 0, size = 0;
    };

    bool chunk_node(uint64_t addr, int rank, std::vector<Chunk> &out, int depth) {
        if (depth > 32) return fail("chunk B-tree too deep");
        uint8_t h[24];
        if (!read_at(addr, h, 24) || std::memcmp(h, "TREE", 4) != 0 || h[4] != 1)
            return fail("bad chunk B-tree node");
        const int level = h[5];
        const uint32_t used = rd16(h + 6);
        const size_t keySize = 8 + 8 * (size_t)(rank + 1);
        std::vector<uint8_t> kc((keySize + 8) * used + keySize);
        if (!read_at(addr + 24, kc.data(), kc.size())) return fail("truncated chunk B-tree node");
        for (uint32_t i = 0; i < used; ++i) {
            const uint8_t *key = kc.data() + (keySize + 8) * i;
            const uint64_t child = rd64(key + keySize);
            if (level > 0) {
                if (!chunk_node(child, rank, out, depth + 1)) return false;
                continue;
            }
            Chunk c;
            c.size = rd32(key);
            c.mask = rd32(key + 4);
            for (int k = 0; k < rank; ++k) c.offset.push_back(rd64(key + 8 + 8 * k));
            c.addr = child;
            out.push_back(c);
        }
        return true;
    }
};

// undoes the filters of one stored chunk (pipeline order reversed, masked filters skipped)
bool unfilter(const Dataset &d, uint32_t mask, std::vector<uint8_t> &buf, size_t expect, std::string &err) {
    for (int k = (int)d.filters.size() - 1; k >= 0; --k) {
        if (mask & (1u << k)) continue;
        const Filter &f = d.filters[k];
        if (f.id == 1) {
            std::vector<uint8_t> out(expect);
            uLongf len = (uLongf)expect;
            const int rc = uncompress(out.data(), &len, buf.data(), (uLong)buf.size());
            if (rc != Z_OK) {
                err = "dataset '" + d.name + "': inflate failed (zlib " + std::to_string(rc) + ")";
                return false;
            }
            out.resize(len);
            buf.swap(out);
        } else if (f.id == 2) {
            const size_t es = f.values.empty() ? type_size(d.type) : f.values[0];
            if (es > 1) {
                const size_t n = buf.size() / es;
                std::vector<uint8_t> out(buf.size());
                for (size_t b = 0; b < es; ++b)
                    for (size_t i = 0; i < n; ++i) out[i * es + b] = buf[b * n + i];
                std::copy(buf.begin() + n * es, buf.end(), out.begin() + n * es);
                buf.swap(out);
            }
        }
    }
    if (buf.size() != expect) {
        err = "dataset '" + d.name + "': a chunk holds " + std::to_string(buf.size()) + " bytes, expected " +
              std::to_string(expect);
        return false;
    }
    return true;
}

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
    uint8_t sb[128] = {0};
    if (!r.read_at(0, sb, 48) || std::memcmp(sb, kSignature, 8) != 0) {
        err = path + ": not an HDF5 file (signature at offset 0)";
        return false;
    }
    uint64_t rootAddr = kUndef;
    const int ver = sb[8];
    if (ver == 0 || ver == 1) {
        // signature, versions (superblock, free space, root symbol table, reserved, shared
        // header), sizes of offsets / lengths, group K values, flags, [v1: indexed storage
        // K + reserved], base / free-space / end-of-file / driver addresses, root entry
        const size_t need = ver == 0 ? 96 : 100;
        if (!r.read_at(0, sb, need)) {
            err = path + ": superblock truncated";
            return false;
        }
        if (sb[13] != 8 || sb[14] != 8) {
            err = path + ": only 8-byte offsets and lengths are supported";
            return false;
        }
        const size_t a = ver == 0 ? 24 : 28;
        if (rd64(sb + a) != 0) {
            err = path + ": non-zero base address is not supported";
            return false;
        }
        r.eof = rd64(sb + a + 16);
        rootAddr = rd64(sb + a + 32 + 8);  // root symbol table entry: name offset, header address
    } else if (ver == 2 || ver == 3) {
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
        rootAddr = rd64(sb + 36);
    } else {
        err = path + ": superblock version " + std::to_string(ver) + " is not supported";
        return false;
    }
    bool isGroup = false;
    Dataset unused;
    if (!r.parse_object(rootAddr, "/", &root, &unused, isGroup, 0) || !isGroup) {
        err = path + ": " + (r.err.empty() ? "root object is not a group" : r.err);
        return false;
    }
    return true;
}

bool read_dataset(const std::string &path, const Dataset &d, void *out, std::string &err) {
    const size_t es = type_size(d.type);
    const size_t bytes = d.count * es;
    if (bytes == 0) return true;
    if (d.layout == 0) {
        if (d.compact.size() != bytes) {
            err = "dataset '" + d.name + "' compact size mismatch";
            return false;
        }
        std::memcpy(out, d.compact.data(), bytes);
        return true;
    }
    Reader r;
    r.f.open(path, std::ios::binary);
    if (!r.f) {
        err = "cannot open " + path;
        return false;
    }
    if (d.layout == 1) {
        if (d.fileOffset == kUndef) {  // never written: the fill value (zero)
            std::memset(out, 0, bytes);
            return true;
        }
        if (!r.read_at(d.fileOffset, out, bytes)) {
            err = "dataset '" + d.name + "' truncated";
            return false;
        }
        return true;
    }
    // chunked: chunks never written read as the fill value (zero)
    const int rank = (int)d.dims.size();
    std::memset(out, 0, bytes);
    if (d.chunkIndex == kUndef) return true;
    std::vector<Reader::Chunk> chunks;
    if (!r.chunk_node(d.chunkIndex, rank, chunks, 0)) {
        err = "dataset '" + d.name + "': " + r.err;
        return false;
    }
    size_t chunkElems = 1;
    for (uint64_t c : d.chunk) chunkElems *= c;
    std::vector<uint8_t> buf;
    uint8_t *dst = static_cast<uint8_t *>(out);
    for (const Reader::Chunk &c : chunks) {
        if (c.size > (size_t)1 << 31) {
            err = "dataset '" + d.name + "': chunk too large";
            return false;
        }
        buf.resize(c.size);
        if (!r.read_at(c.addr, buf.data(), buf.size())) {
            err = "dataset '" + d.name + "': chunk truncated";
            return false;
        }
        if (!unfilter(d, c.mask, buf, chunkElems * es, err)) return false;
        // copy the chunk's rows (runs along the last dimension) inside the extent
        for (int k = 0; k < rank; ++k)
            if (c.offset[k] % d.chunk[k] != 0 || c.offset[k] >= d.dims[k]) {
                err = "dataset '" + d.name + "': chunk offset outside the dataspace";
                return false;
            }
        const uint64_t last = d.chunk[rank - 1];
        const uint64_t run = std::min<uint64_t>(last, d.dims[rank - 1] - c.offset[rank - 1]);
        const size_t rows = chunkElems / last;
        for (size_t row = 0; row < rows; ++row) {
            // row -> chunk coordinates of the leading dimensions
            size_t rem = row, dstIndex = 0;
            bool inside = true;
            std::vector<uint64_t> coord(rank, 0);
            for (int k = rank - 2; k >= 0; --k) {
                coord[k] = rem % d.chunk[k];
                rem /= d.chunk[k];
            }
            for (int k = 0; k < rank - 1; ++k) {
                const uint64_t g = c.offset[k] + coord[k];
                if (g >= d.dims[k]) inside = false;
                dstIndex = dstIndex * d.dims[k] + g;
            }
            if (!inside) continue;
            dstIndex = dstIndex * d.dims[rank - 1] + c.offset[rank - 1];
            std::memcpy(dst + dstIndex * es, buf.data() + row * last * es, run * es);
        }
    }
    return true;
}

}  // namespace h5lite
