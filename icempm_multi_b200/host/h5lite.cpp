// h5lite.cpp -- see h5lite.hpp.  Offsets below are those of the HDF5
// file-format specification (superblock v0/v1, object header v1, B-tree v1,
// local heap, symbol table node, and the message types listed there).
#include "h5lite.hpp"

#include <zlib.h>

#include <algorithm>
#include <cstring>
#include <fstream>
#include <stdexcept>

namespace icy {
namespace h5 {

namespace {

[[noreturn]] void fail(const std::string &m) { throw std::runtime_error("h5lite: " + m); }

uint64_t round8(uint64_t n) { return (n + 7) & ~uint64_t(7); }

const uint8_t kSignature[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

enum : uint16_t {
    MSG_NIL = 0x0, MSG_DATASPACE = 0x1, MSG_DATATYPE = 0x3, MSG_LAYOUT = 0x8, MSG_FILTERS = 0xB,
    MSG_ATTRIBUTE = 0xC, MSG_CONTINUATION = 0x10, MSG_SYMBOL_TABLE = 0x11
};

}  // namespace

File::File(const std::string &path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) fail("cannot open " + path);
    f.seekg(0, std::ios::end);
    std::streamoff n = f.tellg();
    if (n <= 0) fail("empty file " + path);
    buf_.resize((size_t)n);
    f.seekg(0);
    f.read(reinterpret_cast<char *>(buf_.data()), n);
    if (!f) fail("short read of " + path);

    // the superblock sits at 0, 512, 1024, 2048, ...
    uint64_t sb = UINT64_MAX;
    for (uint64_t at = 0; at + 8 <= buf_.size(); at = at ? at * 2 : 512)
        if (std::memcmp(&buf_[at], kSignature, 8) == 0) { sb = at; break; }
    if (sb == UINT64_MAX) fail(path + " is not an HDF5 file");
    need(sb, 24);
    const unsigned ver = buf_[sb + 8];
    if (ver > 1) fail("superblock version " + std::to_string(ver) + " is not supported");
    so_ = buf_[sb + 13];
    sl_ = buf_[sb + 14];
    if (so_ != 8 || sl_ != 8) fail("only 8-byte offsets and lengths are supported");
    uint64_t p = sb + 24 + (ver == 1 ? 4 : 0);
    base_ = u(p, 8);                                   // base address
    p += 4 * so_;                                      // base, free-space, end-of-file, driver
    // root group symbol table entry: name offset, object header, cache type, reserved, scratch
    const uint64_t root_ohdr = u(p + so_, so_);
    const uint32_t cache = (uint32_t)u(p + 2 * so_, 4);
    uint64_t btree = UINT64_MAX, heap = UINT64_MAX;
    if (cache == 1) {
        btree = u(p + 2 * so_ + 8, so_);
        heap = u(p + 2 * so_ + 8 + so_, so_);
    } else {
        for (const Message &m : messages(root_ohdr))
            if (m.type == MSG_SYMBOL_TABLE) { btree = u(m.pos, so_); heap = u(m.pos + so_, so_); }
    }
    if (btree == UINT64_MAX) fail("root group has no symbol table (new-style groups are not supported)");
    read_group(btree, heap);
}

uint64_t File::u(uint64_t pos, unsigned n) const
{
    need(pos, n);
    uint64_t v = 0;
    for (unsigned i = 0; i < n; i++) v |= (uint64_t)buf_[pos + i] << (8 * i);
    return v;
}

void File::need(uint64_t pos, uint64_t n) const
{
    if (pos > buf_.size() || n > buf_.size() - pos) fail("truncated file or bad address");
}

std::vector<File::Message> File::messages(uint64_t ohdr) const
{
    const uint64_t a = base_ + ohdr;
    need(a, 16);
    if (buf_[a] != 1) fail("object header version " + std::to_string(buf_[a]) + " is not supported");
    const unsigned nmsg = (unsigned)u(a + 2, 2);
    std::vector<std::pair<uint64_t, uint64_t>> blocks{{a + 16, u(a + 8, 4)}};
    std::vector<Message> out;
    for (size_t b = 0; b < blocks.size() && out.size() < nmsg; b++) {
        uint64_t q = blocks[b].first;
        const uint64_t end = q + blocks[b].second;
        need(q, blocks[b].second);
        while (q + 8 <= end && out.size() < nmsg) {
            Message m{(uint16_t)u(q, 2), q + 8, (uint16_t)u(q + 2, 2)};
            if (m.pos + m.size > end) fail("object header message overruns its block");
            if (buf_[q + 4] & 0x02) {
                if (m.type == MSG_DATATYPE || m.type == MSG_DATASPACE || m.type == MSG_LAYOUT || m.type == MSG_FILTERS)
                    fail("shared object header messages are not supported");
            }
            if (m.type == MSG_CONTINUATION) blocks.push_back({base_ + u(m.pos, so_), u(m.pos + so_, sl_)});
            out.push_back(m);
            q = m.pos + m.size;
        }
    }
    return out;
}

void File::read_group(uint64_t btree, uint64_t heap)
{
    const uint64_t h = base_ + heap;
    need(h, 8 + 2 * sl_ + so_);
    if (std::memcmp(&buf_[h], "HEAP", 4) != 0) fail("bad local heap signature");
    const uint64_t heap_data = base_ + u(h + 8 + 2 * sl_, so_);

    std::vector<uint64_t> stack{btree};
    while (!stack.empty()) {
        const uint64_t node = base_ + stack.back();
        stack.pop_back();
        need(node, 8 + 2 * so_);
        if (std::memcmp(&buf_[node], "TREE", 4) != 0) fail("bad group B-tree signature");
        if (buf_[node + 4] != 0) fail("group B-tree of the wrong node type");
        const unsigned level = buf_[node + 5], used = (unsigned)u(node + 6, 2);
        uint64_t q = node + 8 + 2 * so_ + sl_;          // past key 0
        for (unsigned i = 0; i < used; i++, q += so_ + sl_) {
            const uint64_t child = u(q, so_);
            if (level > 0) { stack.push_back(child); continue; }
            const uint64_t sn = base_ + child;
            need(sn, 8);
            if (std::memcmp(&buf_[sn], "SNOD", 4) != 0) fail("bad symbol table node signature");
            const unsigned ns = (unsigned)u(sn + 6, 2);
            const uint64_t esz = 2 * so_ + 8 + 16;
            for (unsigned k = 0; k < ns; k++) {
                const uint64_t e = sn + 8 + k * esz;
                const uint64_t name_at = heap_data + u(e, so_);
                need(name_at, 1);
                const void *z = std::memchr(&buf_[name_at], 0, buf_.size() - name_at);
                if (!z) fail("unterminated link name");
                std::string name(reinterpret_cast<const char *>(&buf_[name_at]),
                                 static_cast<const uint8_t *>(z) - &buf_[name_at]);
                entries_.push_back({name, u(e + so_, so_)});
            }
        }
    }
}

std::vector<std::string> File::names() const
{
    std::vector<std::string> v;
    for (auto &e : entries_) v.push_back(e.first);
    return v;
}

bool File::has(const std::string &name) const
{
    for (auto &e : entries_)
        if (e.first == name) return true;
    return false;
}

Datatype File::parse_dtype(uint64_t pos) const
{
    need(pos, 8);
    Datatype t;
    t.cls = buf_[pos] & 0x0f;
    const unsigned bits = buf_[pos + 1];
    t.size = (unsigned)u(pos + 4, 4);
    if (t.cls != 0 && t.cls != 1) fail("datatype class " + std::to_string(t.cls) + " is not supported");
    t.big_endian = bits & 1;
    if (t.cls == 1 && (bits & 0x40)) fail("VAX floating-point order is not supported");
    t.is_signed = (t.cls == 0) && (bits & 0x08);
    if (t.cls == 1 && t.size != 4 && t.size != 8) fail("floating-point size " + std::to_string(t.size));
    if (t.cls == 0 && t.size != 1 && t.size != 2 && t.size != 4 && t.size != 8)
        fail("integer size " + std::to_string(t.size));
    return t;
}

std::vector<uint64_t> File::parse_dataspace(uint64_t pos) const
{
    need(pos, 4);
    const unsigned ver = buf_[pos], rank = buf_[pos + 1];
    std::vector<uint64_t> d;
    uint64_t q;
    if (ver == 1) q = pos + 8;
    else if (ver == 2) {
        if (buf_[pos + 3] == 2) fail("null dataspace");
        q = pos + 4;
    } else fail("dataspace version " + std::to_string(ver));
    for (unsigned i = 0; i < rank; i++) d.push_back(u(q + i * sl_, sl_));
    return d;   // empty = scalar
}

File::Object File::object(const std::string &name) const
{
    uint64_t ohdr = UINT64_MAX;
    for (auto &e : entries_)
        if (e.first == name) ohdr = e.second;
    if (ohdr == UINT64_MAX) fail("no dataset named '" + name + "'");
    Object o;
    bool have_space = false, have_type = false;
    for (const Message &m : messages(ohdr)) {
        const uint64_t p = m.pos;
        switch (m.type) {
        case MSG_DATASPACE: o.dims = parse_dataspace(p); have_space = true; break;
        case MSG_DATATYPE: o.dtype = parse_dtype(p); have_type = true; break;
        case MSG_LAYOUT: {
            const unsigned ver = buf_[p];
            if (ver == 3) {
                o.layout_class = buf_[p + 1];
                if (o.layout_class == 0) {
                    const unsigned n = (unsigned)u(p + 2, 2);
                    need(p + 4, n);
                    o.compact.assign(buf_.begin() + p + 4, buf_.begin() + p + 4 + n);
                } else if (o.layout_class == 1) {
                    o.data_addr = u(p + 2, so_);
                    o.data_size = u(p + 2 + so_, sl_);
                } else if (o.layout_class == 2) {
                    const unsigned nd = buf_[p + 2];
                    o.data_addr = u(p + 3, so_);
                    for (unsigned i = 0; i < nd; i++) o.chunk.push_back((uint32_t)u(p + 3 + so_ + 4 * i, 4));
                } else fail("layout class " + std::to_string(o.layout_class));
            } else if (ver == 1 || ver == 2) {
                const unsigned nd = buf_[p + 1];
                o.layout_class = buf_[p + 2];
                uint64_t q = p + 8;
                if (o.layout_class != 0) { o.data_addr = u(q, so_); q += so_; }
                std::vector<uint32_t> dd;
                for (unsigned i = 0; i < nd; i++) dd.push_back((uint32_t)u(q + 4 * i, 4));
                q += 4 * nd;
                if (o.layout_class == 2) o.chunk = dd;
                else if (o.layout_class == 0) {
                    const unsigned n = (unsigned)u(q, 4);
                    need(q + 4, n);
                    o.compact.assign(buf_.begin() + q + 4, buf_.begin() + q + 4 + n);
                } else o.data_size = UINT64_MAX;   // contiguous: size from the dataspace
            } else fail("layout message version " + std::to_string(ver));
            break;
        }
        case MSG_FILTERS: {
            const unsigned ver = buf_[p], nf = buf_[p + 1];
            uint64_t q = p + (ver == 1 ? 8 : 2);
            for (unsigned i = 0; i < nf; i++) {
                Object::Filter flt;
                flt.id = (uint16_t)u(q, 2);
                unsigned name_len = 0;
                if (ver == 1 || flt.id >= 256) { name_len = (unsigned)u(q + 2, 2); q += 4; }
                else q += 2;
                flt.flags = (uint16_t)u(q, 2);
                const unsigned ncd = (unsigned)u(q + 2, 2);
                q += 4;
                q += ver == 1 ? round8(name_len) : name_len;
                for (unsigned k = 0; k < ncd; k++) flt.cd.push_back((uint32_t)u(q + 4 * k, 4));
                q += 4 * ncd + ((ver == 1 && (ncd & 1)) ? 4 : 0);
                o.filters.push_back(flt);
            }
            break;
        }
        case MSG_ATTRIBUTE: {
            const unsigned ver = buf_[p];
            const unsigned nn = (unsigned)u(p + 2, 2), nt = (unsigned)u(p + 4, 2), ns = (unsigned)u(p + 6, 2);
            uint64_t q = p + 8 + (ver == 3 ? 1 : 0);
            auto adv = [&](unsigned n) { return ver == 1 ? round8(n) : (uint64_t)n; };
            Object::Attr a;
            need(q, nn);
            a.name.assign(reinterpret_cast<const char *>(&buf_[q]), strnlen(reinterpret_cast<const char *>(&buf_[q]), nn));
            q += adv(nn);
            a.dtype = parse_dtype(q);
            q += adv(nt);
            a.dims = parse_dataspace(q);
            q += adv(ns);
            a.data_pos = q;
            if (ver < 1 || ver > 3) fail("attribute message version " + std::to_string(ver));
            o.attrs.push_back(a);
            break;
        }
        default: break;
        }
    }
    if (!have_space || !have_type) fail("'" + name + "' is not a dataset");
    return o;
}

std::vector<uint64_t> File::dims(const std::string &dataset) const { return object(dataset).dims; }
Datatype File::type(const std::string &dataset) const { return object(dataset).dtype; }

std::vector<uint8_t> File::chunk_bytes(const Object &o, uint64_t addr, uint32_t size, uint32_t mask) const
{
    need(base_ + addr, size);
    std::vector<uint8_t> cur(buf_.begin() + base_ + addr, buf_.begin() + base_ + addr + size);
    uint64_t expect = 1;
    for (uint32_t c : o.chunk) expect *= c;
    // filters were applied in pipeline order when writing: undo them in reverse
    for (int i = (int)o.filters.size() - 1; i >= 0; i--) {
        if (mask & (1u << i)) continue;
        const Object::Filter &f = o.filters[i];
        if (f.id == 1) {                           // deflate
            std::vector<uint8_t> out(expect);
            z_stream zs{};
            if (inflateInit(&zs) != Z_OK) fail("inflateInit");
            zs.next_in = cur.data();
            zs.avail_in = (uInt)cur.size();
            zs.next_out = out.data();
            zs.avail_out = (uInt)out.size();
            const int rc = inflate(&zs, Z_FINISH);
            const uint64_t got = zs.total_out;
            inflateEnd(&zs);
            if (rc != Z_STREAM_END) fail("inflate failed on a chunk");
            out.resize(got);
            cur.swap(out);
        } else if (f.id == 2) {                    // shuffle: bytes grouped by byte position
            const unsigned es = f.cd.empty() ? o.dtype.size : f.cd[0];
            if (es > 1) {
                const size_t ne = cur.size() / es;
                std::vector<uint8_t> out(cur.size());
                for (unsigned b = 0; b < es; b++)
                    for (size_t e = 0; e < ne; e++) out[e * es + b] = cur[b * ne + e];
                std::copy(cur.begin() + ne * es, cur.end(), out.begin() + ne * es);
                cur.swap(out);
            }
        } else if (f.id == 3) {                    // fletcher32: checksum appended
            if (cur.size() < 4) fail("fletcher32 chunk too short");
            cur.resize(cur.size() - 4);
        } else {
            fail("filter " + std::to_string(f.id) + " is not supported");
        }
    }
    if (cur.size() < expect) fail("chunk decodes to fewer bytes than its dimensions");
    return cur;
}

std::vector<uint8_t> File::raw(const Object &o) const
{
    uint64_t n = 1;
    for (uint64_t d : o.dims) n *= d;
    const unsigned es = o.dtype.size;
    std::vector<uint8_t> out(n * es, 0);       // unallocated chunks read as the zero fill
    if (o.layout_class == 0) {
        if (o.compact.size() < out.size()) fail("compact data shorter than the dataspace");
        std::copy(o.compact.begin(), o.compact.begin() + out.size(), out.begin());
        return out;
    }
    if (o.layout_class == 1) {
        if (o.data_addr == UINT64_MAX) return out;   // never written
        need(base_ + o.data_addr, out.size());
        std::copy(buf_.begin() + base_ + o.data_addr, buf_.begin() + base_ + o.data_addr + out.size(), out.begin());
        return out;
    }
    // chunked: walk the chunk B-tree; key = chunk size, filter mask, offsets (rank + 1)
    const size_t rank = o.dims.size();
    if (o.chunk.size() != rank + 1) fail("chunk dimensionality does not match the dataspace");
    if (o.data_addr == UINT64_MAX) return out;
    const unsigned key = 8 + 8 * (unsigned)(rank + 1);
    std::vector<uint64_t> stack{o.data_addr};
    while (!stack.empty()) {
        const uint64_t node = base_ + stack.back();
        stack.pop_back();
        need(node, 8 + 2 * so_);
        if (std::memcmp(&buf_[node], "TREE", 4) != 0) fail("bad chunk B-tree signature");
        if (buf_[node + 4] != 1) fail("chunk B-tree of the wrong node type");
        const unsigned level = buf_[node + 5], used = (unsigned)u(node + 6, 2);
        uint64_t q = node + 8 + 2 * so_;
        for (unsigned i = 0; i < used; i++) {
            const uint32_t csize = (uint32_t)u(q, 4), cmask = (uint32_t)u(q + 4, 4);
            std::vector<uint64_t> off(rank);
            for (size_t d = 0; d < rank; d++) off[d] = u(q + 8 + 8 * d, 8);
            const uint64_t child = u(q + key, so_);
            q += key + so_;
            if (level > 0) { stack.push_back(child); continue; }
            const std::vector<uint8_t> c = chunk_bytes(o, child, csize, cmask);
            // copy the part of the chunk inside the dataspace, row by row (last axis contiguous)
            std::vector<uint64_t> idx(rank, 0);
            const uint64_t run = std::min<uint64_t>(o.chunk[rank - 1], o.dims[rank - 1] > off[rank - 1] ?
                                                    o.dims[rank - 1] - off[rank - 1] : 0);
            while (true) {
                bool inside = run > 0;
                uint64_t src = 0, dst = 0;
                for (size_t d = 0; d < rank; d++) {
                    if (off[d] + idx[d] >= o.dims[d]) inside = false;
                    src = src * o.chunk[d] + idx[d];
                    dst = dst * o.dims[d] + off[d] + idx[d];
                }
                if (inside) std::memcpy(&out[dst * es], &c[src * es], run * es);
                size_t d = rank - 1;
                while (d > 0) {
                    if (++idx[d - 1] < o.chunk[d - 1]) break;
                    idx[d - 1] = 0;
                    d--;
                }
                if (d == 0) break;
            }
        }
    }
    return out;
}

namespace {

uint64_t load_le(const uint8_t *p, unsigned n, bool be)
{
    uint64_t v = 0;
    for (unsigned i = 0; i < n; i++) v |= (uint64_t)p[be ? n - 1 - i : i] << (8 * i);
    return v;
}

double to_double(const uint8_t *p, const Datatype &t)
{
    const uint64_t bits = load_le(p, t.size, t.big_endian);
    if (t.cls == 1) {
        if (t.size == 8) { double d; std::memcpy(&d, &bits, 8); return d; }
        uint32_t b32 = (uint32_t)bits;
        float f;
        std::memcpy(&f, &b32, 4);
        return f;
    }
    if (t.is_signed) {
        const unsigned sh = 64 - 8 * t.size;
        return (double)((int64_t)(bits << sh) >> sh);
    }
    return (double)bits;
}

}  // namespace

std::vector<double> File::read_double(const std::string &dataset) const
{
    const Object o = object(dataset);
    const std::vector<uint8_t> r = raw(o);
    std::vector<double> v(r.size() / o.dtype.size);
    for (size_t i = 0; i < v.size(); i++) v[i] = to_double(&r[i * o.dtype.size], o.dtype);
    return v;
}

std::vector<uint64_t> File::read_uint64(const std::string &dataset) const
{
    const Object o = object(dataset);
    if (o.dtype.cls != 0) fail("'" + dataset + "' is not an integer dataset");
    const std::vector<uint8_t> r = raw(o);
    std::vector<uint64_t> v(r.size() / o.dtype.size);
    for (size_t i = 0; i < v.size(); i++) {
        uint64_t b = load_le(&r[i * o.dtype.size], o.dtype.size, o.dtype.big_endian);
        if (o.dtype.is_signed && o.dtype.size < 8) {
            const unsigned sh = 64 - 8 * o.dtype.size;
            b = (uint64_t)((int64_t)(b << sh) >> sh);
        }
        v[i] = b;
    }
    return v;
}

double File::attribute_double(const std::string &dataset, const std::string &attr) const
{
    const Object o = object(dataset);
    for (const Object::Attr &a : o.attrs)
        if (a.name == attr) {
            need(a.data_pos, a.dtype.size);
            return to_double(&buf_[a.data_pos], a.dtype);
        }
    fail("dataset '" + dataset + "' has no attribute '" + attr + "'");
}

}  // namespace h5
}  // namespace icy
