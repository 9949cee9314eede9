// h5file.cu -- the HDF5 writer and reader of h5file.h (host code).
#include "h5file.h"

#include <cstring>

namespace bsn {
namespace h5 {

namespace {
constexpr uint64_t UNDEF = ~0ull;
constexpr uint8_t SIG[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
enum : uint8_t {
    MSG_DATASPACE = 0x01, MSG_LINK_INFO = 0x02, MSG_DATATYPE = 0x03, MSG_FILL = 0x05, MSG_LINK = 0x06,
    MSG_LAYOUT = 0x08, MSG_GROUP_INFO = 0x0A, MSG_ATTRIBUTE = 0x0C, MSG_CONTINUATION = 0x10
};

inline uint32_t rot(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }
}  // namespace

uint32_t lookup3(const uint8_t* k, size_t length, uint32_t initval) {
    uint32_t a, b, c;
    a = b = c = 0xdeadbeefu + (uint32_t)length + initval;
    auto w = [](const uint8_t* p) {
        return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
    };
    while (length > 12) {
        a += w(k); b += w(k + 4); c += w(k + 8);
        a -= c; a ^= rot(c, 4);  c += b;
        b -= a; b ^= rot(a, 6);  a += c;
        c -= b; c ^= rot(b, 8);  b += a;
        a -= c; a ^= rot(c, 16); c += b;
        b -= a; b ^= rot(a, 19); a += c;
        c -= b; c ^= rot(b, 4);  b += a;
        length -= 12;
        k += 12;
    }
    if (length == 0) return c;
    uint8_t t[12] = {0};
    memcpy(t, k, length);   // the tail, zero-extended: the same sums as the byte cases
    a += w(t); b += w(t + 4); c += w(t + 8);
    c ^= b; c -= rot(b, 14);
    a ^= c; a -= rot(c, 11);
    b ^= a; b -= rot(a, 25);
    c ^= b; c -= rot(b, 16);
    a ^= c; a -= rot(c, 4);
    b ^= a; b -= rot(a, 14);
    c ^= b; c -= rot(b, 24);
    return c;
}

uint64_t Dataset::bytes() const {
    uint64_t n = 8;
    for (uint64_t d : dims) n *= d;
    return n;
}

uint64_t RDataset::count() const {
    uint64_t n = 1;
    for (uint64_t d : dims) n *= d;
    return n;
}

Attr attr_f64(const std::string& n, double v) { Attr a; a.name = n; a.kind = F64; a.d = v; return a; }
Attr attr_i64(const std::string& n, int64_t v) { Attr a; a.name = n; a.kind = I64; a.i = v; return a; }
Attr attr_str(const std::string& n, const std::string& v) { Attr a; a.name = n; a.kind = STR; a.s = v; return a; }

// ---------------------------------------------------------------------------
// writer

namespace {

struct Buf {
    std::vector<uint8_t> b;
    void u8(uint8_t v) { b.push_back(v); }
    void u16(uint16_t v) { for (int i = 0; i < 2; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
    void u32(uint32_t v) { for (int i = 0; i < 4; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
    void u64(uint64_t v) { for (int i = 0; i < 8; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
    void bytes(const void* p, size_t n) { b.insert(b.end(), (const uint8_t*)p, (const uint8_t*)p + n); }
    void f64(double v) { uint64_t u; memcpy(&u, &v, 8); u64(u); }
};

// Datatype message body: IEEE float64 / signed int64 little-endian, or a
// null-terminated ASCII string of n bytes
void datatype(Buf& o, Kind k, uint32_t str_size = 0) {
    if (k == F64) {
        o.u8(0x11);                 // version 1, class 1 (floating point)
        o.u8(0x20); o.u8(63); o.u8(0);   // little-endian, implied msb mantissa; sign at bit 63
        o.u32(8);
        o.u16(0); o.u16(64);        // bit offset, precision
        o.u8(52); o.u8(11);         // exponent location, size
        o.u8(0); o.u8(52);          // mantissa location, size
        o.u32(1023);                // exponent bias
    } else if (k == I64) {
        o.u8(0x10);                 // version 1, class 0 (fixed point)
        o.u8(0x08); o.u8(0); o.u8(0);    // little-endian, signed
        o.u32(8);
        o.u16(0); o.u16(64);
    } else {
        o.u8(0x13);                 // version 1, class 3 (string)
        o.u8(0x00); o.u8(0); o.u8(0);    // null terminated, ASCII
        o.u32(str_size);
    }
}
uint32_t datatype_size(Kind k) { return k == F64 ? 20 : (k == I64 ? 12 : 8); }

void dataspace(Buf& o, const std::vector<uint64_t>& dims) {
    o.u8(2);                        // version 2
    o.u8((uint8_t)dims.size());
    o.u8(0);                        // no maximum dimensions
    o.u8(dims.empty() ? 0 : 1);     // scalar or simple
    for (uint64_t d : dims) o.u64(d);
}
uint32_t dataspace_size(size_t rank) { return 4 + 8 * (uint32_t)rank; }

void attribute(Buf& o, const Attr& a) {
    const uint32_t sl = a.kind == STR ? (uint32_t)a.s.size() + 1 : 0;
    o.u8(3); o.u8(0);                          // version 3, flags
    o.u16((uint16_t)(a.name.size() + 1));
    o.u16((uint16_t)datatype_size(a.kind));
    o.u16((uint16_t)dataspace_size(0));
    o.u8(0);                                   // ASCII name
    o.bytes(a.name.c_str(), a.name.size() + 1);
    datatype(o, a.kind, sl);
    dataspace(o, {});
    if (a.kind == F64) o.f64(a.d);
    else if (a.kind == I64) o.u64((uint64_t)a.i);
    else o.bytes(a.s.c_str(), a.s.size() + 1);
}
uint32_t attribute_size(const Attr& a) {
    const uint32_t data = a.kind == STR ? (uint32_t)a.s.size() + 1 : 8;
    return 9 + (uint32_t)a.name.size() + 1 + datatype_size(a.kind) + dataspace_size(0) + data;
}

struct Msg { uint8_t type, flags; Buf body; };

// object header version 2 around the messages (4-byte chunk size, no times)
void object_header(Buf& o, const std::vector<Msg>& msgs) {
    const size_t start = o.b.size();
    o.bytes("OHDR", 4);
    o.u8(2);
    o.u8(0x02);
    uint32_t chunk = 0;
    for (const Msg& m : msgs) chunk += 4 + (uint32_t)m.body.b.size();
    o.u32(chunk);
    for (const Msg& m : msgs) {
        o.u8(m.type);
        o.u16((uint16_t)m.body.b.size());
        o.u8(m.flags);
        o.bytes(m.body.b.data(), m.body.b.size());
    }
    o.u32(lookup3(o.b.data() + start, o.b.size() - start));
}
uint64_t object_header_size(const std::vector<uint32_t>& bodies) {
    uint64_t s = 4 + 1 + 1 + 4 + 4;
    for (uint32_t b : bodies) s += 4 + b;
    return s;
}

uint32_t link_size(const std::string& name) { return 3 + (uint32_t)name.size() + 8; }

// sizes of a group's / dataset's header (addresses are fixed-width)
uint64_t group_header_size(const Group& g) {
    std::vector<uint32_t> b = {18, 2};
    for (const Group& c : g.groups) b.push_back(link_size(c.name));
    for (const Dataset& d : g.dsets) b.push_back(link_size(d.name));
    for (const Attr& a : g.attrs) b.push_back(attribute_size(a));
    return object_header_size(b);
}
uint64_t dataset_header_size(const Dataset& d) {
    std::vector<uint32_t> b = {dataspace_size(d.dims.size()), datatype_size(d.kind), 2, 18};
    for (const Attr& a : d.attrs) b.push_back(attribute_size(a));
    return object_header_size(b);
}

struct Plan {
    std::map<const void*, uint64_t> addr;      // object -> header address
    std::vector<std::pair<const Dataset*, uint64_t>> data;   // dataset -> data address
    uint64_t next = 48;
};

void assign(const Group& g, Plan& P) {
    P.addr[&g] = P.next;
    P.next += group_header_size(g);
    for (const Group& c : g.groups) assign(c, P);
    for (const Dataset& d : g.dsets) {
        P.addr[&d] = P.next;
        P.next += dataset_header_size(d);
    }
}
void assign_data(const Group& g, Plan& P) {
    for (const Group& c : g.groups) assign_data(c, P);
    for (const Dataset& d : g.dsets) {
        P.next = (P.next + 7) & ~7ull;
        P.data.push_back({&d, P.next});
        P.next += d.bytes();
    }
}

void emit(const Group& g, const Plan& P, Buf& o) {
    std::vector<Msg> m;
    Msg li{MSG_LINK_INFO, 0, {}};
    li.body.u8(0); li.body.u8(0); li.body.u64(UNDEF); li.body.u64(UNDEF);
    m.push_back(li);
    Msg gi{MSG_GROUP_INFO, 0, {}};
    gi.body.u8(0); gi.body.u8(0);
    m.push_back(gi);
    auto link = [&](const std::string& name, uint64_t a) {
        Msg l{MSG_LINK, 0, {}};
        l.body.u8(1); l.body.u8(0);            // version 1; 1-byte name length, hard link
        l.body.u8((uint8_t)name.size());
        l.body.bytes(name.data(), name.size());
        l.body.u64(a);
        m.push_back(l);
    };
    for (const Group& c : g.groups) link(c.name, P.addr.at(&c));
    for (const Dataset& d : g.dsets) link(d.name, P.addr.at(&d));
    for (const Attr& a : g.attrs) {
        Msg am{MSG_ATTRIBUTE, 0, {}};
        attribute(am.body, a);
        m.push_back(am);
    }
    object_header(o, m);
    for (const Group& c : g.groups) emit(c, P, o);
    for (const Dataset& d : g.dsets) {
        uint64_t da = 0;
        for (auto& pr : P.data)
            if (pr.first == &d) da = pr.second;
        std::vector<Msg> dm;
        Msg sp{MSG_DATASPACE, 0, {}};
        dataspace(sp.body, d.dims);
        dm.push_back(sp);
        Msg ty{MSG_DATATYPE, 0x01, {}};
        datatype(ty.body, d.kind);
        dm.push_back(ty);
        Msg fv{MSG_FILL, 0x01, {}};
        fv.body.u8(3); fv.body.u8(0x01 | (2 << 2));   // early allocation, fill written if set; none set
        dm.push_back(fv);
        Msg ly{MSG_LAYOUT, 0, {}};
        ly.body.u8(3); ly.body.u8(1); ly.body.u64(da); ly.body.u64(d.bytes());
        dm.push_back(ly);
        for (const Attr& a : d.attrs) {
            Msg am{MSG_ATTRIBUTE, 0, {}};
            attribute(am.body, a);
            dm.push_back(am);
        }
        object_header(o, dm);
    }
}

}  // namespace

namespace {
bool names_fit(const Group& g) {
    for (const Group& c : g.groups)
        if (c.name.empty() || c.name.size() > 255 || !names_fit(c)) return false;
    for (const Dataset& d : g.dsets)
        if (d.name.empty() || d.name.size() > 255) return false;
    return true;
}
}  // namespace

bool write_file(const std::string& path, const Group& root, std::string* err) {
    if (!names_fit(root)) {
        if (err) *err = "group and dataset names must be 1..255 bytes";
        return false;
    }
    Plan P;
    assign(root, P);
    const uint64_t meta_end = P.next;
    assign_data(root, P);
    const uint64_t eof = P.next;
    Buf o;
    o.bytes(SIG, 8);
    o.u8(2); o.u8(8); o.u8(8); o.u8(0);   // superblock version 2, 8-byte offsets and lengths
    o.u64(0);                             // base address
    o.u64(UNDEF);                         // no superblock extension
    o.u64(eof);
    o.u64(P.addr.at(&root));
    o.u32(lookup3(o.b.data(), o.b.size()));
    emit(root, P, o);
    if (o.b.size() != meta_end) {
        if (err) *err = "internal: object header sizes disagree with the plan";
        return false;
    }
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) {
        if (err) *err = "cannot open " + path + " for writing";
        return false;
    }
    bool ok = fwrite(o.b.data(), 1, o.b.size(), f) == o.b.size();
    uint64_t pos = o.b.size();
    static const uint8_t zeros[8] = {0};
    for (auto& pr : P.data) {
        if (!ok) break;
        if (pr.second > pos) ok = fwrite(zeros, 1, pr.second - pos, f) == pr.second - pos;
        const uint64_t n = pr.first->bytes();
        ok = ok && (n == 0 || fwrite(pr.first->data, 1, n, f) == n);
        pos = pr.second + n;
    }
    ok = (fclose(f) == 0) && ok;
    if (!ok && err) *err = "write to " + path + " failed";
    return ok;
}

// ---------------------------------------------------------------------------
// reader

namespace {
struct Cur {
    const uint8_t* p;
    const uint8_t* end;
    bool ok = true;
    bool need(size_t n) { if ((size_t)(end - p) < n) ok = false; return ok; }
    uint64_t un(int n) {
        if (!need(n)) return 0;
        uint64_t v = 0;
        for (int i = 0; i < n; ++i) v |= (uint64_t)p[i] << (8 * i);
        p += n;
        return v;
    }
    void skip(size_t n) { if (need(n)) p += n; }
};

// datatype -> kind and element size (false: not one of the three kinds)
bool parse_datatype(Cur& c, Kind* k, uint32_t* size) {
    uint8_t cv = (uint8_t)c.un(1);
    uint8_t b0 = (uint8_t)c.un(1);
    c.skip(2);
    *size = (uint32_t)c.un(4);
    if (!c.ok) return false;
    const int cls = cv & 0x0f;
    if (cls == 1 && *size == 8 && (b0 & 1) == 0) { c.skip(12); *k = F64; return c.ok; }
    if (cls == 0 && *size == 8 && (b0 & 1) == 0) { c.skip(4); *k = I64; return c.ok; }
    if (cls == 3) { *k = STR; return c.ok; }
    return false;
}
bool parse_dataspace(Cur& c, std::vector<uint64_t>* dims) {
    const int ver = (int)c.un(1);
    const int rank = (int)c.un(1);
    const int flags = (int)c.un(1);
    if (ver == 1) c.skip(5);
    else if (ver == 2) c.skip(1);
    else return false;
    dims->clear();
    for (int i = 0; i < rank; ++i) dims->push_back(c.un(8));
    if (flags & 1) c.skip(8 * (size_t)rank);
    return c.ok;
}
}  // namespace

Reader::~Reader() { if (f_) fclose(f_); }

bool Reader::read_at(uint64_t off, void* dst, uint64_t n) const {
    if (off > eof_ || n > eof_ - off) return false;
    if (fseeko(f_, (off_t)off, SEEK_SET) != 0) return false;
    return fread(dst, 1, n, f_) == n;
}

bool Reader::open(const std::string& path, std::string* err) {
    f_ = fopen(path.c_str(), "rb");
    if (!f_) { if (err) *err = "cannot open " + path; return false; }
    fseeko(f_, 0, SEEK_END);
    eof_ = (uint64_t)ftello(f_);
    uint8_t sb[48];
    if (!read_at(0, sb, 48) || memcmp(sb, SIG, 8) != 0) {
        if (err) *err = path + " is not an HDF5 file";
        return false;
    }
    if (sb[8] != 2 || sb[9] != 8 || sb[10] != 8) {
        if (err) *err = path + ": superblock version " + std::to_string(sb[8]) +
                        " (this reader takes the version-2 files bsn writes)";
        return false;
    }
    uint32_t ck = (uint32_t)sb[44] | ((uint32_t)sb[45] << 8) | ((uint32_t)sb[46] << 16) | ((uint32_t)sb[47] << 24);
    if (lookup3(sb, 44) != ck) { if (err) *err = path + ": superblock checksum mismatch"; return false; }
    Cur c{sb + 36, sb + 44};
    uint64_t root = c.un(8);
    bool is_ds = false;
    RDataset dummy;
    if (!parse_object(root, &root_, &dummy, &is_ds, 0, err)) return false;
    if (is_ds) { if (err) *err = path + ": root object is not a group"; return false; }
    return true;
}

bool Reader::parse_object(uint64_t addr, RGroup* g, RDataset* d, bool* is_dataset, int depth, std::string* err) {
    if (depth > 32) { if (err) *err = "object nesting too deep"; return false; }
    uint8_t h[16];
    if (!read_at(addr, h, 6) || memcmp(h, "OHDR", 4) != 0 || h[4] != 2) {
        if (err) *err = "object header at " + std::to_string(addr) + " is not a version-2 header";
        return false;
    }
    const uint8_t flags = h[5];
    uint64_t off = addr + 6;
    if (flags & 0x20) off += 16;   // times
    if (flags & 0x10) off += 4;    // attribute phase change values
    const int w = 1 << (flags & 3);
    uint8_t wb[8] = {0};
    if (!read_at(off, wb, (uint64_t)w)) { if (err) *err = "truncated object header"; return false; }
    uint64_t chunk = 0;
    for (int i = 0; i < w; ++i) chunk |= (uint64_t)wb[i] << (8 * i);
    off += (uint64_t)w;
    const uint64_t hdr_len = off - addr;
    if (chunk > eof_ || off + chunk + 4 > eof_) {
        if (err) *err = "object header at " + std::to_string(addr) + " runs past the end of the file";
        return false;
    }
    std::vector<uint8_t> all(hdr_len + chunk + 4);
    if (!read_at(addr, all.data(), all.size())) { if (err) *err = "truncated object header"; return false; }
    uint32_t ck = 0;
    for (int i = 0; i < 4; ++i) ck |= (uint32_t)all[hdr_len + chunk + i] << (8 * i);
    if (lookup3(all.data(), hdr_len + chunk) != ck) {
        if (err) *err = "object header checksum mismatch at " + std::to_string(addr);
        return false;
    }
    Cur c{all.data() + hdr_len, all.data() + hdr_len + chunk};
    std::vector<std::pair<std::string, uint64_t>> links;
    std::map<std::string, Attr> attrs;
    bool have_layout = false, have_space = false, have_type = false;
    RDataset ds;
    while (c.ok && c.end - c.p >= 4) {
        const uint8_t type = (uint8_t)c.un(1);
        const uint16_t size = (uint16_t)c.un(2);
        const uint8_t mflags = (uint8_t)c.un(1);
        (void)mflags;
        if (flags & 0x04) c.skip(2);   // creation order
        if (!c.need(size)) break;
        Cur m{c.p, c.p + size};
        c.p += size;
        if (type == MSG_CONTINUATION) { if (err) *err = "continuation blocks are not supported"; return false; }
        if (type == MSG_LINK) {
            const int ver = (int)m.un(1);
            const int lf = (int)m.un(1);
            if (ver != 1) continue;
            int lt = 0;
            if (lf & 0x08) lt = (int)m.un(1);
            if (lf & 0x04) m.skip(8);
            if (lf & 0x10) m.skip(1);
            const uint64_t nl = m.un(1 << (lf & 3));
            if (!m.need(nl)) break;
            std::string name((const char*)m.p, nl);
            m.p += nl;
            if (lt != 0) continue;   // soft / external links are not followed
            links.push_back({name, m.un(8)});
        } else if (type == MSG_ATTRIBUTE) {
            const int ver = (int)m.un(1);
            m.skip(1);
            const uint16_t nsz = (uint16_t)m.un(2), tsz = (uint16_t)m.un(2), ssz = (uint16_t)m.un(2);
            if (ver == 3) m.skip(1);
            else if (ver != 1 && ver != 2) continue;
            auto pad = [&](uint16_t n) { return ver == 1 ? (uint16_t)((n + 7) & ~7) : n; };
            if (!m.need(pad(nsz))) break;
            std::string name((const char*)m.p, nsz ? nsz - 1 : 0);
            m.p += pad(nsz);
            if (!m.need(pad(tsz))) break;
            Cur t{m.p, m.p + tsz};
            m.skip(pad(tsz));
            if (!m.need(pad(ssz))) break;
            Cur s{m.p, m.p + ssz};
            m.skip(pad(ssz));
            Kind k;
            uint32_t es;
            std::vector<uint64_t> dims;
            if (!parse_datatype(t, &k, &es) || !parse_dataspace(s, &dims) || !dims.empty()) continue;
            Attr a;
            a.name = name;
            a.kind = k;
            if (!m.need(es)) break;
            if (k == F64) memcpy(&a.d, m.p, 8);
            else if (k == I64) { uint64_t u = m.un(8); a.i = (int64_t)u; m.p -= 8; }
            else { size_t n = strnlen((const char*)m.p, es); a.s.assign((const char*)m.p, n); }
            attrs[name] = a;
        } else if (type == MSG_DATASPACE) {
            have_space = parse_dataspace(m, &ds.dims);
        } else if (type == MSG_DATATYPE) {
            uint32_t es;
            have_type = parse_datatype(m, &ds.kind, &es) && ds.kind != STR;
        } else if (type == MSG_LAYOUT) {
            const int ver = (int)m.un(1), cls = (int)m.un(1);
            if (ver != 3 || cls != 1) { if (err) *err = "only contiguous datasets are supported"; return false; }
            ds.addr = m.un(8);
            ds.size = m.un(8);
            have_layout = m.ok;
        }
    }
    if (!c.ok) { if (err) *err = "malformed object header at " + std::to_string(addr); return false; }
    if (have_layout) {
        if (!have_space || !have_type || ds.size != 8 * ds.count()) {
            if (err) *err = "dataset at " + std::to_string(addr) + " has no usable dataspace or datatype";
            return false;
        }
        ds.attrs = attrs;
        *d = ds;
        *is_dataset = true;
        return true;
    }
    *is_dataset = false;
    g->attrs = attrs;
    for (auto& l : links) {
        RGroup cg;
        RDataset cd;
        bool cds = false;
        if (!parse_object(l.second, &cg, &cd, &cds, depth + 1, err)) return false;
        if (cds) g->dsets[l.first] = cd;
        else g->groups[l.first] = cg;
    }
    return true;
}

const RGroup* Reader::group(const std::string& path) const {
    const RGroup* g = &root_;
    size_t s = 0;
    while (s < path.size()) {
        size_t e = path.find('/', s);
        if (e == std::string::npos) e = path.size();
        if (e > s) {
            auto it = g->groups.find(path.substr(s, e - s));
            if (it == g->groups.end()) return nullptr;
            g = &it->second;
        }
        s = e + 1;
    }
    return g;
}

const RDataset* Reader::dataset(const std::string& path) const {
    size_t e = path.rfind('/');
    const RGroup* g = e == std::string::npos ? &root_ : group(path.substr(0, e));
    if (!g) return nullptr;
    auto it = g->dsets.find(e == std::string::npos ? path : path.substr(e + 1));
    return it == g->dsets.end() ? nullptr : &it->second;
}

bool Reader::read_data(const RDataset& d, void* dst, uint64_t cap_bytes, std::string* err) const {
    if (d.size > cap_bytes) { if (err) *err = "destination too small for the dataset"; return false; }
    if (!read_at(d.addr, dst, d.size)) { if (err) *err = "dataset data outside the file"; return false; }
    return true;
}

bool get_f64(const std::map<std::string, Attr>& a, const char* name, double* v) {
    auto it = a.find(name);
    if (it == a.end()) return false;
    if (it->second.kind == F64) { *v = it->second.d; return true; }
    if (it->second.kind == I64) { *v = (double)it->second.i; return true; }
    return false;
}
bool get_i64(const std::map<std::string, Attr>& a, const char* name, int64_t* v) {
    auto it = a.find(name);
    if (it == a.end() || it->second.kind != I64) return false;
    *v = it->second.i;
    return true;
}
bool get_str(const std::map<std::string, Attr>& a, const char* name, std::string* v) {
    auto it = a.find(name);
    if (it == a.end() || it->second.kind != STR) return false;
    *v = it->second.s;
    return true;
}

}  // namespace h5
}  // namespace bsn
