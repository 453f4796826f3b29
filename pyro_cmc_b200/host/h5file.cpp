// h5file.cpp -- see h5file.hpp. Field layouts follow the HDF5 file format
// specification: superblock version 2 (48 bytes), version 2 object headers
// ("OHDR", 4-byte chunk size, messages without creation order), messages
// Dataspace (v2), Datatype (v1: fixed-point, floating-point, variable-length
// string over an unsigned byte), Fill Value (v3), Data Layout (v3,
// contiguous), Link Info (v0, compact storage), Group Info (v0), Link (v1,
// hard links) and Attribute (v3); global heap collections ("GCOL", v1).
#include "h5file.hpp"

#include <unistd.h>

#include <cstdio>
#include <cstring>
#include <stdexcept>

namespace CMC {

uint32_t h5_lookup3(const unsigned char* k, size_t length, uint32_t init) {
    auto rot = [](uint32_t x, int r) { return (x << r) | (x >> (32 - r)); };
    uint32_t a, b, c;
    a = b = c = 0xdeadbeefu + uint32_t(length) + init;
    while (length > 12) {
        a += uint32_t(k[0]) | uint32_t(k[1]) << 8 | uint32_t(k[2]) << 16 | uint32_t(k[3]) << 24;
        b += uint32_t(k[4]) | uint32_t(k[5]) << 8 | uint32_t(k[6]) << 16 | uint32_t(k[7]) << 24;
        c += uint32_t(k[8]) | uint32_t(k[9]) << 8 | uint32_t(k[10]) << 16 | uint32_t(k[11]) << 24;
        // mix
        a -= c; a ^= rot(c, 4);  c += b;
        b -= a; b ^= rot(a, 6);  a += c;
        c -= b; c ^= rot(b, 8);  b += a;
        a -= c; a ^= rot(c, 16); c += b;
        b -= a; b ^= rot(a, 19); a += c;
        c -= b; c ^= rot(b, 4);  b += a;
        length -= 12;
        k += 12;
    }
    switch (length) {  // the last 1..12 bytes, fall-through intended
        case 12: c += uint32_t(k[11]) << 24; [[fallthrough]];
        case 11: c += uint32_t(k[10]) << 16; [[fallthrough]];
        case 10: c += uint32_t(k[9]) << 8; [[fallthrough]];
        case 9: c += k[8]; [[fallthrough]];
        case 8: b += uint32_t(k[7]) << 24; [[fallthrough]];
        case 7: b += uint32_t(k[6]) << 16; [[fallthrough]];
        case 6: b += uint32_t(k[5]) << 8; [[fallthrough]];
        case 5: b += k[4]; [[fallthrough]];
        case 4: a += uint32_t(k[3]) << 24; [[fallthrough]];
        case 3: a += uint32_t(k[2]) << 16; [[fallthrough]];
        case 2: a += uint32_t(k[1]) << 8; [[fallthrough]];
        case 1: a += k[0]; break;
        case 0: return c;
    }
    // final
    c ^= b; c -= rot(b, 14);
    a ^= c; a -= rot(c, 11);
    b ^= a; b -= rot(a, 25);
    c ^= b; c -= rot(b, 16);
    a ^= c; a -= rot(c, 4);
    b ^= a; b -= rot(a, 14);
    c ^= b; c -= rot(b, 24);
    return c;
}

namespace {

constexpr uint64_t kUndef = ~uint64_t(0);
using Bytes = std::vector<unsigned char>;

void put8(Bytes& b, unsigned v) { b.push_back(uint8_t(v)); }
void put16(Bytes& b, unsigned v) {
    for (int i = 0; i < 2; ++i) b.push_back(uint8_t(v >> (8 * i)));
}
void put32(Bytes& b, uint32_t v) {
    for (int i = 0; i < 4; ++i) b.push_back(uint8_t(v >> (8 * i)));
}
void put64(Bytes& b, uint64_t v) {
    for (int i = 0; i < 8; ++i) b.push_back(uint8_t(v >> (8 * i)));
}

// Datatype message body for a NumPy-style dtype, and its element size.
Bytes datatype_message(const std::string& dtype, size_t* size) {
    Bytes b;
    if (dtype.size() != 3 || dtype[0] != '<') throw std::invalid_argument("H5File: unsupported dtype " + dtype);
    const char kind = dtype[1];
    const int n = dtype[2] - '0';
    if (kind == 'f' && n == 8) {
        put8(b, 0x11);  // version 1, class 1 (floating point)
        put8(b, 0x20);  // little endian, no padding, mantissa normalisation 2 (implied leading 1)
        put8(b, 63);    // sign bit position
        put8(b, 0);
        put32(b, 8);
        put16(b, 0);     // bit offset
        put16(b, 64);    // precision
        put8(b, 52);     // exponent location
        put8(b, 11);     // exponent size
        put8(b, 0);      // mantissa location
        put8(b, 52);     // mantissa size
        put32(b, 1023);  // exponent bias
    } else if ((kind == 'i' || kind == 'u') && (n == 1 || n == 2 || n == 4 || n == 8)) {
        put8(b, 0x10);                       // version 1, class 0 (fixed point)
        put8(b, kind == 'i' ? 0x08 : 0x00);  // little endian, signed bit 3
        put8(b, 0);
        put8(b, 0);
        put32(b, uint32_t(n));
        put16(b, 0);                // bit offset
        put16(b, unsigned(8 * n));  // precision
    } else {
        throw std::invalid_argument("H5File: unsupported dtype " + dtype);
    }
    *size = size_t(n);
    return b;
}

// Variable-length UTF-8 string over unsigned bytes; elements are 16 bytes
// (length, global heap collection address, object index).
Bytes vlen_string_type() {
    Bytes b;
    put8(b, 0x19);  // version 1, class 9 (variable length)
    put8(b, 0x01);  // type 1: string; padding 0: null terminated
    put8(b, 0x01);  // character set 1: UTF-8
    put8(b, 0);
    put32(b, 16);
    size_t one = 0;
    const Bytes base = datatype_message("<u1", &one);
    b.insert(b.end(), base.begin(), base.end());
    return b;
}

Bytes dataspace_message(const std::vector<uint64_t>& shape) {
    Bytes b;
    put8(b, 2);  // version 2
    put8(b, unsigned(shape.size()));
    put8(b, 0);                      // no maximum dimensions
    put8(b, shape.empty() ? 0 : 1);  // scalar / simple
    for (uint64_t d : shape) put64(b, d);
    return b;
}

void message(Bytes& out, unsigned type, const Bytes& body, unsigned flags = 0) {
    if (body.size() > 0xffff) throw std::runtime_error("H5File: header message too large");
    put8(out, type);
    put16(out, unsigned(body.size()));
    put8(out, flags);
    out.insert(out.end(), body.begin(), body.end());
}

}  // namespace

struct H5File::Node {
    std::string name;
    bool group = true;
    std::vector<std::unique_ptr<Node>> kids;
    struct Attr {
        std::string name;
        Bytes type, space, data;
    };
    std::vector<Attr> attrs;
    // datasets
    Bytes type, space;
    uint64_t data_addr = kUndef, data_size = 0;
    uint64_t header = kUndef;
    bool dirty = true;
};

H5File::H5File(const std::string& path) : path_(path), root_(new Node) {
    fp_ = std::fopen(path.c_str(), "w+b");
    if (!fp_) throw std::runtime_error("Failed to create output file: " + path);
    eof_ = 48;  // the superblock
    Bytes zero(48, 0);
    if (std::fwrite(zero.data(), 1, zero.size(), static_cast<FILE*>(fp_)) != zero.size())
        throw std::runtime_error("H5File: write failed: " + path);
    commit();
}

H5File::~H5File() {
    try {
        close();
    } catch (...) {
    }
}

uint64_t H5File::append(const Bytes& b) {
    FILE* f = static_cast<FILE*>(fp_);
    const uint64_t at = eof_;
    if (std::fseek(f, long(at), SEEK_SET) != 0 || std::fwrite(b.data(), 1, b.size(), f) != b.size())
        throw std::runtime_error("H5File: write failed: " + path_);
    eof_ += b.size();
    return at;
}

uint64_t H5File::append_zeros(uint64_t n) {
    FILE* f = static_cast<FILE*>(fp_);
    const uint64_t at = eof_;
    std::fflush(f);
    if (ftruncate(fileno(f), off_t(at + n)) != 0) throw std::runtime_error("H5File: cannot extend " + path_);
    eof_ += n;
    return at;
}

H5File::Node* H5File::group_at(const std::string& path, bool create) {
    Node* g = root_.get();
    size_t i = 0;
    while (i < path.size()) {
        while (i < path.size() && path[i] == '/') ++i;
        if (i >= path.size()) break;
        size_t j = path.find('/', i);
        if (j == std::string::npos) j = path.size();
        const std::string part = path.substr(i, j - i);
        Node* next = nullptr;
        for (auto& k : g->kids)
            if (k->name == part) next = k.get();
        if (!next) {
            if (!create) return nullptr;
            g->kids.emplace_back(new Node);
            next = g->kids.back().get();
            next->name = part;
            g->dirty = true;
        }
        g = next;
        i = j;
    }
    return g;
}

H5File::Node* H5File::new_dataset(const std::string& path) {
    if (closed_) throw std::runtime_error("H5File: write after close");
    const size_t cut = path.find_last_of('/');
    Node* parent = cut == std::string::npos ? root_.get() : group_at(path.substr(0, cut), true);
    if (!parent->group) throw std::invalid_argument("H5File: " + path + ": parent is a dataset");
    const std::string name = cut == std::string::npos ? path : path.substr(cut + 1);
    for (auto& k : parent->kids)
        if (k->name == name) throw std::invalid_argument("H5File: " + path + " exists");
    parent->kids.emplace_back(new Node);
    Node* d = parent->kids.back().get();
    d->name = name;
    d->group = false;
    parent->dirty = true;
    return d;
}

void H5File::dataset(const std::string& path, const std::string& dtype, const std::vector<uint64_t>& shape,
                     const void* data) {
    Node* d = new_dataset(path);
    size_t es = 0;
    d->type = datatype_message(dtype, &es);
    d->space = dataspace_message(shape);
    uint64_t n = 1;
    for (uint64_t s : shape) n *= s;
    d->data_size = n * es;
    const auto* p = static_cast<const unsigned char*>(data);
    d->data_addr = append(Bytes(p, p + d->data_size));
}

size_t H5File::reserve(const std::string& path, const std::string& dtype, const std::vector<uint64_t>& shape) {
    Node* d = new_dataset(path);
    size_t es = 0;
    d->type = datatype_message(dtype, &es);
    d->space = dataspace_message(shape);
    uint64_t n = 1;
    for (uint64_t s : shape) n *= s;
    d->data_size = n * es;
    d->data_addr = append_zeros(d->data_size);
    reserved_.push_back(d);
    return reserved_.size() - 1;
}

void H5File::write_at(size_t handle, uint64_t off, const void* data, size_t nbytes) {
    if (handle >= reserved_.size()) throw std::invalid_argument("H5File: bad handle");
    const Node* d = reserved_[handle];
    if (off + nbytes > d->data_size) throw std::out_of_range("H5File: slice beyond the reserved dataset");
    FILE* f = static_cast<FILE*>(fp_);
    if (std::fseek(f, long(d->data_addr + off), SEEK_SET) != 0 || std::fwrite(data, 1, nbytes, f) != nbytes)
        throw std::runtime_error("H5File: write failed: " + path_);
    std::fflush(f);
}

void H5File::strings(const std::string& path, const std::vector<std::string>& s) {
    Node* d = new_dataset(path);
    d->type = vlen_string_type();
    d->space = dataspace_message({uint64_t(s.size())});
    // one global heap collection holding every string (object i + 1)
    Bytes objs;
    for (size_t i = 0; i < s.size(); ++i) {
        put16(objs, unsigned(i + 1));
        put16(objs, 1);  // reference count
        put32(objs, 0);
        put64(objs, s[i].size());
        objs.insert(objs.end(), s[i].begin(), s[i].end());
        while (objs.size() % 8) objs.push_back(0);
    }
    const uint64_t used = 16 + objs.size();
    const uint64_t size = used + 16 <= 4096 ? 4096 : used + 16;  // room for the free-space object
    Bytes g{'G', 'C', 'O', 'L'};
    put8(g, 1);
    put8(g, 0);
    put8(g, 0);
    put8(g, 0);
    put64(g, size);
    g.insert(g.end(), objs.begin(), objs.end());
    // object 0: the free space from its own 16-byte header to the end of the
    // collection, header included (a reader steps from the header's start to
    // the collection's end by this size)
    const uint64_t free_bytes = size - g.size();
    put16(g, 0);
    put16(g, 0);
    put32(g, 0);
    put64(g, free_bytes);
    g.resize(size, 0);
    const uint64_t gaddr = append(g);
    Bytes el;
    for (size_t i = 0; i < s.size(); ++i) {
        put32(el, uint32_t(s[i].size()));
        put64(el, gaddr);
        put32(el, uint32_t(i + 1));
    }
    d->data_size = el.size();
    d->data_addr = el.empty() ? append_zeros(0) : append(el);
}

void H5File::attribute(const std::string& path, const std::string& name, const std::string& dtype,
                       const std::vector<uint64_t>& shape, const void* data) {
    if (closed_) throw std::runtime_error("H5File: write after close");
    Node* n = group_at(path, true);
    Node::Attr a;
    a.name = name;
    size_t es = 0;
    a.type = datatype_message(dtype, &es);
    a.space = dataspace_message(shape);
    uint64_t cnt = 1;
    for (uint64_t s : shape) cnt *= s;
    const auto* p = static_cast<const unsigned char*>(data);
    a.data.assign(p, p + cnt * es);
    for (auto& old : n->attrs)
        if (old.name == name) throw std::invalid_argument("H5File: attribute " + name + " exists");
    n->attrs.push_back(std::move(a));
    n->dirty = true;
}

uint64_t H5File::commit_node(Node& n, bool* moved) {
    if (n.group)
        for (auto& k : n.kids) {
            bool km = false;
            commit_node(*k, &km);
            if (km) n.dirty = true;
        }
    *moved = false;
    if (!n.dirty && n.header != kUndef) return n.header;
    Bytes msgs;
    if (n.group) {
        Bytes li;
        put8(li, 0);        // version
        put8(li, 0);        // no creation order
        put64(li, kUndef);  // fractal heap: none (links are stored in this header)
        put64(li, kUndef);  // name index B-tree: none
        message(msgs, 0x0002, li);
        message(msgs, 0x000A, Bytes{0, 0});  // group info
        for (auto& k : n.kids) {
            if (k->name.size() > 255) throw std::invalid_argument("H5File: link name too long");
            Bytes l;
            put8(l, 1);  // version
            put8(l, 0);  // hard link, 1-byte name length, ASCII
            put8(l, unsigned(k->name.size()));
            l.insert(l.end(), k->name.begin(), k->name.end());
            put64(l, k->header);
            message(msgs, 0x0006, l);
        }
    } else {
        message(msgs, 0x0001, n.space);
        message(msgs, 0x0003, n.type, 0x01);    // constant
        message(msgs, 0x0005, Bytes{3, 0x09});  // fill value v3: allocated early, written if set, default value
        Bytes lay;
        put8(lay, 3);
        put8(lay, 1);  // contiguous
        put64(lay, n.data_addr);
        put64(lay, n.data_size);
        message(msgs, 0x0008, lay);
    }
    for (auto& a : n.attrs) {
        Bytes b;
        put8(b, 3);  // version 3
        put8(b, 0);
        put16(b, unsigned(a.name.size() + 1));
        put16(b, unsigned(a.type.size()));
        put16(b, unsigned(a.space.size()));
        put8(b, 0);  // ASCII name
        b.insert(b.end(), a.name.begin(), a.name.end());
        b.push_back(0);
        b.insert(b.end(), a.type.begin(), a.type.end());
        b.insert(b.end(), a.space.begin(), a.space.end());
        b.insert(b.end(), a.data.begin(), a.data.end());
        message(msgs, 0x000C, b);
    }
    Bytes h{'O', 'H', 'D', 'R'};
    put8(h, 2);     // version 2
    put8(h, 0x02);  // chunk 0 size stored in 4 bytes; no times, no creation order
    put32(h, uint32_t(msgs.size()));
    h.insert(h.end(), msgs.begin(), msgs.end());
    put32(h, h5_lookup3(h.data(), h.size(), 0));
    n.header = append(h);
    n.dirty = false;
    *moved = true;
    return n.header;
}

void H5File::write_superblock(uint64_t root_addr) {
    Bytes s{0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    put8(s, 2);        // version 2
    put8(s, 8);        // size of offsets
    put8(s, 8);        // size of lengths
    put8(s, 0);        // consistency flags
    put64(s, 0);       // base address
    put64(s, kUndef);  // superblock extension: none
    put64(s, eof_);
    put64(s, root_addr);
    put32(s, h5_lookup3(s.data(), s.size(), 0));
    FILE* f = static_cast<FILE*>(fp_);
    if (std::fseek(f, 0, SEEK_SET) != 0 || std::fwrite(s.data(), 1, s.size(), f) != s.size())
        throw std::runtime_error("H5File: write failed: " + path_);
    std::fflush(f);
}

void H5File::commit() {
    if (closed_) return;
    bool moved = false;
    const uint64_t root = commit_node(*root_, &moved);
    write_superblock(root);
}

void H5File::close() {
    if (closed_ || !fp_) return;
    commit();
    std::fclose(static_cast<FILE*>(fp_));
    fp_ = nullptr;
    closed_ = true;
}

}  // namespace CMC
