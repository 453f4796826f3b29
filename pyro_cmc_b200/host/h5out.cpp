// h5out.cpp -- HDF5 through H5File, or an .npz writer (zip of .npy members,
// stored, Zip64 when large).
#include "h5out.hpp"

#include <cstdio>
#include <cstring>
#include <stdexcept>

namespace CMC {

namespace {

// CRC-32 (IEEE 802.3, reflected polynomial 0xEDB88320), table driven.
uint32_t crc32_update(uint32_t crc, const unsigned char* p, size_t n) {
    static uint32_t table[256];
    static bool init = false;
    if (!init) {
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t c = i;
            for (int k = 0; k < 8; ++k) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            table[i] = c;
        }
        init = true;
    }
    crc = ~crc;
    for (size_t i = 0; i < n; ++i) crc = table[(crc ^ p[i]) & 0xffu] ^ (crc >> 8);
    return ~crc;
}

void put16(std::vector<unsigned char>& b, uint16_t v) {
    b.push_back(uint8_t(v));
    b.push_back(uint8_t(v >> 8));
}
void put32(std::vector<unsigned char>& b, uint32_t v) {
    for (int i = 0; i < 4; ++i) b.push_back(uint8_t(v >> (8 * i)));
}
void put64(std::vector<unsigned char>& b, uint64_t v) {
    for (int i = 0; i < 8; ++i) b.push_back(uint8_t(v >> (8 * i)));
}

std::string npy_header(const std::string& dtype, const std::vector<uint64_t>& shape) {
    std::string sh = "(";
    for (size_t i = 0; i < shape.size(); ++i) {
        sh += std::to_string(shape[i]);
        if (shape.size() == 1 || i + 1 < shape.size()) sh += ",";
        if (i + 1 < shape.size()) sh += " ";
    }
    sh += ")";
    std::string d = "{'descr': '" + dtype + "', 'fortran_order': False, 'shape': " + sh + ", }";
    // magic(6) + version(2) + len(2) + dict, padded with spaces to a multiple of 64, ending in \n
    size_t total = 10 + d.size() + 1;
    const size_t pad = (64 - total % 64) % 64;
    d += std::string(pad, ' ');
    d += "\n";
    std::string h = "\x93NUMPY";
    h += char(1);
    h += char(0);
    h += char(d.size() & 0xff);
    h += char((d.size() >> 8) & 0xff);
    return h + d;
}

std::string clean(const std::string& path) {
    std::string p = path;
    while (!p.empty() && p[0] == '/') p.erase(0, 1);
    return p;
}

bool ends_with(const std::string& s, const std::string& t) {
    return s.size() >= t.size() && s.compare(s.size() - t.size(), t.size(), t) == 0;
}

}  // namespace

OutFile::OutFile(const std::string& path) : path_(path) {
    if (!ends_with(path, ".npz")) {
        h5_.reset(new H5File(path));
        return;
    }
    fp_ = std::fopen(path.c_str(), "wb");
    if (!fp_) throw std::runtime_error("Failed to create output file: " + path);
}

OutFile::~OutFile() {
    try {
        close();
    } catch (...) {
    }
}

void OutFile::member(const std::string& name, const std::string& dtype, const std::vector<uint64_t>& shape,
                     const void* data, size_t nbytes) {
    if (closed_) throw std::runtime_error("OutFile: write after close");
    const std::string hdr = npy_header(dtype, shape);
    uint32_t crc = crc32_update(0, reinterpret_cast<const unsigned char*>(hdr.data()), hdr.size());
    crc = crc32_update(crc, static_cast<const unsigned char*>(data), nbytes);
    const uint64_t size = hdr.size() + nbytes;
    Entry e{name, crc, size, pos_};
    // local file header with a Zip64 extra field (sizes in the extra field)
    std::vector<unsigned char> lh;
    put32(lh, 0x04034b50);
    put16(lh, 45);  // version needed (Zip64)
    put16(lh, 0);
    put16(lh, 0);  // stored
    put16(lh, 0);
    put16(lh, 0x21);  // 1980-01-01
    put32(lh, crc);
    put32(lh, 0xffffffffu);
    put32(lh, 0xffffffffu);
    put16(lh, uint16_t(name.size()));
    put16(lh, 20);
    lh.insert(lh.end(), name.begin(), name.end());
    put16(lh, 0x0001);
    put16(lh, 16);
    put64(lh, size);
    put64(lh, size);
    FILE* f = static_cast<FILE*>(fp_);
    if (std::fwrite(lh.data(), 1, lh.size(), f) != lh.size() || std::fwrite(hdr.data(), 1, hdr.size(), f) != hdr.size() ||
        (nbytes && std::fwrite(data, 1, nbytes, f) != nbytes))
        throw std::runtime_error("OutFile: write failed: " + path_);
    pos_ += lh.size() + size;
    entries_.push_back(e);
}

void OutFile::dataset(const std::string& path, const std::string& dtype, const std::vector<uint64_t>& shape,
                      const void* data, size_t itemsize) {
    if (h5_) return h5_->dataset(path, dtype, shape, data);
    uint64_t n = 1;
    for (uint64_t s : shape) n *= s;
    member(clean(path) + ".npy", dtype, shape, data, size_t(n) * itemsize);
}

void OutFile::attribute(const std::string& group, const std::string& name, const std::string& dtype,
                        const std::vector<uint64_t>& shape, const void* data, size_t itemsize) {
    if (h5_) return h5_->attribute(group, name, dtype, shape, data);
    uint64_t n = 1;
    for (uint64_t s : shape) n *= s;
    std::string g = clean(group);
    member((g.empty() ? "" : g + "/") + "@" + name + ".npy", dtype, shape, data, size_t(n) * itemsize);
}

void OutFile::dataset_strings(const std::string& path, const std::vector<std::string>& s) {
    if (h5_) return h5_->strings(path, s);
    size_t w = 1;
    for (const auto& x : s) w = std::max(w, x.size());
    std::vector<char> buf(s.size() * w, 0);
    for (size_t i = 0; i < s.size(); ++i) std::memcpy(buf.data() + i * w, s[i].data(), s[i].size());
    dataset(path, "|S" + std::to_string(w), {uint64_t(s.size())}, buf.data(), w);
}

size_t OutFile::reserve(const std::string& path, const std::string& dtype, const std::vector<uint64_t>& shape,
                        size_t itemsize) {
    if (h5_) return h5_->reserve(path, dtype, shape);
    if (closed_) throw std::runtime_error("OutFile: write after close");
    uint64_t n = 1;
    for (uint64_t s : shape) n *= s;
    pending_.push_back(Pending{path, dtype, shape, std::vector<unsigned char>(size_t(n) * itemsize, 0)});
    return pending_.size() - 1;
}

void OutFile::write_slice(size_t handle, uint64_t off, const void* data, size_t nbytes) {
    if (h5_) return h5_->write_at(handle, off, data, nbytes);
    if (handle >= pending_.size()) throw std::invalid_argument("OutFile: bad handle");
    auto& d = pending_[handle].data;
    if (off + nbytes > d.size()) throw std::out_of_range("OutFile: slice beyond the reserved dataset");
    std::memcpy(d.data() + off, data, nbytes);
}

void OutFile::commit() {
    if (h5_) h5_->commit();
}

void OutFile::close() {
    if (h5_) {
        h5_->close();
        return;
    }
    if (closed_ || !fp_) return;
    for (auto& p : pending_) member(clean(p.path) + ".npy", p.dtype, p.shape, p.data.data(), p.data.size());
    pending_.clear();
    FILE* f = static_cast<FILE*>(fp_);
    std::vector<unsigned char> cd;
    for (const auto& e : entries_) {
        put32(cd, 0x02014b50);
        put16(cd, 45);
        put16(cd, 45);
        put16(cd, 0);
        put16(cd, 0);
        put16(cd, 0);
        put16(cd, 0x21);
        put32(cd, e.crc);
        put32(cd, 0xffffffffu);
        put32(cd, 0xffffffffu);
        put16(cd, uint16_t(e.name.size()));
        put16(cd, 28);
        put16(cd, 0);
        put16(cd, 0);
        put16(cd, 0);
        put32(cd, 0);
        put32(cd, 0xffffffffu);
        cd.insert(cd.end(), e.name.begin(), e.name.end());
        put16(cd, 0x0001);
        put16(cd, 24);
        put64(cd, e.size);
        put64(cd, e.size);
        put64(cd, e.offset);
    }
    const uint64_t cd_off = pos_;
    std::vector<unsigned char> end;
    // Zip64 end of central directory record + locator
    put32(end, 0x06064b50);
    put64(end, 44);
    put16(end, 45);
    put16(end, 45);
    put32(end, 0);
    put32(end, 0);
    put64(end, entries_.size());
    put64(end, entries_.size());
    put64(end, cd.size());
    put64(end, cd_off);
    put32(end, 0x07064b50);
    put32(end, 0);
    put64(end, cd_off + cd.size());
    put32(end, 1);
    // classic end of central directory
    put32(end, 0x06054b50);
    put16(end, 0);
    put16(end, 0);
    put16(end, 0xffff);
    put16(end, 0xffff);
    put32(end, 0xffffffffu);
    put32(end, 0xffffffffu);
    put16(end, 0);
    const bool ok = std::fwrite(cd.data(), 1, cd.size(), f) == cd.size() &&
                    std::fwrite(end.data(), 1, end.size(), f) == end.size();
    std::fclose(f);
    fp_ = nullptr;
    closed_ = true;
    if (!ok) throw std::runtime_error("OutFile: write failed: " + path_);
}

}  // namespace CMC
