// BIOM 2.x tables stored in HDF5 files, read without the HDF5 library (the
// format subset is listed in ssu_biom.hpp).  Layouts follow the published
// HDF5 file format specification (superblock, object header, B-tree v1,
// symbol-table node, local and global heap, and the dataspace, datatype,
// data layout, filter pipeline, continuation and symbol-table messages).
#include "ssu_biom.hpp"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>

#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <vector>

namespace ssu {
namespace {

// Read-only view of the file; every access is bounds-checked and throws
// std::runtime_error past the end.
class File {
  public:
    ~File() {
        if (base_) munmap(const_cast<uint8_t *>(base_), size_);
    }
    void open(const std::string &path) {
        const int fd = ::open(path.c_str(), O_RDONLY);
        if (fd < 0) throw std::runtime_error("cannot open the file");
        struct stat st;
        if (fstat(fd, &st) != 0 || st.st_size <= 0) {
            ::close(fd);
            throw std::runtime_error("cannot size the file");
        }
        size_ = static_cast<size_t>(st.st_size);
        void *p = mmap(nullptr, size_, PROT_READ, MAP_PRIVATE, fd, 0);
        ::close(fd);
        if (p == MAP_FAILED) throw std::runtime_error("cannot map the file");
        base_ = static_cast<const uint8_t *>(p);
    }
    const uint8_t *at(uint64_t off, uint64_t n) const {
        if (off > size_ || n > size_ - off) throw std::runtime_error("read past the end of the file");
        return base_ + off;
    }
    uint64_t uint(uint64_t off, unsigned bytes) const {
        const uint8_t *p = at(off, bytes);
        uint64_t v = 0;
        for (unsigned i = 0; i < bytes; i++) v |= static_cast<uint64_t>(p[i]) << (8 * i);
        return v;
    }
    size_t size() const { return size_; }

  private:
    const uint8_t *base_ = nullptr;
    size_t size_ = 0;
};

constexpr uint64_t kUndefined = ~uint64_t(0);

struct Message {
    uint16_t type;
    uint64_t off;  // message data
    uint64_t size;
};

struct Datatype {
    int cls = -1;      // 0 fixed-point, 1 floating-point, 3 string, 9 variable-length
    uint32_t size = 0;
    bool is_signed = false;
    bool big_endian = false;
    int vlen_kind = -1;  // class 9: 0 sequence, 1 string
    int str_pad = 0;     // class 3: 0 null-terminated, 1 null-padded, 2 space-padded
};

struct Dataset {
    std::vector<uint64_t> dims;
    Datatype type;
    int layout = -1;  // 0 compact, 1 contiguous, 2 chunked
    uint64_t addr = kUndefined;
    uint64_t data_size = 0;
    std::vector<uint32_t> chunk;  // chunk dims (element size last)
    std::vector<uint16_t> filters;
    std::vector<std::vector<uint32_t>> filter_values;
};

class Reader {
  public:
    explicit Reader(const std::string &path) { f_.open(path); }

    void superblock() {
        static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
        uint64_t sb = kUndefined;
        for (uint64_t off = 0; off + 8 <= f_.size(); off = off ? off * 2 : 512)
            if (std::memcmp(f_.at(off, 8), sig, 8) == 0) {
                sb = off;
                break;
            }
        if (sb == kUndefined) throw std::runtime_error("not an HDF5 file (no superblock signature)");
        const unsigned version = f_.uint(sb + 8, 1);
        if (version > 1)
            throw std::runtime_error("HDF5 superblock version " + std::to_string(version) +
                                     " is not supported (versions 0 and 1 are)");
        so_ = f_.uint(sb + 13, 1);
        sl_ = f_.uint(sb + 14, 1);
        if ((so_ != 4 && so_ != 8) || (sl_ != 4 && sl_ != 8))
            throw std::runtime_error("unsupported HDF5 offset or length size");
        uint64_t p = sb + 24 + (version == 1 ? 4 : 0);
        base_ = f_.uint(p, so_);
        p += 4 * so_;  // base, free-space, end-of-file and driver-block addresses
        // root group symbol table entry: link name offset, object header address
        root_ = base_ + f_.uint(p + so_, so_);
    }

    // Messages of the version-1 object header at `addr`, continuation blocks
    // followed.
    std::vector<Message> messages(uint64_t addr) const {
        const unsigned version = f_.uint(addr, 1);
        if (version != 1)
            throw std::runtime_error("HDF5 object header version " + std::to_string(version) + " is not supported");
        const uint64_t total = f_.uint(addr + 2, 2);
        std::vector<std::pair<uint64_t, uint64_t>> blocks{{addr + 16, f_.uint(addr + 8, 4)}};
        std::vector<Message> out;
        for (size_t b = 0; b < blocks.size() && out.size() < total; b++) {
            uint64_t p = blocks[b].first;
            const uint64_t end = p + blocks[b].second;
            while (p + 8 <= end && out.size() < total) {
                Message m{static_cast<uint16_t>(f_.uint(p, 2)), p + 8, f_.uint(p + 2, 2)};
                const unsigned flags = f_.uint(p + 4, 1);
                f_.at(m.off, m.size);
                if (flags & 0x2) throw std::runtime_error("shared HDF5 object header messages are not supported");
                if (m.type == 0x10) blocks.emplace_back(base_ + f_.uint(m.off, so_), f_.uint(m.off + so_, sl_));
                out.push_back(m);
                p = m.off + m.size;
            }
            if (blocks.size() > 4096) throw std::runtime_error("too many HDF5 header continuation blocks");
        }
        return out;
    }

    // Object header address of `path` ("/a/b/c") below the root group.
    uint64_t find(const std::string &path) const {
        uint64_t obj = root_;
        size_t pos = 0;
        while (pos < path.size()) {
            if (path[pos] == '/') {
                pos++;
                continue;
            }
            const size_t next = path.find('/', pos);
            const std::string name = path.substr(pos, next == std::string::npos ? std::string::npos : next - pos);
            obj = child(obj, name);
            if (obj == kUndefined) throw std::runtime_error("no object " + path + " in the file");
            pos = next == std::string::npos ? path.size() : next;
        }
        return obj;
    }

    Dataset dataset(uint64_t obj) const {
        Dataset d;
        for (const Message &m : messages(obj)) {
            if (m.type == 0x0001) read_dataspace(m, d);
            else if (m.type == 0x0003) d.type = read_datatype(m.off, m.size);
            else if (m.type == 0x0008) read_layout(m, d);
            else if (m.type == 0x000B) read_filters(m, d);
        }
        if (d.type.cls < 0 || d.layout < 0) throw std::runtime_error("HDF5 dataset without a datatype or layout");
        if (d.layout == 2 && d.dims.size() != 1)
            throw std::runtime_error("only one-dimensional chunked HDF5 datasets are read");
        if (d.type.big_endian && (d.type.cls == 0 || d.type.cls == 1))
            throw std::runtime_error("big-endian HDF5 datasets are not supported");
        return d;
    }

    // The dataset's elements as stored (elements x type size bytes).
    static uint64_t count(const Dataset &d) {
        uint64_t n = 1;
        for (uint64_t x : d.dims) {
            if (x && n > (uint64_t(1) << 40) / x) throw std::runtime_error("HDF5 dataset too large");
            n *= x;
        }
        return n;
    }

    std::vector<uint8_t> raw(const Dataset &d) const {
        const uint64_t n = count(d);
        const uint64_t es = d.type.size;
        if (es == 0 || (n && n > (uint64_t(1) << 40) / es)) throw std::runtime_error("HDF5 dataset too large");
        std::vector<uint8_t> out(n * es, 0);
        if (d.layout == 0 || d.layout == 1) {
            if (d.addr == kUndefined) return out;  // never written: fill value zero
            const uint64_t have = std::min<uint64_t>(d.data_size, out.size());
            std::memcpy(out.data(), f_.at(d.addr, have), have);
            return out;
        }
        if (d.chunk.size() != 2 || d.chunk[1] != es) throw std::runtime_error("unexpected HDF5 chunk shape");
        if (d.addr == kUndefined) return out;
        chunks(d, d.addr, out, 0);
        return out;
    }

    // Elements as doubles (integer or floating-point datasets).
    std::vector<double> doubles(const Dataset &d) const {
        const std::vector<uint8_t> b = raw(d);
        const uint64_t n = count(d);
        std::vector<double> v(n);
        for (uint64_t i = 0; i < n; i++) v[i] = number(b.data() + i * d.type.size, d.type);
        return v;
    }

    std::vector<std::string> strings(const Dataset &d) const {
        const std::vector<uint8_t> b = raw(d);
        const uint64_t n = count(d);
        std::vector<std::string> out(n);
        if (d.type.cls == 3) {
            for (uint64_t i = 0; i < n; i++) {
                const char *s = reinterpret_cast<const char *>(b.data() + i * d.type.size);
                size_t len = d.type.size;
                if (d.type.str_pad == 2) {
                    while (len && s[len - 1] == ' ') len--;
                } else {
                    len = strnlen(s, len);
                }
                out[i].assign(s, len);
            }
        } else if (d.type.cls == 9 && d.type.vlen_kind == 1) {
            const uint64_t es = 4 + so_ + 4;
            if (d.type.size != es) throw std::runtime_error("unexpected HDF5 variable-length string size");
            for (uint64_t i = 0; i < n; i++) {
                const uint8_t *p = b.data() + i * es;
                uint64_t len = 0, coll = 0, idx = 0;
                for (int k = 0; k < 4; k++) len |= static_cast<uint64_t>(p[k]) << (8 * k);
                for (unsigned k = 0; k < so_; k++) coll |= static_cast<uint64_t>(p[4 + k]) << (8 * k);
                for (int k = 0; k < 4; k++) idx |= static_cast<uint64_t>(p[4 + so_ + k]) << (8 * k);
                if (coll == 0 && len == 0) continue;  // empty / null string
                const std::pair<uint64_t, uint64_t> obj = heap_object(base_ + coll, idx);
                out[i].assign(reinterpret_cast<const char *>(f_.at(obj.first, std::min(obj.second, len))),
                              std::min(obj.second, len));
            }
        } else {
            throw std::runtime_error("HDF5 dataset is not a string dataset");
        }
        return out;
    }

  private:
    File f_;
    unsigned so_ = 8, sl_ = 8;
    uint64_t base_ = 0, root_ = 0;
    mutable std::map<uint64_t, std::map<uint64_t, std::pair<uint64_t, uint64_t>>> gheaps_;

    static double number(const uint8_t *p, const Datatype &t) {
        if (t.cls == 1) {
            if (t.size == 8) {
                double v;
                std::memcpy(&v, p, 8);
                return v;
            }
            if (t.size == 4) {
                float v;
                std::memcpy(&v, p, 4);
                return v;
            }
            throw std::runtime_error("unsupported HDF5 floating-point size");
        }
        if (t.cls == 0) {
            uint64_t u = 0;
            for (uint32_t k = 0; k < t.size && k < 8; k++) u |= static_cast<uint64_t>(p[k]) << (8 * k);
            if (t.size == 0 || t.size > 8) throw std::runtime_error("unsupported HDF5 integer size");
            if (t.is_signed && t.size < 8 && (u >> (8 * t.size - 1)) & 1) u |= ~uint64_t(0) << (8 * t.size);
            return t.is_signed ? static_cast<double>(static_cast<int64_t>(u)) : static_cast<double>(u);
        }
        throw std::runtime_error("HDF5 dataset is not numeric");
    }

    // Object header address of the link `name` in the old-style group `grp`.
    uint64_t child(uint64_t grp, const std::string &name) const {
        uint64_t btree = kUndefined, heap = kUndefined;
        for (const Message &m : messages(grp))
            if (m.type == 0x0011) {
                btree = base_ + f_.uint(m.off, so_);
                heap = base_ + f_.uint(m.off + so_, so_);
            }
        if (btree == kUndefined) throw std::runtime_error("HDF5 group without a symbol table (newer group format)");
        if (std::memcmp(f_.at(heap, 4), "HEAP", 4) != 0) throw std::runtime_error("bad HDF5 local heap");
        const uint64_t heap_size = f_.uint(heap + 8, sl_);
        const uint64_t heap_data = base_ + f_.uint(heap + 8 + 2 * sl_, so_);
        return group_lookup(btree, heap_data, heap_size, name, 0);
    }

    uint64_t group_lookup(uint64_t node, uint64_t heap_data, uint64_t heap_size, const std::string &name,
                          int depth) const {
        if (depth > 64) throw std::runtime_error("HDF5 group B-tree too deep");
        if (std::memcmp(f_.at(node, 4), "TREE", 4) != 0 || f_.uint(node + 4, 1) != 0)
            throw std::runtime_error("bad HDF5 group B-tree node");
        const unsigned level = f_.uint(node + 5, 1);
        const uint64_t used = f_.uint(node + 6, 2);
        uint64_t p = node + 8 + 2 * so_;  // past the siblings: key 0
        for (uint64_t i = 0; i < used; i++) {
            const uint64_t child_addr = base_ + f_.uint(p + sl_, so_);
            p += sl_ + so_;
            uint64_t r;
            if (level > 0) {
                r = group_lookup(child_addr, heap_data, heap_size, name, depth + 1);
            } else {
                r = snod_lookup(child_addr, heap_data, heap_size, name);
            }
            if (r != kUndefined) return r;
        }
        return kUndefined;
    }

    uint64_t snod_lookup(uint64_t snod, uint64_t heap_data, uint64_t heap_size, const std::string &name) const {
        if (std::memcmp(f_.at(snod, 4), "SNOD", 4) != 0) throw std::runtime_error("bad HDF5 symbol table node");
        const uint64_t n = f_.uint(snod + 6, 2);
        const uint64_t entry = 2 * so_ + 24;
        for (uint64_t i = 0; i < n; i++) {
            const uint64_t e = snod + 8 + i * entry;
            const uint64_t name_off = f_.uint(e, so_);
            if (name_off >= heap_size) throw std::runtime_error("bad HDF5 link name offset");
            const char *s = reinterpret_cast<const char *>(f_.at(heap_data + name_off, 1));
            const size_t room = heap_size - name_off;
            const size_t len = strnlen(reinterpret_cast<const char *>(f_.at(heap_data + name_off, room)), room);
            if (len == name.size() && std::memcmp(s, name.data(), len) == 0) return base_ + f_.uint(e + so_, so_);
        }
        return kUndefined;
    }

    void read_dataspace(const Message &m, Dataset &d) const {
        const unsigned version = f_.uint(m.off, 1);
        const unsigned rank = f_.uint(m.off + 1, 1);
        uint64_t p;
        if (version == 1) {
            p = m.off + 8;
        } else if (version == 2) {
            p = m.off + 4;
        } else {
            throw std::runtime_error("unsupported HDF5 dataspace message version");
        }
        d.dims.clear();
        for (unsigned r = 0; r < rank; r++) d.dims.push_back(f_.uint(p + r * sl_, sl_));
    }

    Datatype read_datatype(uint64_t off, uint64_t size) const {
        if (size < 8) throw std::runtime_error("short HDF5 datatype message");
        Datatype t;
        const unsigned cv = f_.uint(off, 1);
        t.cls = cv & 0x0F;
        const unsigned b0 = f_.uint(off + 1, 1);
        t.size = static_cast<uint32_t>(f_.uint(off + 4, 4));
        if (t.cls == 0) {
            t.big_endian = b0 & 0x1;
            t.is_signed = b0 & 0x8;
        } else if (t.cls == 1) {
            t.big_endian = b0 & 0x1;
        } else if (t.cls == 3) {
            t.str_pad = b0 & 0x0F;
        } else if (t.cls == 9) {
            t.vlen_kind = b0 & 0x0F;
        }
        return t;
    }

    void read_layout(const Message &m, Dataset &d) const {
        const unsigned version = f_.uint(m.off, 1);
        if (version == 3) {
            d.layout = f_.uint(m.off + 1, 1);
            uint64_t p = m.off + 2;
            if (d.layout == 0) {
                d.data_size = f_.uint(p, 2);
                d.addr = p + 2;  // compact data lives in the message
            } else if (d.layout == 1) {
                const uint64_t a = f_.uint(p, so_);
                d.addr = a == (so_ == 8 ? kUndefined : 0xFFFFFFFFu) ? kUndefined : base_ + a;
                d.data_size = f_.uint(p + so_, sl_);
            } else if (d.layout == 2) {
                const unsigned nd = f_.uint(p, 1);
                const uint64_t a = f_.uint(p + 1, so_);
                d.addr = a == (so_ == 8 ? kUndefined : 0xFFFFFFFFu) ? kUndefined : base_ + a;
                d.chunk.clear();
                for (unsigned i = 0; i < nd; i++) d.chunk.push_back(static_cast<uint32_t>(f_.uint(p + 1 + so_ + 4 * i, 4)));
            } else {
                throw std::runtime_error("unsupported HDF5 layout class");
            }
        } else if (version == 1 || version == 2) {
            const unsigned nd = f_.uint(m.off + 1, 1);
            d.layout = f_.uint(m.off + 2, 1);
            uint64_t p = m.off + 8;
            if (d.layout != 0) {
                const uint64_t a = f_.uint(p, so_);
                d.addr = a == (so_ == 8 ? kUndefined : 0xFFFFFFFFu) ? kUndefined : base_ + a;
                p += so_;
            }
            d.chunk.clear();
            for (unsigned i = 0; i < nd; i++) d.chunk.push_back(static_cast<uint32_t>(f_.uint(p + 4 * i, 4)));
            p += 4 * nd;
            if (d.layout == 0) {
                d.data_size = f_.uint(p, 4);
                d.addr = p + 4;
            } else if (d.layout == 1) {
                d.data_size = kUndefined;  // the dataspace gives the size
            }
        } else {
            throw std::runtime_error("unsupported HDF5 layout message version " + std::to_string(version));
        }
    }

    void read_filters(const Message &m, Dataset &d) const {
        const unsigned version = f_.uint(m.off, 1);
        const unsigned n = f_.uint(m.off + 1, 1);
        uint64_t p = m.off + (version == 1 ? 8 : 2);
        for (unsigned i = 0; i < n; i++) {
            const uint16_t id = static_cast<uint16_t>(f_.uint(p, 2));
            uint64_t name_len = 0;
            if (version == 1 || id >= 256) {
                name_len = f_.uint(p + 2, 2);
                p += 2;
            }
            const uint64_t nvals = f_.uint(p + 4, 2);
            p += 6;
            if (version == 1) name_len = (name_len + 7) / 8 * 8;
            p += name_len;
            std::vector<uint32_t> vals;
            for (uint64_t k = 0; k < nvals; k++) vals.push_back(static_cast<uint32_t>(f_.uint(p + 4 * k, 4)));
            p += 4 * nvals;
            if (version == 1 && (nvals & 1)) p += 4;
            d.filters.push_back(id);
            d.filter_values.push_back(vals);
        }
    }

    // Walk the chunk index (version-1 B-tree, node type 1) of a 1-D dataset.
    void chunks(const Dataset &d, uint64_t node, std::vector<uint8_t> &out, int depth) const {
        if (depth > 64) throw std::runtime_error("HDF5 chunk B-tree too deep");
        if (std::memcmp(f_.at(node, 4), "TREE", 4) != 0 || f_.uint(node + 4, 1) != 1)
            throw std::runtime_error("bad HDF5 chunk B-tree node");
        const unsigned level = f_.uint(node + 5, 1);
        const uint64_t used = f_.uint(node + 6, 2);
        const uint64_t key = 8 + 8 * d.chunk.size();
        uint64_t p = node + 8 + 2 * so_;
        for (uint64_t i = 0; i < used; i++) {
            const uint64_t stored = f_.uint(p, 4);
            const uint32_t mask = static_cast<uint32_t>(f_.uint(p + 4, 4));
            const uint64_t first = f_.uint(p + 8, 8);  // element offset along dimension 0
            const uint64_t child_addr = base_ + f_.uint(p + key, so_);
            p += key + so_;
            if (level > 0) {
                chunks(d, child_addr, out, depth + 1);
                continue;
            }
            std::vector<uint8_t> bytes(f_.at(child_addr, stored), f_.at(child_addr, stored) + stored);
            const uint64_t expect = static_cast<uint64_t>(d.chunk[0]) * d.chunk[1];
            for (size_t k = d.filters.size(); k-- > 0;) {
                if (mask & (1u << k)) continue;
                bytes = unfilter(d.filters[k], d.filter_values[k], bytes, expect);
            }
            const uint64_t es = d.chunk[1];
            if (first >= d.dims[0]) continue;
            const uint64_t count = std::min<uint64_t>(d.chunk[0], d.dims[0] - first);
            if (bytes.size() < count * es) throw std::runtime_error("short HDF5 chunk");
            std::memcpy(out.data() + first * es, bytes.data(), count * es);
        }
    }

    static std::vector<uint8_t> unfilter(uint16_t id, const std::vector<uint32_t> &vals,
                                         const std::vector<uint8_t> &in, uint64_t expect) {
        if (id == 1) {  // deflate (zlib stream)
            std::vector<uint8_t> out(std::max<uint64_t>(expect, 1));
            z_stream z{};
            if (inflateInit(&z) != Z_OK) throw std::runtime_error("zlib initialisation failed");
            z.next_in = const_cast<Bytef *>(in.data());
            z.avail_in = static_cast<uInt>(in.size());
            size_t have = 0;
            int rc = Z_OK;
            while (rc != Z_STREAM_END) {
                if (have == out.size()) out.resize(out.size() * 2);
                z.next_out = out.data() + have;
                z.avail_out = static_cast<uInt>(out.size() - have);
                rc = inflate(&z, Z_NO_FLUSH);
                have = out.size() - z.avail_out;
                if (rc != Z_OK && rc != Z_STREAM_END) {
                    inflateEnd(&z);
                    throw std::runtime_error("corrupt deflate data in an HDF5 chunk");
                }
                if (rc == Z_OK && z.avail_in == 0 && z.avail_out != 0) break;
            }
            inflateEnd(&z);
            out.resize(have);
            return out;
        }
        if (id == 2) {  // shuffle: byte planes back to elements
            const uint32_t es = vals.empty() ? 1 : vals[0];
            if (es <= 1) return in;
            std::vector<uint8_t> out(in.size());
            const size_t n = in.size() / es;
            for (size_t b = 0; b < es; b++)
                for (size_t i = 0; i < n; i++) out[i * es + b] = in[b * n + i];
            std::memcpy(out.data() + n * es, in.data() + n * es, in.size() - n * es);
            return out;
        }
        if (id == 3) {  // Fletcher-32: a 4-byte checksum follows the data
            if (in.size() < 4) throw std::runtime_error("short Fletcher-32 HDF5 chunk");
            return std::vector<uint8_t>(in.begin(), in.end() - 4);
        }
        throw std::runtime_error("HDF5 filter " + std::to_string(id) + " is not supported");
    }

    // (address, size) of object `idx` of the global heap collection at `coll`.
    std::pair<uint64_t, uint64_t> heap_object(uint64_t coll, uint64_t idx) const {
        auto it = gheaps_.find(coll);
        if (it == gheaps_.end()) {
            if (std::memcmp(f_.at(coll, 4), "GCOL", 4) != 0) throw std::runtime_error("bad HDF5 global heap");
            const uint64_t size = f_.uint(coll + 8, sl_);
            std::map<uint64_t, std::pair<uint64_t, uint64_t>> objs;
            uint64_t p = coll + 8 + sl_;
            const uint64_t end = coll + size;
            while (p + 8 + sl_ <= end) {
                const uint64_t id = f_.uint(p, 2);
                const uint64_t osz = f_.uint(p + 8, sl_);
                if (id == 0) break;  // free space to the end of the collection
                objs[id] = {p + 8 + sl_, osz};
                p += 8 + sl_ + (osz + 7) / 8 * 8;
            }
            it = gheaps_.emplace(coll, std::move(objs)).first;
        }
        auto o = it->second.find(idx);
        if (o == it->second.end()) throw std::runtime_error("missing HDF5 global heap object");
        return o->second;
    }
};

}  // namespace

bool read_hdf5_dataset(const std::string &path, const std::string &name, H5Data &out, std::string &err) {
    try {
        Reader r(path);
        r.superblock();
        const Dataset d = r.dataset(r.find(name));
        H5Data o;
        o.dims = d.dims;
        o.is_string = d.type.cls == 3 || (d.type.cls == 9 && d.type.vlen_kind == 1);
        if (o.is_string)
            o.strings = r.strings(d);
        else
            o.values = r.doubles(d);
        out = std::move(o);
        return true;
    } catch (const std::exception &e) {
        err = e.what();
        return false;
    }
}

bool read_biom_hdf5(const std::string &path, Table &out, std::string &err) {
    try {
        Reader r(path);
        r.superblock();
        const std::vector<std::string> obs = r.strings(r.dataset(r.find("/observation/ids")));
        const std::vector<std::string> samples = r.strings(r.dataset(r.find("/sample/ids")));
        const std::vector<double> indptr = r.doubles(r.dataset(r.find("/observation/matrix/indptr")));
        const std::vector<double> indices = r.doubles(r.dataset(r.find("/observation/matrix/indices")));
        const std::vector<double> data = r.doubles(r.dataset(r.find("/observation/matrix/data")));
        if (indptr.size() != obs.size() + 1) throw std::runtime_error("indptr length does not match the observations");
        if (indices.size() != data.size()) throw std::runtime_error("indices and data lengths differ");
        if (obs.size() >= UINT32_MAX || samples.size() >= UINT32_MAX || data.size() >= UINT32_MAX)
            throw std::runtime_error("table too large");
        Table t;
        t.n_obs = static_cast<uint32_t>(obs.size());
        t.n_samples = static_cast<uint32_t>(samples.size());
        t.own_indptr.resize(indptr.size());
        for (size_t i = 0; i < indptr.size(); i++) {
            if (!(indptr[i] >= 0 && indptr[i] <= static_cast<double>(data.size())))
                throw std::runtime_error("indptr entry out of range");
            t.own_indptr[i] = static_cast<uint32_t>(indptr[i]);
        }
        t.own_indices.resize(indices.size());
        for (size_t i = 0; i < indices.size(); i++) {
            if (!(indices[i] >= 0 && indices[i] < static_cast<double>(UINT32_MAX)))
                throw std::runtime_error("sample index out of range");
            t.own_indices[i] = static_cast<uint32_t>(indices[i]);
        }
        t.own_data = data;
        // the ids' bytes, kept by the table; views point into the block
        size_t total = 0;
        for (const std::string &s : obs) total += s.size();
        for (const std::string &s : samples) total += s.size();
        t.own_names.reset(new char[std::max<size_t>(total, 1)]);
        char *w = t.own_names.get();
        for (const std::string &s : obs) {
            std::memcpy(w, s.data(), s.size());
            t.obs_ids.emplace_back(w, s.size());
            w += s.size();
        }
        for (const std::string &s : samples) {
            std::memcpy(w, s.data(), s.size());
            t.sample_ids.emplace_back(w, s.size());
            w += s.size();
        }
        t.adopt();
        t.compute_totals();
        out = std::move(t);
        return true;
    } catch (const std::exception &e) {
        err = e.what();
        return false;
    }
}

}  // namespace ssu
