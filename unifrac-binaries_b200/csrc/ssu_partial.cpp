// Partial result files (format in ssu_partial.hpp): write_partial,
// read_partial, read_partial_header, read_partial_one_stripe and
// validate_partial of the reference's C API (src/api.hpp:816-910), with the
// same status codes.  Unlike the reference, nothing here exits the process or
// leaks on a malformed file, and stripe indices are range-checked.
#include "ssu_partial.hpp"

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>

#include "ssu_lz4.hpp"

namespace ssu {
namespace {

constexpr uint32_t kMagic = 0x088ABA02u;  // PARTIAL_MAGIC_V2, src/api.hpp:23

struct Fd {
    int fd = -1;
    explicit Fd(int f) : fd(f) {}
    ~Fd() {
        if (fd >= 0) ::close(fd);
    }
};

bool read_full(int fd, void *buf, size_t n) {
    uint8_t *p = static_cast<uint8_t *>(buf);
    while (n) {
        const ssize_t r = ::read(fd, p, n);
        if (r <= 0) return false;
        p += r;
        n -= static_cast<size_t>(r);
    }
    return true;
}

bool pread_full(int fd, void *buf, size_t n, uint64_t off) {
    uint8_t *p = static_cast<uint8_t *>(buf);
    while (n) {
        const ssize_t r = ::pread(fd, p, n, static_cast<off_t>(off));
        if (r <= 0) return false;
        p += r;
        off += static_cast<uint64_t>(r);
        n -= static_cast<size_t>(r);
    }
    return true;
}

bool write_full(int fd, const void *buf, size_t n) {
    const uint8_t *p = static_cast<const uint8_t *>(buf);
    while (n) {
        const ssize_t w = ::write(fd, p, n);
        if (w <= 0) return false;
        p += w;
        n -= static_cast<size_t>(w);
    }
    return true;
}

struct Header {
    uint32_t n_samples, n_stripes, stripe_start, stripe_total;
    bool upper;
    std::vector<std::string> ids;
};

// read_partial_header_fd (src/api.cpp:2071-2134): the header checks and the
// sample ids; the file position is left at the first stripe.
IOStatus read_header(int fd, Header &h) {
    uint32_t w[8];
    if (!read_full(fd, w, sizeof(w)) || w[0] != kMagic) return magic_incompatible;
    h.n_samples = w[1];
    h.n_stripes = w[2];
    h.stripe_start = w[3];
    h.stripe_total = w[4];
    h.upper = w[5] != 0;
    if (h.n_samples == 0 || h.n_stripes == 0 || h.stripe_total == 0 || !h.upper) return bad_header;
    if (h.stripe_total >= h.n_samples || h.n_stripes > h.stripe_total || h.stripe_start >= h.stripe_total ||
        h.stripe_start + h.n_stripes > h.stripe_total)
        return bad_header;
    const uint32_t id_bytes = w[6], id_cmp = w[7];
    if (id_bytes == 0 || id_cmp == 0) return bad_header;
    std::vector<uint8_t> cmp(id_cmp), raw(id_bytes);
    if (!read_full(fd, cmp.data(), id_cmp)) return magic_incompatible;
    if (lz4_decompress(cmp.data(), id_cmp, raw.data(), id_bytes) != static_cast<long long>(id_bytes))
        return magic_incompatible;
    const char *p = reinterpret_cast<const char *>(raw.data());
    const char *end = p + id_bytes;
    h.ids.clear();
    h.ids.reserve(h.n_samples);
    for (uint32_t i = 0; i < h.n_samples; i++) {
        const size_t len = strnlen(p, static_cast<size_t>(end - p));
        if (p + len >= end) return magic_incompatible;  // no terminating NUL inside the block
        h.ids.emplace_back(p, len);
        p += len + 1;
    }
    return read_okay;
}

char **ids_to_c(const std::vector<std::string> &ids) {
    char **out = static_cast<char **>(std::malloc(sizeof(char *) * (ids.empty() ? 1 : ids.size())));
    for (size_t i = 0; i < ids.size(); i++) out[i] = strdup(ids[i].c_str());
    return out;
}

IOStatus read_stripe(int fd, uint64_t offset, uint32_t n_samples, double *out, uint64_t *next) {
    uint32_t cmp = 0;
    if (!pread_full(fd, &cmp, 4, offset)) return magic_incompatible;
    const size_t raw = sizeof(double) * static_cast<size_t>(n_samples);
    if (cmp == 0 || cmp > lz4_bound(raw)) return magic_incompatible;
    std::vector<uint8_t> buf(cmp);
    if (!pread_full(fd, buf.data(), cmp, offset + 4)) return magic_incompatible;
    if (lz4_decompress(buf.data(), cmp, reinterpret_cast<uint8_t *>(out), raw) != static_cast<long long>(raw))
        return magic_incompatible;
    if (next) *next = offset + 4 + cmp;
    return read_okay;
}

}  // namespace

IOStatus partial_stripe_offsets(const char *filename, uint64_t first, uint32_t n_stripes,
                                std::vector<uint64_t> &offsets) {
    Fd f(::open(filename, O_RDONLY));
    if (f.fd < 0) return open_error;
    offsets.assign(n_stripes, 0);
    uint64_t off = first;
    for (uint32_t s = 0; s < n_stripes; s++) {
        offsets[s] = off;
        uint32_t cmp = 0;
        if (!pread_full(f.fd, &cmp, 4, off)) return read_error;
        off += 4 + static_cast<uint64_t>(cmp);
    }
    return read_okay;
}

IOStatus partial_read_stripe_at(const char *filename, uint64_t offset, uint32_t n_samples, double *out) {
    Fd f(::open(filename, O_RDONLY));
    if (f.fd < 0) return open_error;
    return read_stripe(f.fd, offset, n_samples, out, nullptr);
}

MergeStatus partial_check(const partial_dyn_mat_t *const *mats, int n, bool verbose) {
    if (n <= 0 || !mats || !mats[0]) {
        if (verbose) std::fprintf(stderr, "Zero or less partials.\n");
        return incomplete_stripe_set;
    }
    const uint32_t n_samples = mats[0]->n_samples;
    const uint32_t total = mats[0]->stripe_total;
    std::vector<bool> seen(total, false);
    uint64_t count = 0;
    for (int i = 0; i < n; i++) {
        const partial_dyn_mat_t *m = mats[i];
        if (!m || m->n_samples != n_samples) {
            if (verbose) std::fprintf(stderr, "Wrong number of samples in %d\n", i);
            return partials_mismatch;
        }
        if (m->stripe_total != total) {
            if (verbose) std::fprintf(stderr, "Wrong number of stripes in %d\n", i);
            return partials_mismatch;
        }
        if (m->is_upper_triangle != mats[0]->is_upper_triangle) {
            if (verbose) std::fprintf(stderr, "Wrong is_upper_triangle in %d\n", i);
            return square_mismatch;
        }
        for (uint32_t j = 0; j < n_samples; j++)
            if (std::strcmp(mats[0]->sample_ids[j], m->sample_ids[j]) != 0) {
                if (verbose) std::fprintf(stderr, "Different sample id %u in %d\n", j, i);
                return sample_id_consistency;
            }
        if (m->stripe_stop > total || m->stripe_start > m->stripe_stop) {
            if (verbose) std::fprintf(stderr, "Stripe range of %d out of bounds\n", i);
            return partials_mismatch;
        }
        for (uint32_t s = m->stripe_start; s < m->stripe_stop; s++) {
            if (seen[s]) {
                if (verbose) std::fprintf(stderr, "Overlap in %d at stripe %u\n", i, s);
                return stripes_overlap;
            }
            seen[s] = true;
            count++;
        }
    }
    if (count != total) {
        if (verbose)
            std::fprintf(stderr, "Insufficient number of stripes found, %llu!=%u\n",
                         static_cast<unsigned long long>(count), total);
        return incomplete_stripe_set;
    }
    return merge_okay;
}

}  // namespace ssu

extern "C" {

IOStatus write_partial(const char *filename, const partial_mat_t *result) {
    if (!filename || !result) return write_error;
    const uint32_t n_stripes = result->stripe_stop - result->stripe_start;
    std::string ids;
    for (uint32_t i = 0; i < result->n_samples; i++) {
        ids.append(result->sample_ids[i]);
        ids.push_back('\0');
    }
    std::vector<uint8_t> cmp(ssu::lz4_bound(ids.size()));
    const size_t id_cmp = ssu::lz4_compress(reinterpret_cast<const uint8_t *>(ids.data()), ids.size(), cmp.data(),
                                            cmp.size());
    if (id_cmp == 0 || ids.size() > UINT32_MAX) return write_error;
    ssu::Fd f(::open(filename, O_WRONLY | O_CREAT | O_TRUNC, S_IRUSR | S_IWUSR));
    if (f.fd < 0) return write_error;
    const uint32_t header[8] = {ssu::kMagic, result->n_samples, n_stripes, result->stripe_start,
                                result->stripe_total, result->is_upper_triangle ? 1u : 0u,
                                static_cast<uint32_t>(ids.size()), static_cast<uint32_t>(id_cmp)};
    if (!ssu::write_full(f.fd, header, sizeof(header)) || !ssu::write_full(f.fd, cmp.data(), id_cmp))
        return write_error;
    const size_t raw = sizeof(double) * static_cast<size_t>(result->n_samples);
    std::vector<uint8_t> block(4 + ssu::lz4_bound(raw));
    for (uint32_t s = 0; s < n_stripes; s++) {
        const size_t c = ssu::lz4_compress(reinterpret_cast<const uint8_t *>(result->stripes[s]), raw,
                                           block.data() + 4, block.size() - 4);
        if (c == 0) return write_error;
        const uint32_t c32 = static_cast<uint32_t>(c);
        std::memcpy(block.data(), &c32, 4);
        if (!ssu::write_full(f.fd, block.data(), 4 + c)) return write_error;
    }
    const uint32_t footer = ssu::kMagic;
    if (!ssu::write_full(f.fd, &footer, 4)) return write_error;
    return write_okay;
}

IOStatus read_partial(const char *filename, partial_mat_t **result) {
    if (!result) return unexpected_end;
    *result = nullptr;
    ssu::Fd f(::open(filename, O_RDONLY));
    if (f.fd < 0) return open_error;
    ssu::Header h;
    IOStatus st = ssu::read_header(f.fd, h);
    if (st != read_okay) return st;
    uint64_t off = static_cast<uint64_t>(::lseek(f.fd, 0, SEEK_CUR));
    partial_mat_t *p = static_cast<partial_mat_t *>(std::calloc(1, sizeof(partial_mat_t)));
    p->n_samples = h.n_samples;
    p->sample_ids = ssu::ids_to_c(h.ids);
    p->stripe_start = h.stripe_start;
    p->stripe_stop = h.stripe_start + h.n_stripes;
    p->stripe_total = h.stripe_total;
    p->is_upper_triangle = h.upper;
    p->stripes = static_cast<double **>(std::calloc(h.n_stripes, sizeof(double *)));
    for (uint32_t s = 0; s < h.n_stripes && st == read_okay; s++) {
        p->stripes[s] = static_cast<double *>(std::malloc(sizeof(double) * h.n_samples));
        st = ssu::read_stripe(f.fd, off, h.n_samples, p->stripes[s], &off);
    }
    uint32_t footer = 0;
    if (st == read_okay && (!ssu::pread_full(f.fd, &footer, 4, off) || footer != ssu::kMagic))
        st = magic_incompatible;
    if (st != read_okay) {
        destroy_partial_mat(&p);
        return st;
    }
    *result = p;
    return read_okay;
}

IOStatus read_partial_header(const char *filename, partial_dyn_mat_t **result) {
    if (!result) return unexpected_end;
    *result = nullptr;
    ssu::Fd f(::open(filename, O_RDONLY));
    if (f.fd < 0) return open_error;
    ssu::Header h;
    const IOStatus st = ssu::read_header(f.fd, h);
    if (st != read_okay) return st;
    partial_dyn_mat_t *p = static_cast<partial_dyn_mat_t *>(std::calloc(1, sizeof(partial_dyn_mat_t)));
    p->n_samples = h.n_samples;
    p->sample_ids = ssu::ids_to_c(h.ids);
    p->stripe_start = h.stripe_start;
    p->stripe_stop = h.stripe_start + h.n_stripes;
    p->stripe_total = h.stripe_total;
    p->is_upper_triangle = h.upper;
    p->stripes = static_cast<double **>(std::calloc(h.n_stripes, sizeof(double *)));
    p->offsets = static_cast<uint64_t *>(std::calloc(h.n_stripes, sizeof(uint64_t)));
    p->offsets[0] = static_cast<uint64_t>(::lseek(f.fd, 0, SEEK_CUR));
    p->filename = strdup(filename);
    *result = p;
    return read_okay;
}

IOStatus read_partial_one_stripe(partial_dyn_mat_t *result, uint32_t stripe_idx) {
    if (!result || !result->filename) return unexpected_end;
    const uint32_t n = result->stripe_stop - result->stripe_start;
    if (stripe_idx >= n) return bad_header;
    if (result->stripes[stripe_idx]) return read_okay;  // read once
    ssu::Fd f(::open(result->filename, O_RDONLY));
    if (f.fd < 0) return open_error;
    // offsets are learned in order: walk from the last known one
    uint32_t s = stripe_idx;
    while (s > 0 && result->offsets[s] == 0) s--;
    for (; s < stripe_idx; s++) {
        uint32_t cmp = 0;
        if (!ssu::pread_full(f.fd, &cmp, 4, result->offsets[s])) return magic_incompatible;
        result->offsets[s + 1] = result->offsets[s] + 4 + cmp;
    }
    double *out = static_cast<double *>(std::malloc(sizeof(double) * result->n_samples));
    const IOStatus st = ssu::read_stripe(f.fd, result->offsets[stripe_idx], result->n_samples, out, nullptr);
    if (st != read_okay) {
        std::free(out);
        return st;
    }
    result->stripes[stripe_idx] = out;
    return read_okay;
}

MergeStatus validate_partial(const partial_dyn_mat_t *const *partial_mats, int n_partials) {
    return ssu::partial_check(partial_mats, n_partials, true);
}

}  // extern "C"
