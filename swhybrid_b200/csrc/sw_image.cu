// sw_image.cu -- the on-disk DB image: one checksummed, mmap-able file with
// the records, their offsets, their titles and the length order.
//
// Replaces the reference's DBmaker output (.seq/.map/.title written by
// FastaFile::makeDatabase/flushOutBatch/flushOutRemain, src/FastaFile.cpp:
// 182-359, read back by DataPool::fill/getTitle, src/DataPool.cpp:171-310).
// Those files hold records in 128-wide length batches (sequence-major bytes),
// the batch map and the titles; this image holds records in FASTA order so a
// hit's index is its FASTA position, plus a title index for DataPool::getTitle
// and the stable longest-first permutation the device layout is built from.
//
// Layout (little-endian; every section starts on a 64-byte boundary):
//   header            128 bytes (ImageHeader)
//   offsets           uint64[n + 1]   record r = residues[offsets[r], offsets[r+1])
//   residues          uint8[n_residues], codes 0..24
//   title_offsets     uint64[n + 1]   title r = titles[title_offsets[r], ...[r+1])
//   titles            bytes (the FASTA header line without '>' and line end)
//   order             uint32[n]       records by length, longest first, stable
// checksum = 64-bit FNV-1a over the bytes after the header, 8 bytes at a time.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/swb200.h"
#include "sw_engine.h"

namespace {

constexpr char kMagic[8] = {'S', 'W', 'B', '2', '0', '0', 'D', 'B'};
constexpr uint32_t kImageVersion = 1;

struct ImageHeader {
    char magic[8];
    uint32_t version;
    uint32_t header_bytes;
    uint64_t n_records;
    uint64_t n_residues;
    uint64_t off_offsets;
    uint64_t off_residues;
    uint64_t off_title_offsets;
    uint64_t off_titles;
    uint64_t titles_bytes;
    uint64_t off_order;
    uint64_t file_bytes;
    uint64_t checksum;
    uint64_t reserved[4];
};
static_assert(sizeof(ImageHeader) == 128, "image header");

using swb::thread_fail;

uint64_t align64(uint64_t x) { return (x + 63) & ~uint64_t(63); }

// FNV-1a over 64-bit words (the tail zero-padded).
struct Hash64 {
    uint64_t h = 0xcbf29ce484222325ull;
    uint8_t tail[8];
    int nt = 0;
    void word(uint64_t w) { h = (h ^ w) * 0x100000001b3ull; }
    void add(const void* p, size_t n) {
        const uint8_t* b = (const uint8_t*)p;
        while (n && nt) {
            tail[nt++] = *b++;
            --n;
            if (nt == 8) {
                uint64_t w;
                memcpy(&w, tail, 8);
                word(w);
                nt = 0;
            }
        }
        for (; n >= 8; n -= 8, b += 8) {
            uint64_t w;
            memcpy(&w, b, 8);
            word(w);
        }
        while (n--) tail[nt++] = *b++;
    }
    uint64_t done() {
        if (nt) {
            memset(tail + nt, 0, 8 - nt);
            uint64_t w;
            memcpy(&w, tail, 8);
            word(w);
            nt = 0;
        }
        return h;
    }
};

struct Writer {
    FILE* f = nullptr;
    uint64_t pos = 0;
    Hash64 hash;
    bool put(const void* p, size_t n) {
        if (n && fwrite(p, 1, n, f) != n) return false;
        hash.add(p, n);
        pos += n;
        return true;
    }
    bool pad() {
        static const uint8_t z[64] = {0};
        return put(z, align64(pos) - pos);
    }
};

// Writes an image from records in memory.  titles / title_offsets may be null
// (empty titles).
sw_status write_image(const char* path, const uint8_t* residues, const uint64_t* offsets,
                      uint64_t n, const char* titles, const uint64_t* title_offsets) {
    if (!path || (n && !offsets)) return thread_fail(SW_ERR_INVALID, "null argument");
    uint64_t total = 0;
    std::vector<uint32_t> len(n);
    for (uint64_t i = 0; i < n; ++i) {
        if (offsets[i + 1] < offsets[i]) return thread_fail(SW_ERR_INVALID, "offsets not monotone at %llu",
                                                     (unsigned long long)i);
        len[i] = (uint32_t)(offsets[i + 1] - offsets[i]);
        total += len[i];
    }
    if (total && !residues) return thread_fail(SW_ERR_INVALID, "null residues");
    const uint8_t* base = n ? residues + offsets[0] : residues;
    for (uint64_t i = 0; i < total; ++i)
        if (base[i] > 24) return thread_fail(SW_ERR_INVALID, "residue code %d at %llu", base[i],
                                      (unsigned long long)i);
    uint64_t tbytes = 0;
    if (title_offsets) {
        for (uint64_t i = 0; i < n; ++i)
            if (title_offsets[i + 1] < title_offsets[i])
                return thread_fail(SW_ERR_INVALID, "title offsets not monotone at %llu",
                            (unsigned long long)i);
        tbytes = n ? title_offsets[n] - title_offsets[0] : 0;
        if (tbytes && !titles) return thread_fail(SW_ERR_INVALID, "null titles");
    }
    std::vector<uint32_t> order(n);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return len[a] > len[b]; });
    ImageHeader h{};
    memcpy(h.magic, kMagic, 8);
    h.version = kImageVersion;
    h.header_bytes = sizeof(ImageHeader);
    h.n_records = n;
    h.n_residues = total;
    h.off_offsets = sizeof(ImageHeader);
    h.off_residues = align64(h.off_offsets + 8 * (n + 1));
    h.off_title_offsets = align64(h.off_residues + total);
    h.off_titles = align64(h.off_title_offsets + 8 * (n + 1));
    h.titles_bytes = tbytes;
    h.off_order = align64(h.off_titles + tbytes);
    h.file_bytes = align64(h.off_order + 4 * n);
    const std::string tmp = std::string(path) + ".tmp";
    Writer w;
    w.f = fopen(tmp.c_str(), "wb");
    if (!w.f) return thread_fail(SW_ERR_INVALID, "cannot create %s", tmp.c_str());
    bool ok = fwrite(&h, sizeof(h), 1, w.f) == 1;
    w.pos = sizeof(h);
    std::vector<uint64_t> o(n + 1, 0);
    for (uint64_t i = 0; i < n; ++i) o[i + 1] = o[i] + len[i];
    ok = ok && w.put(o.data(), 8 * (n + 1)) && w.pad() && w.put(base, total) && w.pad();
    for (uint64_t i = 0; i <= n; ++i)
        o[i] = title_offsets ? title_offsets[i] - title_offsets[0] : 0;
    ok = ok && w.put(o.data(), 8 * (n + 1)) && w.pad();
    ok = ok && w.put(tbytes ? titles + title_offsets[0] : nullptr, tbytes) && w.pad();
    ok = ok && w.put(order.data(), 4 * n) && w.pad();
    h.checksum = w.hash.done();
    ok = ok && w.pos == h.file_bytes && fseek(w.f, 0, SEEK_SET) == 0 &&
         fwrite(&h, sizeof(h), 1, w.f) == 1;
    ok = (fclose(w.f) == 0) && ok;
    if (!ok) {
        unlink(tmp.c_str());
        return thread_fail(SW_ERR_INVALID, "write to %s failed", tmp.c_str());
    }
    if (rename(tmp.c_str(), path) != 0) {
        unlink(tmp.c_str());
        return thread_fail(SW_ERR_INVALID, "cannot rename %s to %s", tmp.c_str(), path);
    }
    return SW_OK;
}

// A mapped image whose header, section bounds, offsets and checksum are
// checked.
struct Mapped {
    const uint8_t* base = nullptr;
    size_t bytes = 0;
    const ImageHeader* h = nullptr;
    void release() {
        if (base) munmap((void*)base, bytes);
        base = nullptr;
    }
};

sw_status map_image(const char* path, bool verify_checksum, Mapped* m) {
    if (!path) return thread_fail(SW_ERR_INVALID, "null path");
    const int fd = open(path, O_RDONLY);
    if (fd < 0) return thread_fail(SW_ERR_INVALID, "cannot open %s", path);
    struct stat st;
    if (fstat(fd, &st) != 0 || st.st_size < (off_t)sizeof(ImageHeader)) {
        close(fd);
        return thread_fail(SW_ERR_FORMAT, "%s: too short for a DB image", path);
    }
    void* p = mmap(nullptr, (size_t)st.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
    close(fd);
    if (p == MAP_FAILED) return thread_fail(SW_ERR_INVALID, "cannot map %s", path);
    m->base = (const uint8_t*)p;
    m->bytes = (size_t)st.st_size;
    m->h = (const ImageHeader*)p;
    const ImageHeader& h = *m->h;
    auto bad = [&](const char* what) {
        m->release();
        return thread_fail(SW_ERR_FORMAT, "%s: %s", path, what);
    };
    if (memcmp(h.magic, kMagic, 8) != 0) return bad("not a DB image (magic)");
    if (h.version != kImageVersion) return bad("unsupported image version");
    if (h.header_bytes != sizeof(ImageHeader) || h.file_bytes != m->bytes)
        return bad("header does not match the file size");
    const uint64_t n = h.n_records;
    if (n >= (1ull << 31)) return bad("record count out of range");
    auto inside = [&](uint64_t off, uint64_t len) {
        return off % 64 == 0 && off >= sizeof(ImageHeader) && off <= h.file_bytes &&
               len <= h.file_bytes - off;
    };
    if (!inside(h.off_offsets, 8 * (n + 1)) || !inside(h.off_residues, h.n_residues) ||
        !inside(h.off_title_offsets, 8 * (n + 1)) || !inside(h.off_titles, h.titles_bytes) ||
        !inside(h.off_order, 4 * n))
        return bad("section outside the file");
    if (verify_checksum) {
        Hash64 hs;
        hs.add(m->base + sizeof(ImageHeader), m->bytes - sizeof(ImageHeader));
        if (hs.done() != h.checksum) return bad("checksum mismatch (file damaged)");
    }
    const uint64_t* off = (const uint64_t*)(m->base + h.off_offsets);
    const uint64_t* toff = (const uint64_t*)(m->base + h.off_title_offsets);
    if (off[0] != 0 || off[n] != h.n_residues || toff[0] != 0 || toff[n] != h.titles_bytes)
        return bad("offset tables inconsistent");
    for (uint64_t i = 0; i < n; ++i)
        if (off[i + 1] < off[i] || toff[i + 1] < toff[i]) return bad("offsets not monotone");
    return SW_OK;
}

// The FASTA letter table of the search path (sw_encode): 23 letters, '@' = 23,
// anything else 24; whitespace is skipped.
struct Alphabet {
    uint8_t code[256];
    bool skip[256];
    Alphabet() {
        static const char* alpha = "ABCDEFGHIKLMNPQRSTVWXYZ";
        memset(code, 24, sizeof(code));
        memset(skip, 0, sizeof(skip));
        for (int i = 0; alpha[i]; ++i) {
            code[(uint8_t)alpha[i]] = (uint8_t)i;
            code[(uint8_t)(alpha[i] - 'A' + 'a')] = (uint8_t)i;
        }
        code[(uint8_t)'@'] = 23;
        for (char c : {' ', '\t', '\r', '\n', '\v', '\f'}) skip[(uint8_t)c] = true;
    }
};

}  // namespace

namespace swb {

namespace {
thread_local std::string t_err;
}

const char* thread_error() { return t_err.c_str(); }

sw_status thread_fail(sw_status st, const char* fmt, ...) {
    char b[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(b, sizeof(b), fmt, ap);
    va_end(ap);
    t_err = b;
    return st;
}

void free_image(sw_ctx* ctx) {
    if (ctx->image) munmap((void*)ctx->image, ctx->image_bytes);
    ctx->image = nullptr;
    ctx->image_bytes = 0;
}

}  // namespace swb

extern "C" sw_status sw_db_write_image(const char* path, const uint8_t* residues,
                                       const uint64_t* offsets, uint64_t n_records,
                                       const char* titles, const uint64_t* title_offsets) {
    return write_image(path, residues, offsets, n_records, titles, title_offsets);
}

extern "C" sw_status sw_fasta_to_image(const char* fasta_path, const char* image_path,
                                       sw_image_info* info) {
    if (!fasta_path || !image_path) return thread_fail(SW_ERR_INVALID, "null path");
    FILE* f = fopen(fasta_path, "rb");
    if (!f) return thread_fail(SW_ERR_INVALID, "cannot open %s", fasta_path);
    static const Alphabet A;
    std::vector<uint8_t> res;
    std::vector<uint64_t> off{0};
    std::string titles;
    std::vector<uint64_t> toff{0};
    std::vector<char> buf(1 << 20);
    bool at_line_start = true, in_title = false, any = false;
    uint64_t line = 1;
    size_t got;
    while ((got = fread(buf.data(), 1, buf.size(), f)) > 0) {
        for (size_t i = 0; i < got; ++i) {
            const char c = buf[i];
            if (in_title) {
                if (c == '\n') {
                    in_title = false;
                    at_line_start = true;
                    ++line;
                } else if (c != '\r') {
                    titles.push_back(c);
                }
                continue;
            }
            if (c == '\n') {
                at_line_start = true;
                ++line;
                continue;
            }
            if (at_line_start && c == '>') {        // a new record: close the previous one
                if (any) {
                    off.push_back(res.size());
                    toff.push_back(titles.size());
                }
                any = true;
                in_title = true;
                at_line_start = false;
                continue;
            }
            at_line_start = false;
            if (A.skip[(uint8_t)c]) continue;
            if (!any) {
                fclose(f);
                return thread_fail(SW_ERR_FORMAT, "%s line %llu: sequence before the first '>' header",
                            fasta_path, (unsigned long long)line);
            }
            res.push_back(A.code[(uint8_t)c]);
        }
    }
    const bool read_error = ferror(f) != 0;
    fclose(f);
    if (read_error) return thread_fail(SW_ERR_INVALID, "read error in %s", fasta_path);
    if (any) {
        off.push_back(res.size());
        toff.push_back(titles.size());
    }
    const uint64_t n = off.size() - 1;
    sw_status st = write_image(image_path, res.data(), off.data(), n, titles.data(), toff.data());
    if (st != SW_OK) return st;
    if (info) return sw_image_get_info(image_path, 1, info);
    return SW_OK;
}

extern "C" sw_status sw_image_get_info(const char* path, int verify_checksum,
                                       sw_image_info* info) {
    if (!info) return thread_fail(SW_ERR_INVALID, "null argument");
    Mapped m;
    sw_status st = map_image(path, verify_checksum != 0, &m);
    if (st != SW_OK) return st;
    info->n_records = m.h->n_records;
    info->n_residues = m.h->n_residues;
    info->file_bytes = m.h->file_bytes;
    info->titles_bytes = m.h->titles_bytes;
    info->checksum = m.h->checksum;
    info->version = m.h->version;
    info->reserved = 0;
    m.release();
    return SW_OK;
}

extern "C" sw_status sw_image_open(const char* path, int verify_checksum, sw_image_view* view) {
    if (!view) return thread_fail(SW_ERR_INVALID, "null argument");
    memset(view, 0, sizeof(*view));
    Mapped m;
    sw_status st = map_image(path, verify_checksum != 0, &m);
    if (st != SW_OK) return st;
    const ImageHeader& h = *m.h;
    view->residues = m.base + h.off_residues;
    view->offsets = (const uint64_t*)(m.base + h.off_offsets);
    view->titles = (const char*)(m.base + h.off_titles);
    view->title_offsets = (const uint64_t*)(m.base + h.off_title_offsets);
    view->order = (const uint32_t*)(m.base + h.off_order);
    view->n_records = h.n_records;
    view->n_residues = h.n_residues;
    view->mapping = m.base;
    view->mapping_bytes = m.bytes;
    return SW_OK;
}

extern "C" void sw_image_close(sw_image_view* view) {
    if (!view || !view->mapping) return;
    munmap((void*)view->mapping, view->mapping_bytes);
    memset(view, 0, sizeof(*view));
}

extern "C" sw_status sw_db_load_image(sw_ctx* ctx, const char* path, int verify_checksum) {
    if (!ctx) return SW_ERR_INVALID;
    if (ctx->serve) return SW_ERR_BUSY;   // the serving loop owns the stream and the DB
    Mapped m;
    sw_status st = map_image(path, verify_checksum != 0, &m);
    if (st != SW_OK) {
        ctx->err = swb::thread_error();
        return st;
    }
    const ImageHeader& h = *m.h;
    st = swb::db_load(ctx, m.base + h.off_residues, (const uint64_t*)(m.base + h.off_offsets),
                      h.n_records, (const uint32_t*)(m.base + h.off_order));
    if (st != SW_OK) {
        m.release();
        return st;
    }
    ctx->image = m.base;          // kept mapped: the titles are read from it
    ctx->image_bytes = m.bytes;
    return SW_OK;
}

extern "C" sw_status sw_db_title(const sw_ctx* ctx, uint64_t record, const char** title,
                                 uint64_t* length) {
    if (!ctx || !title || !length) return SW_ERR_INVALID;
    if (!ctx->db_loaded || !ctx->image) return SW_ERR_STATE;
    const ImageHeader* h = (const ImageHeader*)ctx->image;
    if (record >= h->n_records) return SW_ERR_INVALID;
    const uint64_t* toff = (const uint64_t*)(ctx->image + h->off_title_offsets);
    *title = (const char*)(ctx->image + h->off_titles + toff[record]);
    *length = toff[record + 1] - toff[record];
    return SW_OK;
}
