// vxq.cpp — .vxq files straight into HBM tables.
//
// The file layout follows the reference's storage package:
//   "VXQ1" | row groups | footer body | CRC32(body) u32 | len(body) i64 | "VXQ1"
// (storage/writer.go:41-61, 423-472; storage/reader.go:295-408). A row group
// holds one section per column; a section is a run of blocks of at most 1,024
// rows, each [128-byte validity bitmap][rows × value width][CRC32] for fixed
// width types (storage/rowgroup.go:122-145; writer.go:205-372), or
// [u32 runs][runs × (u32 length, u8 value)][CRC32] for BOOL, where value 0xFF
// is a NULL run (storage/codec.go:253-336). A STRING section is followed by its
// row group's dictionary [u32 n][n × u32 offset][u32 bytes][bytes][CRC32]
// (storage/codec.go:82-99, 233-251); NULL rows carry code 0xFFFFFFFF.
// Integers are little-endian (internal/encoding/binary.go); the CRC is
// CRC-32/IEEE (internal/encoding/crc.go).
//
// The loader maps the file, checks the trailer, footer CRC and every block
// and dictionary CRC it reads (blocks of columns not selected are not read,
// as ColumnReader reads only the sections it opens), decodes the selected
// columns on all host cores, and hands them to the table upload with the
// file's row groups as the table's row groups and its per-row-group
// dictionaries remapped to one global dictionary per column.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "plan.h"

namespace vq {
Table* upload_table(const vexq_column_desc* cols, int32_t ncols, int64_t nrows, int32_t rg_rows, const int8_t* has_null);
}  // namespace vq

using namespace vq;

namespace {

constexpr char kMagic[4] = {'V', 'X', 'Q', '1'};
constexpr int kBlockRows = 1024;     // storage/format.go:8
constexpr int kBitmapBytes = 128;    // storage/format.go:12
constexpr int kTrailer = 16;         // storage/format.go:14
constexpr int kColMetaBytes = 57;    // reader.go:364: 6 × 8 + 1 + 2 × 4

[[noreturn]] void corrupt(const std::string& what) { fail(VEXQ_ECORRUPT, "storage: " + what); }

// ---- CRC-32/IEEE: reflected polynomial 0xEDB88320, initial and final value
// 0xFFFFFFFF. Eight bytes a step through eight 256-entry tables ("slicing by
// 8", Kounavis and Berry, 2005): table k advances a byte by k further bytes of
// zeros, so the eight lookups of one step are independent.
struct Crc32 {
    uint32_t t[8][256];
    Crc32() {
        for (uint32_t i = 0; i < 256; i++) {
            uint32_t c = i;
            for (int b = 0; b < 8; b++) c = (c & 1u) ? (c >> 1) ^ 0xEDB88320u : c >> 1;
            t[0][i] = c;
        }
        for (int k = 1; k < 8; k++)
            for (int i = 0; i < 256; i++) t[k][i] = (t[k - 1][i] >> 8) ^ t[0][t[k - 1][i] & 0xFFu];
    }
    uint32_t operator()(const uint8_t* p, size_t n) const {
        uint32_t c = 0xFFFFFFFFu;
        while (n >= 8) {
            uint32_t lo;
            std::memcpy(&lo, p, 4);  // little-endian host
            lo ^= c;
            c = t[7][lo & 0xFFu] ^ t[6][(lo >> 8) & 0xFFu] ^ t[5][(lo >> 16) & 0xFFu] ^ t[4][lo >> 24] ^ t[3][p[4]] ^
                t[2][p[5]] ^ t[1][p[6]] ^ t[0][p[7]];
            p += 8;
            n -= 8;
        }
        while (n--) c = (c >> 8) ^ t[0][(c ^ *p++) & 0xFFu];
        return c ^ 0xFFFFFFFFu;
    }
};
const Crc32& crc32() {
    static const Crc32 c;
    return c;
}

template <class T>
T rd(const uint8_t* p) {
    T v;
    std::memcpy(&v, p, sizeof v);
    return v;
}

// VerifyTrailing (internal/encoding/crc.go:27-40): the last four bytes are the
// little-endian CRC of the bytes before them.
bool verify_trailing(const uint8_t* p, size_t n) {
    if (n < 4) return false;
    return crc32()(p, n - 4) == rd<uint32_t>(p + n - 4);
}

int value_width(int type) {  // DataType.ValueSize (storage/format.go:46-57)
    switch (type) {
        case VEXQ_TYPE_INT64:
        case VEXQ_TYPE_FLOAT64: return 8;
        case VEXQ_TYPE_DATE:
        case VEXQ_TYPE_STRING: return 4;
        default: return 0;
    }
}

struct ColMeta {
    int64_t off = 0, len = 0, null_count = 0, sum = 0;
    uint64_t min = 0, max = 0;
    bool has_min_max = false;
    uint32_t dict_off = 0, dict_len = 0;
};
struct RowGroup {
    int64_t file_off = 0;
    uint32_t rows = 0;
    std::vector<ColMeta> cols;
};
struct Field {
    std::string name;
    int type = 0, encoding = 0;
    bool nullable = false;
};

// A mapped .vxq file with its parsed footer (Reader.readFooter / parseFooter,
// storage/reader.go:295-408).
struct VxqFile {
    int fd = -1;
    const uint8_t* base = nullptr;
    size_t size = 0;
    std::vector<Field> fields;
    std::vector<RowGroup> rgs;

    explicit VxqFile(const char* path) {
        if (!path) fail(VEXQ_EINVAL, "null path");
        fd = ::open(path, O_RDONLY | O_CLOEXEC);
        if (fd < 0) fail(VEXQ_EINVAL, std::string("storage: open: ") + path + ": " + std::strerror(errno));
        struct stat st;
        if (fstat(fd, &st) != 0) fail(VEXQ_EINVAL, std::string("storage: open: stat: ") + std::strerror(errno));
        size = (size_t)st.st_size;
        if (size > 0) {
            void* m = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
            if (m == MAP_FAILED) fail(VEXQ_EINVAL, std::string("storage: open: mmap: ") + std::strerror(errno));
            base = (const uint8_t*)m;
            madvise(m, size, MADV_WILLNEED);
        }
        parse();
    }
    ~VxqFile() {
        if (base) munmap((void*)base, size);
        if (fd >= 0) ::close(fd);
    }
    VxqFile(const VxqFile&) = delete;
    VxqFile& operator=(const VxqFile&) = delete;

    void parse() {
        if (size < (size_t)kTrailer + sizeof kMagic) corrupt("open: footer: bad magic bytes");
        const uint8_t* tr = base + size - kTrailer;
        if (std::memcmp(tr + 12, kMagic, 4) != 0) corrupt("open: footer: bad magic bytes");
        const uint32_t fcrc = rd<uint32_t>(tr);
        const int64_t flen = rd<int64_t>(tr + 4);
        if (flen < 0 || flen > (int64_t)size - kTrailer - (int64_t)sizeof kMagic) corrupt("open: footer: corrupt footer");
        const uint8_t* b = base + size - kTrailer - flen;
        const uint8_t* end = b + flen;
        if (crc32()(b, (size_t)flen) != fcrc) corrupt("open: footer: checksum mismatch");
        auto need = [&](size_t n, const char* what) {
            if ((size_t)(end - b) < n) corrupt(std::string("open: footer: parse ") + what + ": corrupt footer");
        };
        need(4, "schema");
        const uint32_t ncols = rd<uint32_t>(b);
        b += 4;
        if (ncols > (size_t)(end - b) / 5) corrupt("open: footer: parse schema: corrupt footer");  // 5 bytes a field at least
        fields.resize(ncols);
        for (uint32_t i = 0; i < ncols; i++) {
            need(2, "schema");
            const uint16_t nl = rd<uint16_t>(b);
            b += 2;
            need((size_t)nl + 3, "schema");
            fields[i].name.assign((const char*)b, nl);
            b += nl;
            fields[i].type = b[0];
            fields[i].encoding = b[1];
            fields[i].nullable = (b[2] & 1) != 0;
            b += 3;
        }
        need(4, "row groups");
        const uint32_t nrg = rd<uint32_t>(b);
        b += 4;
        if (nrg > (size_t)(end - b) / (12 + (size_t)ncols * kColMetaBytes))
            corrupt("open: footer: parse row groups: corrupt footer");
        rgs.resize(nrg);
        for (uint32_t r = 0; r < nrg; r++) {
            need(12, "row group");
            rgs[r].file_off = rd<int64_t>(b);
            rgs[r].rows = rd<uint32_t>(b + 8);
            b += 12;
            rgs[r].cols.resize(ncols);
            for (uint32_t c = 0; c < ncols; c++) {
                need(kColMetaBytes, "column meta");
                ColMeta& m = rgs[r].cols[c];
                m.off = rd<int64_t>(b);
                m.len = rd<int64_t>(b + 8);
                m.null_count = rd<int64_t>(b + 16);
                m.sum = rd<int64_t>(b + 24);
                m.min = rd<uint64_t>(b + 32);
                m.max = rd<uint64_t>(b + 40);
                m.has_min_max = b[48] != 0;
                m.dict_off = rd<uint32_t>(b + 49);
                m.dict_len = rd<uint32_t>(b + 53);
                b += kColMetaBytes;
            }
        }
    }
};

// Decoded host columns in the table upload's layout.
struct HostCol {
    int type = 0;
    std::string name;
    std::vector<uint8_t> values;
    std::vector<uint8_t> validity;   // LSB-first, 1 = valid
    std::atomic<bool> any_null{false};
    // STRING: per-row-group dictionaries, flattened
    std::vector<uint32_t> rg_first, str_off;
    std::vector<char> bytes;
    std::vector<std::vector<std::string>> rg_dict;  // filled per row group, flattened after
};

// Sets one validity bit. Row groups whose size is not a multiple of 8 share
// a byte with their neighbour, which another thread may be writing.
inline void set_bit(uint8_t* dst, int64_t r) {
    __atomic_fetch_or(dst + (r >> 3), (uint8_t)(1u << (r & 7)), __ATOMIC_RELAXED);
}

// Copies `rows` validity bits from a block bitmap to row `dst_row` of the
// table bitmap: whole bytes when the row is a multiple of 8.
void put_bits(uint8_t* dst, int64_t dst_row, const uint8_t* src, int rows) {
    int i = 0;
    if ((dst_row & 7) == 0) {
        const int full = rows >> 3;
        std::memcpy(dst + (dst_row >> 3), src, (size_t)full);
        i = full * 8;
    }
    for (; i < rows; i++)
        if ((src[i >> 3] >> (i & 7)) & 1) set_bit(dst, dst_row + i);
}

bool all_valid(const uint8_t* bm, int rows) {
    for (int i = 0; i < (rows >> 3); i++)
        if (bm[i] != 0xFF) return false;
    for (int i = rows & ~7; i < rows; i++)
        if (!((bm[i >> 3] >> (i & 7)) & 1)) return false;
    return true;
}

// One (column, row group) section: every block checked and decoded into the
// column at the row group's first row (ColumnReader.NextBlock,
// storage/rowgroup.go:101-171; DecodeRLEBool, storage/codec.go:292-336;
// UnmarshalDictionary, storage/codec.go:233-251).
// host_blocks = false checks the section's bounds and, for STRING, parses the
// dictionary, leaving the blocks to the device.
void decode_section(const VxqFile& f, int fi, int rg, int64_t row0, HostCol& hc, bool host_blocks = true) {
    const Field& fd = f.fields[fi];
    const ColMeta& m = f.rgs[rg].cols[fi];
    const uint32_t rows = f.rgs[rg].rows;
    auto where = [&](int64_t off) {
        return "rg=" + std::to_string(rg) + " col=" + fd.name + " off=" + std::to_string(off);
    };
    if (m.off < 0 || m.len < 0 || m.off > (int64_t)f.size || m.len > (int64_t)f.size - m.off || (int64_t)m.dict_len > m.len)
        corrupt("read block " + where(m.off) + ": unexpected EOF");
    // STRING: the row group's dictionary first, so codes can be checked
    uint32_t dict_n = 0;
    if (fd.type == VEXQ_TYPE_STRING) {
        std::vector<std::string>& dict = hc.rg_dict[(size_t)rg];
        const int64_t doff = m.off + (int64_t)m.dict_off;
        if (m.dict_len == 0 || (int64_t)m.dict_off > m.len || (int64_t)m.dict_len > m.len - (int64_t)m.dict_off)
            corrupt("read dictionary " + where(doff) + ": unexpected EOF");
        const uint8_t* p = f.base + doff;
        const size_t n = m.dict_len;
        if (!verify_trailing(p, n)) corrupt("unmarshal dict " + where(doff) + ": checksum mismatch");
        const size_t pay = n - 4;
        if (pay < 4) corrupt("unmarshal dict " + where(doff) + ": corrupt footer");
        const uint32_t ne = rd<uint32_t>(p);
        if ((pay - 4) / 4 < (size_t)ne + 1) corrupt("unmarshal dict " + where(doff) + ": corrupt footer");
        const uint8_t* offs = p + 4;
        const uint32_t total = rd<uint32_t>(p + 4 + (size_t)ne * 4);
        const uint8_t* data = p + 8 + (size_t)ne * 4;
        if ((size_t)total > pay - 8 - (size_t)ne * 4) corrupt("unmarshal dict " + where(doff) + ": corrupt footer");
        dict.resize(ne);
        for (uint32_t e = 0; e < ne; e++) {
            // Dictionary.Get (storage/codec.go:170-205): entry e ends where
            // entry e+1 starts, the last one at the end of the data
            const uint32_t a = rd<uint32_t>(offs + (size_t)e * 4);
            const uint32_t b = e + 1 < ne ? rd<uint32_t>(offs + (size_t)(e + 1) * 4) : total;
            if (a > b || b > total) corrupt("unmarshal dict " + where(doff) + ": entry " + std::to_string(e) + " out of range");
            dict[e].assign((const char*)data + a, b - a);
        }
        dict_n = ne;
    }
    const int64_t end = m.off + m.len - (int64_t)m.dict_len;
    int64_t pos = m.off;
    const int w = value_width(fd.type);
    if (!host_blocks) {  // fixed-size blocks: the section must hold all of them
        const int64_t full = rows / kBlockRows, tail = rows % kBlockRows;
        const int64_t need = full * (kBitmapBytes + (int64_t)kBlockRows * w + 4) + (tail ? kBitmapBytes + tail * w + 4 : 0);
        if (need > end - m.off) corrupt("read block " + where(m.off) + ": unexpected EOF");
        return;
    }
    for (uint32_t done = 0; done < rows;) {
        const int n = (int)std::min<uint32_t>(kBlockRows, rows - done);
        const int64_t r = row0 + done;
        if (fd.type == VEXQ_TYPE_BOOL) {
            if (pos + 4 > end) corrupt("read bool block header " + where(pos) + ": unexpected EOF");
            const uint32_t runs = rd<uint32_t>(f.base + pos);
            if (runs > (uint32_t)n) corrupt("read bool block " + where(pos) + ": corrupt footer");
            const int64_t bytes = 4 + (int64_t)runs * 5 + 4;
            if (pos + bytes > end) corrupt("read bool block " + where(pos) + ": unexpected EOF");
            const uint8_t* p = f.base + pos;
            if (!verify_trailing(p, (size_t)bytes)) corrupt("decode rle bool " + where(pos) + ": checksum mismatch");
            int64_t k = 0;
            for (uint32_t u = 0; u < runs; u++) {
                const uint32_t len = rd<uint32_t>(p + 4 + (size_t)u * 5);
                const uint8_t v = p[4 + (size_t)u * 5 + 4];
                if (len > (uint32_t)(n - k)) corrupt("decode rle bool " + where(pos) + ": runs exceed the block's rows");
                for (uint32_t j = 0; j < len; j++, k++) {
                    const int64_t row = r + k;
                    if (v == 0xFF) {
                        hc.any_null = true;
                    } else {
                        hc.values[(size_t)row] = v == 1 ? 1 : 0;
                        set_bit(hc.validity.data(), row);
                    }
                }
            }
            if (k != n) corrupt("decode rle bool " + where(pos) + ": runs cover " + std::to_string(k) + " of " + std::to_string(n) + " rows");
            pos += bytes;
        } else {
            const int64_t bytes = kBitmapBytes + (int64_t)n * w + 4;
            if (pos + bytes > end) corrupt("read block " + where(pos) + ": unexpected EOF");
            const uint8_t* p = f.base + pos;
            if (!verify_trailing(p, (size_t)bytes)) corrupt("crc block " + where(pos) + ": checksum mismatch");
            std::memcpy(hc.values.data() + (size_t)r * w, p + kBitmapBytes, (size_t)n * w);
            if (!all_valid(p, n)) hc.any_null = true;
            put_bits(hc.validity.data(), r, p, n);
            if (fd.type == VEXQ_TYPE_STRING)
                for (int i = 0; i < n; i++)
                    if (((p[i >> 3] >> (i & 7)) & 1) && rd<uint32_t>(p + kBitmapBytes + (size_t)i * 4) >= dict_n)
                        corrupt("crc block " + where(pos) + ": dictionary code out of range");
            pos += bytes;
        }
        done += (uint32_t)n;
    }
}

// Runs fn(task) over [0, n) on up to `threads` host threads.
template <class F>
void parallel_for(size_t n, F&& fn) {
    const size_t threads = std::max<size_t>(1, std::min<size_t>(n, std::max(1u, std::thread::hardware_concurrency())));
    std::atomic<size_t> next{0};
    std::vector<std::string> errs(threads);
    std::vector<int32_t> codes(threads, 0);
    auto work = [&](size_t id) {
        try {
            for (size_t i = next++; i < n; i = next++) fn(i);
        } catch (const Status& s) {
            codes[id] = s.code;
            errs[id] = s.what();
            next = n;
        } catch (const std::exception& e) {
            codes[id] = VEXQ_EINVAL;
            errs[id] = e.what();
            next = n;
        }
    };
    std::vector<std::thread> th;
    for (size_t t = 1; t < threads; t++) th.emplace_back(work, t);
    work(0);
    for (auto& t : th) t.join();
    for (size_t t = 0; t < threads; t++)
        if (codes[t]) fail(codes[t], errs[t]);
}

struct Loaded {
    std::vector<std::unique_ptr<HostCol>> cols;
    std::vector<int> sel;        // file column of each loaded column
    std::vector<int64_t> row0;   // first table row of each row group
    int64_t nrows = 0;
    int32_t rg_rows = VEXQ_ROW_GROUP_ROWS;
    int64_t bytes_checked = 0;
};

// Selected columns decoded from the file. The table's row groups are the
// file's: every row group but the last must hold the same number of rows.
// device = true leaves the fixed-width blocks to k_vxq_blocks (their columns
// get no host arrays); BOOL sections and dictionaries are decoded here.
void load(const VxqFile& f, const char* const* names, int32_t nnames, Loaded& L, bool device = false) {
    std::vector<int> sel;
    if (names) {
        if (nnames < 0) fail(VEXQ_EINVAL, "negative column count");
        for (int32_t i = 0; i < nnames; i++) {
            int idx = -1;
            for (size_t c = 0; c < f.fields.size(); c++)
                if (names[i] && f.fields[c].name == names[i]) { idx = (int)c; break; }
            if (idx < 0) fail(VEXQ_EINVAL, std::string("storage: no column named ") + (names[i] ? names[i] : "(null)"));
            sel.push_back(idx);
        }
    } else {
        for (size_t c = 0; c < f.fields.size(); c++) sel.push_back((int)c);
    }
    for (int c : sel) {
        const int t = f.fields[c].type;
        if (t != VEXQ_TYPE_BOOL && !value_width(t))
            corrupt("column " + f.fields[c].name + ": unknown type " + std::to_string(t));
    }
    const size_t nrg = f.rgs.size();
    std::vector<int64_t> row0(nrg + 1, 0);
    for (size_t r = 0; r < nrg; r++) row0[r + 1] = row0[r] + f.rgs[r].rows;
    L.nrows = row0[nrg];
    if (nrg > 0) {
        L.rg_rows = (int32_t)f.rgs[0].rows;
        if (f.rgs[0].rows == 0) corrupt("row group 0 has no rows");
        for (size_t r = 0; r < nrg; r++) {
            const bool last = r + 1 == nrg;
            if ((!last && f.rgs[r].rows != f.rgs[0].rows) || (last && f.rgs[r].rows > f.rgs[0].rows) || f.rgs[r].rows == 0)
                fail(VEXQ_ENOTSUP, "row group " + std::to_string(r) + " holds " + std::to_string(f.rgs[r].rows) +
                                       " rows: the table's row groups are all " + std::to_string(f.rgs[0].rows) +
                                       " rows but the last");
        }
    }
    for (int c : sel) {
        auto hc = std::make_unique<HostCol>();
        hc->type = f.fields[c].type;
        hc->name = f.fields[c].name;
        const int w = hc->type == VEXQ_TYPE_BOOL ? 1 : value_width(hc->type);
        if (!device || hc->type == VEXQ_TYPE_BOOL) {
            hc->values.assign((size_t)std::max<int64_t>(L.nrows, 1) * w, 0);
            hc->validity.assign((size_t)(L.nrows + 7) / 8 + 1, 0);
        }
        if (hc->type == VEXQ_TYPE_STRING) hc->rg_dict.resize(nrg);
        L.cols.push_back(std::move(hc));
    }
    const size_t ntask = sel.size() * nrg;
    parallel_for(ntask, [&](size_t task) {
        const size_t k = task / std::max<size_t>(nrg, 1), r = task % std::max<size_t>(nrg, 1);
        decode_section(f, sel[k], (int)r, row0[r], *L.cols[k], !device || L.cols[k]->type == VEXQ_TYPE_BOOL);
    });
    L.sel = sel;
    L.row0 = row0;
    for (size_t k = 0; k < sel.size(); k++)
        for (size_t r = 0; r < nrg; r++) L.bytes_checked += f.rgs[r].cols[sel[k]].len;
    // STRING dictionaries flattened into the upload's per-row-group form
    for (auto& hc : L.cols) {
        if (hc->type != VEXQ_TYPE_STRING) continue;
        hc->rg_first.assign(1, 0);
        hc->str_off.assign(1, 0);
        for (size_t r = 0; r < nrg; r++) {
            for (const std::string& s : hc->rg_dict[r]) {
                hc->bytes.insert(hc->bytes.end(), s.begin(), s.end());
                hc->str_off.push_back((uint32_t)hc->bytes.size());
            }
            hc->rg_first.push_back((uint32_t)(hc->str_off.size() - 1));
        }
        if (hc->bytes.empty()) hc->bytes.push_back(0);
        hc->rg_dict.clear();
    }
}

// ---- device decode -----------------------------------------------------------------
// The file's data region is copied to HBM once; one warp then checks and
// scatters each fixed-width block: the CRC-32 of [bitmap][values] (each lane
// folds a contiguous segment with a byte table in shared memory, and the
// segments are joined by the CRC's linearity: crc(A‖B) = crc(A)·x^(8|B|) ⊕
// crc(B) over GF(2) modulo the polynomial, with the 0xFFFFFFFF start value
// entering as 0xFFFFFFFF·x^(8|M|)), the values into the column at the block's
// first row, the validity bits, and for STRING codes the dictionary bound.

struct VxqBlock {
    long long src;       // file offset of the block
    long long dst_row;   // table row of its first row
    int rows;
    int col;             // loaded-column slot
    unsigned dict_n;     // STRING: entries of the row group's dictionary; ~0u otherwise
    int pad;
};
struct VxqDevCol {
    unsigned char* values;
    unsigned* validity;  // zeroed, 4-byte words
    int width;
    int pad;
};
struct VxqPow {
    unsigned x[24];      // x^(8·2^k) mod P, reflected
};

// a·b modulo the CRC polynomial, both in the reflected order (bit 31 = x^0).
__host__ __device__ inline unsigned vq_gf_mul(unsigned a, unsigned b) {
    unsigned p = 0;
    for (int i = 0; i < 32; i++) {
        if (a & (0x80000000u >> i)) p ^= b;
        b = (b & 1u) ? (b >> 1) ^ 0xEDB88320u : b >> 1;
    }
    return p;
}
// x^(8n) modulo the polynomial.
__device__ inline unsigned vq_x8n(unsigned n, const VxqPow& pw) {
    unsigned r = 0x80000000u;
    for (int k = 0; n; k++, n >>= 1)
        if (n & 1u) r = vq_gf_mul(r, pw.x[k]);
    return r;
}

__global__ void __launch_bounds__(256) k_vxq_blocks(const unsigned char* __restrict__ raw, const VxqBlock* __restrict__ blk,
                                                    long long nblk, const VxqDevCol* __restrict__ cols, VxqPow pw,
                                                    unsigned long long* bad, int* has_null) {
    __shared__ unsigned tab[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        unsigned c = (unsigned)i;
        for (int b = 0; b < 8; b++) c = (c & 1u) ? (c >> 1) ^ 0xEDB88320u : c >> 1;
        tab[i] = c;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long b = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < nblk; b += nw) {
        const VxqBlock d = blk[b];
        const VxqDevCol c = cols[d.col];
        const int w = c.width;
        const int len = kBitmapBytes + d.rows * w;
        const unsigned char* p = raw + d.src;
        const int seg = ((len + 31) / 32 + 3) & ~3;
        const int a = min(lane * seg, len), e = min(a + seg, len);
        unsigned r = 0;
        for (int i = a; i < e; i++) r = (r >> 8) ^ tab[(r ^ __ldg(p + i)) & 0xFFu];
        unsigned part = vq_gf_mul(r, vq_x8n((unsigned)(len - e), pw));
        if (lane == 0) part ^= vq_gf_mul(0xFFFFFFFFu, vq_x8n((unsigned)len, pw));
        for (int o = 16; o > 0; o >>= 1) part ^= __shfl_xor_sync(0xffffffffu, part, o);
        const unsigned stored = (unsigned)p[len] | ((unsigned)p[len + 1] << 8) | ((unsigned)p[len + 2] << 16) |
                                ((unsigned)p[len + 3] << 24);
        if ((part ^ 0xFFFFFFFFu) != stored) {
            if (lane == 0) atomicMin(bad, (unsigned long long)b);
            continue;
        }
        // values
        const unsigned char* src = p + kBitmapBytes;
        unsigned char* dst = c.values + d.dst_row * w;
        const int nb = d.rows * w;
        if ((((unsigned long long)src) & 3ull) == 0)
            for (int i = lane; i < nb / 4; i += 32) reinterpret_cast<unsigned*>(dst)[i] = __ldg(reinterpret_cast<const unsigned*>(src) + i);
        else
            for (int i = lane; i < nb; i += 32) dst[i] = __ldg(src + i);
        // validity: whole bytes the block owns as plain stores, the rest as
        // bit ORs into zeroed words (a neighbour may share the byte)
        bool null_seen = false;
        unsigned char* vb = reinterpret_cast<unsigned char*>(c.validity);
        const int own = (d.dst_row & 7) == 0 ? d.rows / 8 : 0;
        for (int i = lane; i < own; i += 32) {
            const unsigned char v = p[i];
            vb[(d.dst_row >> 3) + i] = v;
            null_seen |= v != 0xFFu;
        }
        for (int i = own * 8 + lane; i < d.rows; i += 32) {
            const bool v = (p[i >> 3] >> (i & 7)) & 1;
            null_seen |= !v;
            if (v) {
                const long long row = d.dst_row + i;
                atomicOr(c.validity + (row >> 5), 1u << (row & 31));
            }
        }
        if (__any_sync(0xffffffffu, null_seen) && lane == 0) atomicOr(has_null + d.col, 1);
        // dictionary codes of valid rows within the row group's dictionary
        if (d.dict_n != ~0u) {
            bool out = false;
            for (int i = lane; i < d.rows; i += 32) {
                if (!((p[i >> 3] >> (i & 7)) & 1)) continue;
                const unsigned char* q = src + (size_t)i * 4;
                const unsigned code = (unsigned)q[0] | ((unsigned)q[1] << 8) | ((unsigned)q[2] << 16) | ((unsigned)q[3] << 24);
                out |= code >= d.dict_n;
            }
            if (__any_sync(0xffffffffu, out) && lane == 0) atomicMin(bad + 1, (unsigned long long)b);
        }
    }
}

// The table from a mapped file: BOOL columns and dictionaries decoded on the
// host, every fixed-width block checked and scattered on the device.
Table* load_device(const VxqFile& f, const char* const* names, int32_t nnames) {
    Loaded L;
    load(f, names, nnames, L, true);
    const size_t nrg = f.rgs.size(), ncol = L.cols.size();
    // the data region: everything before the footer (the device copy holds
    // only this, so every block must lie inside it)
    const int64_t flen = rd<int64_t>(f.base + f.size - kTrailer + 4);
    const int64_t data_end = (int64_t)f.size - kTrailer - flen;
    std::vector<VxqBlock> blocks;
    std::vector<int> dev_slot(ncol, -1);
    std::vector<int> slot_col;
    for (size_t k = 0; k < ncol; k++) {
        const HostCol& hc = *L.cols[k];
        if (hc.type == VEXQ_TYPE_BOOL) continue;
        dev_slot[k] = (int)slot_col.size();
        slot_col.push_back((int)k);
        const int w = value_width(hc.type);
        for (size_t r = 0; r < nrg; r++) {
            const ColMeta& m = f.rgs[r].cols[L.sel[k]];
            const unsigned dict_n = hc.type == VEXQ_TYPE_STRING ? hc.rg_first[r + 1] - hc.rg_first[r] : ~0u;
            int64_t pos = m.off;
            for (uint32_t done = 0; done < f.rgs[r].rows;) {
                const int n = (int)std::min<uint32_t>(kBlockRows, f.rgs[r].rows - done);
                if (pos < 0 || pos + kBitmapBytes + (int64_t)n * w + 4 > data_end)
                    corrupt("read block rg=" + std::to_string(r) + " col=" + hc.name + " off=" + std::to_string(pos) +
                            ": outside the data region");
                blocks.push_back(VxqBlock{pos, L.row0[r] + done, n, dev_slot[k], dict_n, 0});
                pos += kBitmapBytes + (int64_t)n * w + 4;
                done += (uint32_t)n;
            }
        }
    }
    // device columns: values and zeroed validity words
    std::vector<DevBuf> vals(slot_col.size()), valid(slot_col.size());
    std::vector<VxqDevCol> dc(slot_col.size());
    const int64_t nrows = L.nrows;
    for (size_t j = 0; j < slot_col.size(); j++) {
        const int w = value_width(L.cols[slot_col[j]]->type);
        vals[j].alloc((size_t)std::max<int64_t>(nrows, 1) * w);
        valid[j].alloc(((size_t)(nrows + 31) / 32 + 1) * 4);
        VQ_CUDA(cudaMemset(valid[j].p, 0, valid[j].n));
        dc[j] = VxqDevCol{vals[j].as<unsigned char>(), valid[j].as<unsigned>(), w, 0};
    }
    std::vector<int> has_null(slot_col.size() + 1, 0);
    if (!blocks.empty()) {
        DevBuf raw(std::max<size_t>((size_t)data_end, 4));
        VQ_CUDA(cudaMemcpy(raw.p, f.base, (size_t)data_end, cudaMemcpyHostToDevice));
        DevBuf d_blk(blocks.size() * sizeof(VxqBlock)), d_col(std::max<size_t>(dc.size(), 1) * sizeof(VxqDevCol));
        DevBuf d_flags(16 + has_null.size() * 4);
        VQ_CUDA(cudaMemcpy(d_blk.p, blocks.data(), d_blk.n, cudaMemcpyHostToDevice));
        VQ_CUDA(cudaMemcpy(d_col.p, dc.data(), dc.size() * sizeof(VxqDevCol), cudaMemcpyHostToDevice));
        VQ_CUDA(cudaMemset(d_flags.p, 0xFF, 16));
        VQ_CUDA(cudaMemset((char*)d_flags.p + 16, 0, has_null.size() * 4));
        VxqPow pw;
        pw.x[0] = 0x00800000u;  // x^8
        for (int k = 1; k < 24; k++) pw.x[k] = vq_gf_mul(pw.x[k - 1], pw.x[k - 1]);
        const long long nb = (long long)blocks.size();
        const int grid = (int)std::min<long long>((nb + 7) / 8, (long long)sm_count() * 8);
        k_vxq_blocks<<<grid, 256>>>(raw.as<unsigned char>(), d_blk.as<VxqBlock>(), nb, d_col.as<VxqDevCol>(), pw,
                                    d_flags.as<unsigned long long>(), (int*)((char*)d_flags.p + 16));
        VQ_CUDA(cudaGetLastError());
        unsigned long long bad[2];
        VQ_CUDA(cudaMemcpy(bad, d_flags.p, 16, cudaMemcpyDeviceToHost));
        VQ_CUDA(cudaMemcpy(has_null.data(), (char*)d_flags.p + 16, has_null.size() * 4, cudaMemcpyDeviceToHost));
        auto where = [&](unsigned long long i) {
            const VxqBlock& b = blocks[(size_t)i];
            const int k = slot_col[(size_t)b.col];
            int rg = 0;
            while (rg + 1 < (int)nrg && L.row0[rg + 1] <= b.dst_row) rg++;
            return "rg=" + std::to_string(rg) + " col=" + L.cols[k]->name + " off=" + std::to_string(b.src);
        };
        if (bad[0] != ~0ull) corrupt("crc block " + where(bad[0]) + ": checksum mismatch");
        if (bad[1] != ~0ull) corrupt("crc block " + where(bad[1]) + ": dictionary code out of range");
    }
    std::vector<vexq_column_desc> d(ncol);
    std::vector<int8_t> nulls(ncol, 0);
    for (size_t k = 0; k < ncol; k++) {
        HostCol& hc = *L.cols[k];
        d[k] = vexq_column_desc{};
        d[k].name = hc.name.c_str();
        d[k].type = hc.type;
        if (dev_slot[k] >= 0) {
            const int j = dev_slot[k];
            nulls[k] = has_null[(size_t)j] ? 1 : 0;
            d[k].values = vals[(size_t)j].p;
            d[k].validity = nulls[k] ? (const uint8_t*)valid[(size_t)j].p : nullptr;
        } else {
            nulls[k] = hc.any_null ? 1 : 0;
            d[k].values = hc.values.data();
            d[k].validity = nulls[k] ? hc.validity.data() : nullptr;
        }
        if (hc.type == VEXQ_TYPE_STRING) {
            d[k].dict_rg_first = hc.rg_first.data();
            d[k].dict_str_off = hc.str_off.data();
            d[k].dict_bytes = hc.bytes.data();
        }
    }
    return upload_table(d.data(), (int32_t)d.size(), L.nrows, L.rg_rows, nulls.data());
}

}  // namespace

extern "C" {

int32_t vexq_vxq_verify(const char* path, vexq_vxq_summary* out) {
    try {
        set_error("");
        if (!out) fail(VEXQ_EINVAL, "null output");
        VxqFile f(path);
        Loaded L;
        load(f, nullptr, 0, L);
        std::memset(out, 0, sizeof *out);
        out->nrows = L.nrows;
        out->ncols = (int32_t)f.fields.size();
        out->n_rg = (int32_t)f.rgs.size();
        out->rg_rows = L.rg_rows;
        out->bytes_checked = L.bytes_checked;
        for (auto& hc : L.cols) out->null_columns += hc->any_null ? 1 : 0;
        return VEXQ_OK;
    } catch (const Status& s) {
        set_error(s.what());
        return s.code;
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return VEXQ_ENOMEM;
    } catch (const std::exception& e) {
        set_error(e.what());
        return VEXQ_EINVAL;
    }
}

int32_t vexq_table_load_vxq(const char* path, const char* const* columns, int32_t ncolumns, vexq_table_t* out) {
    try {
        set_error("");
        if (!out) fail(VEXQ_EINVAL, "null output handle");
        VxqFile f(path);
        Table* t = load_device(f, columns, ncolumns);
        *out = new vexq_table_s{t};
        return VEXQ_OK;
    } catch (const Status& s) {
        set_error(s.what());
        return s.code;
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return VEXQ_ENOMEM;
    } catch (const std::exception& e) {
        set_error(e.what());
        return VEXQ_EINVAL;
    }
}

}  // extern "C"
