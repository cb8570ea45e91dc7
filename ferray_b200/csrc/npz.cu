// npz.cu -- .npz archives (zip files of .npy members) into device buffers.
//
// The reader side of ferray-io/src/npz/mod.rs:88-200 (`NpzFile`): member
// names are the archive's file names with a trailing ".npy" removed
// (mod.rs:130-133); `get(name)` accepts only a listed name and reads the
// member "<name>.npy" (mod.rs:150-167), so a member stored without the
// suffix is listed but cannot be fetched, as in the reference.  The zip
// layer follows the published PKWARE APPNOTE (the reference uses the `zip`
// crate 8.6.0 with `flate2` 1.1.9): the end-of-central-directory record
// (with the ZIP64 locator and record when the archive needs them), central
// directory headers, ZIP64 extra fields (NumPy writes members with
// force_zip64), local headers; methods 0 (stored) and 8 (deflate, inflated
// on the host by zlib) are read, and every member's CRC-32 is checked, as
// the zip crate does when a member is read to its end.  Stored members are
// uploaded straight from the caller's bytes.
#include <cuda_runtime.h>
#include <zlib.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "runtime.h"

namespace fgrt {

namespace {

uint16_t rd16(const unsigned char* p) { return static_cast<uint16_t>(p[0] | (p[1] << 8)); }
uint32_t rd32(const unsigned char* p) {
    return static_cast<uint32_t>(p[0]) | (static_cast<uint32_t>(p[1]) << 8) | (static_cast<uint32_t>(p[2]) << 16) |
           (static_cast<uint32_t>(p[3]) << 24);
}
uint64_t rd64(const unsigned char* p) { return static_cast<uint64_t>(rd32(p)) | (static_cast<uint64_t>(rd32(p + 4)) << 32); }

struct Member {
    std::string name;  // file name in the archive
    uint16_t method;
    uint32_t crc;
    uint64_t csize, usize, local;  // compressed / uncompressed size, local header offset
};

// Central directory of a zip archive held in memory.
fg_status read_directory(const unsigned char* b, size_t len, std::vector<Member>& out) {
    out.clear();
    if (len < 22) return set_error(FG_ERR_INVALID, "npz: not a zip archive (too short)");
    // End of central directory: 22 bytes + a comment of up to 65535 bytes.
    size_t eocd = std::string::npos;
    const size_t lo = len >= 22 + 65535 ? len - 22 - 65535 : 0;
    for (size_t p = len - 22 + 1; p-- > lo;) {
        if (rd32(b + p) == 0x06054b50u && p + 22 + rd16(b + p + 20) == len) {
            eocd = p;
            break;
        }
    }
    if (eocd == std::string::npos) return set_error(FG_ERR_INVALID, "npz: end of central directory not found");
    uint64_t entries = rd16(b + eocd + 10), cd_size = rd32(b + eocd + 12), cd_off = rd32(b + eocd + 16);
    if (entries == 0xFFFF || cd_size == 0xFFFFFFFFu || cd_off == 0xFFFFFFFFu) {
        // ZIP64: locator (20 bytes) just before the end record, then the record
        if (eocd < 20 || rd32(b + eocd - 20) != 0x07064b50u)
            return set_error(FG_ERR_INVALID, "npz: ZIP64 locator missing");
        const uint64_t rec = rd64(b + eocd - 20 + 8);
        if (rec > len || len - rec < 56 || rd32(b + rec) != 0x06064b50u)
            return set_error(FG_ERR_INVALID, "npz: bad ZIP64 end record");
        entries = rd64(b + rec + 32);
        cd_size = rd64(b + rec + 40);
        cd_off = rd64(b + rec + 48);
    }
    if (cd_off > len || cd_size > len - cd_off) return set_error(FG_ERR_INVALID, "npz: central directory out of range");
    if (entries > cd_size / 46) return set_error(FG_ERR_INVALID, "npz: entry count exceeds the central directory");
    size_t p = static_cast<size_t>(cd_off);
    const size_t end = static_cast<size_t>(cd_off + cd_size);
    for (uint64_t i = 0; i < entries; ++i) {
        if (end - p < 46 || rd32(b + p) != 0x02014b50u) return set_error(FG_ERR_INVALID, "npz: bad central directory header");
        Member m;
        const uint16_t flags = rd16(b + p + 8);
        m.method = rd16(b + p + 10);
        m.crc = rd32(b + p + 16);
        m.csize = rd32(b + p + 20);
        m.usize = rd32(b + p + 24);
        const size_t nlen = rd16(b + p + 28), elen = rd16(b + p + 30), clen = rd16(b + p + 32);
        m.local = rd32(b + p + 42);
        if (end - p - 46 < nlen + elen + clen) return set_error(FG_ERR_INVALID, "npz: truncated central directory");
        if (flags & 0x1) return set_error(FG_ERR_UNSUPPORTED, "npz: encrypted members are not supported");
        m.name.assign(reinterpret_cast<const char*>(b + p + 46), nlen);
        // ZIP64 extra field (id 1): the 64-bit values, in this order, of the
        // fields whose 32-bit slot holds 0xFFFFFFFF
        const unsigned char* x = b + p + 46 + nlen;
        for (size_t q = 0; q + 4 <= elen;) {
            const uint16_t id = rd16(x + q), sz = rd16(x + q + 2);
            if (q + 4 + sz > elen) break;
            if (id == 0x0001) {
                const unsigned char* v = x + q + 4;
                size_t k = 0;
                if (m.usize == 0xFFFFFFFFu && k + 8 <= sz) m.usize = rd64(v + k), k += 8;
                if (m.csize == 0xFFFFFFFFu && k + 8 <= sz) m.csize = rd64(v + k), k += 8;
                if (m.local == 0xFFFFFFFFu && k + 8 <= sz) m.local = rd64(v + k), k += 8;
            }
            q += 4 + sz;
        }
        out.push_back(std::move(m));
        p += 46 + nlen + elen + clen;
    }
    return FG_OK;
}

std::string listed_name(const std::string& file) {
    const size_t n = file.size();
    return (n >= 4 && file.compare(n - 4, 4, ".npy") == 0) ? file.substr(0, n - 4) : file;
}

// The member's uncompressed bytes: a pointer into the archive (stored) or
// into `buf` (deflate); CRC-32 checked.
fg_status member_bytes(const unsigned char* b, size_t len, const Member& m, std::vector<unsigned char>& buf,
                       const unsigned char** data, size_t* size) {
    if (m.local > len || len - m.local < 30 || rd32(b + m.local) != 0x04034b50u)
        return set_error(FG_ERR_INVALID, "npz: bad local header for '" + m.name + "'");
    const size_t off = static_cast<size_t>(m.local) + 30 + rd16(b + m.local + 26) + rd16(b + m.local + 28);
    if (off > len || m.csize > len - off) return set_error(FG_ERR_INVALID, "npz: member '" + m.name + "' out of range");
    const unsigned char* src = b + off;
    if (m.method == 0) {
        if (m.csize != m.usize) return set_error(FG_ERR_INVALID, "npz: stored member sizes disagree");
        *data = src;
        *size = static_cast<size_t>(m.usize);
    } else if (m.method == 8) {
        if (m.usize > (1ull << 40)) return set_error(FG_ERR_INVALID, "npz: member too large");
        try {
            buf.resize(static_cast<size_t>(m.usize));
        } catch (const std::bad_alloc&) {
            return set_error(FG_ERR_OOM, "npz: no host memory to inflate '" + m.name + "'");
        }
        z_stream zs;
        std::memset(&zs, 0, sizeof(zs));
        if (inflateInit2(&zs, -15) != Z_OK) return set_error(FG_ERR_INVALID, "npz: inflate init failed");
        size_t in_done = 0, out_done = 0;
        int rc = Z_OK;
        while (rc == Z_OK) {  // chunks of at most 1 GiB (zlib counts in 32 bits)
            const size_t in_chunk = std::min<size_t>(static_cast<size_t>(m.csize) - in_done, 1u << 30);
            const size_t out_chunk = std::min<size_t>(buf.size() - out_done, 1u << 30);
            zs.next_in = const_cast<unsigned char*>(src + in_done);
            zs.avail_in = static_cast<uInt>(in_chunk);
            zs.next_out = buf.data() + out_done;
            zs.avail_out = static_cast<uInt>(out_chunk);
            rc = inflate(&zs, Z_NO_FLUSH);
            in_done += in_chunk - zs.avail_in;
            out_done += out_chunk - zs.avail_out;
            if (rc == Z_OK && in_chunk - zs.avail_in == 0 && out_chunk - zs.avail_out == 0) rc = Z_BUF_ERROR;
        }
        inflateEnd(&zs);
        if (rc != Z_STREAM_END || out_done != buf.size())
            return set_error(FG_ERR_INVALID, "npz: corrupt deflate data in '" + m.name + "'");
        *data = buf.data();
        *size = buf.size();
    } else {
        return set_error(FG_ERR_UNSUPPORTED,
                         "npz: compression method " + std::to_string(m.method) + " of '" + m.name + "' is not supported");
    }
    uLong crc = crc32(0L, Z_NULL, 0);
    for (size_t done = 0; done < *size;) {
        const size_t c = std::min<size_t>(*size - done, 1u << 30);
        crc = crc32(crc, *data + done, static_cast<uInt>(c));
        done += c;
    }
    if (static_cast<uint32_t>(crc) != m.crc) return set_error(FG_ERR_INVALID, "npz: CRC-32 mismatch in '" + m.name + "'");
    return FG_OK;
}

// Member "<name>.npy" for a listed name (mod.rs:150-167).
fg_status find_member(const std::vector<Member>& dir, const char* name, const Member** m) {
    const std::string want(name);
    bool listed = false;
    for (const Member& e : dir)
        if (listed_name(e.name) == want) listed = true;
    if (!listed) return set_error(FG_ERR_INVALID, "npz: array '" + want + "' not found in archive");
    for (const Member& e : dir)
        if (e.name == want + ".npy") {
            *m = &e;
            return FG_OK;
        }
    return set_error(FG_ERR_INVALID, "npz: failed to read entry '" + want + ".npy'");
}

}  // namespace

}  // namespace fgrt

using namespace fgrt;

extern "C" {

fg_status fg_npz_count(const void* bytes, size_t len, size_t* count) {
    if (!bytes || !count) return set_error(FG_ERR_INVALID, "npz: null argument");
    std::vector<Member> dir;
    FG_TRY(read_directory(static_cast<const unsigned char*>(bytes), len, dir));
    *count = dir.size();
    return FG_OK;
}

fg_status fg_npz_name(const void* bytes, size_t len, size_t index, char* out, size_t cap, size_t* name_len) {
    if (!bytes || !name_len) return set_error(FG_ERR_INVALID, "npz: null argument");
    std::vector<Member> dir;
    FG_TRY(read_directory(static_cast<const unsigned char*>(bytes), len, dir));
    if (index >= dir.size()) return set_error(FG_ERR_INVALID, "npz: member index out of range");
    const std::string n = listed_name(dir[index].name);
    *name_len = n.size();
    if (out) {
        if (cap < n.size() + 1) return set_error(FG_ERR_INVALID, "npz: name buffer too small");
        std::memcpy(out, n.c_str(), n.size() + 1);
    }
    return FG_OK;
}

fg_status fg_npz_read(const void* bytes, size_t len, const char* name, void* out, size_t cap, size_t* size) {
    if (!bytes || !name || !size) return set_error(FG_ERR_INVALID, "npz: null argument");
    const unsigned char* b = static_cast<const unsigned char*>(bytes);
    std::vector<Member> dir;
    FG_TRY(read_directory(b, len, dir));
    const Member* m = nullptr;
    FG_TRY(find_member(dir, name, &m));
    std::vector<unsigned char> buf;
    const unsigned char* data = nullptr;
    size_t n = 0;
    FG_TRY(member_bytes(b, len, *m, buf, &data, &n));
    *size = n;
    if (out) {
        if (cap < n) return set_error(FG_ERR_INVALID, "npz: output buffer too small");
        std::memcpy(out, data, n);
    }
    return FG_OK;
}

fg_status fg_npz_upload(fg_ctx* ctx, const void* bytes, size_t len, const char* name, void** dptr, fg_dtype* dtype,
                        int64_t* shape, int* ndim, fg_stream stream) {
    if (!ctx || !bytes || !name || !dptr) return set_error(FG_ERR_INVALID, "npz: null argument");
    *dptr = nullptr;
    const unsigned char* b = static_cast<const unsigned char*>(bytes);
    std::vector<Member> dir;
    FG_TRY(read_directory(b, len, dir));
    const Member* m = nullptr;
    FG_TRY(find_member(dir, name, &m));
    std::vector<unsigned char> buf;
    const unsigned char* data = nullptr;
    size_t n = 0;
    FG_TRY(member_bytes(b, len, *m, buf, &data, &n));
    FG_TRY(fg_npy_upload(ctx, data, n, dptr, dtype, shape, ndim, stream));
    // a pageable source is staged before cudaMemcpyAsync returns, but the
    // inflate buffer dies here: make the copy complete first
    if (!buf.empty()) FG_CUDA(cudaStreamSynchronize(stream_of(ctx, stream)));
    return FG_OK;
}

}  // extern "C"
