// npy.cu -- .npy byte images straight into device buffers (the ingest side of
// the path: served requests can arrive as .npy bytes without a host Array).
//
// Header format as the reference reads it (ferray-io/src/npy/header.rs:32-106):
// magic "\x93NUMPY", version (1|2|3, 0), header length (u16 LE for 1.0, u32
// LE for 2.0 / 3.0, capped at 1 MiB), then a Python dict literal with
// 'descr', 'fortran_order' and 'shape'.  Only the element types the GEMMs
// take are accepted: <f8 <f4 <c16 <c8 |i1 |u1 <i2 <f2 (and '=' / no byte
// order for the same types).
#include <cuda_runtime.h>

#include <cctype>
#include <cstring>
#include <string>

#include "runtime.h"

namespace fgrt {

namespace {

constexpr size_t kMaxHeader = 1u << 20;

// Value text after 'key': in the dict body, or npos.
size_t find_key(const std::string& h, const char* key) {
    const std::string k1 = std::string("'") + key + "'";
    const std::string k2 = std::string("\"") + key + "\"";
    size_t p = h.find(k1);
    size_t len = k1.size();
    if (p == std::string::npos) {
        p = h.find(k2);
        len = k2.size();
    }
    if (p == std::string::npos) return p;
    p += len;
    while (p < h.size() && std::isspace(static_cast<unsigned char>(h[p]))) ++p;
    if (p >= h.size() || h[p] != ':') return std::string::npos;
    ++p;
    while (p < h.size() && std::isspace(static_cast<unsigned char>(h[p]))) ++p;
    return p;
}

fg_status parse_descr(const std::string& d, fg_dtype* dt, size_t* itemsize) {
    if (d.empty()) return set_error(FG_ERR_DTYPE, "npy: empty descr");
    char order = d[0];
    std::string t = d;
    if (order == '<' || order == '>' || order == '|' || order == '=') t = d.substr(1);
    else order = '=';
    if (order == '>' && t != "i1" && t != "u1")
        return set_error(FG_ERR_DTYPE, "npy: big-endian descr '" + d + "' is not supported");
    struct M { const char* t; fg_dtype d; size_t s; };
    static const M map[] = {{"f8", FG_F64, 8}, {"f4", FG_F32, 4}, {"c16", FG_C64, 16}, {"c8", FG_C32, 8},
                            {"i1", FG_I8, 1},  {"u1", FG_U8I8, 1}, {"i2", FG_I16, 2}, {"f2", FG_F16, 2}};
    for (const M& m : map)
        if (t == m.t) {
            *dt = m.d;
            *itemsize = m.s;
            return FG_OK;
        }
    return set_error(FG_ERR_DTYPE, "npy: descr '" + d + "' has no GEMM operand type");
}

}  // namespace

}  // namespace fgrt

using namespace fgrt;

extern "C" {

fg_status fg_npy_parse(const void* bytes, size_t len, fg_dtype* dtype, int64_t* shape, int* ndim,
                       int* fortran_order, size_t* data_offset) {
    if (!bytes || !dtype || !shape || !ndim || !fortran_order || !data_offset)
        return set_error(FG_ERR_INVALID, "npy: null argument");
    const unsigned char* b = static_cast<const unsigned char*>(bytes);
    static const unsigned char magic[6] = {0x93, 'N', 'U', 'M', 'P', 'Y'};
    if (len < 10 || std::memcmp(b, magic, 6) != 0) return set_error(FG_ERR_INVALID, "npy: bad magic number");
    const int major = b[6], minor = b[7];
    if (major < 1 || major > 3 || minor != 0)
        return set_error(FG_ERR_INVALID, "npy: unsupported format version " + std::to_string(major) + "." +
                                             std::to_string(minor));
    size_t hl, pre;
    if (major == 1) {
        hl = static_cast<size_t>(b[8]) | (static_cast<size_t>(b[9]) << 8);
        pre = 10;
    } else {
        if (len < 12) return set_error(FG_ERR_INVALID, "npy: truncated preamble");
        hl = static_cast<size_t>(b[8]) | (static_cast<size_t>(b[9]) << 8) | (static_cast<size_t>(b[10]) << 16) |
             (static_cast<size_t>(b[11]) << 24);
        pre = 12;
        if (hl > kMaxHeader) return set_error(FG_ERR_INVALID, "npy: header length exceeds 1 MiB");
    }
    if (pre + hl > len) return set_error(FG_ERR_INVALID, "npy: truncated header");
    const std::string h(reinterpret_cast<const char*>(b + pre), hl);
    // descr
    size_t p = find_key(h, "descr");
    if (p == std::string::npos || (h[p] != '\'' && h[p] != '"'))
        return set_error(FG_ERR_DTYPE, "npy: missing or structured 'descr'");
    const char q = h[p];
    const size_t e = h.find(q, p + 1);
    if (e == std::string::npos) return set_error(FG_ERR_INVALID, "npy: unterminated descr");
    size_t itemsize = 0;
    FG_TRY(parse_descr(h.substr(p + 1, e - p - 1), dtype, &itemsize));
    // fortran_order
    p = find_key(h, "fortran_order");
    if (p == std::string::npos) return set_error(FG_ERR_INVALID, "npy: missing 'fortran_order'");
    if (h.compare(p, 4, "True") == 0) *fortran_order = 1;
    else if (h.compare(p, 5, "False") == 0) *fortran_order = 0;
    else return set_error(FG_ERR_INVALID, "npy: bad 'fortran_order'");
    // shape: a tuple of non-negative integers
    p = find_key(h, "shape");
    if (p == std::string::npos || h[p] != '(') return set_error(FG_ERR_INVALID, "npy: missing 'shape'");
    const size_t close = h.find(')', p);
    if (close == std::string::npos) return set_error(FG_ERR_INVALID, "npy: unterminated shape");
    int nd = 0;
    unsigned long long count = 1;
    size_t i = p + 1;
    while (i < close) {
        while (i < close && (std::isspace(static_cast<unsigned char>(h[i])) || h[i] == ',')) ++i;
        if (i >= close) break;
        if (!std::isdigit(static_cast<unsigned char>(h[i]))) return set_error(FG_ERR_INVALID, "npy: bad shape");
        unsigned long long v = 0;
        while (i < close && std::isdigit(static_cast<unsigned char>(h[i]))) {
            v = v * 10 + static_cast<unsigned>(h[i] - '0');
            if (v > (1ull << 48)) return set_error(FG_ERR_INVALID, "npy: dimension too large");
            ++i;
        }
        if (nd >= 8) return set_error(FG_ERR_UNSUPPORTED, "npy: more than 8 dimensions");
        shape[nd++] = static_cast<int64_t>(v);
        count *= v;
        if (count > (1ull << 48)) return set_error(FG_ERR_INVALID, "npy: array too large");
    }
    *ndim = nd;
    *data_offset = pre + hl;
    if (len - *data_offset < count * itemsize) return set_error(FG_ERR_SHAPE, "npy: payload shorter than the shape");
    return FG_OK;
}

fg_status fg_npy_upload(fg_ctx* ctx, const void* bytes, size_t len, void** dptr, fg_dtype* dtype,
                        int64_t* shape, int* ndim, fg_stream stream) {
    if (!ctx || !dptr) return set_error(FG_ERR_INVALID, "npy: null argument");
    *dptr = nullptr;
    int fortran = 0;
    size_t off = 0;
    FG_TRY(fg_npy_parse(bytes, len, dtype, shape, ndim, &fortran, &off));
    if (fortran) return set_error(FG_ERR_UNSUPPORTED, "npy: Fortran-order arrays are not supported (row-major only)");
    size_t count = 1;
    for (int i = 0; i < *ndim; ++i) count *= static_cast<size_t>(shape[i]);
    const size_t nbytes = count * in_size(*dtype);
    FG_TRY(fg_buffer_alloc(ctx, std::max<size_t>(nbytes, 1), dptr));
    if (nbytes) {
        const cudaError_t e = cudaMemcpyAsync(*dptr, static_cast<const unsigned char*>(bytes) + off, nbytes,
                                              cudaMemcpyHostToDevice, stream_of(ctx, stream));
        if (e != cudaSuccess) {
            fg_buffer_free(ctx, *dptr);
            *dptr = nullptr;
            return cuda_error(e, "npy upload");
        }
    }
    return FG_OK;
}

}  // extern "C"
