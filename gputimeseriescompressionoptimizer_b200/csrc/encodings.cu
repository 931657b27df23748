// encodings.cu -- host side of every encoding: argument checks, the data-dependent sizes that
// the reference also reads back, allocation of outputs, and the kernel launches.
#include "encodings.hpp"
#include "kernels.hpp"

#include <cstring>

namespace gtsc {

namespace {

DevBuf h2d_small(const void *src, uint64_t bytes, cudaStream_t s)
{
    DevBuf b = dev_alloc(bytes, s);
    if (bytes) GTSC_CUDA(cudaMemcpyAsync(b.get(), src, bytes, cudaMemcpyHostToDevice, s));
    return b;
}

DevBuf empty_buf() { return DevBuf{}; }

// Copy of a view into a fresh 16-byte aligned buffer when the kernels need alignment.
View aligned_input(View in, DevBuf &keep, cudaStream_t s)
{
    if (((uintptr_t)in.ptr & 15) == 0 || in.bytes == 0) return in;
    keep = dev_alloc(in.bytes, s);
    GTSC_CUDA(cudaMemcpyAsync(keep.get(), in.ptr, in.bytes, cudaMemcpyDeviceToDevice, s));
    return View(keep);
}

// Raw bits of the min and max element in order `o` (one D2H read, as the reference's MinMax).
bool column_minmax(View in, int es, Order o, uint64_t *mn, uint64_t *mx, cudaStream_t s)
{
    uint64_t n = in.bytes / es;
    if (n == 0) return false;
    DevBuf acc = dev_alloc(sizeof(MinMaxAcc), s);
    GTSC_CUDA(cudaMemsetAsync(acc.get(), 0, sizeof(MinMaxAcc), s));
    launch_minmax(in.ptr, n, es, o, (MinMaxAcc *)acc.get(), s);
    MinMaxAcc h;
    d2h(&h, acc.get(), sizeof(h), s);
    if (!minmax_result(h, es, o, mn, mx)) {
        uint64_t first = 0;  // every element NaN: thrust would return element 0
        d2h(&first, in.ptr, es, s);
        *mn = *mx = first;
    }
    return true;
}

// ------------------------------------------------------------------------------------ AFL

// AflEncoding::Encode<T> (compression/afl/afl_encoding.cu:15-56)
Parts afl_encode(int dt, View in, cudaStream_t s)
{
    const int es = dtype_size(dt);
    if (is_fp(dt)) fail(GTSC_ERR_TYPE, "afl: floating-point columns are not supported");
    const uint64_t n = in.bytes / es;
    if (n == 0) return {empty_buf(), empty_buf()};
    uint64_t mn, mx;
    column_minmax(in, es, ORD_INT, &mn, &mx, s);
    const int b = bitlen_signed(sext(mn, es), sext(mx, es), es);
    const uint64_t W = 8ull * es;
    const uint64_t words = (b * n + W - 1) / W;
    const uint64_t bytes = words * es;
    uint8_t meta[4] = {(uint8_t)b, (uint8_t)(int8_t)(bytes * 8 - n * (uint64_t)b), 0, 0};
    DevBuf m = h2d_small(meta, 4, s);
    DevBuf out = dev_alloc(bytes, s);
    DevBuf keep;
    View src = aligned_input(in, keep, s);
    launch_afl_pack(src.ptr, n, es, b, out.get(), bytes, s);
    return {m, out};
}

// AflEncoding::Decode<T> / DecodeAfl (afl_encoding.cu:74-113)
DevBuf afl_decode(int dt, View meta, View data, cudaStream_t s)
{
    const int es = dtype_size(dt);
    if (is_fp(dt)) fail(GTSC_ERR_TYPE, "afl: floating-point columns are not supported");
    if (data.bytes == 0) return empty_buf();
    if (meta.bytes < 2) fail(GTSC_ERR_FORMAT, "afl: metadata too short");
    int8_t m[2];
    d2h(m, meta.ptr, 2, s);
    const int b = m[0], rest = m[1];
    if (b < 1 || b > 8 * es) fail(GTSC_ERR_FORMAT, "afl: bad bit width in metadata");
    const int64_t bits = (int64_t)data.bytes * 8 - rest;
    if (bits < 0) fail(GTSC_ERR_FORMAT, "afl: bad rest in metadata");
    const uint64_t n = (uint64_t)bits / b;
    DevBuf out = dev_alloc(n * es, s);
    launch_afl_unpack(data.ptr, data.bytes, n, es, b, out.get(), s);
    return out;
}

// ------------------------------------------------------------------------------------ none

// NoneEncoding (compression/none/none_encoding.cu:13-49): metadata = size_t byte count
Parts none_encode(View in, cudaStream_t s)
{
    uint64_t sz = in.bytes;
    DevBuf m = h2d_small(&sz, 8, s);
    DevBuf out = dev_alloc(in.bytes, s);
    if (in.bytes) GTSC_CUDA(cudaMemcpyAsync(out.get(), in.ptr, in.bytes, cudaMemcpyDeviceToDevice, s));
    return {m, out};
}

DevBuf none_decode(View data, cudaStream_t s)
{
    DevBuf out = dev_alloc(data.bytes, s);
    if (data.bytes) GTSC_CUDA(cudaMemcpyAsync(out.get(), data.ptr, data.bytes, cudaMemcpyDeviceToDevice, s));
    return out;
}

}  // namespace

int n_results(int enc)
{
    switch (enc) {
    case GTSC_DELTA: case GTSC_AFL: case GTSC_SCALE: case GTSC_UNIQUE: case GTSC_FLOAT_TO_INT: case GTSC_CONST:
        return 1;
    case GTSC_RLE: case GTSC_DICT: case GTSC_PATCH: case GTSC_GFC: return 2;
    case GTSC_NONE: return 0;
    default: return -1;
    }
}

int return_type(int enc, int dt, int j)
{
    if (enc == GTSC_RLE && j == 0) return GTSC_INT;
    if (enc == GTSC_FLOAT_TO_INT) return GTSC_INT;
    return dt;
}

Parts encode(int enc, int dt, View in, cudaStream_t s)
{
    if (!dtype_size(dt)) fail(GTSC_ERR_ARG, "unknown data type");
    if (in.bytes && !in.ptr) fail(GTSC_ERR_ARG, "null input");
    if ((uintptr_t)in.ptr % dtype_size(dt)) fail(GTSC_ERR_ARG, "input not aligned to its element size");
    switch (enc) {
    case GTSC_AFL: return afl_encode(dt, in, s);
    case GTSC_NONE: return none_encode(in, s);
    default: fail(GTSC_ERR_UNSUPPORTED, "encoding not available");
    }
}

DevBuf decode(int enc, int dt, const std::vector<View> &in, cudaStream_t s)
{
    if (!dtype_size(dt)) fail(GTSC_ERR_ARG, "unknown data type");
    std::vector<View> v = in;
    while (v.size() < 3) v.push_back(View());
    switch (enc) {
    case GTSC_AFL: return afl_decode(dt, v[0], v[1], s);
    case GTSC_NONE: return none_decode(v[1], s);
    default: fail(GTSC_ERR_UNSUPPORTED, "encoding not available");
    }
}

}  // namespace gtsc
