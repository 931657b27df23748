// encodings.cu -- host side of every encoding: argument checks, the data-dependent sizes that
// the reference also reads back, allocation of outputs, and the kernel launches.
#include "encodings.hpp"
#include "kernels.hpp"
#include "scan.cuh"

#include <array>
#include <cmath>
#include <cstring>
#include <mutex>

namespace gtsc {

namespace {

DevBuf h2d_small(const void *src, uint64_t bytes, cudaStream_t s)
{
    DevBuf b = dev_alloc(bytes, s);
    if (bytes) GTSC_CUDA(cudaMemcpyAsync(b.get(), src, bytes, cudaMemcpyHostToDevice, s));
    return b;
}

DevBuf empty_buf() { return DevBuf{}; }

// A view whose start is aligned to `align` bytes: the view itself, or an aligned copy.
View aligned(View in, int align, DevBuf &keep, cudaStream_t s)
{
    if (in.bytes == 0 || ((uintptr_t)in.ptr % align) == 0) return in;
    keep = dev_alloc(in.bytes, s);
    GTSC_CUDA(cudaMemcpyAsync(keep.get(), in.ptr, in.bytes, cudaMemcpyDeviceToDevice, s));
    return View(keep);
}

DevBuf shrink(DevBuf b, uint64_t bytes)
{
    b.bytes = bytes;
    return b;
}

// small zeroed device scratch for status words / counters
struct Words {
    DevBuf buf;
    explicit Words(cudaStream_t s, int n = 8)
    {
        buf = dev_alloc(8ull * n, s);
        GTSC_CUDA(cudaMemsetAsync(buf.get(), 0, 8ull * n, s));
    }
    unsigned long long *u64(int i) const { return (unsigned long long *)buf.get() + i; }
    uint32_t *u32(int i) const { return (uint32_t *)buf.get() + i; }
};

void check_status_word(uint32_t w, const char *what)
{
    if (w) fail(-(gtsc_status)w, std::string(what) + ": device check failed");
}

uint64_t stencil_count(uint64_t n) { return (n + 7) / 8; }

// elements described by a packed stencil (Stencil::unpack, util/stencil/stencil.cu:70-96)
uint64_t stencil_elems(View packed, cudaStream_t s)
{
    if (packed.bytes < 1) fail(GTSC_ERR_FORMAT, "stencil: empty");
    int8_t rest;
    d2h(&rest, packed.ptr, 1, s);
    int64_t n = (int64_t)(packed.bytes - 1) * 8;
    if (rest) n -= 8 - rest;
    if (n < 0 || rest < 0 || rest > 7) fail(GTSC_ERR_FORMAT, "stencil: bad rest byte");
    return (uint64_t)n;
}

// Raw bits of the min and max element in order `o` (one D2H read, as the reference's MinMax).
void column_minmax(View in, int es, Order o, uint64_t *mn, uint64_t *mx, cudaStream_t s)
{
    const uint64_t n = in.bytes / es;
    Words w(s, 2);
    launch_minmax(in.ptr, n, es, o, (MinMaxAcc *)w.buf.get(), s);
    MinMaxAcc h;
    d2h(&h, w.buf.get(), sizeof(h), s);
    if (!minmax_result(h, es, o, mn, mx)) {
        uint64_t first = 0;  // every element NaN: thrust would return element 0
        d2h(&first, in.ptr, es, s);
        *mn = *mx = first;
    }
}


// ------------------------------------------------------------------------------------ AFL

Parts afl_float_encode(View in, cudaStream_t s);
DevBuf afl_float_decode(View meta, View data, cudaStream_t s);

// AflEncoding::Encode<T> (compression/afl/afl_encoding.cu:15-56)
Parts afl_encode(int dt, View in, cudaStream_t s)
{
    const int es = dtype_size(dt);
    if (dt == GTSC_FLOAT) return afl_float_encode(in, s);
    if (is_fp(dt)) fail(GTSC_ERR_TYPE, "afl: double columns are not supported (EncodeDouble returns no buffers)");
    const uint64_t n = in.bytes / es;
    if (n == 0) return {empty_buf(), empty_buf()};
    DevBuf keep;
    View src = aligned(in, 16, keep, s);
    uint64_t mn, mx;
    column_minmax(src, es, ORD_INT, &mn, &mx, s);
    const int b = bitlen_signed(sext(mn, es), sext(mx, es), es);
    const uint64_t W = 8ull * es;
    const uint64_t words = (b * n + W - 1) / W;
    const uint64_t bytes = words * es;
    uint8_t meta[4] = {(uint8_t)b, (uint8_t)(int8_t)(bytes * 8 - n * (uint64_t)b), 0, 0};
    DevBuf m = h2d_small(meta, 4, s);
    DevBuf out = dev_alloc(bytes, s);
    launch_afl_pack(src.ptr, n, es, b, out.get(), bytes, s);
    return {m, out};
}

// AflEncoding::Decode<T> / DecodeAfl (afl_encoding.cu:74-113)
DevBuf afl_decode(int dt, View meta, View data, cudaStream_t s)
{
    const int es = dtype_size(dt);
    if (dt == GTSC_FLOAT) return afl_float_decode(meta, data, s);
    if (is_fp(dt)) fail(GTSC_ERR_TYPE, "afl: double columns are not supported (DecodeDouble returns no buffer)");
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

// AflEncoding::Encode(SharedCudaPtr<float>) (afl_encoding.cu:116-170).  data = mantissa metadata
// + mantissa words + exponent metadata + exponent words; metadata = size_t mantissa-word bytes, a
// sign byte (1 all positive, 2 all negative, 0: the packed sign stencil follows).  The sign byte is
// decided on the sign bits (the reference's min >= 0 / max < 0 would drop the sign of -0.0 and of
// NaNs).
Parts afl_float_encode(View in, cudaStream_t s)
{
    const uint64_t n = in.bytes / 4;
    if (n == 0) return {empty_buf(), empty_buf()};
    DevBuf mant = dev_alloc(4 * n, s), expo = dev_alloc(4 * n, s);
    DevBuf st = dev_alloc(1 + (n + 7) / 8, s), flags = dev_alloc(4, s);
    GTSC_CUDA(cudaMemsetAsync(flags.get(), 0, 4, s));
    launch_float_split(in.ptr, n, (int32_t *)mant.get(), (int32_t *)expo.get(), st.get(), (uint32_t *)flags.get(), s);
    uint32_t f = 0;
    d2h(&f, flags.get(), 4, s);
    const uint8_t sign = (f & 1) == 0 ? 1 : (f & 2) == 0 ? 2 : 0;
    Parts pm = afl_encode(GTSC_INT, View(mant), s);
    Parts pe = afl_encode(GTSC_INT, View(expo), s);
    const uint64_t msize = pm[1].bytes, esize = pe[1].bytes;
    DevBuf data = dev_alloc(8 + msize + esize, s);
    uint8_t *d = data.get();
    GTSC_CUDA(cudaMemcpyAsync(d, pm[0].get(), 4, cudaMemcpyDeviceToDevice, s));
    if (msize) GTSC_CUDA(cudaMemcpyAsync(d + 4, pm[1].get(), msize, cudaMemcpyDeviceToDevice, s));
    GTSC_CUDA(cudaMemcpyAsync(d + 4 + msize, pe[0].get(), 4, cudaMemcpyDeviceToDevice, s));
    if (esize) GTSC_CUDA(cudaMemcpyAsync(d + 8 + msize, pe[1].get(), esize, cudaMemcpyDeviceToDevice, s));
    const uint64_t sbytes = sign == 0 ? 1 + (n + 7) / 8 : 0;
    DevBuf meta = dev_alloc(9 + sbytes, s);
    uint8_t head[9];
    std::memcpy(head, &msize, 8);
    head[8] = sign;
    GTSC_CUDA(cudaMemcpyAsync(meta.get(), head, 9, cudaMemcpyHostToDevice, s));
    if (sbytes) GTSC_CUDA(cudaMemcpyAsync(meta.get() + 9, st.get(), sbytes, cudaMemcpyDeviceToDevice, s));
    GTSC_CUDA(cudaStreamSynchronize(s));  // `head` is a host stack buffer
    return {meta, data};
}

// AflEncoding::Decode<float> (afl_encoding.cu:189-254)
DevBuf afl_float_decode(View meta, View data, cudaStream_t s)
{
    if (data.bytes == 0) return empty_buf();
    if (meta.bytes < 9 || data.bytes < 8) fail(GTSC_ERR_FORMAT, "afl float: stream too short");
    uint8_t head[9];
    d2h(head, meta.ptr, 9, s);
    uint64_t msize;
    std::memcpy(&msize, head, 8);
    const int sign = (int8_t)head[8];
    if (msize > data.bytes - 8 || sign < 0 || sign > 2) fail(GTSC_ERR_FORMAT, "afl float: bad metadata");
    const uint64_t esize = data.bytes - msize - 8;
    DevBuf m = afl_decode(GTSC_INT, View(data.ptr, 4), View(data.ptr + 4, msize), s);
    DevBuf e = afl_decode(GTSC_INT, View(data.ptr + 4 + msize, 4), View(data.ptr + 8 + msize, esize), s);
    const uint64_t n = m.bytes / 4;
    if (e.bytes / 4 < n) fail(GTSC_ERR_FORMAT, "afl float: fewer exponents than mantissas");
    const uint8_t *stencil = nullptr;
    if (sign == 0) {
        // Stencil(metadata, sizeof(size_t) + 1): rest byte, then the sign bits
        int8_t rest;
        d2h(&rest, meta.ptr + 9, 1, s);
        const int64_t bits = (int64_t)(meta.bytes - 10) * 8 - (rest ? 8 - rest : 0);
        if (meta.bytes < 10 || rest < 0 || rest > 7 || bits < (int64_t)n)
            fail(GTSC_ERR_FORMAT, "afl float: sign stencil too short");
        stencil = meta.ptr + 10;
    }
    DevBuf out = dev_alloc(4 * n, s);
    launch_float_compose((const int32_t *)m.get(), (const int32_t *)e.get(), stencil, sign == 0 ? 0 : sign - 1, n,
                         (uint32_t *)out.get(), s);
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

// ------------------------------------------------------------------------------------ delta

// DeltaEncoding::Encode/Decode (compression/delta/delta_encoding.cu:29-102); float/double use
// their int32/int64 bit patterns (delta_encoding.hpp:57-64), which the byte kernels do anyway.
Parts delta_encode(int dt, View in, cudaStream_t s)
{
    const int es = dtype_size(dt);
    const uint64_t n = in.bytes / es;
    if (n == 0) return {empty_buf(), empty_buf()};
    DevBuf keep;
    View src = aligned(in, 16, keep, s);
    DevBuf m = dev_alloc(es, s);
    GTSC_CUDA(cudaMemcpyAsync(m.get(), src.ptr, es, cudaMemcpyDeviceToDevice, s));
    DevBuf out = dev_alloc((n - 1) * es, s);
    launch_delta_encode(src.ptr, n, es, out.get(), s);
    return {m, out};
}

DevBuf delta_decode(int dt, View meta, View data, cudaStream_t s)
{
    const int es = dtype_size(dt);
    if (meta.bytes == 0) return empty_buf();
    if (meta.bytes < (uint64_t)es) fail(GTSC_ERR_FORMAT, "delta: metadata too short");
    const uint64_t n = data.bytes / es + 1;
    DevBuf keep;
    View d = aligned(data, es, keep, s);
    DevBuf out = dev_alloc(n * es, s);
    const uint64_t tiles = delta_decode_tiles(n);
    DevBuf scratch = dev_alloc(lookback_bytes(tiles), s);
    launch_delta_decode(d.ptr, n, meta.ptr, out.get(), scratch.get(), es, s);
    uint32_t err;
    d2h(&err, lookback_at(scratch.get(), tiles).error, 4, s);
    check_status_word(err, "delta decode");
    return out;
}

// ------------------------------------------------------------------------------------ scale

// ScaleEncoding::Encode (compression/scale/scale_encoding.cu:30-68).  The overflow test at :49-50
// is evaluated with the wrap-around of the reference's x86 host build for int/long.
Parts scale_encode(int dt, View in, cudaStream_t s)
{
    const int es = dtype_size(dt);
    const uint64_t n = in.bytes / es;
    if (n == 0) return {empty_buf(), empty_buf()};
    DevBuf keep;
    View src = aligned(in, 16, keep, s);
    uint64_t mnb, mxb;
    column_minmax(src, es, ORD_INT, &mnb, &mxb, s);
    int64_t mn = sext(mnb, es), mx = sext(mxb, es);
    if (mn < 0) {
        if (es <= 2) {
            const int64_t tmax = es == 1 ? 127 : 32767;
            if ((tmax - mx) < (mn < 0 ? -mn : mn)) mn = 0;
        } else {
            const uint64_t W = 8ull * es;
            const uint64_t msk = W == 64 ? ~0ull : ((1ull << W) - 1);
            const uint64_t tmax = msk >> 1;
            const int64_t diff = sext((tmax - (uint64_t)mx) & msk, es);
            const int64_t absmn = sext((0 - (uint64_t)mn) & msk, es);
            if (diff < absmn) mn = 0;
        }
    }
    uint64_t mnu = (uint64_t)mn;
    DevBuf m = h2d_small(&mnu, es, s);
    DevBuf out = dev_alloc(n * es, s);
    launch_scale(src.ptr, n, es, m.get(), out.get(), true, s);
    return {m, out};
}

DevBuf scale_decode(int dt, View meta, View data, cudaStream_t s)
{
    const int es = dtype_size(dt);
    if (data.bytes == 0) return empty_buf();
    if (meta.bytes < (uint64_t)es) fail(GTSC_ERR_FORMAT, "scale: metadata too short");
    const uint64_t n = data.bytes / es;
    DevBuf keep;
    View d = aligned(data, 16, keep, s);
    DevBuf out = dev_alloc(n * es, s);
    launch_scale(d.ptr, n, es, meta.ptr, out.get(), false, s);
    return out;
}

// ------------------------------------------------------------------------------------ RLE

// RleEncoding::Encode (compression/rle/rle_encode.cu:18-62): meta = int32 run count,
// out1 = int32 lengths, out2 = T values.  No empty-input guard in the reference: n = 0 gives a
// 4-byte zero count and two empty streams.
Parts rle_encode(int dt, View in, cudaStream_t s)
{
    const int es = dtype_size(dt);
    const uint64_t n = in.bytes / es;
    if (n >= (1ull << 31)) fail(GTSC_ERR_CAPACITY, "rle: more than 2^31-1 elements");
    DevBuf keep;
    View src = aligned(in, es, keep, s);
    DevBuf values = dev_alloc(n * es, s), lengths = dev_alloc(4 * n, s), starts = dev_alloc(4 * n, s);
    const uint64_t tiles = rle_tiles(n);
    DevBuf scratch = dev_alloc(lookback_bytes(tiles) + 16, s);
    Words w(s, 1);
    launch_rle_encode(src.ptr, n, es, native_order(dt), values.get(), (int32_t *)lengths.get(),
                      (uint32_t *)starts.get(), w.u64(0), scratch.get(), s);
    unsigned long long runs = 0;
    d2h(&runs, w.u64(0), 8, s);
    if (n) {
        uint32_t err;
        d2h(&err, lookback_at(scratch.get(), tiles).error, 4, s);
        check_status_word(err, "rle encode");
    }
    int32_t r32 = (int32_t)runs;
    DevBuf m = h2d_small(&r32, 4, s);
    return {m, shrink(lengths, 4 * runs), shrink(values, es * runs)};
}

// RleEncoding::Decode (compression/rle/rle_decode.cu:19-73)
DevBuf rle_decode(int dt, View meta, View lengths, View values, cudaStream_t s)
{
    const int es = dtype_size(dt);
    if (lengths.bytes == 0) return empty_buf();
    if (meta.bytes < 4) fail(GTSC_ERR_FORMAT, "rle: metadata too short");
    int32_t runs;
    d2h(&runs, meta.ptr, 4, s);
    if (runs < 0 || (uint64_t)runs * 4 > lengths.bytes || (uint64_t)runs * es > values.bytes)
        fail(GTSC_ERR_FORMAT, "rle: run count exceeds its streams");
    if (runs == 0) return empty_buf();
    DevBuf ends = dev_alloc(8ull * runs, s);
    const uint64_t tiles = rle_tiles(runs);
    DevBuf scratch = dev_alloc(lookback_bytes(tiles), s);
    launch_scan_i32(lengths.ptr, runs, (unsigned long long *)ends.get(), scratch.get(), s);
    unsigned long long n = 0;
    d2h(&n, (unsigned long long *)ends.get() + runs - 1, 8, s);
    uint32_t err;
    d2h(&err, lookback_at(scratch.get(), tiles).error, 4, s);
    check_status_word(err, "rle decode");
    if ((long long)n < 0 || n > (1ull << 40)) fail(GTSC_ERR_FORMAT, "rle: negative or huge run lengths");
    DevBuf out = dev_alloc(n * es, s);
    launch_rle_expand((const unsigned long long *)ends.get(), runs, values.ptr, n, es, out.get(), s);
    return out;
}

// ------------------------------------------------------------------------------------ histogram

// GetMostFrequent(data, k) into dev `top` (k values, es bytes each); returns the scratch so the
// caller can check the overflow word later (after its own synchronisation)
struct TopK {
    DevBuf scratch;
    HistTable table;
    bool full;
};

TopK top_k(View in, int es, Order o, int k, uint8_t *top, bool full, cudaStream_t s)
{
    const uint64_t n = in.bytes / es;
    TopK t;
    t.full = full;
    const uint64_t cap = hist_cap_for(n, full);
    const int grid = hist_grid(n);
    t.scratch = dev_alloc(hist_scratch_bytes(cap, grid), s);
    t.table = hist_table_at(t.scratch.get(), cap, grid);
    launch_hist_topk(in.ptr, n, es, o, k, t.table, grid, top, nullptr, s);
    return t;
}

bool overflowed(const TopK &t, cudaStream_t s)
{
    uint32_t ov = 0;
    d2h(&ov, t.table.overflow, 4, s);
    return ov != 0 && !t.full;
}

// ------------------------------------------------------------------------------------ dict

// DictEncoding::Encode (compression/dict/dict_encoding.cu:66-95) with UniqueEncoding::CompressUnique
// (unique_encoding.cu:88-131) for the 4 most frequent values.
Parts dict_encode(int dt, View in, cudaStream_t s, bool full = false)
{
    const int es = dtype_size(dt);
    const uint64_t n = in.bytes / es;
    if (n == 0) return {empty_buf(), empty_buf(), empty_buf()};
    DevBuf keep;
    View src = aligned(in, 16, keep, s);
    const uint64_t hdr = 16 + 4ull * es;
    const uint64_t max_words = (n + 15) / 16;
    DevBuf out1 = dev_alloc(hdr + 4 * max_words, s);
    GTSC_CUDA(cudaMemsetAsync(out1.get(), 0, hdr + 4 * max_words, s));
    TopK tk = top_k(src, es, native_order(dt), 4, out1.get() + 16, full, s);
    DevBuf meta = dev_alloc(1 + stencil_count(n), s);
    uint8_t rest = (uint8_t)(n % 8);
    GTSC_CUDA(cudaMemcpyAsync(meta.get(), &rest, 1, cudaMemcpyHostToDevice, s));
    DevBuf out2 = dev_alloc(n * es, s);
    const uint64_t tiles = split_tiles(n);
    DevBuf scratch = dev_alloc(lookback_bytes(tiles), s);
    Words w(s, 1);
    SplitArgs a;
    a.order = native_order(dt);
    a.top = out1.get() + 16;
    a.stencil = meta.get() + 1;
    a.no = out2.get();
    a.words = (uint32_t *)(out1.get() + hdr);
    a.yes_count = w.u64(0);
    launch_split(SPLIT_DICT, src.ptr, n, es, a, scratch.get(), s);
    unsigned long long m = 0;
    d2h(&m, w.u64(0), 8, s);
    if (overflowed(tk, s)) return dict_encode(dt, in, s, true);
    uint32_t err;
    d2h(&err, lookback_at(scratch.get(), tiles).error, 4, s);
    check_status_word(err, "dict encode");
    uint64_t sizes[2] = {4, m};
    GTSC_CUDA(cudaMemcpyAsync(out1.get(), sizes, 16, cudaMemcpyHostToDevice, s));
    const uint64_t out1_bytes = m ? hdr + 4 * ((m + 15) / 16) : 0;  // CompressUnique of nothing is empty
    GTSC_CUDA(cudaStreamSynchronize(s));
    return {meta, shrink(out1, out1_bytes), shrink(out2, (n - m) * es)};
}

// DictEncoding::Decode (dict_encoding.cu:103-130)
DevBuf dict_decode(int dt, View meta, View in1, View in2, cudaStream_t s)
{
    const int es = dtype_size(dt);
    if (in1.bytes == 0 && in2.bytes == 0) return empty_buf();
    const uint64_t n = stencil_elems(meta, s);
    uint64_t m = 0;
    const uint64_t hdr = 16 + 4ull * es;
    DevBuf k1;
    View u = aligned(in1, 4, k1, s);
    if (u.bytes) {
        if (u.bytes < 16) fail(GTSC_ERR_FORMAT, "dict: unique header too short");
        uint64_t sz[2];
        d2h(sz, u.ptr, 16, s);
        if (sz[0] != 4) fail(GTSC_ERR_FORMAT, "dict: expected 4 dictionary entries");
        m = sz[1];
        if (hdr + 4 * ((m + 15) / 16) > u.bytes || m > n) fail(GTSC_ERR_FORMAT, "dict: code stream too short");
    }
    DevBuf k2;
    View no = aligned(in2, es, k2, s);
    DevBuf out = dev_alloc(n * es, s);
    const uint64_t tiles = split_tiles(n);
    DevBuf scratch = dev_alloc(lookback_bytes(tiles), s);
    Words w(s, 1);
    MergeArgs a;
    a.order = native_order(dt);
    a.top = u.bytes ? u.ptr + 16 : nullptr;
    a.words = u.bytes ? (const uint32_t *)(u.ptr + hdr) : nullptr;
    a.yes_cap = m;
    a.no = no.ptr;
    a.no_cap = no.bytes / es;
    a.error = w.u32(0);
    launch_merge(SPLIT_DICT, meta.ptr + 1, n, es, a, out.get(), scratch.get(), s);
    uint32_t err[2];
    d2h(&err[0], w.u32(0), 4, s);
    d2h(&err[1], lookback_at(scratch.get(), tiles).error, 4, s);
    check_status_word(err[0], "dict decode");
    check_status_word(err[1], "dict decode");
    return out;
}

// ------------------------------------------------------------------------------------ const

// ConstEncoding::Encode/Decode (compression/const/const_encoding.cu:43-131): meta = T c || packed
// stencil of (x is not c), data = the non-c values in order.
Parts const_encode(int dt, View in, cudaStream_t s, bool full = false)
{
    const int es = dtype_size(dt);
    const uint64_t n = in.bytes / es;
    if (n == 0) return {empty_buf(), empty_buf()};
    DevBuf keep;
    View src = aligned(in, 16, keep, s);
    DevBuf meta = dev_alloc(es + 1 + stencil_count(n), s);
    TopK tk = top_k(src, es, native_order(dt), 1, meta.get(), full, s);
    uint8_t rest = (uint8_t)(n % 8);
    GTSC_CUDA(cudaMemcpyAsync(meta.get() + es, &rest, 1, cudaMemcpyHostToDevice, s));
    DevBuf out1 = dev_alloc(n * es, s);
    const uint64_t tiles = split_tiles(n);
    DevBuf scratch = dev_alloc(lookback_bytes(tiles), s);
    Words w(s, 1);
    SplitArgs a;
    a.order = native_order(dt);
    a.top = meta.get();
    a.stencil = meta.get() + es + 1;
    a.yes = out1.get();
    a.yes_count = w.u64(0);
    launch_split(SPLIT_NOT_CONST, src.ptr, n, es, a, scratch.get(), s);
    unsigned long long m = 0;
    d2h(&m, w.u64(0), 8, s);
    if (overflowed(tk, s)) return const_encode(dt, in, s, true);
    uint32_t err;
    d2h(&err, lookback_at(scratch.get(), tiles).error, 4, s);
    check_status_word(err, "const encode");
    return {meta, shrink(out1, m * es)};
}

DevBuf const_decode(int dt, View meta, View data, cudaStream_t s)
{
    const int es = dtype_size(dt);
    if (meta.bytes == 0) return empty_buf();
    if (meta.bytes < (uint64_t)es + 1) fail(GTSC_ERR_FORMAT, "const: metadata too short");
    const uint64_t n = stencil_elems(View(meta.ptr + es, meta.bytes - es), s);
    DevBuf k1;
    View d = aligned(data, es, k1, s);
    DevBuf out = dev_alloc(n * es, s);
    const uint64_t tiles = split_tiles(n);
    DevBuf scratch = dev_alloc(lookback_bytes(tiles), s);
    Words w(s, 1);
    MergeArgs a;
    a.order = native_order(dt);
    a.top = meta.ptr;
    a.yes = d.ptr;
    a.yes_cap = d.bytes / es;
    a.error = w.u32(0);
    launch_merge(SPLIT_NOT_CONST, meta.ptr + es + 1, n, es, a, out.get(), scratch.get(), s);
    uint32_t err[2];
    d2h(&err[0], w.u32(0), 4, s);
    d2h(&err[1], lookback_at(scratch.get(), tiles).error, 4, s);
    check_status_word(err[0], "const decode");
    check_status_word(err[1], "const decode");
    return out;
}

// ------------------------------------------------------------------------------------ patch

// static_cast<T>(double) as the reference's x86 host build evaluates it (cvttsd2si: truncation,
// INT_MIN for NaN / out of range; narrow integers keep the low bits)
uint64_t cast_double_to_T(double d, int dt)
{
    switch (dt) {
    case GTSC_FLOAT: { float f = (float)d; uint32_t u; memcpy(&u, &f, 4); return u; }
    case GTSC_DOUBLE: { uint64_t u; memcpy(&u, &d, 8); return u; }
    case GTSC_TIME:
        if (!(d >= -9223372036854775808.0 && d < 9223372036854775808.0)) return 0x8000000000000000ull;
        return (uint64_t)(int64_t)d;
    default:
        if (!(d > -2147483649.0 && d < 2147483648.0)) return (uint64_t)(int64_t)INT32_MIN;
        return (uint64_t)(int64_t)(int32_t)d;
    }
}

double T_to_double(uint64_t u, int dt)
{
    switch (dt) {
    case GTSC_FLOAT: { float f; uint32_t v = (uint32_t)u; memcpy(&f, &v, 4); return (double)f; }
    case GTSC_DOUBLE: { double d; memcpy(&d, &u, 8); return d; }
    default: return (double)sext(u, dtype_size(dt));
    }
}

// LowerPatchEncoding::GetOperator<T> (compression/patch/lower_patch_encoding.cu:22-31), factor 0.1,
// with min/max as PatchEncodingFactory<T>::Get passes them (patch_encoding_factory.hpp:40-57)
uint64_t lower_patch_threshold(uint64_t mnb, uint64_t mxb, int dt)
{
    volatile double dmin = T_to_double(mnb, dt), dmax = T_to_double(mxb, dt);
    volatile double span = dmax - dmin;
    const uint64_t dist_bits = cast_double_to_T(span, dt);  // T dist = _max - _min;
    double ddist = is_fp(dt) ? T_to_double(dist_bits, dt) : (double)sext(dist_bits, dtype_size(dt));
    volatile double prod = 0.1 * ddist;
    volatile double t = dmax - prod;
    return cast_double_to_T(t, dt);
}

// OutsidePatchEncoding::GetOperator<T> (compression/patch/outside_patch_encoding.cu:22-31), factor
// 0.1: T dist = _max - _min; low = (T)(_min + 0.1 * dist), high = (T)(_max - 0.1 * dist)
void outside_patch_bounds(uint64_t mnb, uint64_t mxb, int dt, uint64_t *lo, uint64_t *hi)
{
    volatile double dmin = T_to_double(mnb, dt), dmax = T_to_double(mxb, dt);
    volatile double span = dmax - dmin;
    const uint64_t dist_bits = cast_double_to_T(span, dt);
    double ddist = is_fp(dt) ? T_to_double(dist_bits, dt) : (double)sext(dist_bits, dtype_size(dt));
    volatile double prod = 0.1 * ddist;
    volatile double l = dmin + prod, h = dmax - prod;
    *lo = cast_double_to_T(l, dt);
    *hi = cast_double_to_T(h, dt);
}

// LowerPatchEncoding::Encode (lower_patch_encoding.cu:33-67) and, with `outside`,
// OutsidePatchEncoding::Encode (outside_patch_encoding.cu:33-60): the stencil is x < t, or the
// OutsideOperator's low <= x <= high (stencil_operators.hpp:14-25; NaN counts as inside); meta = the
// packed stencil, out1 = the stencil-true values, out2 = the rest, both in order
Parts patch_encode(int dt, View in, cudaStream_t s, bool outside)
{
    const int es = dtype_size(dt);
    const uint64_t n = in.bytes / es;
    if (n == 0) return {empty_buf(), empty_buf(), empty_buf()};
    DevBuf keep;
    View src = aligned(in, 16, keep, s);
    uint64_t mnb, mxb;
    column_minmax(src, es, native_order(dt), &mnb, &mxb, s);
    const uint64_t thr = lower_patch_threshold(mnb, mxb, dt);
    DevBuf meta = dev_alloc(1 + stencil_count(n), s);
    uint8_t rest = (uint8_t)(n % 8);
    GTSC_CUDA(cudaMemcpyAsync(meta.get(), &rest, 1, cudaMemcpyHostToDevice, s));
    DevBuf out1 = dev_alloc(n * es, s), out2 = dev_alloc(n * es, s);
    const uint64_t tiles = split_tiles(n);
    DevBuf scratch = dev_alloc(lookback_bytes(tiles), s);
    Words w(s, 1);
    SplitArgs a;
    a.order = native_order(dt);
    a.thr = thr;
    a.outside = outside;
    if (outside) outside_patch_bounds(mnb, mxb, dt, &a.lo, &a.hi);
    a.stencil = meta.get() + 1;
    a.yes = out1.get();
    a.no = out2.get();
    a.yes_count = w.u64(0);
    launch_split(SPLIT_LOWER, src.ptr, n, es, a, scratch.get(), s);
    unsigned long long m = 0;
    d2h(&m, w.u64(0), 8, s);
    uint32_t err;
    d2h(&err, lookback_at(scratch.get(), tiles).error, 4, s);
    check_status_word(err, "patch encode");
    return {meta, shrink(out1, m * es), shrink(out2, (n - m) * es)};
}

// Lower/OutsidePatchEncoding::Decode (lower_patch_encoding.cu:69-94)
DevBuf patch_decode(int dt, View meta, View in1, View in2, cudaStream_t s)
{
    const int es = dtype_size(dt);
    if (in1.bytes == 0 && in2.bytes == 0) return empty_buf();
    const uint64_t n = stencil_elems(meta, s);
    DevBuf k1, k2;
    View y = aligned(in1, es, k1, s), no = aligned(in2, es, k2, s);
    DevBuf out = dev_alloc(n * es, s);
    const uint64_t tiles = split_tiles(n);
    DevBuf scratch = dev_alloc(lookback_bytes(tiles), s);
    Words w(s, 1);
    MergeArgs a;
    a.order = native_order(dt);
    a.yes = y.ptr;
    a.yes_cap = y.bytes / es;
    a.no = no.ptr;
    a.no_cap = no.bytes / es;
    a.error = w.u32(0);
    launch_merge(SPLIT_LOWER, meta.ptr + 1, n, es, a, out.get(), scratch.get(), s);
    uint32_t err[2];
    d2h(&err[0], w.u32(0), 4, s);
    d2h(&err[1], lookback_at(scratch.get(), tiles).error, 4, s);
    check_status_word(err[0], "patch decode");
    check_status_word(err[1], "patch decode");
    return out;
}

// ------------------------------------------------------------------------------------ GFC

// GfcEncoding::Encode (compression/gfc/gfc_encoding.cpp:15-88); integer types use AFL plus an
// empty third stream (gfc_encoding.cpp:119-166)
Parts gfc_encode(int dt, View in, cudaStream_t s)
{
    if (!is_fp(dt)) {
        Parts p = afl_encode(dt, in, s);
        p.push_back(empty_buf());
        return p;
    }
    const int es = dtype_size(dt);
    const uint64_t n = in.bytes / es;
    if (n == 0) return {empty_buf(), empty_buf(), empty_buf()};
    if (n > (uint64_t)INT32_MAX / 9) fail(GTSC_ERR_CAPACITY, "gfc: column too long for 32-bit stream offsets");
    DevBuf keep;
    View src = aligned(in, es, keep, s);
    const GfcGeom g = gfc_geom(dt == GTSC_DOUBLE, n, 0, 0);
    DevBuf layout = dev_alloc(gfc_scratch_layout_bytes(g), s);
    DevBuf ends = dev_alloc(4ull * g.warps, s);
    DevBuf sizes = dev_alloc(4ull * g.warps, s);
    launch_gfc_compress(src.ptr, g, layout.get(), (int32_t *)ends.get(), (int32_t *)sizes.get(), s);
    DevBuf incl = dev_alloc(8ull * g.warps, s);
    const uint64_t tiles = rle_tiles(g.warps);
    DevBuf scratch = dev_alloc(lookback_bytes(tiles), s);
    launch_scan_i32(sizes.get(), g.warps, (unsigned long long *)incl.get(), scratch.get(), s);
    unsigned long long total = 0;
    d2h(&total, (unsigned long long *)incl.get() + g.warps - 1, 8, s);
    DevBuf out2 = dev_alloc(total, s);
    launch_gfc_compact(layout.get(), g, (const int32_t *)sizes.get(), (const unsigned long long *)incl.get(),
                       out2.get(), s);
    int32_t meta[3] = {g.blocks, g.wpb, (int32_t)n};
    DevBuf m = h2d_small(meta, 12, s);
    return {m, ends, out2};
}

// GfcEncoding::Decode (gfc_encoding.cpp:42-108)
DevBuf gfc_decode(int dt, View meta, View in1, View in2, cudaStream_t s)
{
    if (!is_fp(dt)) return afl_decode(dt, meta, in1, s);
    const int es = dtype_size(dt);
    if (in2.bytes == 0) return empty_buf();
    if (meta.bytes < 12) fail(GTSC_ERR_FORMAT, "gfc: metadata too short");
    int32_t m[3];
    d2h(m, meta.ptr, 12, s);
    if (m[0] <= 0 || m[1] <= 0 || m[2] < 0 || (int64_t)m[0] * m[1] > (1ll << 26))
        fail(GTSC_ERR_FORMAT, "gfc: bad geometry in metadata");
    const GfcGeom g = gfc_geom(dt == GTSC_DOUBLE, (uint64_t)m[2], m[0], m[1]);
    if (in1.bytes < 4ull * g.warps) fail(GTSC_ERR_FORMAT, "gfc: offset stream too short");
    Words w(s, 1);
    DevBuf sizes = dev_alloc(4ull * g.warps, s);
    launch_gfc_sizes(in1.ptr, g, (int32_t *)sizes.get(), w.u32(0), s);
    DevBuf incl = dev_alloc(8ull * g.warps, s);
    const uint64_t tiles = rle_tiles(g.warps);
    DevBuf scratch = dev_alloc(lookback_bytes(tiles), s);
    launch_scan_i32(sizes.get(), g.warps, (unsigned long long *)incl.get(), scratch.get(), s);
    DevBuf out = dev_alloc(g.n * es, s);
    launch_gfc_decompress(in2.ptr, in2.bytes, g, (const int32_t *)sizes.get(), (const unsigned long long *)incl.get(),
                          out.get(), w.u32(0), s);
    uint32_t err;
    d2h(&err, w.u32(0), 4, s);
    check_status_word(err, "gfc decode");
    return out;
}

// ------------------------------------------------------------------------------------ floatToInt

const std::array<int, 11> &precision_table(cudaStream_t s)
{
    static std::array<int, 11> table;
    static std::once_flag once;
    std::call_once(once, [s] {
        DevBuf t = dev_alloc(11 * sizeof(int), s);
        launch_log_table((int *)t.get(), s);
        d2h(table.data(), t.get(), 11 * sizeof(int), s);
    });
    return table;
}

const double kPow10[10] = {1e0, 1e1, 1e2, 1e3, 1e4, 1e5, 1e6, 1e7, 1e8, 1e9};

// FloatEncoding::Encode (compression/float/float_encoding.cu:17-57).  Deviation, to stay lossless:
// when any element would not decode to its exact input bits, the p = 10 raw branch is taken.
Parts f2i_encode(int dt, View in, cudaStream_t s)
{
    const int es = dtype_size(dt);
    const uint64_t n = in.bytes / es;
    if (n == 0) return {empty_buf(), empty_buf()};
    DevBuf keep;
    View src = aligned(in, es, keep, s);
    const Order o = native_order(dt);
    const unsigned grid = stats_grid(n);
    DevBuf acc = dev_alloc(sizeof(StatsAcc) + 8ull * grid, s);
    launch_stats(src.ptr, n, es, o, (StatsAcc *)acc.get(), (double *)(acc.get() + sizeof(StatsAcc)), s);
    StatsAcc h;
    d2h(&h, acc.get(), sizeof(h), s);
    int p = precision_table(s)[h.prec_steps > 10 ? 10 : h.prec_steps];
    bool transform = false;
    if (p < 10) {
        uint64_t mnb = 0, mxb = 0;
        if (!minmax_result(h.mm, es, o, &mnb, &mxb)) {
            d2h(&mnb, src.ptr, es, s);
            mxb = mnb;
        }
        const int scale = (int)kPow10[p];
        bool ok;
        if (dt == GTSC_FLOAT) {
            volatile float a = (float)T_to_double(mnb, dt) * (float)scale;
            volatile float b = (float)T_to_double(mxb, dt) * (float)scale;
            ok = a > (float)INT32_MIN && b < (float)INT32_MAX;
        } else if (dt == GTSC_DOUBLE) {
            volatile double a = T_to_double(mnb, dt) * (double)scale, b = T_to_double(mxb, dt) * (double)scale;
            ok = a > (double)INT32_MIN && b < (double)INT32_MAX;
        } else {
            const int64_t a = sext(mnb, es), b = sext(mxb, es);
            ok = a * scale > INT32_MIN && b * scale < INT32_MAX;
        }
        if (ok) transform = true;
        else p = 10;
    }
    DevBuf out;
    if (transform) {
        out = dev_alloc(4 * n, s);
        Words w(s, 1);
        launch_f2i_encode(src.ptr, n, es, o, p, (int32_t *)out.get(), w.u32(0), s);
        uint32_t lossy = 0;
        d2h(&lossy, w.u32(0), 4, s);
        if (lossy) {
            transform = false;
            p = 10;
        }
    }
    if (!transform) {
        const uint64_t bytes = (n * es) / 4 * 4;  // CastSharedCudaPtr<T,int> keeps whole ints
        out = dev_alloc(bytes, s);
        if (bytes) GTSC_CUDA(cudaMemcpyAsync(out.get(), src.ptr, bytes, cudaMemcpyDeviceToDevice, s));
    }
    DevBuf m = h2d_small(&p, 4, s);
    return {m, out};
}

DevBuf f2i_decode(int dt, View meta, View data, cudaStream_t s)
{
    const int es = dtype_size(dt);
    if (data.bytes == 0) return empty_buf();
    if (meta.bytes < 4) fail(GTSC_ERR_FORMAT, "floatToInt: metadata too short");
    int32_t p;
    d2h(&p, meta.ptr, 4, s);
    if (p < 10) {
        if (p < 0) fail(GTSC_ERR_FORMAT, "floatToInt: negative precision");
        const uint64_t n = data.bytes / 4;
        DevBuf keep;
        View d = aligned(data, 4, keep, s);
        DevBuf out = dev_alloc(n * es, s);
        launch_f2i_decode(d.ptr, n, es, native_order(dt), p, out.get(), s);
        return out;
    }
    const uint64_t n = data.bytes / es;
    DevBuf out = dev_alloc(n * es, s);
    if (n) GTSC_CUDA(cudaMemcpyAsync(out.get(), data.ptr, n * es, cudaMemcpyDeviceToDevice, s));
    return out;
}

}  // namespace

// ------------------------------------------------------------------------------------ statistics

Stats column_stats(int dt, View in, cudaStream_t s)
{
    const int es = dtype_size(dt);
    if (!es) fail(GTSC_ERR_ARG, "unknown data type");
    Stats r{};
    const uint64_t n = in.bytes / es;
    r.size = n;
    if (n == 0) return r;
    DevBuf keep;
    View src = aligned(in, es, keep, s);
    const Order o = native_order(dt);
    const unsigned grid = stats_grid(n);
    DevBuf acc = dev_alloc(sizeof(StatsAcc) + 8ull * grid, s);
    double *partials = (double *)(acc.get() + sizeof(StatsAcc));
    launch_stats(src.ptr, n, es, o, (StatsAcc *)acc.get(), partials, s);
    StatsAcc h;
    d2h(&h, acc.get(), sizeof(h), s);
    std::vector<double> fp(grid);
    if (is_fp(dt)) d2h(fp.data(), partials, 8ull * grid, s);
    uint64_t mnb = 0, mxb = 0;
    if (!minmax_result(h.mm, es, o, &mnb, &mxb)) {
        d2h(&mnb, src.ptr, es, s);
        mxb = mnb;
    }
    r.min = T_to_double(mnb, dt);
    r.max = T_to_double(mxb, dt);
    r.min_bit_cnt = 64;  // BITLEN<double> specialisation (core/cuda_macros.cuh:188-189)
    r.precision = precision_table(s)[h.prec_steps > 10 ? 10 : h.prec_steps];
    r.sorted = h.unsorted ? 0 : 1;
    r.rl_metric = n <= 2 ? 1.0f : (float)((double)(int32_t)h.rl_sum / (double)(n - 2));
    if (dt == GTSC_FLOAT) {
        float sum = 0.0f;
        for (unsigned b = 0; b < grid; b++) sum += (float)fp[b];
        r.mean = (double)(float)(sum / (double)n);
    } else if (dt == GTSC_DOUBLE) {
        double sum = 0.0;
        for (unsigned b = 0; b < grid; b++) sum += fp[b];
        r.mean = sum / (double)n;
    } else {
        const uint64_t msk = es == 8 ? ~0ull : ((1ull << (8 * es)) - 1);
        const double q = (double)sext(h.int_sum & msk, es) / (double)n;
        r.mean = T_to_double(cast_double_to_T(q, dt), dt);
    }
    return r;
}

int precision_of_steps(int steps, cudaStream_t s) { return precision_table(s)[steps > 10 ? 10 : steps]; }

int n_results(int enc)
{
    switch (enc) {
    case GTSC_DELTA: case GTSC_AFL: case GTSC_SCALE: case GTSC_UNIQUE: case GTSC_FLOAT_TO_INT: case GTSC_CONST:
        return 1;
    case GTSC_RLE: case GTSC_DICT: case GTSC_PATCH: case GTSC_PATCH_OUTSIDE: case GTSC_GFC: return 2;
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
    switch (enc) {
    case GTSC_AFL: return afl_encode(dt, in, s);
    case GTSC_NONE: return none_encode(in, s);
    case GTSC_DELTA: return delta_encode(dt, in, s);
    case GTSC_SCALE: return scale_encode(dt, in, s);
    case GTSC_RLE: return rle_encode(dt, in, s);
    case GTSC_DICT: return dict_encode(dt, in, s);
    case GTSC_CONST: return const_encode(dt, in, s);
    case GTSC_PATCH: return patch_encode(dt, in, s, false);
    case GTSC_PATCH_OUTSIDE: return patch_encode(dt, in, s, true);
    case GTSC_FLOAT_TO_INT: return f2i_encode(dt, in, s);
    case GTSC_GFC: return gfc_encode(dt, in, s);
    case GTSC_UNIQUE: return unique_encode(dt, in, s);
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
    case GTSC_DELTA: return delta_decode(dt, v[0], v[1], s);
    case GTSC_SCALE: return scale_decode(dt, v[0], v[1], s);
    case GTSC_RLE: return rle_decode(dt, v[0], v[1], v[2], s);
    case GTSC_DICT: return dict_decode(dt, v[0], v[1], v[2], s);
    case GTSC_CONST: return const_decode(dt, v[0], v[1], s);
    case GTSC_PATCH: case GTSC_PATCH_OUTSIDE: return patch_decode(dt, v[0], v[1], v[2], s);
    case GTSC_FLOAT_TO_INT: return f2i_decode(dt, v[0], v[1], s);
    case GTSC_GFC: return gfc_decode(dt, v[0], v[1], v[2], s);
    case GTSC_UNIQUE: return unique_decode(dt, v[0], v[1], s);
    default: fail(GTSC_ERR_UNSUPPORTED, "encoding not available");
    }
}

}  // namespace gtsc
