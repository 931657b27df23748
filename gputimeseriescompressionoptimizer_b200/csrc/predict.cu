// predict.cu -- Encoding::GetMetadataSize / GetCompressedSize of every encoding (the size
// predictors of compression/*/ *.hpp and *.cu): the byte sizes of [metadata] and of the data
// outputs together, from counting passes instead of an encode.
//
//   none        8, n*es                                        none_encoding.hpp:36-44
//   delta       es, (n-1)*es                                   delta_encoding.hpp:36-46
//   scale       es, n*es                                       scale_encoding.hpp:31-41
//   floatToInt  4, n*es                                        float_encoding.hpp:33-43
//   patch       ceil(n/8)+1, n*es                              patch_encoding.hpp:36-46
//   gfc         12, 0                                          gfc_encoding.hpp:31-35
//   rle         4, runs*(4+es)                                 rle_encode.cu:64-97
//   dict        ceil(n/8)+1, 16 + 4*es + 4*ceil(top/16) + (n-top)*es   dict_encoding.cu:132-161
//   const       ceil(n/8)+es+1, (n-matches)*es                 const_encoding.hpp:32-37, .cu:133-155
//   afl         4 (float: 9), ceil(b*n/W)*es (float: both AFL streams + 8)   afl_encoding.cu:281-343
//   unique      16 + m*es, 4*ceil(n/(32/ALT_BITLEN(m-1)))      unique_encoding.cu:306-326
// An empty column predicts 0 bytes except none (8), gfc (12) and dict (1) metadata, as the
// reference's formulas give (its rle encoder still emits a 4-byte count there).  runs, top,
// matches and m count with the same equality the encoders use (raw bits; NaN equals nothing), so
// the exact predictors equal the encoders' output sizes.  The reference defines rle/dict/const/afl predictors for int and
// float only and throws otherwise; these cover every data type with the same formulas in T units.
#include "encodings.hpp"
#include "kernels.hpp"
#include "predict.hpp"
#include "vec.cuh"

namespace gtsc {

namespace {

__device__ __forceinline__ bool same_bits(uint64_t a, uint64_t b, Order o) { return a == b && !is_nan_bits(a, o); }

// number of i with i == 0 or x[i] != x[i-1]
template <int ES>
__global__ void k_count_heads(const uint8_t *__restrict__ in, uint64_t n, Order o, unsigned long long *cnt)
{
    unsigned long long c = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        c += (i == 0 || !same_bits(ld_elem<ES>(in, i), ld_elem<ES>(in, i - 1), o)) ? 1 : 0;
    for (int d = 16; d; d >>= 1) c += __shfl_down_sync(0xffffffffu, c, d);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(cnt, c);
}

// number of elements equal to one of top[0..k)
template <int ES>
__global__ void k_count_matches(const uint8_t *__restrict__ in, uint64_t n, Order o, const uint8_t *__restrict__ top,
                                int k, unsigned long long *cnt)
{
    uint64_t t[4];
#pragma unroll
    for (int j = 0; j < 4; j++) t[j] = j < k ? ld_unaligned<ES>(top + (uint64_t)j * ES) : 0;
    unsigned long long c = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v = ld_elem<ES>(in, i);
        bool hit = false;
#pragma unroll
        for (int j = 0; j < 4; j++) hit |= j < k && same_bits(v, t[j], o);
        c += hit ? 1 : 0;
    }
    for (int d = 16; d; d >>= 1) c += __shfl_down_sync(0xffffffffu, c, d);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(cnt, c);
}

unsigned count_grid(uint64_t n)
{
    const uint64_t b = (n + 255) / 256;
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(b, (uint64_t)sm_count() * 8));
}

uint64_t count_heads(View in, int es, Order o, cudaStream_t s)
{
    const uint64_t n = in.bytes / es;
    DevBuf c = dev_alloc(8, s);
    GTSC_CUDA(cudaMemsetAsync(c.get(), 0, 8, s));
    auto *cp = (unsigned long long *)c.get();
    switch (es) {
    case 1: k_count_heads<1><<<count_grid(n), 256, 0, s>>>(in.ptr, n, o, cp); break;
    case 2: k_count_heads<2><<<count_grid(n), 256, 0, s>>>(in.ptr, n, o, cp); break;
    case 4: k_count_heads<4><<<count_grid(n), 256, 0, s>>>(in.ptr, n, o, cp); break;
    default: k_count_heads<8><<<count_grid(n), 256, 0, s>>>(in.ptr, n, o, cp); break;
    }
    GTSC_CUDA(cudaGetLastError());
    unsigned long long h = 0;
    d2h(&h, cp, 8, s);
    return h;
}

// elements equal to one of the k most frequent values (k <= 4; the encoders' top-k)
uint64_t count_top(View in, int es, Order o, int k, cudaStream_t s)
{
    const uint64_t n = in.bytes / es;
    DevBuf top = dev_alloc(4 * 8 + 8, s);
    auto *cp = (unsigned long long *)(top.get() + 32);
    GTSC_CUDA(cudaMemsetAsync(top.get(), 0, 40, s));
    for (bool full : {false, true}) {
        const uint64_t cap = hist_cap_for(n, full);
        const int grid = hist_grid(n);
        DevBuf scratch = dev_alloc(hist_scratch_bytes(cap, grid), s);
        const HistTable t = hist_table_at(scratch.get(), cap, grid);
        launch_hist_topk(in.ptr, n, es, o, k, t, grid, top.get(), nullptr, s);
        uint32_t ov = 0;
        d2h(&ov, t.overflow, 4, s);
        if (!ov || full) break;
    }
    switch (es) {
    case 1: k_count_matches<1><<<count_grid(n), 256, 0, s>>>(in.ptr, n, o, top.get(), k, cp); break;
    case 2: k_count_matches<2><<<count_grid(n), 256, 0, s>>>(in.ptr, n, o, top.get(), k, cp); break;
    case 4: k_count_matches<4><<<count_grid(n), 256, 0, s>>>(in.ptr, n, o, top.get(), k, cp); break;
    default: k_count_matches<8><<<count_grid(n), 256, 0, s>>>(in.ptr, n, o, top.get(), k, cp); break;
    }
    GTSC_CUDA(cudaGetLastError());
    unsigned long long h = 0;
    d2h(&h, cp, 8, s);
    return h;
}

// BITLEN of a column's min / max (AflEncoding's b)
int afl_bits(const uint8_t *p, uint64_t n, int es, cudaStream_t s)
{
    DevBuf acc = dev_alloc(sizeof(MinMaxAcc), s);
    GTSC_CUDA(cudaMemsetAsync(acc.get(), 0, sizeof(MinMaxAcc), s));
    launch_minmax(p, n, es, ORD_INT, (MinMaxAcc *)acc.get(), s);
    MinMaxAcc h;
    d2h(&h, acc.get(), sizeof(h), s);
    uint64_t mn = 0, mx = 0;
    minmax_result(h, es, ORD_INT, &mn, &mx);
    return bitlen_signed(sext(mn, es), sext(mx, es), es);
}

int alt_bitlen_u(uint64_t v)
{
    if (v > 0x7fffffffull) return 32;
    int r = 0;
    while (v >> 1) { v >>= 1; r++; }
    return r + 1;
}

}  // namespace

SizePrediction predict_sizes(int enc, int dt, View in, cudaStream_t s)
{
    const int es = dtype_size(dt);
    if (!es) fail(GTSC_ERR_ARG, "unknown data type");
    if (in.bytes % es) fail(GTSC_ERR_ARG, "predict: input is not a whole number of elements");
    const uint64_t n = in.bytes / es, bytes = in.bytes;
    const Order o = native_order(dt);
    if (enc == GTSC_NONE) return {8, bytes};
    if (enc == GTSC_GFC) return {12, 0};          // no empty guard in the reference
    if (n == 0) return {enc == GTSC_DICT ? 1u : 0u, 0};  // dict_encoding.hpp:44-48 has none either
    DevBuf keep;
    if ((uintptr_t)in.ptr % 16) {  // the counting kernels read whole elements
        keep = dev_alloc(bytes, s);
        GTSC_CUDA(cudaMemcpyAsync(keep.get(), in.ptr, bytes, cudaMemcpyDeviceToDevice, s));
        in = View(keep);
    }
    const uint64_t stencil = (n + 7) / 8 + 1;
    switch (enc) {
    case GTSC_DELTA: return {(uint64_t)es, bytes - es};
    case GTSC_SCALE: return {(uint64_t)es, bytes};
    case GTSC_FLOAT_TO_INT: return {4, bytes};
    case GTSC_PATCH: case GTSC_PATCH_OUTSIDE: return {stencil, bytes};
    case GTSC_RLE: return {4, count_heads(in, es, o, s) * (4 + es)};
    case GTSC_DICT: {
        const uint64_t top = count_top(in, es, o, 4, s);
        return {stencil, 16 + 4ull * es + 4 * ((top + 15) / 16) + (n - top) * es};
    }
    case GTSC_CONST: return {stencil + es, (n - count_top(in, es, o, 1, s)) * es};
    case GTSC_AFL: {
        if (dt == GTSC_DOUBLE) fail(GTSC_ERR_TYPE, "afl: double columns are not supported");
        if (dt != GTSC_FLOAT) {
            const uint64_t W = 8ull * es;
            return {4, (afl_bits(in.ptr, n, es, s) * n + W - 1) / W * es};
        }
        DevBuf parts = dev_alloc(8 * n + (n + 7) / 8 + 16, s);
        DevBuf flags = dev_alloc(4, s);
        GTSC_CUDA(cudaMemsetAsync(flags.get(), 0, 4, s));
        int32_t *mant = (int32_t *)parts.get(), *expo = mant + n;
        launch_float_split(in.ptr, n, mant, expo, parts.get() + 8 * n, (uint32_t *)flags.get(), s);
        const uint64_t bm = afl_bits((const uint8_t *)mant, n, 4, s), be = afl_bits((const uint8_t *)expo, n, 4, s);
        return {9, (bm * n + 31) / 32 * 4 + (be * n + 31) / 32 * 4 + 8};
    }
    case GTSC_UNIQUE: {
        const uint64_t m = unique_count(dt, in, s);
        const int per = 32 / alt_bitlen_u(m - 1);
        return {16 + m * es, (n + per - 1) / per * 4};
    }
    default: fail(GTSC_ERR_UNSUPPORTED, "predict: unknown encoding");
    }
}

}  // namespace gtsc
