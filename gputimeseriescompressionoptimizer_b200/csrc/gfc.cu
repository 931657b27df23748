// gfc.cu -- GFC lossless float compression (GfcEncoding, compression/gfc/gfc_encoding.cpp:15-108;
// kernels compression/gfc/gfc_encoding_impl_double.cu:31-148 and gfc_encoding_impl_float.cu:25-145).
//
// Stream layout (kept byte-identical): the column is padded to a multiple of 32 and cut into
// per-warp chunks of `per` values; each chunk is a run of 32-value subchunks.  A subchunk is 16
// header bytes (a nibble per lane: sign bit | byte-count code) followed by each lane's
// |x - last| in its minimal number of little-endian bytes, lanes in order.  `last` is 0 for the
// first subchunk of a chunk and the chunk's 32nd value afterwards (impl_double.cu:86).
//
// The reference computes the lane byte offsets with a shared-memory scan that relies on implicit
// warp synchrony (impl_double.cu:20-29), which is not valid on sm_70+; here they are exact
// __shfl_up_sync scans.  It then compacts the chunks with one cudaMemcpy per chunk
// (impl_double.cu:219-231); here a scan of the chunk sizes and one copy kernel do it.
#include "kernels.hpp"
#include "scan.cuh"
#include "vec.cuh"

namespace gtsc {

namespace {

constexpr int G_THREADS = 256;  // 8 warps per block, one chunk per warp

__device__ __forceinline__ uint64_t cut_at(const GfcGeom &g, int64_t i)
{
    uint64_t c = (uint64_t)(i + 1) * g.per;
    return c < g.npad ? c : g.npad;
}
__device__ __forceinline__ uint64_t chunk_begin(const GfcGeom &g, int64_t w) { return w ? cut_at(g, w - 1) : 0; }
__device__ __forceinline__ uint64_t scratch_start(const GfcGeom &g, int64_t w)
{
    return (chunk_begin(g, w) + 1) / 2 * (uint64_t)g.unit;
}

template <bool DBL>
__global__ void __launch_bounds__(G_THREADS)
k_gfc_compress(const uint8_t *__restrict__ in, GfcGeom g, uint8_t *__restrict__ scratch,
               int32_t *__restrict__ ends, int32_t *__restrict__ sizes)
{
    const int lane = threadIdx.x & 31;
    const int64_t w = ((int64_t)blockIdx.x * G_THREADS + threadIdx.x) >> 5;
    if (w >= g.warps) return;
    const uint64_t cb = chunk_begin(g, w), ce = cut_at(g, w);
    const uint64_t start = scratch_start(g, w);
    uint64_t off = start;
    uint64_t last = 0;
    for (uint64_t s = cb; s < ce; s += 32) {
        const uint64_t i = s + lane;
        uint64_t x = 0;
        if (i < g.n) x = DBL ? ld_elem<8>(in, i) : ld_elem<4>(in, i);
        uint64_t diff;
        uint32_t sign, mb, code;
        if (DBL) {
            diff = x - last;
            sign = (uint32_t)((diff >> 60) & 8);
            if (sign) diff = 0ull - diff;
            const uint32_t lz = (uint32_t)__clzll((long long)diff) >> 3;
            mb = lz == 6 ? 3 : 8 - lz;
            code = mb >= 3 ? mb - 1 : mb;
        } else {
            uint32_t d = (uint32_t)x - (uint32_t)last;
            sign = (d >> 28) & 8;
            if (sign) d = 0u - d;
            mb = 4 - ((uint32_t)__clz((int)d) >> 3);
            code = mb;
            diff = d;
        }
        const uint32_t nib = sign | code;
        // exclusive scan of byte counts across the warp
        uint32_t incl = mb;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        const uint32_t excl = incl - mb;
        const uint32_t prev_nib = __shfl_up_sync(0xffffffffu, nib, 1);
        if (lane & 1) scratch[off + (lane >> 1)] = (uint8_t)(prev_nib | (nib << 4));
        uint8_t *dst = scratch + off + 16 + excl;
        for (uint32_t b = 0; b < mb; b++) dst[b] = (uint8_t)(diff >> (8 * b));
        off += 16 + total;
        if (s == cb) last = __shfl_sync(0xffffffffu, x, 31);
    }
    if (lane == 31) {
        ends[w] = (int32_t)off;
        sizes[w] = (int32_t)(off - start);
    }
}

// copies chunk w's payload from the scratch layout to its compacted position
__global__ void __launch_bounds__(G_THREADS)
k_gfc_compact(const uint8_t *__restrict__ scratch, GfcGeom g, const int32_t *__restrict__ sizes,
              const unsigned long long *__restrict__ incl, uint8_t *__restrict__ out)
{
    const int lane = threadIdx.x & 31;
    const int64_t w = ((int64_t)blockIdx.x * G_THREADS + threadIdx.x) >> 5;
    if (w >= g.warps) return;
    const uint64_t size = (uint64_t)sizes[w];
    const uint64_t dst0 = incl[w] - size;
    const uint8_t *src = scratch + scratch_start(g, w);
    for (uint64_t b = lane; b < size; b += 32) out[dst0 + b] = src[b];
}

// sizes of the chunks of a stream from its absolute end offsets (out1)
__global__ void k_gfc_sizes(const uint8_t *__restrict__ ends, GfcGeom g, int32_t *__restrict__ sizes,
                            uint32_t *__restrict__ error)
{
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= g.warps) return;
    const int64_t e = (int32_t)ld_unaligned<4>(ends + 4 * w);
    const int64_t sz = e - (int64_t)scratch_start(g, w);
    const uint64_t subs = (cut_at(g, w) - chunk_begin(g, w)) / 32;
    const int64_t max_sz = (int64_t)(subs * (16 + 32 * (g.dbl ? 8 : 4)));
    if (sz < 0 || sz > max_sz) atomicExch(error, (uint32_t)(-GTSC_ERR_FORMAT));
    sizes[w] = sz < 0 ? 0 : (int32_t)sz;
}

template <bool DBL>
__global__ void __launch_bounds__(G_THREADS)
k_gfc_decompress(const uint8_t *__restrict__ payload, uint64_t payload_bytes, GfcGeom g,
                 const int32_t *__restrict__ sizes, const unsigned long long *__restrict__ incl,
                 uint8_t *__restrict__ out, uint32_t *__restrict__ error)
{
    const int lane = threadIdx.x & 31;
    const int64_t w = ((int64_t)blockIdx.x * G_THREADS + threadIdx.x) >> 5;
    if (w >= g.warps) return;
    const uint64_t cb = chunk_begin(g, w), ce = cut_at(g, w);
    const uint64_t size = (uint64_t)sizes[w];
    const uint64_t end = incl[w];
    if (end > payload_bytes || end < size) {
        if (lane == 0) atomicExch(error, (uint32_t)(-GTSC_ERR_FORMAT));
        return;
    }
    uint64_t pos = end - size;
    uint64_t last = 0;
    for (uint64_t s = cb; s < ce; s += 32) {
        if (pos + 16 > end) {
            if (lane == 0) atomicExch(error, (uint32_t)(-GTSC_ERR_FORMAT));
            return;
        }
        const uint32_t hb = __ldg(payload + pos + (lane >> 1));
        const uint32_t nib = (hb >> (4 * (lane & 1))) & 15u;
        const uint32_t code = nib & 7u;
        uint32_t mb = DBL ? (code >= 2 ? code + 1 : code) : code;
        if (!DBL && mb > 4) {
            atomicExch(error, (uint32_t)(-GTSC_ERR_FORMAT));
            mb = 4;
        }
        uint32_t incl_b = mb;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, incl_b, o);
            if (lane >= o) incl_b += y;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl_b, 31);
        if (pos + 16 + total > end) {
            if (lane == 0) atomicExch(error, (uint32_t)(-GTSC_ERR_FORMAT));
            return;
        }
        const uint8_t *src = payload + pos + 16 + (incl_b - mb);
        uint64_t diff = 0;
        for (int b = (int)mb - 1; b >= 0; b--) diff = (diff << 8) | __ldg(src + b);
        if (nib & 8u) diff = 0ull - diff;
        uint64_t x = last + diff;
        if (!DBL) x &= 0xffffffffull;
        const uint64_t i = s + lane;
        if (i < g.n) {
            if (DBL) st_elem<8>(out, i, x);
            else st_elem<4>(out, i, x);
        }
        pos += 16 + total;
        if (s == cb) last = __shfl_sync(0xffffffffu, x, 31);
    }
    if (lane == 0 && pos != end) atomicExch(error, (uint32_t)(-GTSC_ERR_FORMAT));
}

unsigned g_grid(int64_t warps) { return (unsigned)((warps * 32 + G_THREADS - 1) / G_THREADS); }

}  // namespace

GfcGeom gfc_geom(bool dbl, uint64_t n, int blocks, int wpb)
{
    GfcGeom g;
    g.dbl = dbl;
    g.n = n;
    g.npad = (n + 31) & ~31ull;
    g.unit = dbl ? 17 : 9;
    if (blocks > 0) {
        g.blocks = blocks;
        g.wpb = wpb;
    } else {
        g.wpb = dbl ? 16 : 32;                      // gfc_encoding.cpp:30-33, 77-80
        const uint64_t sub = dbl ? 64 : 32;
        const uint64_t bs = (uint64_t)g.wpb * sub * 32;
        g.blocks = (int)((n + bs - 1) / bs);
    }
    g.warps = (int64_t)g.blocks * g.wpb;
    uint64_t per = g.warps ? (g.npad + g.warps - 1) / g.warps : 32;  // impl_double.cu:170-172
    if (per < 32) per = 32;
    g.per = (per + 31) & ~31ull;
    return g;
}

uint64_t gfc_scratch_layout_bytes(const GfcGeom &g) { return (g.npad + 1) / 2 * g.unit + 64; }

void launch_gfc_compress(const uint8_t *in, const GfcGeom &g, uint8_t *layout, int32_t *ends, int32_t *sizes,
                         cudaStream_t s)
{
    if (g.warps == 0) return;
    if (g.dbl) k_gfc_compress<true><<<g_grid(g.warps), G_THREADS, 0, s>>>(in, g, layout, ends, sizes);
    else k_gfc_compress<false><<<g_grid(g.warps), G_THREADS, 0, s>>>(in, g, layout, ends, sizes);
    GTSC_CUDA(cudaGetLastError());
}

void launch_gfc_compact(const uint8_t *layout, const GfcGeom &g, const int32_t *sizes,
                        const unsigned long long *incl, uint8_t *out, cudaStream_t s)
{
    if (g.warps == 0) return;
    k_gfc_compact<<<g_grid(g.warps), G_THREADS, 0, s>>>(layout, g, sizes, incl, out);
    GTSC_CUDA(cudaGetLastError());
}

void launch_gfc_sizes(const uint8_t *ends, const GfcGeom &g, int32_t *sizes, uint32_t *error, cudaStream_t s)
{
    if (g.warps == 0) return;
    k_gfc_sizes<<<(unsigned)((g.warps + 255) / 256), 256, 0, s>>>(ends, g, sizes, error);
    GTSC_CUDA(cudaGetLastError());
}

void launch_gfc_decompress(const uint8_t *payload, uint64_t payload_bytes, const GfcGeom &g, const int32_t *sizes,
                           const unsigned long long *incl, uint8_t *out, uint32_t *error, cudaStream_t s)
{
    if (g.warps == 0) return;
    if (g.dbl)
        k_gfc_decompress<true><<<g_grid(g.warps), G_THREADS, 0, s>>>(payload, payload_bytes, g, sizes, incl, out, error);
    else
        k_gfc_decompress<false><<<g_grid(g.warps), G_THREADS, 0, s>>>(payload, payload_bytes, g, sizes, incl, out, error);
    GTSC_CUDA(cudaGetLastError());
}

}  // namespace gtsc
