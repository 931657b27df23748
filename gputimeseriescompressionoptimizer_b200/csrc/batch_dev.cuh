// batch_dev.cuh -- device helpers shared by the batched pass kernels.
#pragma once

#include "batch.hpp"
#include "kernels.hpp"
#include "scan.cuh"
#include "vec.cuh"

namespace gtsc {

constexpr int kBThreads = 256;
static_assert(kBTile == kBThreads * kBVPT, "tile = threads x values per thread");

// Loads elements [base, base + VPT) of a stream (zeros past n): 16-byte vector loads when the
// whole run is in range and the stream is 16-byte aligned, else element loads (byte loads when
// the stream is not even element aligned, as streams inside a blob may be).
template <int ES, int VPT>
__device__ __forceinline__ void load_run(const uint8_t *p, uint64_t base, uint64_t n, uint64_t (&v)[VPT])
{
    if (base + VPT <= n && ((uintptr_t)p & 15) == 0) {
        constexpr int PER = 16 / ES;
        static_assert(VPT % PER == 0, "a run is whole 16-byte chunks");
#pragma unroll
        for (int c = 0; c < VPT / PER; c++) {
            const uint4 q = ld_chunk(p + (base + (uint64_t)c * PER) * ES);
#pragma unroll
            for (int j = 0; j < PER; j++) v[c * PER + j] = chunk_elem<ES>(q, j);
        }
    } else if (((uintptr_t)p & (ES - 1)) == 0) {
#pragma unroll
        for (int j = 0; j < VPT; j++) v[j] = base + j < n ? ld_elem<ES>(p, base + j) : 0;
    } else {
#pragma unroll
        for (int j = 0; j < VPT; j++) v[j] = base + j < n ? ld_unaligned<ES>(p + (base + j) * ES) : 0;
    }
}

// element i of a shared-memory array of ES-byte elements
template <int ES>
__device__ __forceinline__ uint64_t ld_elem_sm(const uint8_t *sm, uint64_t i)
{
    if (ES == 1) return sm[i];
    if (ES == 2) return ((const uint16_t *)sm)[i];
    if (ES == 4) return ((const uint32_t *)sm)[i];
    return ((const unsigned long long *)sm)[i];
}

// element i of a stream that may not be element aligned (streams inside a blob)
template <int ES>
__device__ __forceinline__ uint64_t ld_elem_any(const uint8_t *p, uint64_t i, bool aligned)
{
    return aligned ? ld_elem<ES>(p, i) : ld_unaligned<ES>(p + i * ES);
}

// Stores elements [base, min(base + VPT, n)) to an element-aligned stream (16-byte stores when the
// whole run is in range and the stream is 16-byte aligned).
template <int ES, int VPT>
__device__ __forceinline__ void store_run(uint8_t *p, uint64_t base, uint64_t n, const uint64_t (&v)[VPT])
{
    if (base + VPT <= n && ((uintptr_t)p & 15) == 0) {
        constexpr int PER = 16 / ES;
#pragma unroll
        for (int c = 0; c < VPT / PER; c++)
            reinterpret_cast<uint4 *>(p + (base + (uint64_t)c * PER) * ES)[0] = make_chunk<ES>(v + c * PER);
    } else {
#pragma unroll
        for (int j = 0; j < VPT; j++)
            if (base + j < n) st_elem<ES>(p, base + j, v[j]);
    }
}

// ------------------------------------------------------------------------------- warp exchange
// A warp's 32 * VPT consecutive elements pass between the blocked arrangement of the scan passes
// (lane l holds elements [VPT l, VPT l + VPT) of the warp's run) and a striped one (the warp's k-th
// access covers 32 consecutive 16-byte chunks) through a per-warp shared-memory tile.  A blocked
// 16-byte access by a warp touches one half of 32 different sectors; the striped access touches
// whole consecutive sectors, with a quarter of the L2 requests.  The tile holds one row of VPT
// elements per lane; the 16-byte chunks of row r are permuted by an XOR with (r / G) mod (chunks
// per row), G = 8 / chunks per row, so that the blocked accesses of eight consecutive lanes (one
// shared-memory wavefront of 16-byte accesses) fall in eight distinct 16-byte bank groups, while a
// striped access still covers whole rows.  The warp's lanes all take part; no block barrier is
// involved.  `xs` is the block's exchange area (16-byte aligned, kXchgBlockBytes), one tile per
// warp.  Used where it measured faster: the RLE expansion's output and the split's and RLE heads'
// source runs.  Not in the delta decode: there it sped up the many-column step but slowed one long
// column's decode by a quarter (its stores leave the block later, and one column's tiles form a
// single look-back chain).
constexpr int kXchgWarpBytes = 32 * (int)kBVPT * 8;
constexpr int kXchgBlockBytes = kBThreads / 32 * kXchgWarpBytes;

template <int ES, int VPT>
__device__ __forceinline__ uint8_t *xchg_tile(uint8_t *xs)
{
    static_assert(32 * VPT * ES <= kXchgWarpBytes, "exchange tile too small");
    static_assert((VPT * ES) % 16 == 0 && VPT * ES / 16 <= 8, "a lane's row is 1 to 8 whole 16-byte chunks");
    return xs + (threadIdx.x >> 5) * kXchgWarpBytes;
}

// byte offset of 16-byte chunk c of row r in a warp's tile
template <int ES, int VPT>
__device__ __forceinline__ uint32_t xchg_chunk(uint32_t r, uint32_t c)
{
    constexpr uint32_t CPR = VPT * ES / 16, G = 8 / CPR;
    return (r * CPR + (c ^ ((r / G) & (CPR - 1)))) * 16;
}

// byte offset of 16-byte chunk q of the warp's run
template <int ES, int VPT>
__device__ __forceinline__ uint32_t xchg_chunk_at(uint32_t q)
{
    constexpr uint32_t CPR = VPT * ES / 16;
    return xchg_chunk<ES, VPT>(q / CPR, q % CPR);
}

// Elements [wb, wb + 32 VPT) of a 16-byte aligned stream (the run lies inside it and wb * ES is a
// multiple of 16) into the blocked arrangement, loaded as 32 consecutive 16-byte chunks per access.
template <int ES, int VPT>
__device__ __forceinline__ void load_run_warp(const uint8_t *p, uint64_t wb, uint64_t (&v)[VPT], uint8_t *xs)
{
    constexpr int PER = 16 / ES, CPR = VPT * ES / 16;
    uint8_t *w = xchg_tile<ES, VPT>(xs);
    const uint32_t lane = threadIdx.x & 31;
    const uint4 *src = reinterpret_cast<const uint4 *>(p + wb * ES);
    __syncwarp();  // earlier reads of the tile by other lanes are done
#pragma unroll
    for (int k = 0; k < CPR; k++) {
        const uint32_t q = 32 * k + lane;
        *reinterpret_cast<uint4 *>(w + xchg_chunk_at<ES, VPT>(q)) = ldg(src + q);
    }
    __syncwarp();
#pragma unroll
    for (int c = 0; c < CPR; c++) {
        const uint4 q = *reinterpret_cast<const uint4 *>(w + xchg_chunk<ES, VPT>(lane, c));
#pragma unroll
        for (int j = 0; j < PER; j++) v[c * PER + j] = chunk_elem<ES>(q, j);
    }
}

// Elements [wb, wb + 32 VPT) of a 16-byte aligned stream (the run lies inside it and wb * ES is a
// multiple of 16) from the blocked arrangement, stored as 32 consecutive 16-byte chunks per access.
template <int ES, int VPT>
__device__ __forceinline__ void store_run_warp(uint8_t *p, uint64_t wb, const uint64_t (&v)[VPT], uint8_t *xs)
{
    constexpr int PER = 16 / ES, CPR = VPT * ES / 16;
    uint8_t *w = xchg_tile<ES, VPT>(xs);
    const uint32_t lane = threadIdx.x & 31;
    __syncwarp();  // earlier reads of the tile by other lanes are done
#pragma unroll
    for (int c = 0; c < CPR; c++)
        *reinterpret_cast<uint4 *>(w + xchg_chunk<ES, VPT>(lane, c)) = make_chunk<ES>(v + c * PER);
    __syncwarp();
    uint4 *dst = reinterpret_cast<uint4 *>(p + wb * ES);
#pragma unroll
    for (int k = 0; k < CPR; k++) {
        const uint32_t q = 32 * k + lane;
        dst[q] = *reinterpret_cast<const uint4 *>(w + xchg_chunk_at<ES, VPT>(q));
    }
}

__device__ __forceinline__ void set_status(uint32_t *status, gtsc_status code)
{
    atomicCAS(status, 0u, (uint32_t)(-code));
}

__device__ __forceinline__ bool bsame(uint64_t a, uint64_t b, Order o) { return a == b && !is_nan_bits(a, o); }

__device__ __forceinline__ uint64_t wrap_es(uint64_t v, int es) { return es == 8 ? v : (v & ((1ull << (8 * es)) - 1)); }

// block-wide min/max of order keys (all threads call; result valid in thread 0)
__device__ __forceinline__ void block_minmax(uint64_t &kmin, uint64_t &kmax)
{
    __shared__ uint64_t smin[kBThreads / 32], smax[kBThreads / 32];
    for (int off = 16; off > 0; off >>= 1) {
        const uint64_t a = __shfl_xor_sync(0xffffffffu, kmin, off);
        const uint64_t b = __shfl_xor_sync(0xffffffffu, kmax, off);
        kmin = a < kmin ? a : kmin;
        kmax = b > kmax ? b : kmax;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { smin[warp] = kmin; smax[warp] = kmax; }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int w = 1; w < kBThreads / 32; w++) {
            kmin = smin[w] < kmin ? smin[w] : kmin;
            kmax = smax[w] > kmax ? smax[w] : kmax;
        }
    __syncthreads();
}

// raw bits of min / max from an accumulator; false when nothing (non-NaN) was seen
__device__ __forceinline__ bool acc_minmax(const MinMaxAcc *acc, int es, Order o, uint64_t &mn, uint64_t &mx)
{
    const unsigned long long a = acc->nkmin, b = acc->kmax;
    if (a == 0 && b == 0) return false;
    mn = order_unkey(~(uint64_t)a, es, o);
    mx = order_unkey(b, es, o);
    return true;
}

// ScaleEncoding's min with the overflow rule of scale_encoding.cu:49-50 (x86 wrap for int/long)
__device__ __forceinline__ uint64_t scale_min(uint64_t mnb, uint64_t mxb, int es)
{
    int64_t mn = sext(mnb, es), mx = sext(mxb, es);
    if (mn < 0) {
        if (es <= 2) {
            const int64_t tmax = es == 1 ? 127 : 32767;
            if ((tmax - mx) < (mn < 0 ? -mn : mn)) mn = 0;
        } else {
            const uint64_t msk = es == 8 ? ~0ull : ((1ull << (8 * es)) - 1);
            const uint64_t tmax = msk >> 1;
            const int64_t diff = sext((tmax - (uint64_t)mx) & msk, es);
            const int64_t absmn = sext((0 - (uint64_t)mn) & msk, es);
            if (diff < absmn) mn = 0;
        }
    }
    return wrap_es((uint64_t)mn, es);
}

// static_cast<T>(double) as the reference's x86 host build evaluates it (cvttsd2si)
__device__ __forceinline__ uint64_t d_cast_double_to_T(double d, int dt, int es)
{
    if (dt == GTSC_FLOAT) return __float_as_uint(__double2float_rn(d));
    if (dt == GTSC_DOUBLE) return (uint64_t)__double_as_longlong(d);
    if (dt == GTSC_TIME) {
        if (!(d >= -9223372036854775808.0 && d < 9223372036854775808.0)) return 0x8000000000000000ull;
        return (uint64_t)__double2ll_rz(d);
    }
    (void)es;
    if (!(d > -2147483649.0 && d < 2147483648.0)) return (uint64_t)(int64_t)INT32_MIN;
    return (uint64_t)(int64_t)__double2int_rz(d);
}
__device__ __forceinline__ double d_T_to_double(uint64_t u, int dt, int es)
{
    if (dt == GTSC_FLOAT) return (double)__uint_as_float((uint32_t)u);
    if (dt == GTSC_DOUBLE) return __longlong_as_double((long long)u);
    if (dt == GTSC_TIME) return __ll2double_rn((long long)u);
    return (double)sext(u, es);
}
// LowerPatchEncoding::GetOperator<T> (lower_patch_encoding.cu:22-31), factor 0.1, x86 casts
__device__ __forceinline__ uint64_t d_patch_threshold(uint64_t mnb, uint64_t mxb, int dt, int es)
{
    const double dmin = d_T_to_double(mnb, dt, es), dmax = d_T_to_double(mxb, dt, es);
    const uint64_t dist_bits = d_cast_double_to_T(__dsub_rn(dmax, dmin), dt, es);
    const double ddist = (dt == GTSC_FLOAT || dt == GTSC_DOUBLE) ? d_T_to_double(dist_bits, dt, es)
                                                                   : (double)sext(dist_bits, es);
    return d_cast_double_to_T(__dsub_rn(dmax, __dmul_rn(0.1, ddist)), dt, es);
}

// OutsidePatchEncoding::GetOperator<T> (outside_patch_encoding.cu:22-31), factor 0.1, x86 casts:
// low = (T)(min + 0.1 * dist), high = (T)(max - 0.1 * dist) with T dist = max - min
__device__ __forceinline__ void d_outside_patch_bounds(uint64_t mnb, uint64_t mxb, int dt, int es, uint64_t &lo,
                                                       uint64_t &hi)
{
    const double dmin = d_T_to_double(mnb, dt, es), dmax = d_T_to_double(mxb, dt, es);
    const uint64_t dist_bits = d_cast_double_to_T(__dsub_rn(dmax, dmin), dt, es);
    const double ddist = (dt == GTSC_FLOAT || dt == GTSC_DOUBLE) ? d_T_to_double(dist_bits, dt, es)
                                                                   : (double)sext(dist_bits, es);
    const double prod = __dmul_rn(0.1, ddist);
    lo = d_cast_double_to_T(__dadd_rn(dmin, prod), dt, es);
    hi = d_cast_double_to_T(__dsub_rn(dmax, prod), dt, es);
}

// (int)(logf(10^k) / logf(10)) with CUDA's logf (cuda_array_statistics.cu:43)
__device__ __forceinline__ int d_precision_of(int steps)
{
    long long e = 1;
    for (int i = 0; i < steps; i++) e *= 10;
    return (int)(logf((float)e) / logf(10.0f));
}

__device__ __forceinline__ int d_precision_steps(float x)
{
    long long e = 1;
    int k = 0;
    while (true) {
        const float fe = (float)e;
        const float q = __fdiv_rn(roundf(__fmul_rn(x, fe)), fe);
        if (!(q != x && e < 10000000000ll)) break;
        e *= 10;
        ++k;
    }
    return k;
}

// GFC geometry (gfc_encoding.cpp:29-33 / 76-80, impl_double.cu:156-179)
struct DGfc {
    uint64_t n, npad, per;
    int64_t warps;
    int blocks, wpb, unit;
};
__device__ __forceinline__ DGfc d_gfc_geom(bool dbl, uint64_t n, int blocks, int wpb)
{
    DGfc g;
    g.n = n;
    g.npad = (n + 31) & ~31ull;
    g.unit = dbl ? 17 : 9;
    if (blocks > 0) {
        g.blocks = blocks;
        g.wpb = wpb;
    } else {
        g.wpb = dbl ? 16 : 32;
        const uint64_t bs = (uint64_t)g.wpb * (dbl ? 64 : 32) * 32;
        g.blocks = (int)((n + bs - 1) / bs);
    }
    g.warps = (int64_t)g.blocks * g.wpb;
    uint64_t per = g.warps ? (g.npad + g.warps - 1) / g.warps : 32;
    if (per < 32) per = 32;
    g.per = (per + 31) & ~31ull;
    return g;
}
__device__ __forceinline__ uint64_t d_gfc_cut(const DGfc &g, int64_t i)
{
    const uint64_t c = (uint64_t)(i + 1) * g.per;
    return c < g.npad ? c : g.npad;
}
__device__ __forceinline__ uint64_t d_gfc_begin(const DGfc &g, int64_t w) { return w ? d_gfc_cut(g, w - 1) : 0; }
__device__ __forceinline__ uint64_t d_gfc_start(const DGfc &g, int64_t w) { return (d_gfc_begin(g, w) + 1) / 2 * (uint64_t)g.unit; }

// ------------------------------------------------------------------------------- input views
// A pass's input is S[it.in[0]] seen through it.vop[]: the constants of the scale ops and the
// view's length, computed once per block.
struct ViewCtx {
    uint64_t c[kMaxViewOps];
    uint64_t n;      // view elements
    uint64_t n_src;  // source elements
    int nd;          // delta ops (source elements read past the view's end)
    bool plain;
};

template <int ES>
__device__ __forceinline__ ViewCtx view_ctx(const BItem &it, const StreamDesc &src)
{
    ViewCtx v;
    v.n_src = src.len / ES;
    v.nd = 0;
    v.plain = it.vop[0] == V_NONE;
#pragma unroll
    for (int k = 0; k < kMaxViewOps; k++) {
        v.c[k] = 0;
        if (it.vop[k] == V_DELTA) ++v.nd;
        else if (it.vop[k] == V_SCALE) {
            uint64_t mnb = 0, mxb = 0;
            acc_minmax((const MinMaxAcc *)it.vscr[k], ES, ORD_INT, mnb, mxb);
            v.c[k] = scale_min(mnb, mxb, ES);
        }
    }
    v.n = v.n_src > (uint64_t)v.nd ? v.n_src - v.nd : 0;
    return v;
}

// view elements [base, base + VPT) (garbage at and past the view's end)
template <int ES, int VPT>
__device__ __forceinline__ void load_view(const BItem &it, const ViewCtx &vc, const uint8_t *src, uint64_t base,
                                          uint64_t (&v)[VPT])
{
    if (vc.plain) {
        load_run<ES, VPT>(src, base, vc.n_src, v);
        return;
    }
    uint64_t x[VPT + kMaxViewOps];
    uint64_t head[VPT];
    load_run<ES, VPT>(src, base, vc.n_src, head);
#pragma unroll
    for (int j = 0; j < VPT; j++) x[j] = head[j];
#pragma unroll
    for (int j = 0; j < kMaxViewOps; j++)
        x[VPT + j] = j < vc.nd && base + VPT + j < vc.n_src ? ld_elem<ES>(src, base + VPT + j) : 0;
#pragma unroll
    for (int k = 0; k < kMaxViewOps; k++) {
        if (it.vop[k] == V_DELTA) {
#pragma unroll
            for (int j = 0; j + 1 < VPT + kMaxViewOps; j++) x[j] = wrap_es(x[j + 1] - x[j], ES);
        } else if (it.vop[k] == V_SCALE) {
#pragma unroll
            for (int j = 0; j < VPT + kMaxViewOps; j++) x[j] = wrap_es(x[j] - vc.c[k], ES);
        }
    }
#pragma unroll
    for (int j = 0; j < VPT; j++) v[j] = x[j];
}

// load_view for passes whose block has `xs` (kXchgBlockBytes of shared memory, free at this point):
// a warp whose source run lies wholly inside the source and starts 16-byte aligned loads it through
// the warp exchange, as whole consecutive sectors; other warps load blocked.  Every lane of the
// block calls it.
template <int ES, int VPT>
__device__ __forceinline__ void load_view_x(const BItem &it, const ViewCtx &vc, const uint8_t *src, uint64_t base,
                                            uint64_t (&v)[VPT], uint8_t *xs)
{
    const uint64_t wb = base - (uint64_t)(threadIdx.x & 31) * VPT;
    if (!(wb + 32 * VPT <= vc.n_src && ((uintptr_t)src & 15) == 0)) {  // warp-uniform
        load_view<ES, VPT>(it, vc, src, base, v);
        return;
    }
    if (vc.plain) {
        load_run_warp<ES, VPT>(src, wb, v, xs);
        return;
    }
    uint64_t x[VPT + kMaxViewOps];
    uint64_t head[VPT];
    load_run_warp<ES, VPT>(src, wb, head, xs);
#pragma unroll
    for (int j = 0; j < VPT; j++) x[j] = head[j];
#pragma unroll
    for (int j = 0; j < kMaxViewOps; j++)
        x[VPT + j] = j < vc.nd && base + VPT + j < vc.n_src ? ld_elem<ES>(src, base + VPT + j) : 0;
#pragma unroll
    for (int k = 0; k < kMaxViewOps; k++) {
        if (it.vop[k] == V_DELTA) {
#pragma unroll
            for (int j = 0; j + 1 < VPT + kMaxViewOps; j++) x[j] = wrap_es(x[j + 1] - x[j], ES);
        } else if (it.vop[k] == V_SCALE) {
#pragma unroll
            for (int j = 0; j < VPT + kMaxViewOps; j++) x[j] = wrap_es(x[j] - vc.c[k], ES);
        }
    }
#pragma unroll
    for (int j = 0; j < VPT; j++) v[j] = x[j];
}

// view element i (i < vc.n)
template <int ES>
__device__ __forceinline__ uint64_t view_elem(const BItem &it, const ViewCtx &vc, const uint8_t *src, uint64_t i)
{
    if (vc.plain) return ld_elem<ES>(src, i);
    uint64_t x[kMaxViewOps + 1];
#pragma unroll
    for (int j = 0; j <= kMaxViewOps; j++) x[j] = j <= vc.nd && i + j < vc.n_src ? ld_elem<ES>(src, i + j) : 0;
#pragma unroll
    for (int k = 0; k < kMaxViewOps; k++) {
        if (it.vop[k] == V_DELTA) {
#pragma unroll
            for (int j = 0; j < kMaxViewOps; j++) x[j] = wrap_es(x[j + 1] - x[j], ES);
        } else if (it.vop[k] == V_SCALE) {
#pragma unroll
            for (int j = 0; j <= kMaxViewOps; j++) x[j] = wrap_es(x[j] - vc.c[k], ES);
        }
    }
    return x[0];
}

// ------------------------------------------------------------------------------- decode views
// A decode input read through its DView (or plainly through in[slot]).
struct DViewCtx {
    const uint8_t *p;      // plain: the stream; AFL: the packed words (rounded down to 4 bytes)
    uint64_t n;            // elements
    uint64_t bytes;        // AFL: readable bytes from p
    uint64_t off_bits;     // AFL: bit offset of value 0 from p
    uint64_t mask;
    uint64_t c0, c1;       // constants added (0 when absent: addition of 0 is the identity)
    int b;                 // AFL bit width; 0 = plain
    bool aligned;          // plain: element aligned
};

// a plain stream that is not element aligned (a none leaf inside a blob) is read like a packed
// stream of full-width values: whole 4-byte words and funnel shifts instead of ES byte loads
template <int ES>
__device__ __forceinline__ void dview_plain(DViewCtx &v, const uint8_t *ptr, uint64_t len)
{
    v.n = len / ES;
    v.aligned = ((uintptr_t)ptr & (ES - 1)) == 0;
    if (v.aligned) {
        v.p = ptr;
        return;
    }
    const uintptr_t mis = (uintptr_t)ptr & 3;
    v.p = ptr - mis;
    v.bytes = len + mis;
    v.off_bits = 8 * mis;
    v.b = 8 * ES;
    v.mask = ES == 8 ? ~0ull : ((1ull << (8 * ES)) - 1);
}

// ok = false when AFL metadata is malformed (the view is then empty)
template <int ES>
__device__ __forceinline__ DViewCtx dview_ctx(const BItem &it, const StreamDesc *S, int slot, bool &ok)
{
    DViewCtx v{};
    ok = true;
    const DView &d = it.dv[slot - 1];
    if (d.data < 0) {  // no view: the input stream itself
        const StreamDesc in = S[it.in[slot]];
        dview_plain<ES>(v, in.ptr, in.len);
        return v;
    }
    const StreamDesc data = S[d.data];
    if (d.afl_meta < 0) {
        dview_plain<ES>(v, data.ptr, data.len);
    } else {
        const StreamDesc meta = S[d.afl_meta];
        if (data.len) {
            const int b = meta.len >= 2 ? (int8_t)meta.ptr[0] : 0, rest = meta.len >= 2 ? (int8_t)meta.ptr[1] : 0;
            const int64_t bits = (int64_t)data.len * 8 - rest;
            if (b < 1 || b > 8 * ES || bits < 0) {
                ok = false;
            } else {
                const uintptr_t mis = (uintptr_t)data.ptr & 3;
                v.p = data.ptr - mis;
                v.bytes = data.len + mis;
                v.off_bits = 8 * mis;
                v.b = b;
                v.mask = b >= 64 ? ~0ull : ((1ull << b) - 1);
                v.n = (uint64_t)bits / b;
            }
        }
    }
    if (d.add[0] >= 0) {
        const StreamDesc m = S[d.add[0]];
        v.c0 = m.len >= (uint64_t)ES ? ld_unaligned<ES>(m.ptr) : 0;
    }
    if (d.add[1] >= 0) {
        const StreamDesc m = S[d.add[1]];
        v.c1 = m.len >= (uint64_t)ES ? ld_unaligned<ES>(m.ptr) : 0;
    }
    return v;
}

template <int ES>
__device__ __forceinline__ uint64_t dview_elem(const DViewCtx &v, uint64_t i)
{
    uint64_t x;
    if (v.b == 0) {
        x = v.aligned ? ld_elem<ES>(v.p, i) : ld_unaligned<ES>(v.p + i * ES);
    } else {
        const StreamReader rd{(const uint32_t *)v.p, v.bytes};
        const uint64_t pos = v.off_bits + i * (uint64_t)v.b;
        const uint64_t w = pos >> 5;
        const uint32_t s = (uint32_t)(pos & 31);
        if (v.b <= 32) {
            const uint32_t lo = rd.word(w);
            const uint32_t hi = (s + v.b > 32) ? rd.word(w + 1) : 0u;
            x = __funnelshift_r(lo, hi, s) & v.mask;
        } else {
            const uint64_t q0 = (uint64_t)rd.word(w) | ((uint64_t)rd.word(w + 1) << 32);
            uint64_t y = q0 >> s;
            if (s + v.b > 64) y |= (uint64_t)rd.word(w + 2) << (64 - s);
            x = y & v.mask;
        }
    }
    return wrap_es(x + v.c0 + v.c1, ES);
}

// elements [base, base + VPT) of the view (0 past its end)
template <int ES, int VPT>
__device__ __forceinline__ void load_dview(const DViewCtx &v, uint64_t base, uint64_t (&out)[VPT])
{
    if (v.b == 0 && v.aligned) {
        load_run<ES, VPT>(v.p, base, v.n, out);
        const uint64_t c = v.c0 + v.c1;
#pragma unroll
        for (int j = 0; j < VPT; j++) out[j] = wrap_es(out[j] + c, ES);
        return;
    }
#pragma unroll
    for (int j = 0; j < VPT; j++) out[j] = base + j < v.n ? dview_elem<ES>(v, base + j) : 0;
}

// the stage kernel skeleton: finds this block's (item, tile).  DYN passes take tiles in claim
// order from a counter (look-back needs every predecessor claimed first), the others use the
// block index; item_of[t] is the item of global tile t (one table per launch), and for DYN launches
// item_of[grid + c] is the tile taken by the c-th claim.
// copies items[k] into the block's shared descriptor (every thread of the block calls it; the
// caller makes sure no thread still reads the previous one); fields are then read from shared
// memory instead of every thread loading the whole descriptor into registers
static __shared__ __align__(16) unsigned long long s_item_words[sizeof(BItem) / 8];  // raw: BItem has initialisers

__device__ __forceinline__ const BItem &shared_item_ref() { return *reinterpret_cast<const BItem *>(s_item_words); }

__device__ __forceinline__ const BItem &shared_item(const BItem *items, uint32_t k)
{
    static_assert(sizeof(BItem) % 8 == 0, "BItem is copied in 8-byte words");
    constexpr int W = (int)(sizeof(BItem) / 8);
    if (threadIdx.x < W)
        s_item_words[threadIdx.x] = ldg((const unsigned long long *)(items + k) + threadIdx.x);
    __syncthreads();
    return shared_item_ref();
}

// GFC: inclusive scan of the chunk sizes (compress: this node's; decode: p[1]); a pass of both the
// compress and the decode step, so it lives here
__device__ inline void p_gfc_scan(const BItem &it, uint32_t tile, StreamDesc *S, bool dbl, bool decode)
{
    __shared__ unsigned long long ws[32];
    __shared__ unsigned long long s_prefix;
    uint64_t n;
    int blocks = 0, wpb = 0;
    if (decode) {
        const StreamDesc m = S[it.in[0]];
        if (m.len < 12) return;
        blocks = (int32_t)ld_unaligned<4>(m.ptr);
        wpb = (int32_t)ld_unaligned<4>(m.ptr + 4);
        n = (uint64_t)(int32_t)ld_unaligned<4>(m.ptr + 8);
        if (blocks <= 0 || wpb <= 0) return;
    } else {
        int nd = 0;
        for (int k = 0; k < kMaxViewOps; k++) nd += it.vop[k] == V_DELTA;
        const uint64_t n_src = S[it.in[0]].len / (dbl ? 8 : 4);
        n = n_src > (uint64_t)nd ? n_src - nd : 0;
    }
    const DGfc g = d_gfc_geom(dbl, n, blocks, wpb);
    // decode: p[3] = the chunks the scratch holds (a larger count is reported by the sizes pass)
    if (decode && (uint64_t)g.warps > it.p[3]) return;
    if (tile > 0 && (uint64_t)tile * kBTile >= (uint64_t)g.warps) return;  // past the chunks
    const int32_t *sizes = (const int32_t *)(it.scratch + it.p[1]);
    unsigned long long *incl = (unsigned long long *)(it.scratch + it.p[2]);
    Lookback lb = lookback_at(it.scratch + it.p[0], it.tiles);
    const uint64_t base = (uint64_t)tile * kBTile + (uint64_t)threadIdx.x * kBVPT;
    unsigned long long v[kBVPT], local = 0;
#pragma unroll
    for (int j = 0; j < (int)kBVPT; j++) {
        v[j] = base + j < (uint64_t)g.warps ? (unsigned long long)(uint32_t)sizes[base + j] : 0ull;
        local += v[j];
    }
    unsigned long long total;
    const unsigned long long excl = block_exclusive_scan<kBThreads>(local, ws, total);
    if (threadIdx.x < 32) {
        const unsigned long long e = lookback_exclusive(lb, tile, total);
        if (threadIdx.x == 0) s_prefix = e;
    }
    __syncthreads();
    unsigned long long acc = s_prefix + excl;
#pragma unroll
    for (int j = 0; j < (int)kBVPT; j++) {
        acc += v[j];
        if (base + j < (uint64_t)g.warps) incl[base + j] = acc;
    }
}

// ------------------------------------------------------------------------------- persistent step
// Helpers of the persistent kernels (batch.hpp, PUnit); all of them run on thread 0 of a block.

// waits until the item's column has finished the entries of its earlier levels; bounded: gives up
// with GTSC_ERR_TIMEOUT after kSpinLimit polls, or at once when another block recorded an error
__device__ __forceinline__ void persist_wait(const PersistArgs &a, const PItem &pi)
{
    uint32_t spins = 0;
    while (*(volatile const uint32_t *)(a.done + pi.col) < pi.wait) {
        if (*(volatile const uint32_t *)a.status != 0u) break;
        if (++spins > kSpinLimit) {
            set_status(a.status, GTSC_ERR_TIMEOUT);
            break;
        }
        __nanosleep(spins < 64 ? 32 : 256);
    }
    __threadfence();  // acquire: what the earlier levels wrote is visible to this block from here
}

// counts `pend` finished entries of `item` (after the block's barrier behind its last tile)
__device__ __forceinline__ void persist_flush(const PersistArgs &a, int item, uint32_t &pend)
{
    if (item >= 0 && pend) {
        __threadfence();  // release: this block's writes before the count
        atomicAdd(a.done + a.pitems[item].col, pend);
    }
    pend = 0;
}

// The persistent loop shared by the compress and the decode kernel.  A block claims one queue unit
// at a time, when it needs one: one tile of a look-back pass (its successors wait on it, so it is
// never held behind other work of the same block -- claiming the next unit ahead measured 3x
// slower for that reason), up to kPersistChunk consecutive tiles of any other pass.  The unit table
// gives the unit's first (item, tile) and its tile count, so a claim costs one 8-byte load; the
// look-back passes' units are already in the stage launch's claim order (tile j of every item
// before tile j + 1 of any, each item's tiles in order).  Thread 0 does the bookkeeping: it keeps
// the current item's fields in registers and walks past tiles beyond an item's real extent without
// involving the block.  EXTENT(op, item, S) gives an item's tiles that do work (the level
// schedule's streaming passes skip the others), RUN(op, item, tile) runs one tile with the whole
// block.
template <class Extent, class Run>
__device__ __forceinline__ void persist_loop(const PersistArgs &a, Extent extent, Run run)
{
    __shared__ uint32_t s_tile;
    __shared__ int s_item, s_op, s_new, s_run;
    int cur = -1;       // thread 0: the item whose tiles it is counting
    int loaded = -1;    // thread 0: the item in the block's shared descriptor
    uint32_t pend = 0;  // thread 0: finished tiles of cur not counted yet
    uint32_t cur_ext = 0, cur_tiles = 0;
    int cur_op = 0;
    for (;;) {
        // thread 0: claim a unit (all threads learn through s_run whether there was one)
        int gi = 0;
        uint32_t tile = 0, cnt = 0;
        if (threadIdx.x == 0) {
            const uint32_t u = atomicAdd(a.qcounter, 1u);
            if (u < a.total) {
                const PUnit pu = a.units[u];
                gi = (int)pu.item;
                tile = pu.tile_count & 0x0fffffffu;
                cnt = pu.tile_count >> 28;
            }
        }
        const bool have = cnt > 0;
        for (;;) {
            if (threadIdx.x == 0) {
                s_run = have ? 0 : -1;
                while (cnt > 0) {
                    if (gi != cur) {
                        persist_flush(a, cur, pend);
                        persist_wait(a, a.pitems[gi]);
                        cur = gi;
                        const BItem &gitem = a.items[gi];
                        cur_tiles = gitem.tiles;
                        cur_op = gitem.op;
                        // the extent is cached per item (a stale read only recomputes the same value)
                        uint32_t x = a.ext[gi];
                        if (x == 0) {
                            x = 1 + extent(cur_op, gitem, a.S);
                            a.ext[gi] = x;
                        }
                        cur_ext = x - 1;
                    }
                    if (tile >= cur_tiles) {  // the unit goes on with the launch's next item
                        ++gi;
                        tile = 0;
                        continue;
                    }
                    const uint32_t my = tile++;
                    --cnt;
                    if (my < cur_ext) {
                        s_run = 1;
                        s_item = gi;
                        s_op = cur_op;
                        s_tile = my;
                        s_new = gi != loaded;
                        loaded = gi;
                        break;
                    }
                    ++pend;  // past the item's real length: nothing to do
                }
            }
            __syncthreads();
            if (s_run <= 0) break;
            if (s_new) shared_item(a.items, (uint32_t)s_item);
            run(s_op, shared_item_ref(), s_tile);
            __syncthreads();  // the next tile reuses the shared memory and the descriptor
            if (threadIdx.x == 0) ++pend;
        }
        if (s_run < 0) break;  // the queue is exhausted
        __syncthreads();       // every thread has read s_run before thread 0 writes it again
    }
    if (threadIdx.x == 0) persist_flush(a, cur, pend);
}

template <bool DYN>
__device__ __forceinline__ const BItem &locate(const BItem *items, const uint32_t *item_of, uint32_t *counter,
                                               uint32_t &tile)
{
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_idx;
    if (threadIdx.x == 0) {
        // DYN launches: the claim order (items interleaved round-robin, each item's tiles in order)
        // follows the launch's tile -> item table
        const uint32_t t = DYN ? item_of[gridDim.x + atomicAdd(counter, 1u)] : blockIdx.x;
        const uint32_t idx = item_of[t];
        s_idx = idx;
        s_tile = (uint32_t)(t - items[idx].tile_base);
    }
    __syncthreads();
    tile = s_tile;
    return shared_item(items, s_idx);
}

}  // namespace gtsc
