// batch_decode.cu -- decode passes of the batched engine, plus the kernels that frame compressed
// columns (assembly) and locate their nodes again (parse).
//
// Framed output: for every column, a uint64 blob length followed by the column's serialized tree
// (the reference's per-column-chunk file framing, optimizer/compression_task.cpp:35-40, with
// the blob of CompressionTree::Compress).
//
// As in batch_kernels.cu, batch_persist_d.cu compiles the decode passes a second time (with
// GTSC_PERSISTENT_TU and coherent loads) for the persistent decode kernel; the stage kernels and the
// framing kernels are built only here.
#include "batch_dev.cuh"

#include <algorithm>

namespace gtsc {

namespace {

// ------------------------------------------------------------------------------- block copy
// Copies n bytes from src to dst (any alignment) with the whole block: byte head up to a 4-byte
// aligned destination, then 32-bit words assembled from the two source words that cover them.
// Source words are read at most 3 bytes past its end, inside the same aligned word.
__device__ void block_copy(uint8_t *dst, const uint8_t *src, uint64_t n)
{
    const uint64_t head = (4 - ((uintptr_t)dst & 3)) & 3;
    const uint64_t h = head < n ? head : n;
    if (threadIdx.x < h) dst[threadIdx.x] = src[threadIdx.x];
    if (n <= h) return;
    uint8_t *d = dst + h;
    const uint8_t *sp = src + h;
    const uint64_t words = (n - h) / 4;
    const uint32_t sh = 8 * (uint32_t)((uintptr_t)sp & 3);
    const uint32_t *sw = (const uint32_t *)((uintptr_t)sp & ~(uintptr_t)3);
    uint32_t *dw = (uint32_t *)d;
    // eight words a thread are loaded before any of them is stored, so the loads are in flight
    // together whatever the compiler assumes about the two buffers overlapping
    constexpr int U = 8;
    uint64_t k = threadIdx.x;
    if (sh == 0) {
        for (; k + (U - 1) * kBThreads < words; k += U * kBThreads) {
            uint32_t r[U];
#pragma unroll
            for (int u = 0; u < U; u++) r[u] = ldg(sw + k + u * kBThreads);
#pragma unroll
            for (int u = 0; u < U; u++) dw[k + u * kBThreads] = r[u];
        }
        for (; k < words; k += kBThreads) dw[k] = ldg(sw + k);
    } else {
        for (; k + (U - 1) * kBThreads < words; k += U * kBThreads) {
            uint32_t r[U], q[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                r[u] = ldg(sw + k + u * kBThreads);
                q[u] = ldg(sw + k + u * kBThreads + 1);
            }
#pragma unroll
            for (int u = 0; u < U; u++) dw[k + u * kBThreads] = __funnelshift_r(r[u], q[u], sh);
        }
        for (; k < words; k += kBThreads) dw[k] = __funnelshift_r(ldg(sw + k), ldg(sw + k + 1), sh);
    }
    const uint64_t tail = (n - h) - 4 * words;
    if (threadIdx.x < tail) d[4 * words + threadIdx.x] = sp[4 * words + threadIdx.x];
}

constexpr uint64_t kCopyPiece = 1ull << 16;  // bytes of one copy tile (one block each)

// ------------------------------------------------------------------------------- none / copy
// in[0] = source stream, out[0] = destination stream; p[0] = destination byte offset inside it
__device__ void p_none_copy(const BItem &it, uint32_t tile, StreamDesc *S, uint32_t *status)
{
    const StreamDesc in = S[it.in[0]];
    const uint64_t off = (uint64_t)tile * kCopyPiece;
    if (in.len > S[it.out[0]].cap) {
        if (tile == 0 && threadIdx.x == 0) set_status(status, GTSC_ERR_CAPACITY);
        return;
    }
    if (tile == 0 && threadIdx.x == 0) S[it.out[0]].len = in.len;
    if (off >= in.len) return;
    const uint64_t n = in.len - off < kCopyPiece ? in.len - off : kCopyPiece;
    block_copy(S[it.out[0]].ptr + off, in.ptr + off, n);
}

// ------------------------------------------------------------------------------- AFL unpack
template <int ES>
__device__ void p_afl_unpack(const BItem &it, uint32_t tile, StreamDesc *S, uint32_t *status)
{
    const StreamDesc meta = S[it.in[0]], data = S[it.in[1]];
    StreamDesc &out = S[it.out[0]];
    if (data.len == 0) {
        if (tile == 0 && threadIdx.x == 0) out.len = 0;
        return;
    }
    if (meta.len < 2) {
        if (tile == 0 && threadIdx.x == 0) set_status(status, GTSC_ERR_FORMAT);
        return;
    }
    const int b = (int8_t)meta.ptr[0], rest = (int8_t)meta.ptr[1];
    const int64_t bits = (int64_t)data.len * 8 - rest;
    if (b < 1 || b > 8 * ES || bits < 0) {
        if (tile == 0 && threadIdx.x == 0) set_status(status, GTSC_ERR_FORMAT);
        return;
    }
    const uint64_t n = (uint64_t)bits / b;
    if (n * ES > out.cap) {
        if (tile == 0 && threadIdx.x == 0) set_status(status, GTSC_ERR_CAPACITY);
        return;
    }
    if (tile == 0 && threadIdx.x == 0) out.len = n * ES;
    const uintptr_t mis = (uintptr_t)data.ptr & 3;
    const StreamReader rd{(const uint32_t *)(data.ptr - mis), data.len + mis};
    const uint64_t off_bits = 8 * mis;
    const uint64_t mask = b >= 64 ? ~0ull : ((1ull << b) - 1);
    const uint64_t base = (uint64_t)tile * kBTile + (uint64_t)threadIdx.x * kBVPT;
    if (base >= n) return;
    uint64_t v[kBVPT];
#pragma unroll
    for (int j = 0; j < (int)kBVPT; j++) {
        v[j] = 0;
        const uint64_t i = base + j;
        if (i >= n) continue;
        const uint64_t p = off_bits + i * (uint64_t)b;
        const uint64_t w = p >> 5;
        const uint32_t s = (uint32_t)(p & 31);
        if (b <= 32) {
            const uint32_t lo = rd.word(w);
            const uint32_t hi = (s + b > 32) ? rd.word(w + 1) : 0u;
            v[j] = __funnelshift_r(lo, hi, s) & mask;
        } else {
            const uint64_t q0 = (uint64_t)rd.word(w) | ((uint64_t)rd.word(w + 1) << 32);
            uint64_t x = q0 >> s;
            if (s + b > 64) x |= (uint64_t)rd.word(w + 2) << (64 - s);
            v[j] = x & mask;
        }
    }
    store_run<ES, kBVPT>(out.ptr, base, n, v);
}

// ------------------------------------------------------------------------------- delta decode
template <int ES>
__device__ void p_delta_dec(const BItem &it, uint32_t tile, StreamDesc *S, uint32_t *status)
{
    __shared__ unsigned long long ws[32];
    __shared__ unsigned long long s_prefix;
    const StreamDesc meta = S[it.in[0]];
    bool ok;
    const DViewCtx dv = dview_ctx<ES>(it, S, 1, ok);
    StreamDesc &out = S[it.out[0]];
    const uint64_t n = meta.len ? dv.n + 1 : 0;
    if (!ok || n * ES > out.cap) {  // item-uniform: no tile of this item enters the look-back
        if (tile == 0 && threadIdx.x == 0) set_status(status, ok ? GTSC_ERR_CAPACITY : GTSC_ERR_FORMAT);
        return;
    }
    if (tile == 0 && threadIdx.x == 0) out.len = n * ES;
    // a tile past the output has no successor waiting on its look-back descriptor
    if (tile > 0 && (uint64_t)tile * kBTile >= n) return;
    Lookback lb = lookback_at(it.scratch + it.p[0], it.tiles);
    const uint64_t m = n ? n - 1 : 0;
    const uint64_t base = (uint64_t)tile * kBTile + (uint64_t)threadIdx.x * kBVPT;
    uint64_t v[kBVPT];
    load_dview<ES, kBVPT>(dv, base, v);
#pragma unroll
    for (int j = 0; j < (int)kBVPT; j++)
        if (base + j >= m) v[j] = 0;
    unsigned long long local = 0;
#pragma unroll
    for (int j = 0; j < (int)kBVPT; j++) local += v[j];
    unsigned long long total;
    const unsigned long long excl = block_exclusive_scan<kBThreads>(local, ws, total);
    if (threadIdx.x < 32) {
        const unsigned long long e = lookback_exclusive(lb, tile, total);
        if (threadIdx.x == 0) s_prefix = e;
    }
    __syncthreads();
    if (base >= n) return;
    unsigned long long acc = ld_unaligned<ES>(meta.ptr) + s_prefix + excl;
    uint64_t o[kBVPT];
#pragma unroll
    for (int j = 0; j < (int)kBVPT; j++) {
        o[j] = wrap_es(acc, ES);
        acc += v[j];
    }
    store_run<ES, kBVPT>(out.ptr, base, n, o);
}

// ------------------------------------------------------------------------------- scale add
template <int ES>
__device__ void p_scale_add(const BItem &it, uint32_t tile, StreamDesc *S, uint32_t *status)
{
    const StreamDesc meta = S[it.in[0]];
    bool ok;
    const DViewCtx dv = dview_ctx<ES>(it, S, 1, ok);
    StreamDesc &out = S[it.out[0]];
    const uint64_t n = dv.n;
    if (!ok || n * ES > out.cap || (n && meta.len < (uint64_t)ES)) {
        if (tile == 0 && threadIdx.x == 0) set_status(status, GTSC_ERR_FORMAT);
        return;
    }
    if (tile == 0 && threadIdx.x == 0) out.len = n * ES;
    const uint64_t mn = ld_unaligned<ES>(meta.ptr);
    // block-striped: the k-th access of a warp covers 32 consecutive elements
    const uint64_t t0 = (uint64_t)tile * kBTile + threadIdx.x;
#pragma unroll 4
    for (int j = 0; j < (int)kBVPT; j++) {
        const uint64_t i = t0 + (uint64_t)j * kBThreads;
        if (i >= n) break;
        st_elem<ES>(out.ptr, i, wrap_es(dview_elem<ES>(dv, i) + mn, ES));
    }
}

// ------------------------------------------------------------------------------- merge
// elements [p0, p0 + cnt) of a decode view into shared memory at element slot `at`; unpacked views
// take plain loads, packed ones the view's bit extraction
template <int ES>
__device__ __forceinline__ void stage_view(const DViewCtx &v, uint64_t p0, uint32_t cnt, uint8_t *sm, uint32_t at)
{
    if (v.b == 0) {
        const uint64_t c = v.c0 + v.c1;
        for (uint32_t i = threadIdx.x; i < cnt; i += kBThreads)
            st_elem<ES>(sm, at + i, wrap_es(ld_elem<ES>(v.p, p0 + i) + c, ES));  // plain views are aligned
    } else {
        for (uint32_t i = threadIdx.x; i < cnt; i += kBThreads) st_elem<ES>(sm, at + i, dview_elem<ES>(v, p0 + i));
    }
}

// Merge tiles find their offsets in the match / non-match streams without a look-back chain: a
// counting pass (B_MERGE_COUNT, any order) stores each tile's number of stencil matches and adds it
// to its group of kMergeGroup tiles; a merge tile's exclusive prefix is then the sum of the groups
// before its own plus the tiles before it inside its group.  Scratch at it.p[0]: 16 bytes, the
// group sums (u64), then the tile counts (u32) -- within the look-back area's 16 + 16 * tiles.
constexpr uint32_t kMergeGroup = 64;

__device__ __forceinline__ unsigned long long *merge_groups(const BItem &it)
{
    return (unsigned long long *)(it.scratch + it.p[0] + 16);  // p[1] = tiles of kBTile elements
}
__device__ __forceinline__ uint32_t *merge_counts(const BItem &it)
{
    return (uint32_t *)(it.scratch + it.p[0] + 16 + 8ull * ((it.p[1] + kMergeGroup - 1) / kMergeGroup));
}

// the stencil of a merge node and the element count its rest byte gives (0 when malformed)
template <int ES>
__device__ __forceinline__ const uint8_t *merge_stencil(const BItem &it, const StreamDesc &meta, uint64_t &n)
{
    const uint8_t *stencil = it.mode == SPLIT_NOT_CONST ? meta.ptr + ES : meta.ptr;
    const uint64_t sbytes = it.mode == SPLIT_NOT_CONST ? (meta.len > (uint64_t)ES ? meta.len - ES : 0) : meta.len;
    n = 0;
    if (sbytes >= 1) {
        const int rest = (int8_t)stencil[0];
        int64_t nn = (int64_t)(sbytes - 1) * 8;
        if (rest) nn -= 8 - rest;
        if (nn >= 0 && rest >= 0 && rest <= 7) n = (uint64_t)nn;
    }
    return stencil;
}

template <int ES>
__device__ void p_merge_count(const BItem &it, uint32_t tile, StreamDesc *S)
{
    __shared__ unsigned long long ws[32];
    uint64_t n;
    const uint8_t *stencil = merge_stencil<ES>(it, S[it.in[0]], n);
    const uint64_t base = (uint64_t)tile * kBTile + (uint64_t)threadIdx.x * kBVPT;
    uint32_t bits = 0;
#pragma unroll
    for (int q = 0; q < (int)kBVPT / 8; q++)
        if (base + 8 * q < n) bits |= (uint32_t)stencil[1 + base / 8 + q] << (8 * q);
    const uint32_t valid_mask = base >= n ? 0u : (n - base >= kBVPT ? (1u << kBVPT) - 1 : ((1u << (n - base)) - 1));
    unsigned long long total;
    block_exclusive_scan<kBThreads>((unsigned long long)__popc(bits & valid_mask), ws, total);
    if (threadIdx.x == 0) {
        merge_counts(it)[tile] = (uint32_t)total;
        if (total) atomicAdd(merge_groups(it) + tile / kMergeGroup, total);
    }
}

// matches before `tile` (its exclusive prefix) from the counting pass; the same in every thread
__device__ __forceinline__ unsigned long long merge_prefix(const BItem &it, uint32_t tile, unsigned long long *ws)
{
    const uint32_t g = tile / kMergeGroup;
    const unsigned long long *groups = merge_groups(it);
    const uint32_t *counts = merge_counts(it);
    unsigned long long part = 0;
    for (uint32_t k = threadIdx.x; k < g; k += kBThreads) part += groups[k];
    for (uint32_t k = g * kMergeGroup + threadIdx.x; k < tile; k += kBThreads) part += counts[k];
    unsigned long long total;
    block_exclusive_scan<kBThreads>(part, ws, total);
    return total;
}

// The counting launch of the merges: one warp per tile (512 stencil bytes, 16 per lane), so no
// block barrier sits between a tile's loads and its count.
__global__ void __launch_bounds__(kBThreads)
k_merge_count(const BItem *items, const uint32_t *item_of, StreamDesc *S, const uint32_t *status, uint32_t total_tiles)
{
    if (*(volatile const uint32_t *)(status + 1)) return;
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (kBThreads / 32);
    for (uint32_t t = blockIdx.x * (kBThreads / 32) + (threadIdx.x >> 5); t < total_tiles; t += warps) {
        const BItem &it = items[item_of[t]];
        const uint32_t tile = t - (uint32_t)it.tile_base;
        uint64_t n;
        const uint8_t *stencil;
        switch (it.es) {
        case 1: stencil = merge_stencil<1>(it, S[it.in[0]], n); break;
        case 2: stencil = merge_stencil<2>(it, S[it.in[0]], n); break;
        case 4: stencil = merge_stencil<4>(it, S[it.in[0]], n); break;
        default: stencil = merge_stencil<8>(it, S[it.in[0]], n); break;
        }
        const uint64_t e0 = (uint64_t)tile * kBTile + (uint64_t)lane * 128;  // this lane's 128 elements
        uint32_t c = 0;
        if (e0 < n) {
            const uint64_t valid = n - e0 < 128 ? n - e0 : 128;
            const uint8_t *b = stencil + 1 + e0 / 8;
            for (uint32_t q = 0; q < (valid + 7) / 8; q++) {
                uint32_t byte = b[q];
                const uint64_t left = valid - 8ull * q;
                if (left < 8) byte &= (1u << left) - 1;
                c += __popc(byte);
            }
        }
        for (int o = 16; o; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
        if (lane == 0) {
            merge_counts(it)[tile] = c;
            if (c) atomicAdd(merge_groups(it) + tile / kMergeGroup, (unsigned long long)c);
        }
    }
}

// Shared staging of the merge and the RLE expansion, declared once at file scope: a __shared__
// array inside a function template is one array per instantiation (per element size), which a
// kernel running every pass kind for every element size could not hold.
static __shared__ uint32_t s_merge_codes[kBTile / 16 + 2];              // the tile's dictionary code words
static __shared__ uint16_t s_merge_bits[kBThreads], s_merge_excl[kBThreads];  // stencil bits, matches before
static __shared__ uint16_t s_rle_end[kBTile + 2];                       // the tile's run ends

template <int ES>
__device__ void p_merge(const BItem &it, uint32_t stile, StreamDesc *S, uint32_t *status, uint8_t *sm)
{
    // a block merges kBMergeSub consecutive tiles of its item; the setup below is done once for them
    __shared__ unsigned long long ws[32];
    const int mode = it.mode;
    const StreamDesc meta = S[it.in[0]];
    // dictionary: in1 is the packed code stream (read plainly); otherwise both inputs may be views
    const StreamDesc in1 = mode == SPLIT_DICT ? S[it.in[1]] : StreamDesc{nullptr, 0, 0, 0};
    bool ok1 = true, ok2 = true;
    DViewCtx v1{}, v2{};
    if (mode != SPLIT_DICT) v1 = dview_ctx<ES>(it, S, 1, ok1);
    if (mode != SPLIT_NOT_CONST) v2 = dview_ctx<ES>(it, S, 2, ok2);
    StreamDesc &out = S[it.out[0]];
    if (!ok1 || !ok2) {
        if (stile == 0 && threadIdx.x == 0) set_status(status, GTSC_ERR_FORMAT);
        return;
    }
    const uint64_t len1 = mode == SPLIT_DICT ? in1.len : v1.n * ES, len2 = v2.n * ES;
    // empty-input rules of the three Decode()s
    const bool empty = mode == SPLIT_NOT_CONST ? meta.len == 0 : (len1 == 0 && len2 == 0);
    const uint8_t *stencil = mode == SPLIT_NOT_CONST ? meta.ptr + ES : meta.ptr;
    const uint64_t sbytes = mode == SPLIT_NOT_CONST ? (meta.len > (uint64_t)ES ? meta.len - ES : 0) : meta.len;
    uint64_t n = 0;
    if (!empty) {
        if (sbytes < 1) {
            if (stile == 0 && threadIdx.x == 0) set_status(status, GTSC_ERR_FORMAT);
            return;
        }
        const int rest = (int8_t)stencil[0];
        int64_t nn = (int64_t)(sbytes - 1) * 8;
        if (rest) nn -= 8 - rest;
        if (nn < 0 || rest < 0 || rest > 7) {
            if (stile == 0 && threadIdx.x == 0) set_status(status, GTSC_ERR_FORMAT);
            return;
        }
        n = (uint64_t)nn;
    }
    if (n * ES > out.cap) {
        if (stile == 0 && threadIdx.x == 0) set_status(status, GTSC_ERR_CAPACITY);
        return;
    }
    if (stile == 0 && threadIdx.x == 0) out.len = n * ES;
    // dictionary stream: 16-byte header, 4 values, codes
    uint64_t top[4] = {0, 0, 0, 0}, yes_cap = 0, no_cap = v2.n;
    const uint8_t *codes = nullptr;
    if (mode == SPLIT_DICT) {
        if (in1.len >= 16 + 4ull * ES) {
            const uint64_t m = ld_unaligned<8>(in1.ptr + 8);
            for (int k = 0; k < 4; k++) top[k] = ld_unaligned<ES>(in1.ptr + 16 + k * ES);
            codes = in1.ptr + 16 + 4 * ES;
            yes_cap = (in1.len - 16 - 4ull * ES) / 4 * 16;
            if (m < yes_cap) yes_cap = m;
        }
    } else if (mode == SPLIT_NOT_CONST) {
        if (meta.len >= (uint64_t)ES) top[0] = ld_unaligned<ES>(meta.ptr);
        yes_cap = v1.n;
    } else {
        yes_cap = v1.n;
    }
    bool bad = false;
    for (uint32_t sub = 0; sub < kBMergeSub; sub++) {
    const uint32_t tile = stile * kBMergeSub + sub;
    if ((uint64_t)tile * kBTile >= n) break;  // past the output
    const uint64_t base = (uint64_t)tile * kBTile + (uint64_t)threadIdx.x * kBVPT;
    const uint32_t valid_mask = base >= n ? 0u : (n - base >= kBVPT ? (1u << kBVPT) - 1 : ((1u << (n - base)) - 1));
    uint32_t bits = 0;
#pragma unroll
    for (int q = 0; q < (int)kBVPT / 8; q++)
        if (base + 8 * q < n) bits |= (uint32_t)stencil[1 + base / 8 + q] << (8 * q);
    bits &= valid_mask;
    unsigned long long total;
    const unsigned long long excl = block_exclusive_scan<kBThreads>((unsigned long long)__popc(bits), ws, total);
    const unsigned long long prefix = merge_prefix(it, tile, ws);
    // the tile's runs of both streams are staged in shared memory with coalesced loads (matches
    // first, then the rest), then every thread assembles its values from there
    const uint64_t tile_base = (uint64_t)tile * kBTile;
    const uint64_t tile_n = tile_base < n ? (n - tile_base < kBTile ? n - tile_base : kBTile) : 0;
    const uint64_t ny = total, nn = tile_n - ny;
    const uint64_t yes0 = prefix, no0 = tile_base - (tile_base < n ? yes0 : 0);
    // dictionary: the code words of the tile's matches, staged once (coalesced, whole words)
    uint32_t *s_codes = s_merge_codes;
    const uint64_t w0 = yes0 >> 4;
    if (mode == SPLIT_DICT && ny) {
        const uint64_t nw = ((yes0 + ny + 15) >> 4) - w0;
        const uint64_t avail = in1.len >= 16 + 4ull * ES ? (in1.len - 16 - 4ull * ES) / 4 : 0;
        const bool al = ((uintptr_t)codes & 3) == 0;
        for (uint64_t k = threadIdx.x; k < nw; k += kBThreads) {
            const uint64_t w = w0 + k;
            s_codes[k] = w >= avail ? 0u : al ? ldg((const uint32_t *)codes + w) : (uint32_t)ld_unaligned<4>(codes + 4 * w);
        }
    }
    // in-tile counts fit 32 bits; a stream position past the stream's end is corrupt input
    const uint32_t ny32 = (uint32_t)ny, nn32 = (uint32_t)nn;
    if (mode != SPLIT_DICT) {
        const uint32_t ok = yes_cap > yes0 ? (uint32_t)(yes_cap - yes0 < ny ? yes_cap - yes0 : ny) : 0u;
        bad |= ok < ny32;
        stage_view<ES>(v1, yes0, ok, sm, 0);
    }
    if (mode != SPLIT_NOT_CONST) {
        const uint32_t ok = no_cap > no0 ? (uint32_t)(no_cap - no0 < nn ? no_cap - no0 : nn) : 0u;
        bad |= ok < nn32;
        stage_view<ES>(v2, no0, ok, sm, ny32);
    }
    // every thread's 16 stencil bits and the matches before them, for the striped assembly below
    uint16_t *s_bits = s_merge_bits, *s_excl = s_merge_excl;
    s_bits[threadIdx.x] = (uint16_t)bits;
    s_excl[threadIdx.x] = (uint16_t)excl;
    __syncthreads();
    // step j writes elements j * 256 + t: consecutive threads read consecutive staged values (no
    // bank conflicts) and store consecutive outputs (coalesced)
    const uint32_t y0 = (uint32_t)(yes0 & 15);
    const uint32_t lim = yes_cap > yes0 ? (uint32_t)(yes_cap - yes0 < kBTile ? yes_cap - yes0 : kBTile) : 0u;
    uint8_t *dst = out.ptr + tile_base * ES;
#pragma unroll 4
    for (uint32_t e = threadIdx.x; e < (uint32_t)tile_n; e += kBThreads) {
        const uint32_t o = e >> 4, q = e & 15;
        const uint32_t bb = s_bits[o];
        const uint32_t r = s_excl[o] + __popc(bb & ((1u << q) - 1));  // matches before e in the tile
        uint64_t val;
        if ((bb >> q) & 1u) {
            if (mode == SPLIT_DICT) {
                bad |= r >= lim;
                const uint32_t y = y0 + r;
                const uint32_t c = (s_codes[y >> 4] >> (2 * (y & 15))) & 3u;  // select, not an indexed array
                val = c == 0 ? top[0] : c == 1 ? top[1] : c == 2 ? top[2] : top[3];
            } else {
                val = ld_elem_sm<ES>(sm, r);
            }
        } else {
            val = mode == SPLIT_NOT_CONST ? top[0] : ld_elem_sm<ES>(sm, ny32 + (e - r));
        }
        st_elem<ES>(dst, e, val);
    }
    __syncthreads();  // the next tile restages the shared buffers
    }
    if (bad) set_status(status, GTSC_ERR_FORMAT);
}

// ------------------------------------------------------------------------------- RLE decode
// node scratch: p[0] look-back, p[1] run ends (u64)
__device__ void p_rle_scan(const BItem &it, uint32_t tile, StreamDesc *S, uint32_t *status)
{
    __shared__ unsigned long long ws[32];
    __shared__ unsigned long long s_prefix;
    const StreamDesc meta = S[it.in[0]];
    bool ok1, ok2;
    const DViewCtx lengths = dview_ctx<4>(it, S, 1, ok1);  // int32 run lengths
    uint64_t n_values = 0;
    switch (it.es) {  // the values' count (their element size is the node's)
    case 1: n_values = dview_ctx<1>(it, S, 2, ok2).n; break;
    case 2: n_values = dview_ctx<2>(it, S, 2, ok2).n; break;
    case 4: n_values = dview_ctx<4>(it, S, 2, ok2).n; break;
    default: n_values = dview_ctx<8>(it, S, 2, ok2).n; break;
    }
    int64_t runs = 0;
    if (!ok1 || !ok2) {
        if (tile == 0 && threadIdx.x == 0) set_status(status, GTSC_ERR_FORMAT);
    } else if (lengths.n) {
        runs = meta.len >= 4 ? (int32_t)ld_unaligned<4>(meta.ptr) : -1;
        if (runs < 0 || (uint64_t)runs > lengths.n || (uint64_t)runs > n_values) {
            if (tile == 0 && threadIdx.x == 0) set_status(status, GTSC_ERR_FORMAT);
            runs = 0;
        }
    }
    unsigned long long *ends = (unsigned long long *)(it.scratch + it.p[1]);
    if (tile > 0 && (uint64_t)tile * kBTile >= (uint64_t)runs) return;  // past the runs
    Lookback lb = lookback_at(it.scratch + it.p[0], it.tiles);
    const uint64_t base = (uint64_t)tile * kBTile + (uint64_t)threadIdx.x * kBVPT;
    long long v[kBVPT];
    unsigned long long local = 0;
    bool neg = false;
#pragma unroll
    for (int j = 0; j < (int)kBVPT; j++) {
        v[j] = base + j < (uint64_t)runs ? (long long)(int32_t)dview_elem<4>(lengths, base + j) : 0;
        neg |= v[j] < 0;
        local += (unsigned long long)v[j];
    }
    if (neg) set_status(status, GTSC_ERR_FORMAT);
    unsigned long long total;
    const unsigned long long excl = block_exclusive_scan<kBThreads>(local, ws, total);
    if (threadIdx.x < 32) {
        const unsigned long long e = lookback_exclusive(lb, tile, total);
        if (threadIdx.x == 0) s_prefix = e;
    }
    __syncthreads();
    unsigned long long acc = s_prefix + excl;
    unsigned long long *first_run = (unsigned long long *)(it.scratch + it.p[3]);
#pragma unroll
    for (int j = 0; j < (int)kBVPT; j++) {
        acc += (unsigned long long)v[j];
        if (base + j < (uint64_t)runs) {
            ends[base + j] = acc;
            // the expand tiles whose first element lies in this run start from it
            if (v[j] > 0)
                for (uint64_t t = (acc - (unsigned long long)v[j] + kBTile - 1) / kBTile; t <= (acc - 1) / kBTile && t < it.tiles; t++)
                    first_run[t] = base + j;
        }
    }
    // p[2] holds the run count for the expand pass
    if (tile == 0 && threadIdx.x == 0) *(unsigned long long *)(it.scratch + it.p[2]) = (unsigned long long)runs;
}

template <int ES>
__device__ void p_rle_expand(const BItem &it, uint32_t tile, StreamDesc *S, uint32_t *status, uint8_t *xs)
{
    // the tile's run ends relative to its first element, clamped to kBTile (at most kBTile + 1 runs)
    uint16_t *s_end = s_rle_end;
    bool ok;
    const DViewCtx values = dview_ctx<ES>(it, S, 2, ok);
    StreamDesc &out = S[it.out[0]];
    const uint64_t runs = *(const unsigned long long *)(it.scratch + it.p[2]);
    const unsigned long long *ends = (const unsigned long long *)(it.scratch + it.p[1]);
    const uint64_t n = runs ? ends[runs - 1] : 0;
    if (n * ES > out.cap) {
        if (tile == 0 && threadIdx.x == 0) set_status(status, GTSC_ERR_CAPACITY);
        return;
    }
    if (tile == 0 && threadIdx.x == 0) out.len = n * ES;
    const uint64_t t0 = (uint64_t)tile * kBTile;
    if (t0 >= n) return;
    // the scan pass recorded the run holding each tile's first element
    const unsigned long long *first_run = (const unsigned long long *)(it.scratch + it.p[3]);
    uint64_t r_lo = first_run[tile];
    uint64_t r_hi = t0 + kBTile < n && tile + 1 < it.tiles ? first_run[tile + 1] + 1 : runs;
    if (r_hi > runs) r_hi = runs;
    if (r_lo > r_hi) r_lo = r_hi;  // only on corrupt lengths (reported by the scan pass)
    // <= kBTile + 1 when ends rise by at least 1 per run; corrupt zero-length runs are cut off
    const uint32_t m = (uint32_t)(r_hi - r_lo < kBTile + 2 ? r_hi - r_lo : kBTile + 2);
    for (uint32_t k = threadIdx.x; k < m; k += kBThreads) {
        const uint64_t e = ends[r_lo + k] - t0;
        s_end[k] = (uint16_t)(e < kBTile ? e : kBTile);
    }
    __syncthreads();
    const uint32_t b = threadIdx.x * kBVPT;  // relative to t0
    const uint64_t base = t0 + b;
    const uint64_t wb = base - (uint64_t)(threadIdx.x & 31) * kBVPT;  // the warp's first element
    // warp-uniform: the warp's whole run is inside the output and the output is 16-byte aligned
    const bool wfull = wb + 32 * kBVPT <= n && ((uintptr_t)out.ptr & 15) == 0;
    if (!wfull && base >= n) return;
    uint32_t lo = 0, hi = m;  // first staged run ending after b
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s_end[mid] > b) hi = mid;
        else lo = mid + 1;
    }
    // a run's value is read (through the values' view, which may unpack it) once per run, not per
    // element: the thread's 16 elements usually lie in one or two runs
    uint64_t v[kBVPT];
    uint64_t last_r = ~0ull, last_v = 0;
#pragma unroll
    for (int j = 0; j < (int)kBVPT; j++) {
        while (lo < m && s_end[lo] <= b + j) ++lo;
        const uint64_t r = r_lo + lo;
        const bool in = base + j < n && lo < m && r < values.n;
        if (in && r != last_r) {
            last_v = dview_elem<ES>(values, r);
            last_r = r;
        }
        v[j] = in ? last_v : 0;
    }
    if (wfull)
        store_run_warp<ES, kBVPT>(out.ptr, wb, v, xs);
    else
        store_run<ES, kBVPT>(out.ptr, base, n, v);
    (void)status;
}

// ------------------------------------------------------------------------------- floatToInt
template <int ES>
__device__ void p_f2i_dec(const BItem &it, uint32_t tile, StreamDesc *S, uint32_t *status)
{
    __shared__ double p10[10];
    if (threadIdx.x < 10) {
        double v = 1.0;
        for (unsigned i = 0; i < threadIdx.x; i++) v *= 10.0;
        p10[threadIdx.x] = v;
    }
    __syncthreads();
    const StreamDesc meta = S[it.in[0]];
    bool ok;
    const DViewCtx d = dview_ctx<4>(it, S, 1, ok);  // the child's int32 stream
    StreamDesc &out = S[it.out[0]];
    if (!ok) {
        if (tile == 0 && threadIdx.x == 0) set_status(status, GTSC_ERR_FORMAT);
        return;
    }
    if (d.n == 0) {
        if (tile == 0 && threadIdx.x == 0) out.len = 0;
        return;
    }
    const int p = meta.len >= 4 ? (int32_t)ld_unaligned<4>(meta.ptr) : -1;
    if (p < 0) {
        if (tile == 0 && threadIdx.x == 0) set_status(status, GTSC_ERR_FORMAT);
        return;
    }
    const uint64_t n = p < 10 ? d.n : d.n * 4 / ES;
    if (n * ES > out.cap) {
        if (tile == 0 && threadIdx.x == 0) set_status(status, GTSC_ERR_CAPACITY);
        return;
    }
    if (tile == 0 && threadIdx.x == 0) out.len = n * ES;
    // block-striped: the k-th access of a warp covers 32 consecutive elements
    const uint64_t t0 = (uint64_t)tile * kBTile + threadIdx.x;
    const Order o = (Order)it.order;
    for (int j = 0; j < (int)kBVPT; j++) {
        const uint64_t i = t0 + (uint64_t)j * kBThreads;
        if (i >= n) break;
        uint64_t v;
        if (p < 10) {
            const int k = (int32_t)dview_elem<4>(d, i);
            if (o == ORD_F32) v = __float_as_uint(__double2float_rn(__ddiv_rn((double)__int2float_rn(k), p10[p])));
            else if (o == ORD_F64) v = (uint64_t)__double_as_longlong(__ddiv_rn((double)k, p10[p]));
            else if (ES == 8) v = (uint64_t)__double2ll_rz(__ddiv_rn((double)k, p10[p]));
            else v = (uint64_t)(long long)__double2int_rz(__ddiv_rn((double)sext((uint64_t)(long long)k, ES), p10[p]));
        } else if (ES == 8) {  // raw bytes: two int32 per element
            v = dview_elem<4>(d, 2 * i) | (dview_elem<4>(d, 2 * i + 1) << 32);
        } else if (ES == 4) {
            v = dview_elem<4>(d, i);
        } else {  // 1- and 2-byte elements inside the int32 words
            constexpr uint64_t emask = ES >= 8 ? ~0ull : ((1ull << (8 * (ES % 8))) - 1);
            const uint64_t byte = i * ES;
            v = (dview_elem<4>(d, byte / 4) >> (8 * (byte % 4))) & emask;
        }
        st_elem<ES>(out.ptr, i, v);
    }
}

// ------------------------------------------------------------------------------- GFC decode
// node scratch: p[0] look-back, p[1] sizes (int32), p[2] inclusive ends (u64)
__device__ bool gfc_meta(const StreamDesc &m, bool dbl, DGfc &g)
{
    if (m.len < 12) return false;
    const int blocks = (int32_t)ld_unaligned<4>(m.ptr), wpb = (int32_t)ld_unaligned<4>(m.ptr + 4);
    const int nn = (int32_t)ld_unaligned<4>(m.ptr + 8);
    if (blocks <= 0 || wpb <= 0 || nn < 0 || (int64_t)blocks * wpb > (1ll << 26)) return false;
    g = d_gfc_geom(dbl, (uint64_t)nn, blocks, wpb);
    return true;
}

__device__ void p_gfc_sizes(const BItem &it, uint32_t tile, StreamDesc *S, uint32_t *status)
{
    const bool dbl = it.es == 8;
    const StreamDesc meta = S[it.in[0]], ends = S[it.in[1]], payload = S[it.in[2]];
    if (payload.len == 0) return;
    DGfc g;
    if (!gfc_meta(meta, dbl, g) || ends.len < 4ull * g.warps || (uint64_t)g.warps > it.p[3]) {
        if (tile == 0 && threadIdx.x == 0) set_status(status, GTSC_ERR_FORMAT);
        return;
    }
    int32_t *sizes = (int32_t *)(it.scratch + it.p[1]);
    const uint64_t w0 = (uint64_t)tile * kBTile;
    for (uint64_t w = w0 + threadIdx.x; w < (uint64_t)g.warps && w < w0 + kBTile; w += kBThreads) {
        const int64_t e = (int32_t)ld_unaligned<4>(ends.ptr + 4 * w);
        const int64_t sz = e - (int64_t)d_gfc_start(g, (int64_t)w);
        const uint64_t subs = (d_gfc_cut(g, (int64_t)w) - d_gfc_begin(g, (int64_t)w)) / 32;
        if (sz < 0 || sz > (int64_t)(subs * (16 + 32 * (dbl ? 8 : 4)))) {
            set_status(status, GTSC_ERR_FORMAT);
            sizes[w] = 0;
        } else {
            sizes[w] = (int32_t)sz;
        }
    }
}

// A warp's GFC decode reads its chunk through a ring of four 512-byte segments in shared memory,
// filled by cp.async (16 bytes a lane) up to three segments ahead of the subchunk being parsed.
constexpr uint32_t kGfcSeg = 512, kGfcRing = 4 * kGfcSeg;

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t n)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <bool DBL>
__device__ void p_gfc_dec(const BItem &it, uint32_t tile, StreamDesc *S, uint32_t *status, uint8_t *sm)
{
    const StreamDesc meta = S[it.in[0]], payload = S[it.in[2]];
    StreamDesc &out = S[it.out[0]];
    if (payload.len == 0) {
        if (tile == 0 && threadIdx.x == 0) out.len = 0;
        return;
    }
    DGfc g;
    if (!gfc_meta(meta, DBL, g) || (uint64_t)g.warps > it.p[3]) return;  // reported by p_gfc_sizes
    constexpr int ES = DBL ? 8 : 4;
    if (g.n * ES > out.cap) {
        if (tile == 0 && threadIdx.x == 0) set_status(status, GTSC_ERR_CAPACITY);
        return;
    }
    if (tile == 0 && threadIdx.x == 0) out.len = g.n * ES;
    const int lane = threadIdx.x & 31;
    const int64_t w = (int64_t)tile * kBGfcChunks + (threadIdx.x >> 5);
    if (w >= g.warps) return;
    const int32_t *sizes = (const int32_t *)(it.scratch + it.p[1]);
    const unsigned long long *incl = (const unsigned long long *)(it.scratch + it.p[2]);
    const uint64_t size = (uint64_t)(uint32_t)sizes[w], end = incl[w];
    if (end > payload.len || end < size) {
        if (lane == 0) set_status(status, GTSC_ERR_FORMAT);
        return;
    }
    const uint64_t cb = d_gfc_begin(g, w), ce = d_gfc_cut(g, w);
    uint64_t pos = end - size, last = 0;
    const uint32_t mis = (uint32_t)((uintptr_t)payload.ptr & 15);
    const uint8_t *base = payload.ptr - mis;  // 16-byte aligned; stream bytes count from here
    const uint64_t nbytes = payload.len + mis, seg0 = (pos + mis) & ~15ull, lim = end + mis;
    uint32_t *ring = (uint32_t *)(sm + (threadIdx.x >> 5) * kGfcRing);
    const uint32_t ring_s = (uint32_t)__cvta_generic_to_shared(ring);
    uint32_t issued = 0;  // segments requested (one commit group each, empty past the chunk)
    auto issue = [&]() {
        const uint64_t sb = seg0 + (uint64_t)issued * kGfcSeg;
        if (sb < lim) {
            const uint64_t b = sb + 16 * lane;
            const uint32_t n = b >= nbytes ? 0u : (uint32_t)min((uint64_t)16, nbytes - b);
            cp_async16(ring_s + (issued & 3) * kGfcSeg + 16 * lane, n ? base + b : base, n);
        }
        cp_async_commit();
        issued++;
    };
    issue();
    issue();
    issue();
    for (uint64_t s = cb; s < ce; s += 32) {
        if (pos + 16 > end) {
            if (lane == 0) set_status(status, GTSC_ERR_FORMAT);
            cp_async_wait<0>();
            return;
        }
        // a subchunk reads ring bytes [rel, rel + 284): its 16-byte header, at most 32 x 8 payload
        // bytes and the two words after the last one
        const uint32_t rel = (uint32_t)(pos + mis - seg0), kcur = rel / kGfcSeg, kneed = (rel + 283) / kGfcSeg;
        __syncwarp();  // the segments before kcur are no longer read: their slots can be refilled
        while (issued < kcur + 4) issue();
        const uint32_t pend = issued - 1 - kneed;  // groups newer than the last one needed
        if (pend >= 3) cp_async_wait<3>();
        else if (pend == 2) cp_async_wait<2>();
        else if (pend == 1) cp_async_wait<1>();
        else cp_async_wait<0>();
        __syncwarp();
        const uint32_t hb = rel + (lane >> 1);
        const uint32_t nib = (ring[(hb >> 2) & 511] >> (8 * (hb & 3) + 4 * (lane & 1))) & 15u;
        const uint32_t code = nib & 7u;
        uint32_t mb = DBL ? (code >= 2 ? code + 1 : code) : code;
        if (!DBL && mb > 4) {
            set_status(status, GTSC_ERR_FORMAT);
            mb = 4;
        }
        uint32_t inc = mb;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, inc, 31);
        if (pos + 16 + total > end) {
            if (lane == 0) set_status(status, GTSC_ERR_FORMAT);
            cp_async_wait<0>();
            return;
        }
        // the lane's mb little-endian bytes from three ring words (bytes past mb are masked off)
        const uint32_t q = rel + 16 + (inc - mb), sh = 8 * (q & 3), qw = q >> 2;
        const uint32_t w0 = ring[qw & 511], w1 = ring[(qw + 1) & 511], w2 = ring[(qw + 2) & 511];
        uint64_t diff = ((uint64_t)__funnelshift_r(w1, w2, sh) << 32) | __funnelshift_r(w0, w1, sh);
        diff = mb ? diff & (~0ull >> (64 - 8 * mb)) : 0ull;
        if (nib & 8u) diff = 0ull - diff;
        uint64_t x = last + diff;
        if (!DBL) x &= 0xffffffffull;
        if (s + lane < g.n) st_elem<ES>(out.ptr, s + lane, x);
        pos += 16 + total;
        if (s == cb) last = __shfl_sync(0xffffffffu, x, 31);
    }
    cp_async_wait<0>();
    if (lane == 0 && pos != end) set_status(status, GTSC_ERR_FORMAT);
}

// ------------------------------------------------------------------------------- dispatch
// A framed buffer that does not parse leaves blob-resident stream pointers unset, so status[1]
// (set only by the parse kernel, which runs before every decode stage) turns all stages off.
__device__ __forceinline__ void parse_fail(uint32_t *status)
{
    set_status(status, GTSC_ERR_FORMAT);
    atomicExch(status + 1, 1u);
}

// elements a decode input holds (a DView or in[slot]); 0 when its AFL metadata is malformed
__device__ __forceinline__ uint64_t dview_len(const BItem &it, const StreamDesc *S, int slot, int es)
{
    const DView &d = it.dv[slot - 1];
    if (d.data < 0) return S[it.in[slot]].len / es;
    const StreamDesc data = S[d.data];
    if (d.afl_meta < 0) return data.len / es;
    const StreamDesc meta = S[d.afl_meta];
    if (!data.len || meta.len < 2) return 0;
    const int b = (int8_t)meta.ptr[0], rest = (int8_t)meta.ptr[1];
    const int64_t bits = (int64_t)data.len * 8 - rest;
    return (b < 1 || b > 8 * es || bits < 0) ? 0 : (uint64_t)bits / b;
}

// Tiles of an item that do work in a decode pass (tile 0 always runs: it sets the output length).
template <int OP>
__device__ __forceinline__ uint32_t dec_extent(const BItem &it, const StreamDesc *S)
{
    auto cdiv = [](uint64_t a, uint64_t b) { return (a + b - 1) / b; };
    uint64_t e = it.tiles;
    if constexpr (OP == B_SCALE_ADD) {
        e = cdiv(dview_len(it, S, 1, it.es), kBTile);
    } else if constexpr (OP == B_AFL_UNPACK) {
        const StreamDesc data = S[it.in[1]], meta = S[it.in[0]];
        uint64_t n = 0;
        if (data.len && meta.len >= 2) {
            const int b = (int8_t)meta.ptr[0], rest = (int8_t)meta.ptr[1];
            const int64_t bits = (int64_t)data.len * 8 - rest;
            if (b >= 1 && b <= 8 * it.es && bits >= 0) n = (uint64_t)bits / b;
        }
        e = cdiv(n, kBTile);
    } else if constexpr (OP == B_RLE_EXPAND) {
        const uint64_t runs = *(const unsigned long long *)(it.scratch + it.p[2]);
        const uint64_t n = runs ? ((const unsigned long long *)(it.scratch + it.p[1]))[runs - 1] : 0;
        e = cdiv(n, kBTile);
    } else if constexpr (OP == B_MERGE_COUNT) {
        uint64_t n;
        switch (it.es) {
        case 1: merge_stencil<1>(it, S[it.in[0]], n); break;
        case 2: merge_stencil<2>(it, S[it.in[0]], n); break;
        case 4: merge_stencil<4>(it, S[it.in[0]], n); break;
        default: merge_stencil<8>(it, S[it.in[0]], n); break;
        }
        e = cdiv(n, kBTile);
    } else if constexpr (OP == B_F2I_DEC) {
        const StreamDesc meta = S[it.in[0]];
        const int p = meta.len >= 4 ? (int32_t)ld_unaligned<4>(meta.ptr) : 0;
        const uint64_t k = dview_len(it, S, 1, 4);
        e = cdiv(p < 10 ? k : k * 4 / it.es, kBTile);
    }
    if (e == 0) e = 1;
    return (uint32_t)(e < it.tiles ? e : it.tiles);
}

template <int OP>
__device__ __forceinline__ void run_dec(const BItem &it, uint32_t tile, StreamDesc *S, uint32_t *status,
                                        unsigned char *smem);

constexpr bool dec_persistent(int op)
{
    return op == B_AFL_UNPACK || op == B_SCALE_ADD || op == B_F2I_DEC || op == B_RLE_EXPAND || op == B_MERGE_COUNT;
}

// One launch of a decode pass over every item: look-back passes one tile per block in claim order,
// the others persistent over the tiles (see k_bstage).
template <int OP>
__global__ void __launch_bounds__(kBThreads, 5)
k_bdec(const BItem *items, const uint32_t *item_of, StreamDesc *S, uint32_t *counter, uint32_t *status,
       uint32_t total_tiles)
{
    constexpr bool DYN = OP == B_DELTA_DEC || OP == B_RLE_SCAN;
    constexpr int kSmem = OP == B_MERGE                             ? 8 * kBTile
                          : OP == B_GFC_DEC                         ? kGfcRing * (kBThreads / 32)
                          : OP == B_RLE_EXPAND                      ? kXchgBlockBytes  // warp exchange
                                                                    : 16;
    __shared__ __align__(16) unsigned char smem[kSmem];
    if (*(volatile uint32_t *)(status + 1)) return;
    if constexpr (!dec_persistent(OP)) {
        uint32_t tile;
        const BItem &it = locate<DYN>(items, item_of, counter, tile);
        if (tile >= it.tiles) return;
        run_dec<OP>(it, tile, S, status, smem);
    } else {
        uint32_t t = blockIdx.x;
        uint32_t cur = 0xffffffffu;  // the item in the shared descriptor
        while (t < total_tiles) {
            const uint32_t k = item_of[t];
            if (k != cur) {
                __syncthreads();  // nobody reads the previous descriptor any more
                shared_item(items, k);
                cur = k;
            }
            const BItem &it = shared_item_ref();
            const uint32_t tile = t - (uint32_t)it.tile_base;
            if (tile >= dec_extent<OP>(it, S)) {
                const uint64_t next = it.tile_base + it.tiles;
                if (next >= total_tiles) break;
                t = (uint32_t)(next + (blockIdx.x + gridDim.x - next % gridDim.x) % gridDim.x);
                continue;
            }
            run_dec<OP>(it, tile, S, status, smem);
            __syncthreads();
            t += gridDim.x;
        }
    }
}

template <int OP>
__device__ __forceinline__ void run_dec(const BItem &it, uint32_t tile, StreamDesc *S, uint32_t *status,
                                        unsigned char *smem)
{
#define GTSC_ES_SWITCH(CALL)                       \
    switch (it.es) {                               \
    case 1: { constexpr int E = 1; CALL; } break;  \
    case 2: { constexpr int E = 2; CALL; } break;  \
    case 4: { constexpr int E = 4; CALL; } break;  \
    default: { constexpr int E = 8; CALL; } break; \
    }
    if constexpr (OP == B_NONE_COPY) p_none_copy(it, tile, S, status);
    else if constexpr (OP == B_AFL_UNPACK) { GTSC_ES_SWITCH(p_afl_unpack<E>(it, tile, S, status)) }
    else if constexpr (OP == B_DELTA_DEC) { GTSC_ES_SWITCH(p_delta_dec<E>(it, tile, S, status)) }
    else if constexpr (OP == B_SCALE_ADD) { GTSC_ES_SWITCH(p_scale_add<E>(it, tile, S, status)) }
    else if constexpr (OP == B_MERGE) { GTSC_ES_SWITCH(p_merge<E>(it, tile, S, status, smem)) }
    else if constexpr (OP == B_MERGE_COUNT) { GTSC_ES_SWITCH(p_merge_count<E>(it, tile, S)) }
    else if constexpr (OP == B_RLE_SCAN) p_rle_scan(it, tile, S, status);
    else if constexpr (OP == B_RLE_EXPAND) { GTSC_ES_SWITCH(p_rle_expand<E>(it, tile, S, status, smem)) }
    else if constexpr (OP == B_F2I_DEC) { GTSC_ES_SWITCH(p_f2i_dec<E>(it, tile, S, status)) }
    else if constexpr (OP == B_GFC_SIZES) p_gfc_sizes(it, tile, S, status);
    else if constexpr (OP == B_GFC_DEC) {
        if (it.es == 8) p_gfc_dec<true>(it, tile, S, status, smem);
        else p_gfc_dec<false>(it, tile, S, status, smem);
    }
#undef GTSC_ES_SWITCH
}

#ifdef GTSC_PERSISTENT_TU
// ------------------------------------------------------------------------------- persistent step
constexpr size_t kPersistSmemD = std::max<size_t>({8 * kBTile, kGfcRing * (kBThreads / 32), kXchgBlockBytes});

__device__ __forceinline__ uint32_t persist_extent_d(int op, const BItem &it, const StreamDesc *S)
{
    switch (op) {
    case B_AFL_UNPACK: return dec_extent<B_AFL_UNPACK>(it, S);
    case B_SCALE_ADD: return dec_extent<B_SCALE_ADD>(it, S);
    case B_F2I_DEC: return dec_extent<B_F2I_DEC>(it, S);
    case B_RLE_EXPAND: return dec_extent<B_RLE_EXPAND>(it, S);
    case B_MERGE_COUNT: return dec_extent<B_MERGE_COUNT>(it, S);
    default: return it.tiles;
    }
}

// The whole decode step in one launch (batch.hpp, PUnit); the merges' counting pass is the
// queue's first launch.
__global__ void __launch_bounds__(kBThreads, 4) k_bpersist_d(PersistArgs a)
{
    __shared__ __align__(16) unsigned char smem[kPersistSmemD];
    if (*(volatile uint32_t *)(a.status + 1)) return;  // the frames did not parse
    persist_loop(
        a, [](int op, const BItem &it, const StreamDesc *S) { return persist_extent_d(op, it, S); },
        [&](int op, const BItem &it, uint32_t tile) {
            switch (op) {
#define GTSC_RUN(OPC) case OPC: run_dec<OPC>(it, tile, a.S, a.status, smem); break;
                GTSC_RUN(B_NONE_COPY)
                GTSC_RUN(B_AFL_UNPACK)
                GTSC_RUN(B_DELTA_DEC)
                GTSC_RUN(B_SCALE_ADD)
                GTSC_RUN(B_MERGE)
                GTSC_RUN(B_MERGE_COUNT)
                GTSC_RUN(B_RLE_SCAN)
                GTSC_RUN(B_RLE_EXPAND)
                GTSC_RUN(B_F2I_DEC)
                GTSC_RUN(B_GFC_SIZES)
                GTSC_RUN(B_GFC_DEC)
#undef GTSC_RUN
            case B_GFC_SCAN: p_gfc_scan(it, tile, a.S, it.es == 8, it.mode != 0); break;
            default: set_status(a.status, GTSC_ERR_ARG); break;
            }
        });
}

#else

// ------------------------------------------------------------------------------- framing
// Framed buffer: uint64 column count C, uint64 blob bytes of every column (the directory), then the
// C blobs back to back.  The directory lets decode find every column without walking the blobs.
// Per column: pre-order nodes; node k of column c is cols[c].first + k in the node table.
__device__ __forceinline__ uint64_t frame_header_bytes(int ncols) { return 8 + 8 * (uint64_t)ncols; }

// col_off[0..ncols] = blob offsets, col_off[ncols] = total framed bytes; writes the directory
__global__ void k_frame_sizes(const BColumnDev *cols, int ncols, const BNodeDev *nodes, const StreamDesc *S,
                              unsigned long long *col_off, unsigned long long *total, uint8_t *framed)
{
    // one block: thread t sums its columns' blob sizes, then an exclusive scan gives offsets
    __shared__ unsigned long long ws[32];
    const int per = (ncols + kBThreads - 1) / kBThreads;
    unsigned long long mine = 0;
    for (int c = threadIdx.x * per; c < ncols && c < (int)(threadIdx.x + 1) * per; c++) {
        unsigned long long sz = 0;
        for (int k = 0; k < cols[c].n_nodes; k++) {
            const BNodeDev &nd = nodes[cols[c].first + k];
            sz += 8 + (nd.meta >= 0 ? S[nd.meta].len : 8);
            if (nd.data >= 0) sz += S[nd.data].len;
        }
        col_off[c] = sz;  // temporarily the blob size
        mine += sz;
    }
    unsigned long long tot;
    unsigned long long excl = block_exclusive_scan<kBThreads>(mine, ws, tot) + frame_header_bytes(ncols);
    unsigned long long *dir = (unsigned long long *)framed;  // the framed buffer is 256-byte aligned
    for (int c = threadIdx.x * per; c < ncols && c < (int)(threadIdx.x + 1) * per; c++) {
        const unsigned long long sz = col_off[c];
        dir[1 + c] = sz;
        col_off[c] = excl;
        excl += sz;
    }
    if (threadIdx.x == 0) {
        dir[0] = (unsigned long long)ncols;
        col_off[ncols] = tot + frame_header_bytes(ncols);
        *total = tot + frame_header_bytes(ncols);
    }
}

// one thread per column: node headers and the destinations of every segment
__global__ void k_frame_layout(const BColumnDev *cols, int ncols, BNodeDev *nodes, const StreamDesc *S,
                               const unsigned long long *col_off, uint8_t *framed)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncols) return;
    unsigned long long pos = col_off[c];
    for (int k = 0; k < cols[c].n_nodes; k++) {
        BNodeDev &nd = nodes[cols[c].first + k];
        const uint64_t ml = nd.meta >= 0 ? S[nd.meta].len : 8;
        const uint8_t h[8] = {(uint8_t)nd.enc, (uint8_t)(nd.enc >> 8), (uint8_t)nd.dt, (uint8_t)(nd.dt >> 8),
                              (uint8_t)ml, (uint8_t)(ml >> 8), (uint8_t)(ml >> 16), (uint8_t)(ml >> 24)};
        for (int b = 0; b < 8; b++) framed[pos + b] = h[b];
        nd.meta_dst = pos + 8;
        if (nd.meta < 0) {  // NoneEncoding metadata: size_t byte count of the data
            const uint64_t ds = S[nd.data].len;
            for (int b = 0; b < 8; b++) framed[pos + 8 + b] = (uint8_t)(ds >> (8 * b));
        }
        pos += 8 + ml;
        if (nd.data >= 0) {
            nd.data_dst = pos;
            pos += S[nd.data].len;
        }
    }
}

// copy items: p[0] = node table index, p[1] = 0 copy the node's metadata, 1 its data
__global__ void __launch_bounds__(kBThreads)
k_frame_copy(const BItem *items, const uint32_t *item_of, const BNodeDev *nodes, const StreamDesc *S, uint8_t *framed)
{
    uint32_t tile;
    const BItem &it = locate<false>(items, item_of, nullptr, tile);
    const BNodeDev &nd = nodes[it.p[0]];
    const StreamDesc src = S[it.p[1] ? nd.data : nd.meta];
    const uint64_t dst = it.p[1] ? nd.data_dst : nd.meta_dst;
    const uint64_t off = (uint64_t)tile * kCopyPiece;
    if (off >= src.len) return;
    const uint64_t n = src.len - off < kCopyPiece ? src.len - off : kCopyPiece;
    block_copy(framed + dst + off, src.ptr + off, n);
}

// decode, one block: reads the directory of the framed buffer into col_off[0..ncols]
__global__ void k_parse_directory(int ncols, unsigned long long *col_off, const uint8_t *const *framed_p,
                                  const unsigned long long *framed_bytes_p, uint32_t *status)
{
    __shared__ unsigned long long ws[32];
    __shared__ int s_bad;
    const uint8_t *framed = *framed_p;
    const uint64_t fb = *framed_bytes_p;
    const uint64_t hdr = frame_header_bytes(ncols);
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    // every length is at most fb < 2^40, so the sums below cannot wrap (ncols < 2^24)
    if (fb < hdr || fb >= (1ull << 40) || ld_unaligned<8>(framed) != (uint64_t)ncols) {
        if (threadIdx.x == 0) parse_fail(status);
        return;
    }
    const int per = (ncols + kBThreads - 1) / kBThreads;
    unsigned long long mine = 0;
    for (int c = threadIdx.x * per; c < ncols && c < (int)(threadIdx.x + 1) * per; c++) {
        const uint64_t len = ld_unaligned<8>(framed + 8 + 8 * (uint64_t)c);
        if (len > fb) s_bad = 1;
        mine += len > fb ? fb : len;
    }
    unsigned long long tot;
    unsigned long long excl = block_exclusive_scan<kBThreads>(mine, ws, tot) + hdr;
    for (int c = threadIdx.x * per; c < ncols && c < (int)(threadIdx.x + 1) * per; c++) {
        const uint64_t len = ld_unaligned<8>(framed + 8 + 8 * (uint64_t)c);
        col_off[c] = excl;
        excl += len > fb ? fb : len;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        col_off[ncols] = tot + hdr;
        if (s_bad || tot + hdr > fb) parse_fail(status);
    }
}

// decode, one thread per column: walks the column's blob and points its meta / data streams into it
__global__ void k_parse_frames(const BColumnDev *cols, int ncols, const BNodeDev *nodes, StreamDesc *S,
                               const unsigned long long *col_off, const uint8_t *const *framed_p, uint32_t *status)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncols) return;
    if (*(volatile uint32_t *)(status + 1)) return;  // the directory did not parse
    const uint8_t *framed = *framed_p;
    uint64_t pos = col_off[c];
    const uint64_t end = col_off[c + 1];
    for (int k = 0; k < cols[c].n_nodes; k++) {
        const BNodeDev &nd = nodes[cols[c].first + k];
        if (pos + 8 > end) { parse_fail(status); return; }
        const int enc = (int16_t)ld_unaligned<2>(framed + pos), dt = (int16_t)ld_unaligned<2>(framed + pos + 2);
        const int64_t ml = (int32_t)ld_unaligned<4>(framed + pos + 4);
        if (enc != nd.enc || dt != nd.dt || ml < 0 || pos + 8 + (uint64_t)ml > end) {
            parse_fail(status);
            return;
        }
        if (nd.meta >= 0) {
            S[nd.meta].ptr = (uint8_t *)framed + pos + 8;
            S[nd.meta].len = (uint64_t)ml;
        }
        pos += 8 + (uint64_t)ml;
        if (nd.data >= 0) {
            if (ml < 8) { parse_fail(status); return; }
            const uint64_t ds = ld_unaligned<8>(framed + pos - ml);
            if (ds > end - pos) { parse_fail(status); return; }
            S[nd.data].ptr = (uint8_t *)framed + pos;
            S[nd.data].len = ds;
            pos += ds;
        }
    }
    if (pos != end) parse_fail(status);
}

__global__ void k_zero_ranges(const unsigned long long *ranges, int n)
{
    // ranges: (pointer, bytes) pairs; bytes are multiples of 4 and pointers 4-byte aligned
    for (int r = blockIdx.x; r < n; r += gridDim.x) {
        uint32_t *p = (uint32_t *)ranges[2 * r];
        const uint64_t words = ranges[2 * r + 1] / 4;
        for (uint64_t k = threadIdx.x; k < words; k += blockDim.x) p[k] = 0u;
    }
}

#endif  // GTSC_PERSISTENT_TU

}  // namespace

#ifndef GTSC_PERSISTENT_TU
// as many blocks as fit at once for the streaming decode passes, else one block per tile
template <class K>
unsigned stage_grid_dec(K kernel, int op, uint64_t total_tiles)
{
    if (!dec_persistent(op)) return (unsigned)total_tiles;
    int per_sm = 0;
    GTSC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBThreads, 0));
    const uint64_t resident = (uint64_t)(per_sm > 1 ? per_sm : 1) * (uint64_t)sm_count();
    return (unsigned)(total_tiles < resident ? total_tiles : resident);
}

void launch_batch_decode_stage(int op, const BItem *d_items, const uint32_t *d_item_of, int n_items,
                               uint64_t total_tiles, StreamDesc *d_streams, uint32_t *d_counter, uint32_t *d_status,
                               cudaStream_t s)
{
    if (n_items == 0 || total_tiles == 0) return;
    if (total_tiles > 0x7fffffffull) fail(GTSC_ERR_CAPACITY, "batch: too many tiles in one stage");
    switch (op) {
#define GTSC_STAGE(OPC)                                                                                            \
    case OPC: {                                                                                                    \
        const unsigned g = stage_grid_dec(k_bdec<OPC>, OPC, total_tiles);                                          \
        k_bdec<OPC><<<g, kBThreads, 0, s>>>(d_items, d_item_of, d_streams, d_counter, d_status, (uint32_t)total_tiles); \
        break;                                                                                                     \
    }
        GTSC_STAGE(B_NONE_COPY)
        GTSC_STAGE(B_AFL_UNPACK)
        GTSC_STAGE(B_DELTA_DEC)
        GTSC_STAGE(B_SCALE_ADD)
        GTSC_STAGE(B_MERGE)
    case B_MERGE_COUNT: {
        int per_sm = 0;
        GTSC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_merge_count, kBThreads, 0));
        const uint64_t warps = (total_tiles + kBThreads / 32 - 1) / (kBThreads / 32);
        const uint64_t resident = (uint64_t)std::max(per_sm, 1) * (uint64_t)sm_count();
        const unsigned g = (unsigned)std::min<uint64_t>(warps, resident);
        k_merge_count<<<g, kBThreads, 0, s>>>(d_items, d_item_of, d_streams, d_status, (uint32_t)total_tiles);
        break;
    }
        GTSC_STAGE(B_RLE_SCAN)
        GTSC_STAGE(B_RLE_EXPAND)
        GTSC_STAGE(B_F2I_DEC)
        GTSC_STAGE(B_GFC_SIZES)
        GTSC_STAGE(B_GFC_DEC)
#undef GTSC_STAGE
    default: fail(GTSC_ERR_ARG, "batch: unknown pass");
    }
    GTSC_CUDA(cudaGetLastError());
}

uint64_t batch_copy_piece() { return kCopyPiece; }

void launch_frame_sizes(const BColumnDev *cols, int ncols, const BNodeDev *nodes, const StreamDesc *S,
                        unsigned long long *col_off, unsigned long long *total, uint8_t *framed, cudaStream_t s)
{
    k_frame_sizes<<<1, kBThreads, 0, s>>>(cols, ncols, nodes, S, col_off, total, framed);
    GTSC_CUDA(cudaGetLastError());
}

void launch_frame_layout(const BColumnDev *cols, int ncols, BNodeDev *nodes, const StreamDesc *S,
                         const unsigned long long *col_off, uint8_t *framed, cudaStream_t s)
{
    k_frame_layout<<<(ncols + 127) / 128, 128, 0, s>>>(cols, ncols, nodes, S, col_off, framed);
    GTSC_CUDA(cudaGetLastError());
}

void launch_frame_copy(const BItem *items, const uint32_t *item_of, int n_items, uint64_t total_tiles,
                       const BNodeDev *nodes, const StreamDesc *S, uint8_t *framed, cudaStream_t s)
{
    if (!n_items || !total_tiles) return;
    k_frame_copy<<<(unsigned)total_tiles, kBThreads, 0, s>>>(items, item_of, nodes, S, framed);
    GTSC_CUDA(cudaGetLastError());
}

void launch_parse_frames(const BColumnDev *cols, int ncols, const BNodeDev *nodes, StreamDesc *S,
                         unsigned long long *col_off, const uint8_t *const *framed_p,
                         const unsigned long long *framed_bytes_p, uint32_t *status, cudaStream_t s)
{
    k_parse_directory<<<1, kBThreads, 0, s>>>(ncols, col_off, framed_p, framed_bytes_p, status);
    GTSC_CUDA(cudaGetLastError());
    k_parse_frames<<<(ncols + 127) / 128, 128, 0, s>>>(cols, ncols, nodes, S, col_off, framed_p, status);
    GTSC_CUDA(cudaGetLastError());
}

void launch_zero_ranges(const unsigned long long *ranges, int n, cudaStream_t s)
{
    if (!n) return;
    k_zero_ranges<<<n < 1024 ? n : 1024, 256, 0, s>>>(ranges, n);
    GTSC_CUDA(cudaGetLastError());
}

#else

void launch_batch_persistent_d(const PersistArgs &a, cudaStream_t s)
{
    if (a.total == 0) return;
    int per_sm = 0;
    GTSC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bpersist_d, kBThreads, 0));
    const uint64_t grid = std::min<uint64_t>((uint64_t)std::max(per_sm, 1) * (uint64_t)sm_count(),
                                             (uint64_t)a.total);
    k_bpersist_d<<<(unsigned)grid, kBThreads, 0, s>>>(a);
    GTSC_CUDA(cudaGetLastError());
}

#endif  // GTSC_PERSISTENT_TU

}  // namespace gtsc
