// batch_kernels.cu -- the compress passes of the batched engine.
//
// Each pass is one templated stage kernel launched with one block per (item, tile); the block finds
// its item by binary search over the items' first tiles.  Passes that rank elements across tiles
// (split, RLE heads, GFC offsets) claim tiles from a counter and chain them with the decoupled
// look-back of scan.cuh, per item.  Every pass reads its input length from the stream table and
// writes its outputs' lengths there; tile 0 (or the tile that ends the input) writes metadata.
// Byte layouts are the per-encoding ones of encodings.cu (and of the reference).
//
// The stage kernels read their inputs through the read-only path (every input was written by an
// earlier launch).  batch_persist_c.cu compiles this file a second time, with GTSC_PERSISTENT_TU and
// coherent loads, for the persistent kernel, in which later passes read what earlier passes of the
// same launch wrote.
#include "batch_dev.cuh"

#include <algorithm>
#include <type_traits>

namespace gtsc {

namespace {

// ------------------------------------------------------------------------------- min / max
// VPT values of a view starting at base (zeros past the view): one vector run when a run is whole
// 16-byte chunks, else element loads
template <int ES, int VPT>
__device__ __forceinline__ void load_view_any(const BItem &it, const ViewCtx &vc, const uint8_t *src, uint64_t base,
                                              uint64_t (&v)[VPT])
{
    if constexpr ((VPT * ES) % 16 == 0) {
        load_view<ES, VPT>(it, vc, src, base, v);
    } else {
#pragma unroll
        for (int j = 0; j < VPT; j++) v[j] = base + j < vc.n ? view_elem<ES>(it, vc, src, base + j) : 0;
    }
}

// A tile of it.p[0] values (the tuned min/max tile; a multiple of kBThreads * VPT): rounds of VPT
// consecutive values a thread, two rounds loaded before either is reduced.
template <int ES, int VPT>
__device__ void p_minmax_v(const BItem &it, uint32_t tile, StreamDesc *S)
{
    const StreamDesc in = S[it.in[0]];
    const ViewCtx vc = view_ctx<ES>(it, in);
    const uint64_t n = vc.n;
    const uint64_t T = it.p[0];
    const uint64_t t0 = (uint64_t)tile * T;
    if (t0 >= n) return;
    const uint64_t end = n < t0 + T ? n : t0 + T;
    const Order o = (Order)it.order;
    constexpr uint64_t R = (uint64_t)kBThreads * VPT;  // values of one round of the block
    uint64_t kmin = ~0ull, kmax = 0;
    if constexpr (ES <= 4) {
        // 32-bit keys of the same order (sign bit flipped for integers, order_key's map for floats),
        // turned into the accumulator's 64-bit keys once per thread
        const bool f32 = o == ORD_F32;
        constexpr uint32_t SH = 32 - 8 * ES;
        uint32_t k32min = ~0u, k32max = 0;
        bool seen = false;
        auto key32 = [&](uint32_t u) {
            if (f32) return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
            return (uint32_t)((int32_t)(u << SH) >> SH) ^ 0x80000000u;
        };
        for (uint64_t b0 = t0 + (uint64_t)threadIdx.x * VPT; b0 < end; b0 += 2 * R) {
            const uint64_t b1 = b0 + R;
            uint32_t u[2][VPT];
            {
                uint64_t v[VPT];
                load_view_any<ES, VPT>(it, vc, in.ptr, b0, v);
#pragma unroll
                for (int j = 0; j < VPT; j++) u[0][j] = (uint32_t)v[j];
                if (b1 < end) load_view_any<ES, VPT>(it, vc, in.ptr, b1, v);
#pragma unroll
                for (int j = 0; j < VPT; j++) u[1][j] = (uint32_t)v[j];
            }
#pragma unroll
            for (int r = 0; r < 2; r++) {
                const uint64_t base = r ? b1 : b0;
                const uint32_t cnt = base >= end ? 0u : end - base < (uint64_t)VPT ? (uint32_t)(end - base) : VPT;
#pragma unroll
                for (int j = 0; j < VPT; j++) {
                    const bool ok = (uint32_t)j < cnt && !(f32 && (u[r][j] & 0x7fffffffu) > 0x7f800000u);
                    const uint32_t k = key32(u[r][j]);
                    k32min = ok && k < k32min ? k : k32min;
                    k32max = ok && k > k32max ? k : k32max;
                    seen |= ok;
                }
            }
        }
        if (seen) {
            const uint32_t umin = f32 ? ((k32min & 0x80000000u) ? (k32min ^ 0x80000000u) : ~k32min)
                                      : (k32min ^ 0x80000000u);
            const uint32_t umax = f32 ? ((k32max & 0x80000000u) ? (k32max ^ 0x80000000u) : ~k32max)
                                      : (k32max ^ 0x80000000u);
            kmin = order_key(umin, 4, o);  // umin / umax are sign-extended to 32 bits
            kmax = order_key(umax, 4, o);
        }
    } else {
        for (uint64_t base = t0 + (uint64_t)threadIdx.x * VPT; base < end; base += R) {
            uint64_t v[VPT];
            load_view_any<ES, VPT>(it, vc, in.ptr, base, v);
#pragma unroll
            for (int j = 0; j < VPT; j++) {
                if (base + j >= end || is_nan_bits(v[j], o)) continue;
                const uint64_t k = order_key(v[j], ES, o);
                kmin = k < kmin ? k : kmin;
                kmax = k > kmax ? k : kmax;
            }
        }
    }
    block_minmax(kmin, kmax);
    if (threadIdx.x == 0) {
        MinMaxAcc *acc = (MinMaxAcc *)it.scratch;
        if (kmin != ~0ull) atomicMax(&acc->nkmin, (unsigned long long)~kmin);
        if (kmax != 0) atomicMax(&acc->kmax, (unsigned long long)kmax);
    }
}

// the min/max pass with the tuned values per thread (it.p[1]: 1, 2, 4, 8 or 16)
template <int ES>
__device__ void p_minmax(const BItem &it, uint32_t tile, StreamDesc *S)
{
    switch (it.p[1]) {
    case 1: p_minmax_v<ES, 1>(it, tile, S); break;
    case 2: p_minmax_v<ES, 2>(it, tile, S); break;
    case 4: p_minmax_v<ES, 4>(it, tile, S); break;
    case 8: p_minmax_v<ES, 8>(it, tile, S); break;
    default: p_minmax_v<ES, 16>(it, tile, S); break;
    }
}

// ------------------------------------------------------------------------------- delta
template <int ES>
__device__ void p_delta_enc(const BItem &it, uint32_t tile, StreamDesc *S)
{
    const StreamDesc in = S[it.in[0]];
    const ViewCtx vc = view_ctx<ES>(it, in);
    const uint64_t n = vc.n;
    if (tile == 0 && threadIdx.x == 0) {
        StreamDesc &m = S[it.out[0]];
        if (n) {
            st_elem<ES>(m.ptr, 0, view_elem<ES>(it, vc, in.ptr, 0));
            m.len = ES;
            S[it.out[1]].len = (n - 1) * ES;
        } else {
            m.len = 0;
            S[it.out[1]].len = 0;
        }
    }
    const uint64_t m = n ? n - 1 : 0;
    const uint64_t base = (uint64_t)tile * kBTile + (uint64_t)threadIdx.x * kBVPT;
    if (base >= m) return;
    uint64_t v[kBVPT];
    load_view<ES, kBVPT>(it, vc, in.ptr, base, v);
    const uint64_t next = base + kBVPT < n ? view_elem<ES>(it, vc, in.ptr, base + kBVPT) : 0;
    uint64_t d[kBVPT];
#pragma unroll
    for (int j = 0; j + 1 < (int)kBVPT; j++) d[j] = wrap_es(v[j + 1] - v[j], ES);
    d[kBVPT - 1] = wrap_es(next - v[kBVPT - 1], ES);
    store_run<ES, kBVPT>(S[it.out[1]].ptr, base, m, d);
}

// ------------------------------------------------------------------------------- scale
template <int ES>
__device__ void p_scale_sub(const BItem &it, uint32_t tile, StreamDesc *S)
{
    const StreamDesc in = S[it.in[0]];
    const ViewCtx vc = view_ctx<ES>(it, in);
    const uint64_t n = vc.n;
    uint64_t mnb = 0, mxb = 0;
    acc_minmax((const MinMaxAcc *)it.scratch, ES, ORD_INT, mnb, mxb);
    const uint64_t mn = scale_min(mnb, mxb, ES);
    if (tile == 0 && threadIdx.x == 0) {
        if (n) {
            st_elem<ES>(S[it.out[0]].ptr, 0, mn);
            S[it.out[0]].len = ES;
        } else {
            S[it.out[0]].len = 0;
        }
        S[it.out[1]].len = n * ES;
    }
    const uint64_t base = (uint64_t)tile * kBTile + (uint64_t)threadIdx.x * kBVPT;
    if (base >= n) return;
    uint64_t v[kBVPT];
    load_view<ES, kBVPT>(it, vc, in.ptr, base, v);
#pragma unroll
    for (int j = 0; j < (int)kBVPT; j++) v[j] = wrap_es(v[j] - mn, ES);
    store_run<ES, kBVPT>(S[it.out[1]].ptr, base, n, v);
}

// ------------------------------------------------------------------------------- AFL pack
__device__ __forceinline__ uint32_t afl_slot(uint32_t i) { return i + (i >> 4); }
template <int ES>
__device__ void p_afl_pack(const BItem &it, uint32_t tile, StreamDesc *S, unsigned long long *sv)
{
    const StreamDesc in = S[it.in[0]];
    const ViewCtx vc = view_ctx<ES>(it, in);
    const uint64_t n = vc.n;
    uint64_t mnb = 0, mxb = 0;
    int b;
    if (it.vflags & 1) {
        // the view ends with a scale by c = scale_min(min, max) of the scale's input: c = 0 leaves
        // [min, max]; c = min maps onto [0, max - min], unless max - min passes the type's largest
        // value (scale_min keeps c = min for the most negative min): then values wrap negative
        // and the width is the full word, as BITLEN gives for any negative minimum
        // the last scale of the view (static indices: no local-memory copy of the context)
        uint64_t c = 0;
        const uint8_t *scr = nullptr;
#pragma unroll
        for (int k = 0; k < kMaxViewOps; k++)
            if (it.vop[k] == V_SCALE) {
                c = vc.c[k];
                scr = it.vscr[k];
            }
        acc_minmax((const MinMaxAcc *)scr, ES, ORD_INT, mnb, mxb);
        if (c == 0) {
            b = bitlen_signed(sext(mnb, ES), sext(mxb, ES), ES);
        } else {
            const uint64_t span = (uint64_t)sext(mxb, ES) - (uint64_t)sext(mnb, ES);
            const uint64_t tmax = (ES == 8 ? ~0ull : ((1ull << (8 * ES)) - 1)) >> 1;
            b = span > tmax ? 8 * ES : bitlen_signed(0, (int64_t)span, ES);
        }
    } else {
        acc_minmax((const MinMaxAcc *)it.scratch, ES, ORD_INT, mnb, mxb);
        b = bitlen_signed(sext(mnb, ES), sext(mxb, ES), ES);
    }
    const uint64_t W = 8ull * ES;
    const uint64_t out_bytes = n ? (b * n + W - 1) / W * ES : 0;
    if (tile == 0 && threadIdx.x == 0) {
        StreamDesc &m = S[it.out[0]];
        if (n) {
            m.ptr[0] = (uint8_t)b;
            m.ptr[1] = (uint8_t)(int8_t)(out_bytes * 8 - n * (uint64_t)b);
            m.ptr[2] = 0;
            m.ptr[3] = 0;
            m.len = 4;
        } else {
            m.len = 0;
        }
        S[it.out[1]].len = out_bytes;
    }
    const uint64_t t0 = (uint64_t)tile * kBTile;
    if (t0 >= n) return;
    uint8_t *out = S[it.out[1]].ptr;
    if constexpr (ES <= 4) {
        // b <= 32.  Thread t packs its 16 values (tile bits [16 b t, 16 b (t + 1))) into a register
        // and stores whole words to the tile's words in shared memory; the word it shares with the
        // thread before it (a start inside a word) and the one it shares with the thread after it
        // (an end inside a word) are or-ed in.  Word w sits at w + w / 32, so that threads storing
        // b / 2 words apart spread over the banks.  A tile's output starts on a word: 4096 b / 32.
        uint32_t *ow = (uint32_t *)sv;
        auto slot = [](uint32_t w) { return w + (w >> 5); };
        const uint32_t vmask32 = b >= 32 ? ~0u : ((1u << b) - 1);
        uint64_t v[kBVPT];
        const uint64_t base = t0 + (uint64_t)threadIdx.x * kBVPT;
        load_view<ES, kBVPT>(it, vc, in.ptr, base, v);
        const uint32_t bit0 = threadIdx.x * kBVPT * (uint32_t)b;
        if (bit0 & 31) ow[slot(bit0 >> 5)] = 0;
        __syncthreads();
        uint32_t wi = bit0 >> 5, fill = bit0 & 31;
        bool shared_first = fill != 0;
        uint64_t acc = 0;
#pragma unroll
        for (int j = 0; j < (int)kBVPT; j++) {
            const uint32_t u = base + j < n ? ((uint32_t)v[j] & vmask32) : 0u;
            acc |= (uint64_t)u << fill;
            fill += (uint32_t)b;
            if (fill >= 32) {
                if (shared_first) atomicOr(&ow[slot(wi)], (uint32_t)acc);
                else ow[slot(wi)] = (uint32_t)acc;
                shared_first = false;
                ++wi;
                acc >>= 32;
                fill -= 32;
            }
        }
        if (fill) atomicOr(&ow[slot(wi)], (uint32_t)acc);
        __syncthreads();
        const uint64_t total_words = (out_bytes + 3) / 4;
        const uint64_t w0 = t0 * (uint64_t)b / 32;
        uint64_t w_end = w0 + 128u * (uint32_t)b;
        if (w_end > total_words) w_end = total_words;
        for (uint64_t w = w0 + threadIdx.x; w < w_end; w += kBThreads) {
            const uint32_t word = ow[slot((uint32_t)(w - w0))];
            if (4 * w + 4 <= out_bytes) {
                reinterpret_cast<uint32_t *>(out)[w] = word;
            } else {
                for (int k = 0; k < 4; k++)
                    if (4 * w + k < out_bytes) out[4 * w + k] = (uint8_t)(word >> (8 * k));
            }
        }
        return;
    }
    const uint64_t vmask = b >= 64 ? ~0ull : ((1ull << b) - 1);
    const uint64_t cnt = n - t0 < kBTile ? n - t0 : kBTile;
    // the tile's values in shared memory, skewed by one slot per 16 values (afl_slot) so that a
    // thread's run of 16 and the word gather below both spread over the banks
    if (vc.plain && cnt == kBTile && ((uintptr_t)in.ptr & 15) == 0) {
        const uint8_t *src = in.ptr + t0 * ES;
        constexpr int PER = 16 / ES;
        for (int c = threadIdx.x; c < (int)kBTile / PER; c += kBThreads) {
            const uint4 v = ld_chunk(src + 16 * c);
#pragma unroll
            for (int j = 0; j < PER; j++) sv[afl_slot(c * PER + j)] = chunk_elem<ES>(v, j) & vmask;
        }
    } else {
        uint64_t v[kBVPT];
        const uint64_t base = t0 + (uint64_t)threadIdx.x * kBVPT;
        load_view<ES, kBVPT>(it, vc, in.ptr, base, v);
#pragma unroll
        for (int j = 0; j < (int)kBVPT; j++) {
            const uint32_t i = threadIdx.x * kBVPT + j;
            sv[afl_slot(i)] = base + j < n ? (v[j] & vmask) : 0ull;
        }
    }
    if (threadIdx.x < 4) sv[afl_slot(kBTile + threadIdx.x)] = 0;
    __syncthreads();
    const uint64_t total_words = (out_bytes + 3) / 4;
    const uint64_t w0 = t0 * (uint64_t)b / 32;
    uint64_t w_end = (t0 + kBTile) * (uint64_t)b / 32;
    if (w_end > total_words) w_end = total_words;
    for (uint64_t w = w0 + threadIdx.x; w < w_end; w += kBThreads) {
        const uint32_t p = (uint32_t)(w - w0) * 32u;
        uint32_t a = p / (uint32_t)b;
        const uint32_t s = p - a * (uint32_t)b;
        uint64_t acc = sv[afl_slot(a)] >> s;
        int filled = b - (int)s;
        ++a;
        while (filled < 32) {
            acc |= sv[afl_slot(a)] << filled;
            filled += b;
            ++a;
        }
        const uint32_t word = (uint32_t)acc;
        if (4 * w + 4 <= out_bytes) {
            reinterpret_cast<uint32_t *>(out)[w] = word;
        } else {
            for (int k = 0; k < 4; k++)
                if (4 * w + k < out_bytes) out[4 * w + k] = (uint8_t)(word >> (8 * k));
        }
    }
}

// ------------------------------------------------------------------------------- histogram
__device__ __forceinline__ uint64_t bhash(uint64_t k)
{
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

struct HTab {
    BHistHdr *hdr;
    unsigned long long *keys;
    unsigned int *counts;
    unsigned int *used;
    unsigned long long *nan;   // 4 per histogram tile
    unsigned long long *part;  // top-k partials: 4 x (key, bits, count) per histogram tile
    uint64_t cap;
};
__device__ __forceinline__ HTab htab(const BItem &it)
{
    // p[0] = table capacity, p[1] = histogram tiles, p[2] = table offset in the node scratch
    HTab t;
    t.cap = it.p[0];
    uint8_t *b = it.scratch + it.p[2];
    t.hdr = (BHistHdr *)b;
    t.keys = (unsigned long long *)(b + 16);
    t.counts = (unsigned int *)(b + 16 + 8 * t.cap);
    t.used = (unsigned int *)(b + 16 + 12 * t.cap);
    t.nan = (unsigned long long *)(b + 16 + 16 * t.cap);
    t.part = t.nan + 4 * it.p[1];
    return t;
}

__device__ void g_insert(const HTab &t, unsigned long long key, unsigned int c, uint32_t *status)
{
    constexpr unsigned long long EMPTY = ~0ull;
    if (key == EMPTY) {
        atomicAdd(&t.hdr->special, c);
        return;
    }
    const uint64_t mask = t.cap - 1;
    uint64_t h = bhash(key) & mask;
    for (uint64_t probe = 0; probe < t.cap && probe < 8192; probe++) {
        const unsigned long long prev = atomicCAS(t.keys + h, EMPTY, key);
        if (prev == EMPTY) {
            const unsigned int u = atomicAdd(&t.hdr->used, 1u);
            t.used[u] = (unsigned int)h;
            atomicAdd(t.counts + h, c);
            return;
        }
        if (prev == key) {
            atomicAdd(t.counts + h, c);
            return;
        }
        h = (h + 1) & mask;
    }
    atomicExch(&t.hdr->overflow, 1u);
    set_status(status, GTSC_ERR_CAPACITY);
}

// Adds P (key, count) pairs of a thread to the node's global table (a zero count adds nothing).
// Each key's first slot is read with a plain load, all P loads in flight together: after a
// column's first tiles most keys are already there, and their counts are then added with
// reductions that nothing waits for.  A key not at its first slot takes the full insert.  (Keys
// never move once set, so a slot read holding the key is the key's slot.)
template <int P>
__device__ __forceinline__ void g_insert_many(const HTab &t, const unsigned long long (&key)[P],
                                              const uint32_t (&cnt)[P], uint32_t *status)
{
    constexpr unsigned long long EMPTY = ~0ull;
    const uint64_t mask = t.cap - 1;
    uint64_t h[P];
    unsigned long long cur[P];
#pragma unroll
    for (int j = 0; j < P; j++) {
        h[j] = bhash(key[j]) & mask;
        cur[j] = cnt[j] && key[j] != EMPTY ? *(volatile const unsigned long long *)(t.keys + h[j]) : EMPTY;
    }
#pragma unroll
    for (int j = 0; j < P; j++) {
        if (!cnt[j]) continue;
        if (key[j] != EMPTY && cur[j] == key[j]) atomicAdd(t.counts + h[j], cnt[j]);
        else g_insert(t, key[j], cnt[j], status);
    }
}

template <int ES>
__device__ void p_hist(const BItem &it, uint32_t tile, StreamDesc *S, uint32_t *status, unsigned char *smem)
{
    constexpr unsigned long long EMPTY = ~0ull;
    unsigned long long *skeys = (unsigned long long *)smem;
    unsigned int *scounts = (unsigned int *)(smem + 8 * kBHistSmem);
    unsigned long long(*snan)[4] = (unsigned long long(*)[4])(smem + 8 * kBHistPacked);
    const StreamDesc in = S[it.in[0]];
    const ViewCtx vc = view_ctx<ES>(it, in);
    const uint64_t n = vc.n;
    const uint64_t HT = it.p[3];  // the tuned histogram tile
    const uint64_t t0 = (uint64_t)tile * HT;
    const HTab t = htab(it);
    const Order o = (Order)it.order;
    if (it.mode == 4 && t0 < n) {
        // dict: clear this tile's share of the 2-bit code words (out1 after its 16 + 4*es header)
        uint32_t *words = (uint32_t *)(S[it.out[1]].ptr + 16 + 4 * ES);
        const uint64_t e_end = n < t0 + HT ? n : t0 + HT;
        for (uint64_t w = t0 / 16 + threadIdx.x; w < (e_end + 15) / 16; w += kBThreads) words[w] = 0u;
    }
    unsigned long long nan_min[4] = {EMPTY, EMPTY, EMPTY, EMPTY};
    if (ES <= 4 && t0 < n) {
        // values of up to 4 bytes: 32-bit keys and 16-bit counts (a tile holds at most
        // kBHistTileMax = 32768 values, so a count never wraps), two counts a word, as many slots as
        // the block's shared buffer holds (5456: a 32K tile of Zipf ids, 3,500-4,000 distinct
        // values, leaves the table under 3/4 full, so few inserts run out of probes).  A value
        // already in the table costs a plain key read and one 32-bit atomicAdd.  0xffffffff marks an
        // empty slot, so that value itself is counted apart.  Each thread reads 16 consecutive bytes
        // a round (one vector load), two rounds in flight before either is inserted; slots are
        // chosen by a multiplicative hash scaled to the table.
        constexpr uint32_t SL = kBHistSlots16;
        static_assert(6 * SL <= 8 * kBHistPacked, "the table fits the shared buffer");
        static_assert(kBHistTileMax <= 65535, "a 16-bit count holds a tile's values");
        uint32_t *k32 = (uint32_t *)smem;
        uint32_t *c16w = k32 + SL;
        __shared__ uint32_t s_ones;
        for (int i = threadIdx.x; i < (int)SL; i += kBThreads) k32[i] = 0xffffffffu;
        for (int i = threadIdx.x; i < (int)SL / 2; i += kBThreads) c16w[i] = 0u;
        if (threadIdx.x == 0) s_ones = 0;
        __syncthreads();
        const uint64_t end = n < t0 + HT ? n : t0 + HT;
        constexpr int VPT = 16 / ES;
        constexpr uint64_t R = (uint64_t)kBThreads * VPT;  // values of one round of the block
        // a thread counts a run of equal values in registers and inserts the run once when the
        // value changes (a constant or run-heavy column then costs a compare per value)
        uint32_t run_key = 0, run_cnt = 0;
        auto add = [&](uint32_t kk, uint32_t c) {
            uint32_t h = (uint32_t)(((uint64_t)(kk * 0x9E3779B1u) * SL) >> 32);
            for (int p = 0; p < 8; p++) {
                uint32_t cur = ((volatile uint32_t *)k32)[h];
                if (cur == 0xffffffffu) cur = atomicCAS(&k32[h], 0xffffffffu, kk);
                if (cur == 0xffffffffu || cur == kk) {
                    atomicAdd(&c16w[h >> 1], c << (16 * (h & 1)));
                    return;
                }
                h = h + 1 == SL ? 0 : h + 1;
            }
            g_insert(t, (unsigned long long)kk, c, status);
        };
        auto insert = [&](uint32_t kk, bool valid) {
            if (!valid) return;
            if (run_cnt && kk == run_key) {  // run_key is never a NaN or 0xffffffff
                ++run_cnt;
                return;
            }
            if (ES == 4 && is_nan_bits(kk, o)) {
                unsigned long long k = order_key(kk, ES, o);
#pragma unroll
                for (int j = 0; j < 4; j++)
                    if (k < nan_min[j]) { const unsigned long long x = nan_min[j]; nan_min[j] = k; k = x; }
                return;
            }
            if (kk == 0xffffffffu) {
                atomicAdd(&s_ones, 1u);
                return;
            }
            if (run_cnt) add(run_key, run_cnt);
            run_key = kk;
            run_cnt = 1;
        };
        const uint32_t lane = threadIdx.x & 31u;
        const uint64_t wfirst = t0 + (uint64_t)(threadIdx.x - lane) * VPT;
        for (uint64_t w0 = wfirst; w0 < end; w0 += 2 * R) {
            const uint64_t b0 = w0 + (uint64_t)lane * VPT, b1 = b0 + R;
            uint32_t u[2][VPT];
            {
                uint64_t v[VPT];
                if (b0 < end) load_view_any<ES, VPT>(it, vc, in.ptr, b0, v);
#pragma unroll
                for (int j = 0; j < VPT; j++) u[0][j] = (uint32_t)v[j];
                if (b1 < end) load_view_any<ES, VPT>(it, vc, in.ptr, b1, v);
#pragma unroll
                for (int j = 0; j < VPT; j++) u[1][j] = (uint32_t)v[j];
            }
#pragma unroll
            for (int r = 0; r < 2; r++) {
                const uint64_t base = r ? b1 : b0;
                const uint32_t cnt = base >= end ? 0u : end - base < (uint64_t)VPT ? (uint32_t)(end - base) : VPT;
#pragma unroll
                for (int j = 0; j < VPT; j++) insert(u[r][j], (uint32_t)j < cnt);
            }
        }
        if (run_cnt) add(run_key, run_cnt);
        __syncthreads();
        for (int i0 = threadIdx.x; i0 < (int)SL; i0 += 4 * kBThreads) {
            unsigned long long k[4];
            uint32_t c[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int i = i0 + j * kBThreads;
                const uint32_t kk = i < (int)SL ? k32[i] : 0xffffffffu;
                k[j] = kk;
                c[j] = kk != 0xffffffffu ? (c16w[i >> 1] >> (16 * (i & 1))) & 0xffffu : 0u;
            }
            g_insert_many<4>(t, k, c, status);
        }
        if (threadIdx.x == 0 && s_ones) g_insert(t, 0xffffffffull, s_ones, status);
    } else if (t0 < n) {
        // 8-byte values: 64-bit keys, two values a round (one 16-byte load), two rounds in flight
        for (int i = threadIdx.x; i < (int)kBHistSmem; i += kBThreads) {
            skeys[i] = EMPTY;
            scounts[i] = 0;
        }
        __syncthreads();
        const uint64_t end = n < t0 + HT ? n : t0 + HT;
        constexpr int VPT = 2;
        constexpr uint64_t R = (uint64_t)kBThreads * VPT;
        constexpr uint32_t HSH = 32 - 11;  // log2(kBHistSmem) = 11
        static_assert(kBHistSmem == 2048, "the slot hash takes the top 11 bits");
        const uint32_t lane = threadIdx.x & 31u;
        unsigned long long run_key = 0;
        uint32_t run_cnt = 0;
        auto add = [&](unsigned long long key, uint32_t c) {
            if (key != EMPTY) {
                uint32_t h = ((uint32_t)(key ^ (key >> 32)) * 0x9E3779B1u) >> HSH;
                for (int p = 0; p < 8; p++) {
                    unsigned long long cur = ((volatile unsigned long long *)skeys)[h];
                    if (cur == EMPTY) cur = atomicCAS(&skeys[h], EMPTY, key);
                    if (cur == EMPTY || cur == key) {
                        atomicAdd(&scounts[h], c);
                        return;
                    }
                    h = (h + 1) & (kBHistSmem - 1);
                }
            }
            g_insert(t, key, c, status);
        };
        auto insert = [&](unsigned long long key, bool valid) {
            if (!valid) return;
            if (run_cnt && key == run_key) {  // run_key is never a NaN
                ++run_cnt;
                return;
            }
            if (is_nan_bits(key, o)) {
                unsigned long long k = order_key(key, ES, o);
#pragma unroll
                for (int j = 0; j < 4; j++)
                    if (k < nan_min[j]) { const unsigned long long x = nan_min[j]; nan_min[j] = k; k = x; }
                return;
            }
            if (run_cnt) add(run_key, run_cnt);
            run_key = key;
            run_cnt = 1;
        };
        const uint64_t wfirst = t0 + (uint64_t)(threadIdx.x - lane) * VPT;
        for (uint64_t w0 = wfirst; w0 < end; w0 += 2 * R) {
            const uint64_t b0 = w0 + (uint64_t)lane * VPT, b1 = b0 + R;
            uint64_t u[2][VPT];
            if (b0 < end) load_view_any<ES, VPT>(it, vc, in.ptr, b0, u[0]);
            if (b1 < end) load_view_any<ES, VPT>(it, vc, in.ptr, b1, u[1]);
#pragma unroll
            for (int r = 0; r < 2; r++) {
                const uint64_t base = r ? b1 : b0;
                const uint32_t cnt = base >= end ? 0u : end - base < (uint64_t)VPT ? (uint32_t)(end - base) : VPT;
#pragma unroll
                for (int j = 0; j < VPT; j++) insert(u[r][j], (uint32_t)j < cnt);
            }
        }
        if (run_cnt) add(run_key, run_cnt);
        __syncthreads();
        for (int i0 = threadIdx.x; i0 < (int)kBHistSmem; i0 += 4 * kBThreads) {
            unsigned long long k[4];
            uint32_t c[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int i = i0 + j * kBThreads;
                k[j] = i < (int)kBHistSmem ? skeys[i] : EMPTY;
                c[j] = k[j] != EMPTY ? scounts[i] : 0u;
            }
            g_insert_many<4>(t, k, c, status);
        }
    }
    // this tile's 4 smallest NaN sort keys
    for (int off = 16; off > 0; off >>= 1) {
        unsigned long long other[4], merged[4];
#pragma unroll
        for (int j = 0; j < 4; j++) other[j] = __shfl_xor_sync(0xffffffffu, nan_min[j], off);
        int a = 0, b2 = 0;
#pragma unroll
        for (int j = 0; j < 4; j++) merged[j] = (nan_min[a] <= other[b2]) ? nan_min[a++] : other[b2++];
#pragma unroll
        for (int j = 0; j < 4; j++) nan_min[j] = merged[j];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        for (int j = 0; j < 4; j++) snan[warp][j] = nan_min[j];
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long best[4] = {EMPTY, EMPTY, EMPTY, EMPTY};
        for (int w = 0; w < kBThreads / 32; w++)
            for (int j = 0; j < 4; j++) {
                unsigned long long k = snan[w][j];
                for (int q = 0; q < 4; q++)
                    if (k < best[q]) { const unsigned long long x = best[q]; best[q] = k; k = x; }
            }
        for (int j = 0; j < 4; j++) t.nan[4 * tile + j] = best[j];
    }
}

struct Cand {
    unsigned long long key, bits;
    unsigned int count;
};
__device__ __forceinline__ bool cbetter(const Cand &a, const Cand &b)
{
    return a.count > b.count || (a.count == b.count && a.count != 0 && a.key < b.key);
}
__device__ __forceinline__ void cpush(Cand *l, const Cand &c)
{
    if (!cbetter(c, l[3])) return;
    l[3] = c;
#pragma unroll
    for (int i = 3; i > 0; i--)
        if (cbetter(l[i], l[i - 1])) { const Cand x = l[i]; l[i] = l[i - 1]; l[i - 1] = x; }
}

// The k most frequent values of an item, then the table is cleared for the next step.  The item's
// blocks (one per histogram tile) each take a slice of the used-slot list (and of the NaN lists),
// reduce it to a top-4, clear their slots and write the top-4 to the partial list; the last block
// to finish (threadfence + counter) merges the partials, writes the result and resets the header.
__device__ __forceinline__ void topk_block_reduce(Cand *l, Cand *sc)
{
    for (int j = 0; j < 4; j++) sc[threadIdx.x * 4 + j] = l[j];
    __syncthreads();
    for (int width = kBThreads / 2; width > 0; width >>= 1) {
        if ((int)threadIdx.x < width) {
            Cand mine[4] = {sc[threadIdx.x * 4], sc[threadIdx.x * 4 + 1], sc[threadIdx.x * 4 + 2], sc[threadIdx.x * 4 + 3]};
            for (int j = 0; j < 4; j++) cpush(mine, sc[(threadIdx.x + width) * 4 + j]);
            for (int j = 0; j < 4; j++) sc[threadIdx.x * 4 + j] = mine[j];
        }
        __syncthreads();
    }
}

template <int ES>
__device__ void p_topk(const BItem &it, uint32_t tile, StreamDesc *S, unsigned char *smem)
{
    constexpr unsigned long long EMPTY = ~0ull;
    __shared__ bool s_last;
    Cand *sc = (Cand *)smem;
    const HTab t = htab(it);
    const Order o = (Order)it.order;
    const uint32_t T = it.tiles;
    const unsigned int used = t.hdr->used;
    const uint64_t slice = (used + T - 1) / T;
    const uint64_t lo = (uint64_t)tile * slice, hi = lo + slice < used ? lo + slice : used;
    const uint64_t nan_n = 4 * it.p[1], nslice = (nan_n + T - 1) / T;
    const uint64_t nlo = (uint64_t)tile * nslice, nhi = nlo + nslice < nan_n ? nlo + nslice : nan_n;
    Cand l[4];
    for (int j = 0; j < 4; j++) l[j] = Cand{EMPTY, 0, 0};
    for (uint64_t i = lo + threadIdx.x; i < hi; i += kBThreads) {
        const unsigned int h = t.used[i];
        const unsigned long long k = t.keys[h];
        cpush(l, Cand{order_key(k, ES, o), k, t.counts[h]});
    }
    if (tile == 0 && threadIdx.x == 0 && t.hdr->special) cpush(l, Cand{order_key(EMPTY, ES, o), EMPTY, t.hdr->special});
    for (uint64_t i = nlo + threadIdx.x; i < nhi; i += kBThreads) {
        const unsigned long long k = t.nan[i];
        if (k != EMPTY) cpush(l, Cand{k, order_unkey(k, ES, o), 1u});
    }
    topk_block_reduce(l, sc);
    // clear this slice of the table for the next step
    for (uint64_t i = lo + threadIdx.x; i < hi; i += kBThreads) {
        const unsigned int h = t.used[i];
        t.keys[h] = EMPTY;
        t.counts[h] = 0;
    }
    unsigned long long *part = t.part + (uint64_t)tile * 12;
    if (threadIdx.x < 4) {
        part[3 * threadIdx.x] = sc[threadIdx.x].key;
        part[3 * threadIdx.x + 1] = sc[threadIdx.x].bits;
        part[3 * threadIdx.x + 2] = sc[threadIdx.x].count;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(&t.hdr->pad, 1u) == T - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    for (int j = 0; j < 4; j++) l[j] = Cand{EMPTY, 0, 0};
    for (uint64_t i = threadIdx.x; i < 4ull * T; i += kBThreads) {
        const volatile unsigned long long *q = t.part + 3 * i;
        cpush(l, Cand{q[0], q[1], (unsigned int)q[2]});
    }
    __syncthreads();
    topk_block_reduce(l, sc);
    if (threadIdx.x == 0) {
        const int k = it.mode;  // 1: const -> meta[0..es), 4: dict -> out1[16 ..)
        uint8_t *dst = k == 1 ? S[it.out[0]].ptr : S[it.out[1]].ptr + 16;
        for (int j = 0; j < k; j++) st_elem<ES>(dst, j, sc[j].count ? sc[j].bits : 0ull);
        t.hdr->used = 0;
        t.hdr->special = 0;
        t.hdr->overflow = 0;
        t.hdr->pad = 0;
    }
}

// ------------------------------------------------------------------------------- split
__device__ __forceinline__ uint32_t spad(uint32_t x) { return x + (x >> 4); }

template <int ES>
__device__ void p_split(const BItem &it, uint32_t tile, StreamDesc *S, uint32_t *status, unsigned char *sm)
{
    __shared__ unsigned long long ws[32];
    __shared__ unsigned long long s_prefix;
    const int mode = it.mode;
    const StreamDesc in = S[it.in[0]];
    const ViewCtx vc = view_ctx<ES>(it, in);
    const uint64_t n = vc.n;
    const Order o = (Order)it.order;
    Lookback lb = lookback_at(it.scratch + it.p[0], it.tiles);
    // stencil location and the values matched against
    uint8_t *meta = S[it.out[0]].ptr;
    uint8_t *stencil = mode == SPLIT_NOT_CONST ? meta + ES + 1 : meta + 1;
    uint64_t top[4] = {0, 0, 0, 0}, thr = 0, lo = 0;
    const bool outside = mode == SPLIT_LOWER && it.p[1] != 0;
    if (mode == SPLIT_LOWER) {
        uint64_t mnb = 0, mxb = 0;
        if (!acc_minmax((const MinMaxAcc *)it.scratch, ES, o, mnb, mxb) && n) mnb = mxb = view_elem<ES>(it, vc, in.ptr, 0);
        if (outside) d_outside_patch_bounds(mnb, mxb, it.dt, ES, lo, thr);  // thr: the high bound
        else thr = d_patch_threshold(mnb, mxb, it.dt, ES);
    } else if (mode == SPLIT_NOT_CONST) {
        top[0] = ld_elem<ES>(meta, 0);
    } else {
        const uint8_t *tp = S[it.out[1]].ptr + 16;
        for (int k = 0; k < 4; k++) top[k] = ld_unaligned<ES>(tp + k * ES);
    }
    if (tile == 0 && threadIdx.x == 0) {
        (mode == SPLIT_NOT_CONST ? meta[ES] : meta[0]) = (uint8_t)(n % 8);
        if (n == 0) {
            S[it.out[0]].len = 0;
            S[it.out[1]].len = 0;
            if (mode != SPLIT_NOT_CONST) S[it.out[2]].len = 0;
        }
    }
    // a tile past the input has no successor waiting on its look-back descriptor (every later
    // tile is past the input too), so it leaves at once; grids are sized for the worst case
    if (tile > 0 && (uint64_t)tile * kBTile >= n) return;
    const uint64_t base = (uint64_t)tile * kBTile + (uint64_t)threadIdx.x * kBVPT;
    uint64_t v[kBVPT];
    load_view_x<ES, kBVPT>(it, vc, in.ptr, base, v, sm);  // sm is free until the staging below
    uint32_t bits = 0, codes = 0;
    if (mode == SPLIT_LOWER && outside) {
        // OutsideOperator (stencil_operators.hpp:14-25): false when x > high or x < low
#pragma unroll
        for (int j = 0; j < (int)kBVPT; j++)
            bits |= (uint32_t)!(lt_native(thr, v[j], ES, o) || lt_native(v[j], lo, ES, o)) << j;
    } else if (mode == SPLIT_LOWER) {
#pragma unroll
        for (int j = 0; j < (int)kBVPT; j++) bits |= (uint32_t)lt_native(v[j], thr, ES, o) << j;
    } else {
        // equal bits and not NaN (bsame): NaN-ness once per value, not once per candidate
        const bool fp = o != ORD_INT;
#pragma unroll
        for (int j = 0; j < (int)kBVPT; j++) {
            const bool nan = fp && is_nan_bits(v[j], o);
            if (mode == SPLIT_NOT_CONST) {
                bits |= (uint32_t)(nan || v[j] != top[0]) << j;
            } else {
                const uint32_t e0 = v[j] == top[0], e1 = v[j] == top[1], e2 = v[j] == top[2], e3 = v[j] == top[3];
                bits |= (uint32_t)(!nan && (e0 | e1 | e2 | e3)) << j;
                codes |= (nan ? 0u : (e1 | (e2 << 1) | (e3 * 3u))) << (2 * j);
            }
        }
    }
    if (base < n) {
        const uint64_t valid = n - base;
        if (valid < kBVPT) {  // Stencil::pack's index clamp: the last element fills the last byte
            const uint32_t last = (bits >> (valid - 1)) & 1u;
            for (int j = (int)valid; j < (int)kBVPT; j++) bits = (bits & ~(1u << j)) | (last << j);
        }
#pragma unroll
        for (int q = 0; q < (int)kBVPT / 8; q++)
            if (base + 8 * q < n) stencil[base / 8 + q] = (uint8_t)(bits >> (8 * q));
    }
    const uint32_t valid_mask = base >= n ? 0u : (n - base >= kBVPT ? (1u << kBVPT) - 1 : ((1u << (n - base)) - 1));
    const uint32_t yes_bits = bits & valid_mask;
    if (it.p[2] | it.p[3]) {
        // min / max of the matches and of the rest, for the AFL children that read them (integer
        // order, as their own min/max pass would compute it); only the classes with such a child
        const bool fold_y = it.p[2] != 0, fold_n = it.p[3] != 0;
        uint64_t ymin = ~0ull, ymax = 0, nmin = ~0ull, nmax = 0;
#pragma unroll
        for (int j = 0; j < (int)kBVPT; j++) {
            const uint64_t k = order_key(v[j], ES, ORD_INT);
            const bool in = (valid_mask >> j) & 1u, y = (yes_bits >> j) & 1u;
            if (fold_y && in && y) { ymin = k < ymin ? k : ymin; ymax = k > ymax ? k : ymax; }
            if (fold_n && in && !y) { nmin = k < nmin ? k : nmin; nmax = k > nmax ? k : nmax; }
        }
        block_minmax(ymin, ymax);
        block_minmax(nmin, nmax);
        if (threadIdx.x == 0) {
            MinMaxAcc *ay = (MinMaxAcc *)it.p[2], *an = (MinMaxAcc *)it.p[3];
            if (ay && ymin != ~0ull) atomicMax(&ay->nkmin, (unsigned long long)~ymin);
            if (ay && ymax != 0) atomicMax(&ay->kmax, (unsigned long long)ymax);
            if (an && nmin != ~0ull) atomicMax(&an->nkmin, (unsigned long long)~nmin);
            if (an && nmax != 0) atomicMax(&an->kmax, (unsigned long long)nmax);
        }
    }
    unsigned long long total;
    const unsigned long long excl = block_exclusive_scan<kBThreads>((unsigned long long)__popc(yes_bits), ws, total);
    if (threadIdx.x < 32) {
        const unsigned long long e = lookback_exclusive(lb, tile, total);
        if (threadIdx.x == 0) s_prefix = e;
    }
    __syncthreads();
    // the tile's values go to shared memory in output order (matches first, then the rest), then
    // the block writes both runs with coalesced stores
    const uint64_t tile_base = (uint64_t)tile * kBTile;
    const uint64_t tile_n = tile_base < n ? (n - tile_base < kBTile ? n - tile_base : kBTile) : 0;
    const uint64_t ny = total, nn = tile_n - ny;
    const uint64_t yes0 = s_prefix, no0 = tile_base - (tile_base < n ? yes0 : 0);
    // staged at spad(position): one spare slot per 16, so the runs of consecutive threads (16 apart
    // when most values match) fall into different banks.  Only the runs that are written are
    // staged: a dictionary writes codes for its matches, a const node only its mismatches.
    uint32_t ly = (uint32_t)excl, ln = threadIdx.x * kBVPT - (uint32_t)excl;
    const uint32_t ny32 = (uint32_t)ny;
    const bool stage_y = mode != SPLIT_DICT, stage_n = mode != SPLIT_NOT_CONST;
#pragma unroll
    for (int j = 0; j < (int)kBVPT; j++) {
        if (!((valid_mask >> j) & 1u)) break;
        if ((yes_bits >> j) & 1u) {
            if (stage_y) st_elem<ES>(sm, spad(ly), v[j]);
            ++ly;
        } else {
            if (stage_n) st_elem<ES>(sm, spad(ny32 + ln), v[j]);
            ++ln;
        }
    }
    if (mode == SPLIT_DICT) {
        // 2-bit codes of this thread's matches: at most two code words; a word wholly inside the
        // thread's range is stored, a shared one is merged with atomicOr (the words start zeroed)
        uint32_t *words = (uint32_t *)(S[it.out[1]].ptr + 16 + 4 * ES);
        const uint64_t y0 = yes0 + excl, y1 = y0 + __popc(yes_bits);
        uint32_t acc0 = 0u, acc1 = 0u;  // the first and the second code word of the range
        uint32_t r = (uint32_t)(y0 & 15);  // position inside the first word (at most 15 + 16 < 32)
#pragma unroll
        for (int j = 0; j < (int)kBVPT; j++)
            if ((yes_bits >> j) & 1u) {
                const uint32_t bits2 = ((codes >> (2 * j)) & 3u) << (2 * (r & 15));
                if (r < 16) acc0 |= bits2;
                else acc1 |= bits2;
                ++r;
            }
        if (y1 > y0) {
            for (uint64_t w = y0 >> 4; w <= (y1 - 1) >> 4; w++) {
                const uint32_t a = w == (y0 >> 4) ? acc0 : acc1;
                if (16 * w >= y0 && 16 * w + 16 <= y1) words[w] = a;
                else if (a) atomicOr(words + w, a);
            }
        }
    }
    __syncthreads();
    if (mode != SPLIT_DICT) {
        uint8_t *yes = S[it.out[1]].ptr + yes0 * ES;
        for (uint32_t i = threadIdx.x; i < ny32; i += kBThreads) st_elem<ES>(yes, i, ld_elem_sm<ES>(sm, spad(i)));
    }
    if (mode != SPLIT_NOT_CONST) {
        uint8_t *no = S[it.out[2]].ptr + no0 * ES;
        const uint32_t nn32 = (uint32_t)nn;
        for (uint32_t i = threadIdx.x; i < nn32; i += kBThreads)
            st_elem<ES>(no, i, ld_elem_sm<ES>(sm, spad(ny32 + i)));
    }
    const uint64_t yes_pos = yes0 + ny;
    if (base < n && base + kBVPT >= n) {  // the thread holding the last element: lengths and headers
        const uint64_t m = yes_pos;  // this is the last tile: its matches end the match stream
        if (mode == SPLIT_LOWER) {
            S[it.out[0]].len = 1 + (n + 7) / 8;
            S[it.out[1]].len = m * ES;
            S[it.out[2]].len = (n - m) * ES;
        } else if (mode == SPLIT_NOT_CONST) {
            S[it.out[0]].len = ES + 1 + (n + 7) / 8;
            S[it.out[1]].len = m * ES;
        } else {
            uint64_t *sz = (uint64_t *)S[it.out[1]].ptr;
            sz[0] = 4;
            sz[1] = m;
            S[it.out[0]].len = 1 + (n + 7) / 8;
            S[it.out[1]].len = m ? 16 + 4 * ES + 4 * ((m + 15) / 16) : 0;
            S[it.out[2]].len = (n - m) * ES;
        }
    }
    (void)status;
}

// ------------------------------------------------------------------------------- RLE
template <int ES>
__device__ void p_rle_heads(const BItem &it, uint32_t tile, StreamDesc *S, uint8_t *xs)
{
    __shared__ unsigned long long ws[32];
    __shared__ unsigned long long s_prefix;
    const StreamDesc in = S[it.in[0]];
    const ViewCtx vc = view_ctx<ES>(it, in);
    const uint64_t n = vc.n;
    const Order o = (Order)it.order;
    Lookback lb = lookback_at(it.scratch + it.p[0], it.tiles);
    uint32_t *starts = (uint32_t *)(it.scratch + it.p[1]);
    if (n == 0) {
        if (tile == 0 && threadIdx.x == 0) {
            *(int32_t *)S[it.out[0]].ptr = 0;
            S[it.out[0]].len = 4;
            S[it.out[1]].len = 0;
            S[it.out[2]].len = 0;
        }
        return;
    }
    if ((uint64_t)tile * kBTile >= n) return;  // past the input: no successor needs this tile
    const uint64_t base = (uint64_t)tile * kBTile + (uint64_t)threadIdx.x * kBVPT;
    uint64_t v[kBVPT];
    load_view_x<ES, kBVPT>(it, vc, in.ptr, base, v, xs);
    const uint64_t prev = base > 0 && base - 1 < n ? view_elem<ES>(it, vc, in.ptr, base - 1) : 0;
    uint32_t heads = 0;
#pragma unroll
    for (int j = 0; j < (int)kBVPT; j++) {
        const uint64_t i = base + j;
        if (i < n && (i == 0 || !bsame(v[j], j ? v[j - 1] : prev, o))) heads |= 1u << j;
    }
    unsigned long long total;
    const unsigned long long excl = block_exclusive_scan<kBThreads>((unsigned long long)__popc(heads), ws, total);
    if (threadIdx.x < 32) {
        const unsigned long long e = lookback_exclusive(lb, tile, total);
        if (threadIdx.x == 0) s_prefix = e;
    }
    __syncthreads();
    uint64_t r = s_prefix + excl;
    uint8_t *values = S[it.out[2]].ptr;
#pragma unroll
    for (int j = 0; j < (int)kBVPT; j++)
        if ((heads >> j) & 1u) {
            st_elem<ES>(values, r, v[j]);
            starts[r] = (uint32_t)(base + j);
            ++r;
        }
    if (base < n && base + kBVPT >= n) {
        *(int32_t *)S[it.out[0]].ptr = (int32_t)r;
        S[it.out[0]].len = 4;
        S[it.out[1]].len = 4 * r;
        S[it.out[2]].len = ES * r;
    }
}

__device__ void p_rle_lengths(const BItem &it, uint32_t tile, StreamDesc *S)
{
    int nd = 0;
    for (int k = 0; k < kMaxViewOps; k++) nd += it.vop[k] == V_DELTA;
    const uint64_t n_src = S[it.in[0]].len / it.es;
    const uint64_t n = n_src > (uint64_t)nd ? n_src - nd : 0;
    const uint64_t runs = S[it.out[1]].len / 4;
    const uint32_t *starts = (const uint32_t *)(it.scratch + it.p[1]);
    int32_t *lengths = (int32_t *)S[it.out[1]].ptr;
    const uint64_t r0 = (uint64_t)tile * kBTile;
    for (uint64_t r = r0 + threadIdx.x; r < runs && r < r0 + kBTile; r += kBThreads) {
        const uint64_t next = r + 1 < runs ? starts[r + 1] : n;
        lengths[r] = (int32_t)(next - starts[r]);
    }
}

// ------------------------------------------------------------------------------- floatToInt
__device__ __forceinline__ const double *pow10_table()
{
    __shared__ double t[10];
    if (threadIdx.x < 10) {
        double v = 1.0;
        for (unsigned i = 0; i < threadIdx.x; i++) v *= 10.0;
        t[threadIdx.x] = v;
    }
    __syncthreads();
    return t;
}

template <int ES>
__device__ __forceinline__ double as_double(uint64_t u, Order o)
{
    if (o == ORD_F32) return (double)__uint_as_float((uint32_t)u);
    if (o == ORD_F64) return __longlong_as_double((long long)u);
    if (ES == 8) return __ll2double_rn((long long)u);
    return (double)sext(u, ES);
}

template <int ES>
__device__ __forceinline__ float as_float_T(uint64_t u, Order o)
{
    if (o == ORD_F32) return __uint_as_float((uint32_t)u);
    if (o == ORD_F64) return __double2float_rn(__longlong_as_double((long long)u));
    if (ES == 8) return __ll2float_rn((long long)u);
    return __int2float_rn((int)sext(u, ES));
}

template <int ES>
__device__ __forceinline__ uint64_t f2i_dec_one(int k, int p, Order o, const double *p10)
{
    if (o == ORD_F32) return __float_as_uint(__double2float_rn(__ddiv_rn((double)__int2float_rn(k), p10[p])));
    if (o == ORD_F64) return (uint64_t)__double_as_longlong(__ddiv_rn((double)k, p10[p]));
    if (ES == 8) return (uint64_t)__double2ll_rz(__ddiv_rn((double)k, p10[p]));
    const long long t = sext((uint64_t)(long long)k, ES);
    return (uint64_t)(long long)__double2int_rz(__ddiv_rn((double)t, p10[p]));
}

// node scratch of floatToInt: StatsAcc at 0, lossy flag at 64
template <int ES>
__device__ void p_f2i_stats(const BItem &it, uint32_t tile, StreamDesc *S)
{
    const StreamDesc in = S[it.in[0]];
    const uint64_t n = in.len / ES;
    const uint64_t t0 = (uint64_t)tile * kBTile;
    if (t0 >= n) return;
    const Order o = (Order)it.order;
    uint64_t kmin = ~0ull, kmax = 0;
    int steps = 0;
    const uint64_t end = n < t0 + kBTile ? n : t0 + kBTile;
    for (uint64_t i = t0 + threadIdx.x; i < end; i += kBThreads) {
        const uint64_t u = ld_elem<ES>(in.ptr, i);
        if (!is_nan_bits(u, o)) {
            const uint64_t k = order_key(u, ES, o);
            kmin = k < kmin ? k : kmin;
            kmax = k > kmax ? k : kmax;
        }
        const int s = d_precision_steps(as_float_T<ES>(u, o));
        steps = s > steps ? s : steps;
    }
    for (int off = 16; off > 0; off >>= 1) {
        const int x = __shfl_xor_sync(0xffffffffu, steps, off);
        steps = x > steps ? x : steps;
    }
    __shared__ int s_steps[kBThreads / 32];
    if ((threadIdx.x & 31) == 0) s_steps[threadIdx.x >> 5] = steps;
    block_minmax(kmin, kmax);
    if (threadIdx.x == 0) {
        for (int w = 1; w < kBThreads / 32; w++) steps = s_steps[w] > steps ? s_steps[w] : steps;
        StatsAcc *acc = (StatsAcc *)it.scratch;
        if (kmin != ~0ull) atomicMax(&acc->mm.nkmin, (unsigned long long)~kmin);
        if (kmax != 0) atomicMax(&acc->mm.kmax, (unsigned long long)kmax);
        atomicMax(&acc->prec_steps, (unsigned int)steps);
    }
}

// FloatEncoding::Encode's decision (float_encoding.cu:29-43) from the stats pass
template <int ES>
__device__ __forceinline__ int f2i_decide(const BItem &it, const uint8_t *col, uint64_t n, bool &transform)
{
    const StatsAcc *acc = (const StatsAcc *)it.scratch;
    const Order o = (Order)it.order;
    const unsigned steps = acc->prec_steps > 10 ? 10 : acc->prec_steps;
    int p = d_precision_of((int)steps);
    transform = false;
    if (p < 10 && n) {
        uint64_t mnb = 0, mxb = 0;
        if (!acc_minmax(&acc->mm, ES, o, mnb, mxb)) mnb = mxb = ld_elem<ES>(col, 0);
        long long sc = 1;
        for (int i = 0; i < p; i++) sc *= 10;
        bool ok;
        if (o == ORD_F32) {
            const float a = __fmul_rn(__uint_as_float((uint32_t)mnb), (float)sc);
            const float b = __fmul_rn(__uint_as_float((uint32_t)mxb), (float)sc);
            ok = a > -2147483648.0f && b < 2147483648.0f;
        } else if (o == ORD_F64) {
            const double a = __dmul_rn(__longlong_as_double((long long)mnb), (double)sc);
            const double b = __dmul_rn(__longlong_as_double((long long)mxb), (double)sc);
            ok = a > -2147483648.0 && b < 2147483647.0;
        } else {
            ok = sext(mnb, ES) * sc > (long long)INT32_MIN && sext(mxb, ES) * sc < (long long)INT32_MAX;
        }
        if (ok) transform = true;
        else p = 10;
    }
    return p;
}

// the raw branch (p = 10): the bytes of the tile's elements that fall in the stream's whole 32-bit
// words (`words`), block-striped; whole words when the input is 4-byte aligned (the output, a node
// stream, always is), else bytes
template <int ES>
__device__ __forceinline__ void f2i_copy_words(uint8_t *out, const uint8_t *in, uint32_t tile, uint64_t words)
{
    constexpr uint64_t B = (uint64_t)kBTile * ES;  // bytes of one tile
    const uint64_t b0 = (uint64_t)tile * B, b1 = b0 + B < 4 * words ? b0 + B : 4 * words;
    if (((uintptr_t)in & 3) == 0) {
        for (uint64_t w = b0 / 4 + threadIdx.x; w < b1 / 4; w += kBThreads)
            ((uint32_t *)out)[w] = ldg((const uint32_t *)in + w);
    } else {
        for (uint64_t b = b0 + threadIdx.x; b < b1; b += kBThreads) out[b] = ldg(in + b);
    }
}

template <int ES>
__device__ void p_f2i_enc(const BItem &it, uint32_t tile, StreamDesc *S)
{
    const double *p10 = pow10_table();
    const StreamDesc in = S[it.in[0]];
    const uint64_t n = in.len / ES;
    bool transform;
    const int p = f2i_decide<ES>(it, in.ptr, n, transform);
    if (tile == 0 && threadIdx.x == 0) {
        if (n) {
            *(int32_t *)S[it.out[0]].ptr = p;
            S[it.out[0]].len = 4;
            S[it.out[1]].len = transform ? 4 * n : (n * ES) / 4 * 4;
        } else {
            S[it.out[0]].len = 0;
            S[it.out[1]].len = 0;
        }
    }
    // block-striped: the k-th access of a warp covers 32 consecutive elements (or words)
    const uint64_t t0 = (uint64_t)tile * kBTile;
    if (t0 >= n) return;
    uint8_t *out = S[it.out[1]].ptr;
    if (transform) {
        const Order o = (Order)it.order;
        const uint64_t wm = ES == 8 ? ~0ull : ((1ull << (8 * ES)) - 1);
        bool bad = false;
        for (int j = 0; j < (int)kBVPT; j++) {
            const uint64_t i = t0 + (uint64_t)j * kBThreads + threadIdx.x;
            if (i >= n) break;
            const uint64_t u = ld_elem<ES>(in.ptr, i);
            const int k = (int)(long long)__double2ll_rn(__dmul_rn(as_double<ES>(u, o), p10[p]));
            ((int32_t *)out)[i] = k;
            if (((f2i_dec_one<ES>(k, p, o, p10) ^ u) & wm) != 0) bad = true;
        }
        if (bad) atomicExch((unsigned int *)(it.scratch + 64), 1u);
    } else {
        f2i_copy_words<ES>(out, in.ptr, tile, (n * ES) / 4);
    }
}

// the lossless check failed: the raw p = 10 branch
template <int ES>
__device__ void p_f2i_raw(const BItem &it, uint32_t tile, StreamDesc *S)
{
    if (*(volatile unsigned int *)(it.scratch + 64) == 0) return;
    const StreamDesc in = S[it.in[0]];
    const uint64_t n = in.len / ES;
    const uint64_t bytes = (n * ES) / 4 * 4;
    if (tile == 0 && threadIdx.x == 0) {
        *(int32_t *)S[it.out[0]].ptr = 10;
        S[it.out[1]].len = bytes;
    }
    f2i_copy_words<ES>(S[it.out[1]].ptr, in.ptr, tile, bytes / 4);
}

// ------------------------------------------------------------------------------- GFC
// node scratch of GFC: p[0] look-back, p[1] chunk sizes (int32), p[2] inclusive ends (u64), p[3] layout

// A double chunk is built in a 1 KB ring of the warp's shared memory and stored in 512-byte blocks,
// 16 bytes a lane (its payload bytes, up to 8 a lane, would otherwise be that many partial global
// stores); a float chunk, at most 4 bytes a lane, is stored directly.  Positions count bytes from
// the 16-byte aligned address at or below the chunk's start; only the bytes in [lo, hi) are stored.
constexpr uint32_t kGfcStage = 1024;

__device__ __forceinline__ void gfc_flush(uint8_t *al, const uint8_t *ring, uint32_t b, uint32_t lo, uint32_t hi,
                                          int lane)
{
    const uint32_t p = b + 16 * (uint32_t)lane;
    if (p >= lo && p + 16 <= hi) {
        *(uint4 *)(al + p) = *(const uint4 *)(ring + (p & (kGfcStage - 1)));
    } else {
        for (uint32_t k = 0; k < 16; k++)
            if (p + k >= lo && p + k < hi) al[p + k] = ring[(p + k) & (kGfcStage - 1)];
    }
}

template <bool DBL>
__device__ void p_gfc_compress(const BItem &it, uint32_t tile, StreamDesc *S, uint8_t *sm)
{
    const StreamDesc in = S[it.in[0]];
    const ViewCtx vc = view_ctx<DBL ? 8 : 4>(it, in);
    const uint64_t n = vc.n;
    const DGfc g = d_gfc_geom(DBL, n, 0, 0);
    if (tile == 0 && threadIdx.x == 0) {
        if (n) {
            int32_t *m = (int32_t *)S[it.out[0]].ptr;
            m[0] = g.blocks;
            m[1] = g.wpb;
            m[2] = (int32_t)n;
            S[it.out[0]].len = 12;
            S[it.out[1]].len = 4 * (uint64_t)g.warps;
        } else {
            S[it.out[0]].len = 0;
            S[it.out[1]].len = 0;
            S[it.out[2]].len = 0;
        }
    }
    const int lane = threadIdx.x & 31;
    const int64_t w = (int64_t)tile * kBGfcChunks + (threadIdx.x >> 5);
    if (w >= g.warps) return;
    uint8_t *layout = it.scratch + it.p[3];
    int32_t *sizes = (int32_t *)(it.scratch + it.p[1]);
    int32_t *ends = (int32_t *)S[it.out[1]].ptr;
    const uint64_t cb = d_gfc_begin(g, w), ce = d_gfc_cut(g, w);
    const uint64_t start = d_gfc_start(g, w);
    uint64_t last = 0;
    uint8_t *ring = sm + (threadIdx.x >> 5) * kGfcStage;
    const uint32_t mis = (uint32_t)((uintptr_t)(layout + start) & 15);
    uint8_t *al = layout + start - mis;
    uint32_t fr = mis, flushed = 0;  // positions: the next subchunk's header, the bytes stored
    // values of the next 4 subchunks are in flight while one is encoded
    uint64_t xb[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const uint64_t i = cb + 32 * q + lane;
        xb[q] = cb + 32 * q < ce && i < n ? view_elem<DBL ? 8 : 4>(it, vc, in.ptr, i) : 0;
    }
    for (uint64_t s0 = cb; s0 < ce; s0 += 128)
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const uint64_t s = s0 + 32 * q;
        if (s >= ce) break;
        const uint64_t x = xb[q];
        {
            const uint64_t i = s + 128 + lane;
            xb[q] = s + 128 < ce && i < n ? view_elem<DBL ? 8 : 4>(it, vc, in.ptr, i) : 0;
        }
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
        uint32_t incl = mb;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        const uint32_t prev_nib = __shfl_up_sync(0xffffffffu, nib, 1);
        const uint32_t pl = fr + 16 + (incl - mb);
        if constexpr (DBL) {
            if (lane & 1) ring[(fr + (lane >> 1)) & (kGfcStage - 1)] = (uint8_t)(prev_nib | (nib << 4));
            for (uint32_t b = 0; b < mb; b++) ring[(pl + b) & (kGfcStage - 1)] = (uint8_t)(diff >> (8 * b));
        } else {
            if (lane & 1) al[fr + (lane >> 1)] = (uint8_t)(prev_nib | (nib << 4));
            for (uint32_t b = 0; b < mb; b++) al[pl + b] = (uint8_t)(diff >> (8 * b));
        }
        fr += 16 + total;  // at most 272 bytes a subchunk: the ring holds [flushed, fr) below 784 bytes
        if (s == cb) last = __shfl_sync(0xffffffffu, x, 31);
        if constexpr (DBL) {
            __syncwarp();
            if (fr - flushed >= 512) {
                gfc_flush(al, ring, flushed, mis, 0xffffffffu, lane);
                flushed += 512;
                __syncwarp();
            }
        }
    }
    if (DBL && flushed < fr) gfc_flush(al, ring, flushed, mis, fr, lane);
    if (lane == 31) {
        ends[w] = (int32_t)(start + fr - mis);
        sizes[w] = (int32_t)(fr - mis);
    }
}

// one warp copies n bytes between any addresses: head bytes up to a 4-byte aligned destination,
// then whole words funnel-shifted out of aligned source words, then the tail.  Eight words a lane
// are loaded before any is stored, so the loads are in flight together.
__device__ __forceinline__ void warp_copy(uint8_t *dst, const uint8_t *src, uint64_t n, int lane)
{
    const uint64_t head = (4 - ((uintptr_t)dst & 3)) & 3;
    const uint64_t h = head < n ? head : n;
    if ((uint64_t)lane < h) dst[lane] = src[lane];
    if (n <= h) return;
    uint32_t *d = (uint32_t *)(dst + h);
    const uint8_t *sp = src + h;
    const uint64_t words = (n - h) / 4;
    const uint32_t sh = 8 * (uint32_t)((uintptr_t)sp & 3);
    const uint32_t *sw = (const uint32_t *)((uintptr_t)sp & ~(uintptr_t)3);
    constexpr int U = 8;
    uint64_t k = lane;
    if (sh == 0) {
        for (; k + (U - 1) * 32 < words; k += U * 32) {
            uint32_t r[U];
#pragma unroll
            for (int u = 0; u < U; u++) r[u] = ldg(sw + k + u * 32);
#pragma unroll
            for (int u = 0; u < U; u++) d[k + u * 32] = r[u];
        }
        for (; k < words; k += 32) d[k] = ldg(sw + k);
    } else {
        for (; k + (U - 1) * 32 < words; k += U * 32) {
            uint32_t r[U], q[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                r[u] = ldg(sw + k + u * 32);
                q[u] = ldg(sw + k + u * 32 + 1);
            }
#pragma unroll
            for (int u = 0; u < U; u++) d[k + u * 32] = __funnelshift_r(r[u], q[u], sh);
        }
        for (; k < words; k += 32) d[k] = __funnelshift_r(ldg(sw + k), ldg(sw + k + 1), sh);
    }
    const uint64_t tail = (n - h) - 4 * words;
    if ((uint64_t)lane < tail) ((uint8_t *)d)[4 * words + lane] = sp[4 * words + lane];
}

template <bool DBL>
__device__ void p_gfc_compact(const BItem &it, uint32_t tile, StreamDesc *S)
{
    int nd = 0;
    for (int k = 0; k < kMaxViewOps; k++) nd += it.vop[k] == V_DELTA;
    const uint64_t n_src = S[it.in[0]].len / (DBL ? 8 : 4);
    const uint64_t n = n_src > (uint64_t)nd ? n_src - nd : 0;
    const DGfc g = d_gfc_geom(DBL, n, 0, 0);
    const int lane = threadIdx.x & 31;
    const int64_t w = (int64_t)tile * kBGfcChunks + (threadIdx.x >> 5);
    if (w >= g.warps) return;
    const int32_t *sizes = (const int32_t *)(it.scratch + it.p[1]);
    const unsigned long long *incl = (const unsigned long long *)(it.scratch + it.p[2]);
    const uint8_t *layout = it.scratch + it.p[3];
    const uint64_t size = (uint64_t)(uint32_t)sizes[w];
    const uint64_t dst0 = incl[w] - size;
    const uint8_t *src = layout + d_gfc_start(g, w);
    uint8_t *out = S[it.out[2]].ptr;
    warp_copy(out + dst0, src, size, lane);
    if (w == g.warps - 1 && lane == 0) S[it.out[2]].len = incl[w];
}

// ------------------------------------------------------------------------------- view nodes
// Metadata of a delta / scale node whose output is only read through its child's view: delta's
// first value, scale's minimum (scale_min of its min / max).  One thread per item.
template <int ES>
__device__ void p_vmeta(const BItem &it, StreamDesc *S)
{
    if (threadIdx.x != 0) return;
    const StreamDesc in = S[it.in[0]];
    const ViewCtx vc = view_ctx<ES>(it, in);
    StreamDesc &m = S[it.out[0]];
    if (vc.n == 0) {
        m.len = 0;
        return;
    }
    uint64_t v;
    if (it.mode == GTSC_DELTA) {
        v = view_elem<ES>(it, vc, in.ptr, 0);
    } else {
        uint64_t mnb = 0, mxb = 0;
        acc_minmax((const MinMaxAcc *)it.scratch, ES, ORD_INT, mnb, mxb);
        v = scale_min(mnb, mxb, ES);
    }
    st_elem<ES>(m.ptr, 0, v);
    m.len = ES;
}

// ------------------------------------------------------------------------------- dispatch
constexpr size_t stage_smem(int op)
{
    return op == B_AFL_PACK ? 8 * (kBTile + kBTile / 16 + 8)
         : op == B_HIST     ? 8 * kBHistPacked + 8 * 4 * (kBThreads / 32)
         : op == B_TOPK     ? sizeof(Cand) * kBThreads * 4
         : op == B_SPLIT    ? 8 * (kBTile + kBTile / 16)  // >= kXchgBlockBytes (its loads)
         : op == B_RLE_HEADS ? kXchgBlockBytes
         : op == B_GFC_COMPRESS ? kGfcStage * (kBThreads / 32)
                            : 16;
}
static_assert(stage_smem(B_SPLIT) >= kXchgBlockBytes, "the split loads through the warp exchange");

// Tiles of an item that do work in a pass (the grid is sized for worst-case capacities; the real
// stream lengths are only known on the device).  Tile 0 of a pass that writes metadata always
// runs.  Passes not listed run every reserved tile.
template <int OP>
__device__ __forceinline__ uint32_t stage_extent(const BItem &it, const StreamDesc *S)
{
    auto cdiv = [](uint64_t a, uint64_t b) { return (a + b - 1) / b; };
    auto view_n = [&]() {
        int nd = 0;
        for (int k = 0; k < kMaxViewOps; k++) nd += it.vop[k] == V_DELTA;
        const uint64_t n_src = S[it.in[0]].len / it.es;
        return n_src > (uint64_t)nd ? n_src - nd : 0;
    };
    uint64_t e = it.tiles;
    if constexpr (OP == B_MINMAX) e = cdiv(view_n(), it.p[0]);  // the tuned min/max tile
    else if constexpr (OP == B_DELTA_ENC) {
        const uint64_t n = view_n();
        e = cdiv(n ? n - 1 : 0, kBTile);
        if (e == 0) e = 1;
    } else if constexpr (OP == B_SCALE_SUB || OP == B_AFL_PACK || OP == B_F2I_ENC || OP == B_F2I_RAW) {
        e = cdiv(view_n(), kBTile);
        if (e == 0) e = 1;
    } else if constexpr (OP == B_F2I_STATS) e = cdiv(view_n(), kBTile);
    else if constexpr (OP == B_RLE_LENGTHS) e = cdiv(S[it.out[1]].len / 4, kBTile);
    else if constexpr (OP == B_GFC_COMPRESS || OP == B_GFC_COMPACT) {
        const DGfc g = d_gfc_geom(it.es == 8, view_n(), 0, 0);
        e = cdiv((uint64_t)g.warps, kBGfcChunks);
        if (OP == B_GFC_COMPRESS && e == 0) e = 1;
    }
    return (uint32_t)(e < it.tiles ? e : it.tiles);
}

template <int OP>
__device__ __forceinline__ void run_stage(const BItem &it, uint32_t tile, StreamDesc *S, uint32_t *status,
                                          unsigned char *smem);

// passes whose tiles all do the same streaming work run persistent grids (see stage_grid)
constexpr bool stage_persistent(int op)
{
    return op == B_MINMAX || op == B_DELTA_ENC || op == B_SCALE_SUB || op == B_AFL_PACK || op == B_F2I_STATS ||
           op == B_F2I_ENC || op == B_F2I_RAW || op == B_RLE_LENGTHS;
}

// One launch of a pass over every item.  Look-back passes take one tile per block in claim order;
// the others are persistent: an occupancy-sized grid strides over the tiles, skipping from a tile
// past its item's real extent straight to its first tile of the next item.
// resident blocks per SM the compiler keeps registers for (measured per pass on the mixed workload)
constexpr int stage_min_blocks(int op)
{
    // the histogram at 4 (64 registers, no spills) measured 6 % faster than at 5 (48 registers, spilling)
    return op == B_SPLIT || op == B_GFC_COMPRESS || op == B_TOPK || op == B_HIST ? 4 : 5;
}

template <int OP>
__global__ void __launch_bounds__(kBThreads, stage_min_blocks(OP))
k_bstage(const BItem *items, const uint32_t *item_of, StreamDesc *S, uint32_t *counter, uint32_t *status,
         uint32_t total_tiles)
{
    constexpr bool DYN = OP == B_SPLIT || OP == B_RLE_HEADS || OP == B_GFC_SCAN;
    __shared__ __align__(16) unsigned char smem[stage_smem(OP)];
    if constexpr (!stage_persistent(OP)) {
        uint32_t tile;
        const BItem &it = locate<DYN>(items, item_of, counter, tile);
        if (tile >= it.tiles) return;
        run_stage<OP>(it, tile, S, status, smem);
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
            if (tile >= stage_extent<OP>(it, S)) {
                const uint64_t next = it.tile_base + it.tiles;  // the next item's first tile
                if (next >= total_tiles) break;
                t = (uint32_t)(next + (blockIdx.x + gridDim.x - next % gridDim.x) % gridDim.x);
                continue;
            }
            run_stage<OP>(it, tile, S, status, smem);
            __syncthreads();  // the next tile reuses the shared memory
            t += gridDim.x;
        }
    }
}

template <int OP>
__device__ __forceinline__ void run_stage(const BItem &it, uint32_t tile, StreamDesc *S, uint32_t *status,
                                          unsigned char *smem)
{
#define GTSC_ES_SWITCH(CALL)                       \
    switch (it.es) {                               \
    case 1: { constexpr int E = 1; CALL; } break;  \
    case 2: { constexpr int E = 2; CALL; } break;  \
    case 4: { constexpr int E = 4; CALL; } break;  \
    default: { constexpr int E = 8; CALL; } break; \
    }
    if constexpr (OP == B_MINMAX) { GTSC_ES_SWITCH(p_minmax<E>(it, tile, S)) }
    else if constexpr (OP == B_DELTA_ENC) { GTSC_ES_SWITCH(p_delta_enc<E>(it, tile, S)) }
    else if constexpr (OP == B_SCALE_SUB) { GTSC_ES_SWITCH(p_scale_sub<E>(it, tile, S)) }
    else if constexpr (OP == B_AFL_PACK) { GTSC_ES_SWITCH(p_afl_pack<E>(it, tile, S, (unsigned long long *)smem)) }
    else if constexpr (OP == B_HIST) { GTSC_ES_SWITCH(p_hist<E>(it, tile, S, status, smem)) }
    else if constexpr (OP == B_TOPK) { GTSC_ES_SWITCH(p_topk<E>(it, tile, S, smem)) }
    else if constexpr (OP == B_VMETA) { GTSC_ES_SWITCH(p_vmeta<E>(it, S)) }
    else if constexpr (OP == B_SPLIT) { GTSC_ES_SWITCH(p_split<E>(it, tile, S, status, smem)) }
    else if constexpr (OP == B_RLE_HEADS) { GTSC_ES_SWITCH(p_rle_heads<E>(it, tile, S, smem)) }
    else if constexpr (OP == B_RLE_LENGTHS) { p_rle_lengths(it, tile, S); }
    else if constexpr (OP == B_F2I_STATS) { GTSC_ES_SWITCH(p_f2i_stats<E>(it, tile, S)) }
    else if constexpr (OP == B_F2I_ENC) { GTSC_ES_SWITCH(p_f2i_enc<E>(it, tile, S)) }
    else if constexpr (OP == B_F2I_RAW) { GTSC_ES_SWITCH(p_f2i_raw<E>(it, tile, S)) }
    else if constexpr (OP == B_GFC_COMPRESS) {
        if (it.es == 8) p_gfc_compress<true>(it, tile, S, smem);
        else p_gfc_compress<false>(it, tile, S, smem);
    } else if constexpr (OP == B_GFC_SCAN) {
        p_gfc_scan(it, tile, S, it.es == 8, it.mode != 0);
    } else if constexpr (OP == B_GFC_COMPACT) {
        if (it.es == 8) p_gfc_compact<true>(it, tile, S);
        else p_gfc_compact<false>(it, tile, S);
    }
#undef GTSC_ES_SWITCH
}

#ifdef GTSC_PERSISTENT_TU
// ------------------------------------------------------------------------------- persistent step
constexpr size_t persist_smem_c()
{
    size_t m = 16;
    for (int op = 0; op <= B_GFC_COMPACT; op++) m = stage_smem(op) > m ? stage_smem(op) : m;
    return m;
}

// tiles of an item that do work: the streaming passes skip tiles past the real length, as their
// stage launches do; every other pass runs all its tiles
__device__ __forceinline__ uint32_t persist_extent_c(int op, const BItem &it, const StreamDesc *S)
{
    switch (op) {
    case B_MINMAX: return stage_extent<B_MINMAX>(it, S);
    case B_DELTA_ENC: return stage_extent<B_DELTA_ENC>(it, S);
    case B_SCALE_SUB: return stage_extent<B_SCALE_SUB>(it, S);
    case B_AFL_PACK: return stage_extent<B_AFL_PACK>(it, S);
    case B_F2I_STATS: return stage_extent<B_F2I_STATS>(it, S);
    case B_F2I_ENC: return stage_extent<B_F2I_ENC>(it, S);
    case B_F2I_RAW: return stage_extent<B_F2I_RAW>(it, S);
    case B_RLE_LENGTHS: return stage_extent<B_RLE_LENGTHS>(it, S);
    default: return it.tiles;
    }
}

// The whole compress step in one launch: every pass kind behind one switch, tiles pulled from the
// queue of batch.hpp (PUnit).
__global__ void __launch_bounds__(kBThreads, 4) k_bpersist_c(PersistArgs a)
{
    __shared__ __align__(16) unsigned char smem[persist_smem_c()];
    persist_loop(
        a, [](int op, const BItem &it, const StreamDesc *S) { return persist_extent_c(op, it, S); },
        [&](int op, const BItem &it, uint32_t tile) {
        switch (op) {
#define GTSC_RUN(OPC) case OPC: run_stage<OPC>(it, tile, a.S, a.status, smem); break;
            GTSC_RUN(B_MINMAX)
            GTSC_RUN(B_DELTA_ENC)
            GTSC_RUN(B_SCALE_SUB)
            GTSC_RUN(B_AFL_PACK)
            GTSC_RUN(B_HIST)
            GTSC_RUN(B_TOPK)
            GTSC_RUN(B_SPLIT)
            GTSC_RUN(B_RLE_HEADS)
            GTSC_RUN(B_RLE_LENGTHS)
            GTSC_RUN(B_F2I_STATS)
            GTSC_RUN(B_F2I_ENC)
            GTSC_RUN(B_F2I_RAW)
            GTSC_RUN(B_GFC_COMPRESS)
            GTSC_RUN(B_GFC_SCAN)
            GTSC_RUN(B_GFC_COMPACT)
            GTSC_RUN(B_VMETA)
#undef GTSC_RUN
        default: set_status(a.status, GTSC_ERR_ARG); break;
        }
    });
}

#endif  // GTSC_PERSISTENT_TU

}  // namespace

#ifdef GTSC_PERSISTENT_TU
void launch_batch_persistent_c(const PersistArgs &a, cudaStream_t s)
{
    if (a.total == 0) return;
    int per_sm = 0;
    GTSC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bpersist_c, kBThreads, 0));
    const uint64_t grid = std::min<uint64_t>((uint64_t)std::max(per_sm, 1) * (uint64_t)sm_count(),
                                             (uint64_t)a.total);
    k_bpersist_c<<<(unsigned)grid, kBThreads, 0, s>>>(a);
    GTSC_CUDA(cudaGetLastError());
}
#else

void launch_batch_decode_stage(int op, const BItem *d_items, const uint32_t *d_item_of, int n_items,
                               uint64_t total_tiles, StreamDesc *d_streams, uint32_t *d_counter, uint32_t *d_status,
                               cudaStream_t s);

// Grid of a stage launch: as many blocks as can be resident at once for the streaming passes (the
// kernel strides over the tiles), else one block per tile (look-back passes claim each tile once).
template <class K>
unsigned stage_grid(K kernel, int op, uint64_t total_tiles)
{
    // persistent where every tile does the same streaming work; one block per tile where tiles differ
    // a lot (GFC chunks, histograms, top-k) and independent blocks balance better
    if (!stage_persistent(op)) return (unsigned)total_tiles;
    int per_sm = 0;
    GTSC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBThreads, 0));
    const uint64_t resident = (uint64_t)std::max(per_sm, 1) * (uint64_t)sm_count();
    return (unsigned)std::min<uint64_t>(total_tiles, resident);
}

void launch_batch_stage(int op, const BItem *d_items, const uint32_t *d_item_of, int n_items, uint64_t total_tiles,
                        StreamDesc *d_streams, uint32_t *d_counter, uint32_t *d_status, cudaStream_t s)
{
    if (n_items == 0 || total_tiles == 0) return;
    if (total_tiles > 0x7fffffffull) fail(GTSC_ERR_CAPACITY, "batch: too many tiles in one stage");
    switch (op) {
#define GTSC_STAGE(OPC)                                                                                              \
    case OPC: {                                                                                                      \
        const unsigned g = stage_grid(k_bstage<OPC>, OPC, total_tiles);                                              \
        k_bstage<OPC><<<g, kBThreads, 0, s>>>(d_items, d_item_of, d_streams, d_counter, d_status, (uint32_t)total_tiles); \
        break;                                                                                                       \
    }
        GTSC_STAGE(B_MINMAX)
        GTSC_STAGE(B_DELTA_ENC)
        GTSC_STAGE(B_SCALE_SUB)
        GTSC_STAGE(B_AFL_PACK)
        GTSC_STAGE(B_HIST)
        GTSC_STAGE(B_TOPK)
        GTSC_STAGE(B_SPLIT)
        GTSC_STAGE(B_RLE_HEADS)
        GTSC_STAGE(B_RLE_LENGTHS)
        GTSC_STAGE(B_F2I_STATS)
        GTSC_STAGE(B_F2I_ENC)
        GTSC_STAGE(B_F2I_RAW)
        GTSC_STAGE(B_GFC_COMPRESS)
        GTSC_STAGE(B_GFC_SCAN)
        GTSC_STAGE(B_GFC_COMPACT)
        GTSC_STAGE(B_VMETA)
#undef GTSC_STAGE
    default:
        launch_batch_decode_stage(op, d_items, d_item_of, n_items, total_tiles, d_streams, d_counter, d_status, s);
        return;
    }
    GTSC_CUDA(cudaGetLastError());
}

#endif  // GTSC_PERSISTENT_TU

}  // namespace gtsc
