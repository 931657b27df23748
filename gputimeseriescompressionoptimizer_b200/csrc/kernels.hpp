// kernels.hpp -- host launchers of the device kernels (one declaration per kernel family).
#pragma once

#include "common.cuh"

namespace gtsc {

// ---- min / max (minmax.cu) ---------------------------------------------------------------
// Folds the elements of in[0..n) into *acc (which the caller zeroes first) in order `o`.
// Floating NaNs are skipped.  `in` must be aligned to the element size.
void launch_minmax(const uint8_t *in, uint64_t n, int es, Order o, MinMaxAcc *acc, cudaStream_t s);
// Host-side decode of an accumulator (raw bits of min and max); `first` = bits of element 0,
// used when every element was NaN.  Returns false when nothing was seen.
bool minmax_result(const MinMaxAcc &acc, int es, Order o, uint64_t *mn, uint64_t *mx);

// ---- AFL fixed-width packing (afl.cu) ------------------------------------------------------
// Packs in[0..n) (elements of es bytes) at b bits each into the little-endian LSB-first
// bitstream out[0..out_bytes).  `in` and `out` 16-byte aligned.
void launch_afl_pack(const uint8_t *in, uint64_t n, int es, int b, uint8_t *out, uint64_t out_bytes,
                     cudaStream_t s);
// Unpacks n values of b bits starting at stream byte 0 of `stream` (any alignment) into out.
void launch_afl_unpack(const uint8_t *stream, uint64_t stream_bytes, uint64_t n, int es, int b,
                       uint8_t *out, cudaStream_t s);

// ---- delta / scale (delta_scale.cu) ---------------------------------------------------------
// delta encode: out[i] = in[i+1] - in[i], i < n-1 (in 16-byte aligned)
void launch_delta_encode(const uint8_t *in, uint64_t n, int es, uint8_t *out, cudaStream_t s);
// delta decode: out[k] = first + sum(d[0..k-1]), k < n; scratch = lookback_bytes(delta_decode_tiles(n))
uint64_t delta_decode_tiles(uint64_t n);
void launch_delta_decode(const uint8_t *d, uint64_t n, const uint8_t *first, uint8_t *out,
                         uint8_t *scratch, int es, cudaStream_t s);
// scale: out[i] = in[i] -/+ *min_p (min_p any alignment)
void launch_scale(const uint8_t *in, uint64_t n, int es, const uint8_t *min_p, uint8_t *out, bool encode,
                  cudaStream_t s);

// ---- split / merge (split.cu) -----------------------------------------------------------------
enum SplitMode : int { SPLIT_LOWER = 0, SPLIT_NOT_CONST = 1, SPLIT_DICT = 2 };
struct SplitArgs {
    Order order = ORD_INT;
    uint64_t thr = 0;                        // SPLIT_LOWER: threshold bits (x < thr in T order)
    bool outside = false;                    // SPLIT_LOWER of the outside patch: !(x > hi || x < lo)
    uint64_t lo = 0, hi = 0;                 //   its bounds (bits, T order)
    const uint8_t *top = nullptr;            // NOT_CONST: 1 value, DICT: 4 values (device, any alignment)
    uint8_t *stencil = nullptr;              // packed stencil bytes (after the rest byte)
    uint8_t *yes = nullptr, *no = nullptr;   // ordered outputs (yes unused for DICT, no for NOT_CONST)
    uint32_t *words = nullptr;               // DICT: zeroed 2-bit code words
    unsigned long long *yes_count = nullptr; // device: number of stencil-true elements
};
struct MergeArgs {
    Order order = ORD_INT;
    const uint8_t *top = nullptr;
    const uint8_t *yes = nullptr, *no = nullptr;
    const uint32_t *words = nullptr;
    uint64_t yes_cap = 0, no_cap = 0;        // elements available (DICT: codes) -- reads stay inside
    uint32_t *error = nullptr;               // set to GTSC_ERR_FORMAT (negated) when a cap is exceeded
};
uint64_t split_tiles(uint64_t n);

// ---- histogram / top-k (hist.cu) ---------------------------------------------------------------
struct HistTable {
    unsigned long long *keys = nullptr;   // cap entries, ~0 = empty
    unsigned int *counts = nullptr;
    uint64_t cap = 0;                     // power of two
    unsigned int *special = nullptr;      // occurrences of the value whose bits are all ones
    unsigned int *overflow = nullptr;     // set when an insert found no slot
    unsigned long long *nan_keys = nullptr;  // 4 smallest NaN sort keys per block
    uint8_t *partial = nullptr;           // per-block top-4 lists
};
uint64_t hist_cap_for(uint64_t n, bool full);
int hist_grid(uint64_t n);
uint64_t hist_scratch_bytes(uint64_t cap, int grid);
HistTable hist_table_at(uint8_t *scratch, uint64_t cap, int grid);
// top-k values (k <= 4, es bytes each) by count desc then value asc; unused slots 0
void launch_hist_topk(const uint8_t *in, uint64_t n, int es, Order o, int k, const HistTable &t, int grid,
                      uint8_t *top_out, unsigned long long *count_out, cudaStream_t s);

// ---- RLE and scans (rle.cu) ----------------------------------------------------------------------
uint64_t rle_tiles(uint64_t n);
// scratch = lookback_bytes(rle_tiles(n)); starts: n uint32; runs: device count
void launch_rle_encode(const uint8_t *in, uint64_t n, int es, Order o, uint8_t *values, int32_t *lengths,
                       uint32_t *starts, unsigned long long *runs, uint8_t *scratch, cudaStream_t s);
// inclusive scan of n int32 (any alignment) into uint64; scratch = lookback_bytes(rle_tiles(n))
void launch_scan_i32(const uint8_t *in, uint64_t n, unsigned long long *out, uint8_t *scratch, cudaStream_t s);
void launch_rle_expand(const unsigned long long *ends, uint64_t runs, const uint8_t *values, uint64_t n, int es,
                       uint8_t *out, cudaStream_t s);

// ---- GFC (gfc.cu) ----------------------------------------------------------------------------------
struct GfcGeom {
    bool dbl = true;
    uint64_t n = 0, npad = 0, per = 32;
    int blocks = 0, wpb = 0, unit = 17;
    int64_t warps = 0;
};
GfcGeom gfc_geom(bool dbl, uint64_t n, int blocks, int wpb);
uint64_t gfc_scratch_layout_bytes(const GfcGeom &g);
void launch_gfc_compress(const uint8_t *in, const GfcGeom &g, uint8_t *layout, int32_t *ends, int32_t *sizes,
                         cudaStream_t s);
void launch_gfc_compact(const uint8_t *layout, const GfcGeom &g, const int32_t *sizes,
                        const unsigned long long *incl, uint8_t *out, cudaStream_t s);
void launch_gfc_sizes(const uint8_t *ends, const GfcGeom &g, int32_t *sizes, uint32_t *error, cudaStream_t s);
void launch_gfc_decompress(const uint8_t *payload, uint64_t payload_bytes, const GfcGeom &g, const int32_t *sizes,
                           const unsigned long long *incl, uint8_t *out, uint32_t *error, cudaStream_t s);

// ---- statistics / floatToInt (stats.cu) -------------------------------------------------------------
struct StatsAcc {
    MinMaxAcc mm;
    unsigned long long rl_sum;
    unsigned long long int_sum;
    unsigned int prec_steps;
    unsigned int unsorted;
};
unsigned stats_grid(uint64_t n);
// fsum_partial: stats_grid(n) doubles
void launch_stats(const uint8_t *in, uint64_t n, int es, Order o, StatsAcc *acc, double *fsum_partial,
                  cudaStream_t s);
void launch_log_table(int *table, cudaStream_t s);
void launch_f2i_encode(const uint8_t *in, uint64_t n, int es, Order o, int p, int32_t *out, unsigned int *lossy,
                       cudaStream_t s);
void launch_f2i_decode(const uint8_t *in, uint64_t n, int es, Order o, int p, uint8_t *out, cudaStream_t s);
// scratch = lookback_bytes(split_tiles(n))
void launch_split(int mode, const uint8_t *in, uint64_t n, int es, const SplitArgs &a, uint8_t *scratch,
                  cudaStream_t s);
void launch_merge(int mode, const uint8_t *stencil, uint64_t n, int es, const MergeArgs &a, uint8_t *out,
                  uint8_t *scratch, cudaStream_t s);

// AflEncoding's float path (afl_float.cu): split into mantissa / exponent int32 arrays and the sign
// stencil (1 + ceil(n/8) bytes); flags |= 1 when a sign bit is set, |= 2 when one is clear
void launch_float_split(const uint8_t *in, uint64_t n, int32_t *mant, int32_t *expo, uint8_t *stencil,
                        uint32_t *flags, cudaStream_t s);
// the inverse; stencil = the packed sign bits (without its rest byte), or null and `fill` for all
void launch_float_compose(const int32_t *mant, const int32_t *expo, const uint8_t *stencil, int fill, uint64_t n,
                          uint32_t *out, cudaStream_t s);

// aligned AFL layout (afl32.cu): words of a stream of n elements at b bits (element units)
uint64_t afl32_words(uint64_t n, int b, int es);
void launch_afl32_pack(const uint8_t *in, uint64_t n, int es, int b, uint8_t *out, uint64_t words, cudaStream_t s);
void launch_afl32_unpack(const uint8_t *comp, uint64_t words, uint64_t n, int es, int b, uint8_t *out, cudaStream_t s);
// random access: out[t] = element (idx ? idx[t] : t) of an FL (omega 1) or aligned (omega 32) stream
void launch_afl_values(const uint8_t *comp, uint64_t words, int es, int b, int omega, const uint64_t *idx,
                       uint64_t n, uint8_t *out, cudaStream_t s);

}  // namespace gtsc
