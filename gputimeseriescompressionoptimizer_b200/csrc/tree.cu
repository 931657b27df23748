// tree.cu -- compression-tree serialization over the GPU encodings.
//
// Serialized tree (CompressionNode::Compress / PrepareMetadata, tree/compression_node.cpp:84-138):
// pre-order, node := {int16 EncodingType, int16 DataType, int32 MetadataLength} || metadata ||
// (none ? data[*(size_t*)metadata] : child_1 .. child_k).
//
// Decompression: the reference reads every node header with its own device-to-host copy
// (tree/compression_tree.cpp:105-146).  Here one single-thread kernel walks the blob and writes a
// node table (offsets of each node's metadata and data), the host reads the table once and decodes
// bottom-up directly from views into the blob.
#include "kernels.hpp"
#include "tree.hpp"
#include "vec.cuh"

#include <cstring>

namespace gtsc {

// Encoding::GetCompressionRatio (compression/encoding.hpp:78-84)
double compression_ratio(uint64_t in, uint64_t out) { return (out == 0 || out > in) ? 1.0 : (double)in / (double)out; }

namespace {

constexpr int kMaxNodes = 1024;
constexpr int kMaxDepth = 64;

struct ParsedNode {
    int32_t enc, dt, parent, pad;
    uint64_t meta_off, meta_len, data_off, data_len;
};

__device__ int nres_dev(int enc)
{
    switch (enc) {
    case GTSC_DELTA: case GTSC_AFL: case GTSC_SCALE: case GTSC_UNIQUE: case GTSC_FLOAT_TO_INT: case GTSC_CONST:
        return 1;
    case GTSC_RLE: case GTSC_DICT: case GTSC_PATCH: case GTSC_GFC: return 2;
    case GTSC_NONE: return 0;
    default: return -1;
    }
}

__global__ void k_parse_tree(const uint8_t *__restrict__ blob, uint64_t bytes, ParsedNode *nodes, int *count,
                             uint32_t *error)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int stack_node[kMaxDepth], stack_left[kMaxDepth];
    int depth = 0, cnt = 0;
    uint64_t pos = 0;
    int parent = -1;
    while (true) {
        // parse the node at pos
        if (cnt >= kMaxNodes || pos + 8 > bytes) { *error = (uint32_t)(-GTSC_ERR_FORMAT); return; }
        const int enc = (int16_t)ld_unaligned<2>(blob + pos);
        const int dt = (int16_t)ld_unaligned<2>(blob + pos + 2);
        const int64_t ml = (int32_t)ld_unaligned<4>(blob + pos + 4);
        const int r = nres_dev(enc);
        if (r < 0 || dt < 0 || dt > 5 || ml < 0 || pos + 8 + (uint64_t)ml > bytes) {
            *error = (uint32_t)(-GTSC_ERR_FORMAT);
            return;
        }
        ParsedNode nd;
        nd.enc = enc; nd.dt = dt; nd.parent = parent; nd.pad = 0;
        nd.meta_off = pos + 8;
        nd.meta_len = (uint64_t)ml;
        pos += 8 + (uint64_t)ml;
        nd.data_off = pos;
        nd.data_len = 0;
        if (enc == GTSC_NONE) {
            if (ml < 8) { *error = (uint32_t)(-GTSC_ERR_FORMAT); return; }
            const uint64_t ds = ld_unaligned<8>(blob + nd.meta_off);
            if (ds > bytes - pos) { *error = (uint32_t)(-GTSC_ERR_FORMAT); return; }
            nd.data_len = ds;
            pos += ds;
        }
        nodes[cnt] = nd;
        const int me = cnt++;
        if (r > 0) {
            if (depth >= kMaxDepth) { *error = (uint32_t)(-GTSC_ERR_FORMAT); return; }
            stack_node[depth] = me;
            stack_left[depth] = r;
            depth++;
        }
        // next node: first pending child of the deepest open node
        while (depth > 0 && stack_left[depth - 1] == 0) depth--;
        if (depth == 0) break;
        stack_left[depth - 1]--;
        parent = stack_node[depth - 1];
    }
    if (pos != bytes) { *error = (uint32_t)(-GTSC_ERR_FORMAT); return; }
    *count = cnt;
}

// ----------------------------------------------------------------------- compress

struct Seg {
    const uint8_t *src;  // device pointer, or nullptr for host header bytes
    uint64_t host_off;   // offset into the host header staging
    uint64_t bytes;
};

uint64_t seg_bytes(const std::vector<Seg> &segs, size_t from)
{
    uint64_t b = 0;
    for (size_t k = from; k < segs.size(); k++) b += segs[k].bytes;
    return b;
}

void compress_rec(const Tree &t, int &i, View in, std::vector<Seg> &segs, std::vector<uint8_t> &hdrs,
                  std::vector<DevBuf> &keep, cudaStream_t s, std::vector<double> *ratios)
{
    if (i >= t.size()) fail(GTSC_ERR_ARG, "tree: incomplete node list");
    const int enc = t.enc[i], dt = t.dt[i];
    const int me = i;
    const size_t seg0 = segs.size();
    ++i;
    auto push_hdr = [&](int32_t meta_len) {
        // both patch variants serialise as EncodingType::patch
        int16_t h[2] = {(int16_t)(enc == GTSC_PATCH_OUTSIDE ? GTSC_PATCH : enc), (int16_t)dt};
        size_t off = hdrs.size();
        hdrs.resize(off + 8);
        memcpy(hdrs.data() + off, h, 4);
        memcpy(hdrs.data() + off + 4, &meta_len, 4);
        segs.push_back(Seg{nullptr, off, 8});
    };
    if (enc == GTSC_NONE) {  // NoneEncoding: size_t byte count, then the bytes themselves
        push_hdr(8);
        size_t off = hdrs.size();
        hdrs.resize(off + 8);
        uint64_t b = in.bytes;
        memcpy(hdrs.data() + off, &b, 8);
        segs.push_back(Seg{nullptr, off, 8});
        if (in.bytes) segs.push_back(Seg{in.ptr, 0, in.bytes});
        if (ratios) (*ratios)[me] = compression_ratio(in.bytes, seg_bytes(segs, seg0));
        return;
    }
    Parts p = encode(enc, dt, in, s);
    for (auto &b : p) keep.push_back(b);
    const int r = n_results(enc);
    push_hdr((int32_t)p[0].bytes);
    if (p[0].bytes) segs.push_back(Seg{p[0].get(), 0, p[0].bytes});
    for (int j = 0; j < r; j++) compress_rec(t, i, View(p[j + 1]), segs, hdrs, keep, s, ratios);
    // CompressionNode::Compress (tree/compression_node.cpp:103-135): input over everything the
    // subtree wrote, headers included
    if (ratios) (*ratios)[me] = compression_ratio(in.bytes, seg_bytes(segs, seg0));
}

// ----------------------------------------------------------------------- decompress

DevBuf decode_node(const std::vector<ParsedNode> &nd, const std::vector<std::vector<int>> &kids, int i,
                   const uint8_t *blob, cudaStream_t s, int depth)
{
    if (depth > kMaxDepth) fail(GTSC_ERR_FORMAT, "tree: too deep");
    const ParsedNode &n = nd[i];
    if (n.enc == GTSC_NONE) {  // NoneEncoding::Decode copies the data
        DevBuf out = dev_alloc(n.data_len, s);
        if (n.data_len) GTSC_CUDA(cudaMemcpyAsync(out.get(), blob + n.data_off, n.data_len, cudaMemcpyDeviceToDevice, s));
        return out;
    }
    std::vector<DevBuf> child;
    std::vector<View> in;
    in.push_back(View(blob + n.meta_off, n.meta_len));
    for (int k : kids[i]) {
        const ParsedNode &c = nd[k];
        if (c.enc == GTSC_NONE) {
            in.push_back(View(blob + c.data_off, c.data_len));  // decode straight from the blob
        } else {
            child.push_back(decode_node(nd, kids, k, blob, s, depth + 1));
            in.push_back(View(child.back()));
        }
    }
    return decode(n.enc, n.dt, in, s);
}

}  // namespace

// ----------------------------------------------------------------------- public

Tree tree_from_nodes(const int16_t *pairs, int n_nodes)
{
    if (!pairs || n_nodes <= 0 || n_nodes > kMaxNodes) fail(GTSC_ERR_ARG, "tree: bad node list");
    Tree t;
    int need = 1;
    for (int i = 0; i < n_nodes; i++) {
        const int enc = pairs[2 * i], dt = pairs[2 * i + 1];
        if (need == 0) fail(GTSC_ERR_ARG, "tree: nodes after the last subtree");
        const int r = n_results(enc);
        if (r < 0 || !dtype_size(dt)) fail(GTSC_ERR_ARG, "tree: unknown encoding or data type");
        need += r - 1;
        t.enc.push_back((int16_t)enc);
        t.dt.push_back((int16_t)dt);
    }
    if (need != 0) fail(GTSC_ERR_ARG, "tree: a node misses children (leaves must be none)");
    return t;
}

void tree_to_nodes(const Tree &t, int16_t *pairs)
{
    for (int i = 0; i < t.size(); i++) {
        pairs[2 * i] = t.enc[i];
        pairs[2 * i + 1] = t.dt[i];
    }
}

static void from_path_rec(const int16_t *encs, int n, int &id, int dt, Tree &t, int depth)
{
    if (id >= n || depth > kMaxDepth) fail(GTSC_ERR_ARG, "path: too short");
    const int enc = encs[id];
    const int r = n_results(enc);
    if (r < 0) fail(GTSC_ERR_ARG, "path: unknown encoding");
    t.enc.push_back((int16_t)enc);
    t.dt.push_back((int16_t)dt);
    for (int j = 0; j < r; j++) {
        ++id;
        from_path_rec(encs, n, id, return_type(enc, dt, j), t, depth + 1);
    }
}

Tree tree_from_path(const int16_t *encs, int n, int dtype)
{
    if (!dtype_size(dtype)) fail(GTSC_ERR_ARG, "path: unknown data type");
    Tree t;
    int id = 0;
    from_path_rec(encs, n, id, dtype, t, 0);
    if (id != n - 1) fail(GTSC_ERR_ARG, "path: extra entries");
    return t;
}

Tree leaf_tree(int enc, int dtype)
{
    Tree t;
    t.enc.push_back((int16_t)enc);
    t.dt.push_back((int16_t)dtype);
    for (int j = 0; j < n_results(enc); j++) {
        t.enc.push_back(GTSC_NONE);
        t.dt.push_back((int16_t)dtype);
    }
    return t;
}

DevBuf tree_compress(const Tree &t, View in, cudaStream_t s, std::vector<double> *ratios)
{
    std::vector<Seg> segs;
    std::vector<uint8_t> hdrs;
    std::vector<DevBuf> keep;
    int i = 0;
    if (ratios) ratios->assign(t.size(), 1.0);
    compress_rec(t, i, in, segs, hdrs, keep, s, ratios);
    if (i != t.size()) fail(GTSC_ERR_ARG, "tree: extra nodes");
    uint64_t total = 0;
    for (auto &g : segs) total += g.bytes;
    DevBuf blob = dev_alloc(total, s);
    DevBuf staging = dev_alloc(hdrs.size(), s);
    if (!hdrs.empty()) GTSC_CUDA(cudaMemcpyAsync(staging.get(), hdrs.data(), hdrs.size(), cudaMemcpyHostToDevice, s));
    uint64_t off = 0;
    for (auto &g : segs) {
        const uint8_t *src = g.src ? g.src : staging.get() + g.host_off;
        GTSC_CUDA(cudaMemcpyAsync(blob.get() + off, src, g.bytes, cudaMemcpyDeviceToDevice, s));
        off += g.bytes;
    }
    GTSC_CUDA(cudaStreamSynchronize(s));  // `keep` and `hdrs` die here
    return blob;
}

DevBuf tree_decompress(View blob, int *dtype, cudaStream_t s)
{
    if (blob.bytes < 8) fail(GTSC_ERR_FORMAT, "tree: blob too short");
    DevBuf table = dev_alloc(sizeof(ParsedNode) * kMaxNodes + 16, s);
    int *cnt = (int *)(table.get() + sizeof(ParsedNode) * kMaxNodes);
    uint32_t *err = (uint32_t *)(cnt + 1);
    GTSC_CUDA(cudaMemsetAsync(cnt, 0, 16, s));
    k_parse_tree<<<1, 1, 0, s>>>(blob.ptr, blob.bytes, (ParsedNode *)table.get(), cnt, err);
    GTSC_CUDA(cudaGetLastError());
    int hc[2];
    d2h(hc, cnt, 8, s);
    if (hc[1]) fail(-(gtsc_status)hc[1], "tree: corrupt blob");
    if (hc[0] <= 0) fail(GTSC_ERR_FORMAT, "tree: no nodes");
    std::vector<ParsedNode> nd(hc[0]);
    d2h(nd.data(), table.get(), sizeof(ParsedNode) * hc[0], s);
    std::vector<std::vector<int>> kids(hc[0]);
    for (int k = 1; k < hc[0]; k++) kids[nd[k].parent].push_back(k);
    if (dtype) *dtype = nd[0].dt;
    DevBuf out = decode_node(nd, kids, 0, blob.ptr, s, 0);
    GTSC_CUDA(cudaStreamSynchronize(s));
    return out;
}

uint64_t predicted_metadata_size(int enc, int dt, View in, cudaStream_t s)
{
    const int es = dtype_size(dt);
    const uint64_t bytes = in.bytes, elems = bytes / es;
    switch (enc) {
    case GTSC_NONE: return 8;                                            // none_encoding.hpp:36-39
    case GTSC_DELTA: case GTSC_SCALE: return bytes ? (uint64_t)es : 0;
    case GTSC_RLE: case GTSC_FLOAT_TO_INT: return bytes ? 4 : 0;
    case GTSC_AFL:                                                       // afl_encoding.cu:281-293
        if (!bytes) return 0;
        if (dt == GTSC_INT) return 4;
        if (dt == GTSC_FLOAT) return 9;
        fail(GTSC_ERR_UNSUPPORTED, "afl: no metadata-size predictor for this type");
    case GTSC_DICT: return (elems + 7) / 8 + 1;                          // dict_encoding.hpp:44-48
    case GTSC_PATCH: case GTSC_PATCH_OUTSIDE: return bytes ? (elems + 7) / 8 + 1 : 0;
    case GTSC_CONST: return bytes ? (elems + 7) / 8 + es + 1 : 0;
    case GTSC_GFC: return 12;
    default: (void)s; fail(GTSC_ERR_UNSUPPORTED, "no metadata-size predictor for this encoding");
    }
}

static uint64_t predict_rec(const Tree &t, int &i, int type, View in, cudaStream_t s)
{
    if (i >= t.size()) fail(GTSC_ERR_ARG, "tree: incomplete node list");
    const int enc = t.enc[i];
    ++i;
    uint64_t size = predicted_metadata_size(enc, type, in, s) + 8;
    if (enc == GTSC_NONE) return size + in.bytes;  // NoneEncoding::GetCompressedSize
    Parts p = encode(enc, type, in, s);
    for (int j = 0; j < n_results(enc); j++) size += predict_rec(t, i, return_type(enc, type, j), View(p[j + 1]), s);
    return size;
}

uint64_t tree_predict_size(const Tree &t, View in, cudaStream_t s)
{
    int i = 0;
    uint64_t sz = predict_rec(t, i, t.dt[0], in, s);
    if (i != t.size()) fail(GTSC_ERR_ARG, "tree: extra nodes");
    return sz;
}

}  // namespace gtsc
