// batch.cu -- compiles many columns' compression trees into stages of batched passes, owns their
// device memory, and records each step (compress / decompress) once as a CUDA graph.
//
// Compile: every node of every tree gets its output streams with worst-case capacities (computed
// from the column length), a scratch area (accumulators, look-back state, hash table, GFC layout)
// and a list of passes.  A pass's level is one more than the pass it waits for (the previous pass of
// its node, or the pass that produced its input); passes with the same (level, kind) form one
// launch over all columns.  Capacities only bound memory and grids: the real lengths are written
// by the passes into the device stream table, so a step never waits for the host.
#include "batch.hpp"
#include "encodings.hpp"
#include "kernels.hpp"
#include "scan.cuh"

#include <algorithm>
#include <chrono>
#include <functional>
#include <map>
#include <tuple>

namespace gtsc {

namespace {

__global__ void k_set_streams(const unsigned long long *vals, const int *sids, int n, StreamDesc *S)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    S[sids[i]].ptr = (uint8_t *)vals[2 * i];
    S[sids[i]].len = vals[2 * i + 1];
}

uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }
uint64_t cdiv(uint64_t a, uint64_t b) { return (a + b - 1) / b; }
bool aligned16(const void *p) { return ((uintptr_t)p & 15) == 0; }

struct HNode {
    int col = 0, enc = 0, dt = 0, es = 0;
    int parent = -1;
    std::vector<int> kids;
    int in_sid = -1;                  // compress input
    int out_sid[3] = {-1, -1, -1};    // compress outputs: meta, out1, out2
    int dec_meta_sid = -1;            // decode: the node's metadata inside the blob
    int dec_data_sid = -1;            // decode (none leaves): the data inside the blob
    int dec_out_sid = -1;             // decode: this node's decoded stream
    uint64_t in_cap = 0;              // bytes
    uint64_t scratch = 0;             // offset in the arena
    uint64_t c_bytes = 0, d_bytes = 0;
    // compress scratch layout
    uint64_t lb_off = 64, tab_off = 0, starts_off = 0, g_sizes = 0, g_incl = 0, g_layout = 0, tab_cap = 0;
    uint64_t hist_tiles = 0, split_tiles = 0, gfc_warps = 0;
    // decode scratch layout (relative to scratch)
    uint64_t dlb_off = 0, dends_off = 0, druns_off = 0, dtiles_off = 0, dsizes_off = 0, dincl_off = 0;
    int last_c_level = 0, last_d_level = 0;
    // compress input view: the node reads stream in_sid through vop[] (V_SCALE ops take their
    // constant from scale node vnode[k]); a virtual node's own output is never written, its child
    // reads it as this node's view plus this node's operation
    int8_t vop[kMaxViewOps] = {V_NONE, V_NONE, V_NONE};
    int vnode[kMaxViewOps] = {-1, -1, -1};
    bool virt = false;
    // decode: a node whose decoded output its parent reads through a DView (an AFL node over its
    // packed bits, a scale node as an addition) has no decode pass and no output stream
    bool dvirt = false;
    DView dview;        // how the parent reads this node's decoded output
    int d_ready = 0;    // decode level from which that output can be read
};

struct Pass {
    int level;
    int op;
    int node;
    BItem item;
};

int view_ops(const int8_t *vop)
{
    int k = 0;
    while (k < kMaxViewOps && vop[k] != V_NONE) ++k;
    return k;
}

// encodings whose compress passes read their input through a view
bool view_consumer(int enc)
{
    return enc == GTSC_AFL || enc == GTSC_GFC || enc == GTSC_DICT || enc == GTSC_CONST || enc == GTSC_PATCH ||
           enc == GTSC_PATCH_OUTSIDE || enc == GTSC_RLE || enc == GTSC_DELTA || enc == GTSC_SCALE;
}

struct Launch {
    int op;
    int first, count;
    uint64_t tiles;
    uint64_t map_off;  // this launch's tile -> item table in the item_of array
    int level;
};

// passes whose tiles chain through a decoupled look-back (claimed in order from a counter)
bool dyn_pass(int op)
{
    return op == B_SPLIT || op == B_RLE_HEADS || op == B_GFC_SCAN || op == B_DELTA_DEC || op == B_RLE_SCAN;
}

constexpr uint32_t kMinMaxTileMin = 1024;  // the smallest min/max tile (tiles are reserved for it)

uint64_t gfc_warps_for(bool dbl, uint64_t n)
{
    const uint64_t wpb = dbl ? 16 : 32;
    const uint64_t bs = wpb * (dbl ? 64 : 32) * 32;
    return cdiv(n, bs) * wpb;
}

}  // namespace

class BatchEngine {
public:
    std::vector<HNode> nodes;
    std::vector<StreamDesc> streams;        // host image of the table
    std::vector<int> col_root;              // root node of each column
    std::vector<int> col_in_sid, col_out_sid;
    std::vector<uint64_t> col_bytes;
    std::vector<BColumnDev> cols_dev;
    std::vector<BNodeDev> nodes_c, nodes_d;  // framing (compress) / parse (decode) node tables
    std::vector<Pass> pass_c, pass_d;
    std::vector<BItem> items_c, items_d, items_copy;
    std::vector<int> item_col_c, item_col_d;  // each item's column
    std::vector<Launch> launch_c, launch_d;
    // the persistent schedule (batch.hpp, PUnit) of each phase
    std::vector<PUnit> punit_c, punit_d;
    std::vector<PItem> pitem_c, pitem_d;
    uint32_t q_total_c = 0, q_total_d = 0;
    PUnit *d_punit_c = nullptr, *d_punit_d = nullptr;
    PItem *d_pitem_c = nullptr, *d_pitem_d = nullptr;
    uint32_t *d_done_c = nullptr, *d_done_d = nullptr, *d_ext_c = nullptr, *d_ext_d = nullptr;
    uint32_t *d_queue = nullptr;  // [0] compress claim counter, [1] decode claim counter
    BatchTuning tune;             // launch parameters (schedule, tile sizes)
    std::vector<BatchColumn> src_cols;  // the columns (current inputs) and trees, for re-tuning
    std::vector<Tree> src_trees;
    std::vector<uint32_t> item_of;           // tile -> item tables of every launch, back to back
    uint64_t copy_map_off = 0;
    uint32_t *d_item_of = nullptr;
    uint64_t copy_tiles = 0, framed_cap = 0;
    std::vector<unsigned long long> zero_c, zero_d;  // (ptr, bytes) pairs
    std::vector<std::pair<uint64_t, uint64_t>> hist_tables;  // (offset, cap) to initialise

    DevBuf arena, tables;
    StreamDesc *d_streams = nullptr;
    BItem *d_items_c = nullptr, *d_items_d = nullptr, *d_items_copy = nullptr;
    BColumnDev *d_cols = nullptr;
    BNodeDev *d_nodes_c = nullptr, *d_nodes_d = nullptr;
    unsigned long long *d_col_off = nullptr, *d_col_off_d = nullptr, *d_total = nullptr;
    unsigned long long *d_zero_c = nullptr, *d_zero_d = nullptr;
    unsigned long long *d_set_vals = nullptr, *d_frame_len = nullptr;
    int *d_set_sids = nullptr;
    uint8_t **d_frame_ptr = nullptr;
    uint32_t *d_status = nullptr, *d_counters = nullptr;
    uint8_t *d_framed = nullptr;
    int n_counters = 0;
    cudaGraphExec_t graph_c[2] = {nullptr, nullptr}, graph_d[2] = {nullptr, nullptr};  // [persistent]

    int new_stream(uint64_t cap)
    {
        streams.push_back(StreamDesc{nullptr, 0, cap, 0});
        return (int)streams.size() - 1;
    }

    void build_node(const Tree &t, int &k, int col, int parent, int in_sid, uint64_t in_cap, int depth,
                    const int8_t *in_vop, const int *in_vnode);
    int folded_minmax(int id) const;
    void plan_passes();
    void layout(cudaStream_t s);
    void capture(cudaStream_t s);
    void record_compress(cudaStream_t s, const std::function<void(int)> &mark, bool pers);
    void record_decompress(cudaStream_t s, const std::function<void(int)> &mark, bool pers);
    void plan_persistent(const std::vector<Launch> &launches, const std::vector<BItem> &items,
                         const std::vector<int> &item_col, std::vector<PUnit> &units, std::vector<PItem> &pi,
                         uint32_t &total);
    PersistArgs persist_args(bool compress) const;
};

// ---------------------------------------------------------------------------------- compile

void BatchEngine::build_node(const Tree &t, int &k, int col, int parent, int in_sid, uint64_t in_cap, int depth,
                             const int8_t *in_vop, const int *in_vnode)
{
    if (k >= t.size() || depth > 64) fail(GTSC_ERR_ARG, "batch: incomplete tree");
    HNode nd;
    nd.col = col;
    nd.enc = t.enc[k];
    nd.dt = t.dt[k];
    nd.es = dtype_size(nd.dt);
    nd.parent = parent;
    nd.in_sid = in_sid;
    nd.in_cap = in_cap;
    for (int j = 0; j < kMaxViewOps; j++) {
        nd.vop[j] = in_vop ? in_vop[j] : (int8_t)V_NONE;
        nd.vnode[j] = in_vnode ? in_vnode[j] : -1;
    }
    ++k;
    // a delta / scale whose one child reads through views is not materialised
    const int nops = view_ops(nd.vop);
    nd.virt = (nd.enc == GTSC_DELTA || nd.enc == GTSC_SCALE) && k < t.size() && view_consumer(t.enc[k]) &&
              nops < kMaxViewOps;
    const int id = (int)nodes.size();
    nodes.push_back(nd);
    if (parent >= 0) nodes[parent].kids.push_back(id);
    HNode &me = nodes[id];
    const uint64_t es = me.es, n = in_cap / es;
    uint64_t cap[3] = {0, 0, 0};
    switch (me.enc) {
    case GTSC_NONE: break;
    case GTSC_DELTA: case GTSC_SCALE: cap[0] = es; cap[1] = in_cap; break;
    case GTSC_AFL: cap[0] = 4; cap[1] = in_cap + es; break;
    case GTSC_RLE: cap[0] = 4; cap[1] = 4 * n; cap[2] = in_cap; break;
    case GTSC_DICT: cap[0] = 2 + cdiv(n, 8); cap[1] = 20 + 4 * es + 4 * cdiv(n, 16); cap[2] = in_cap; break;
    case GTSC_CONST: cap[0] = es + 2 + cdiv(n, 8); cap[1] = in_cap; break;
    case GTSC_PATCH: case GTSC_PATCH_OUTSIDE: cap[0] = 2 + cdiv(n, 8); cap[1] = in_cap; cap[2] = in_cap; break;
    case GTSC_FLOAT_TO_INT: cap[0] = 4; cap[1] = std::max<uint64_t>(4 * n, in_cap); break;
    case GTSC_GFC:
        if (is_fp(me.dt)) {
            cap[0] = 12;
            cap[1] = 4 * gfc_warps_for(me.dt == GTSC_DOUBLE, n);
            cap[2] = cdiv((n + 31) & ~31ull, 32) * (16 + 32 * es);
        } else {
            cap[0] = 4;
            cap[1] = in_cap + es;
        }
        break;
    default: fail(GTSC_ERR_ARG, "batch: unsupported encoding in tree");
    }
    if (me.enc == GTSC_AFL && is_fp(me.dt))
        fail(GTSC_ERR_UNSUPPORTED, "batch: AFL of a floating-point node runs on the per-column path only");
    const int r = n_results(me.enc);
    if (me.virt) cap[1] = 0;  // read through the child's view, never written
    if (me.enc != GTSC_NONE)
        for (int j = 0; j <= r; j++) nodes[id].out_sid[j] = new_stream(cap[j]);
    // decode-side streams
    if (nodes[id].enc == GTSC_NONE) nodes[id].dec_data_sid = new_stream(0);
    else nodes[id].dec_meta_sid = new_stream(0);
    if (parent >= 0) nodes[id].dec_out_sid = new_stream(in_cap);
    if (nodes[id].virt) {
        int8_t cv[kMaxViewOps];
        int cn[kMaxViewOps];
        for (int j = 0; j < kMaxViewOps; j++) {
            cv[j] = nodes[id].vop[j];
            cn[j] = nodes[id].vnode[j];
        }
        const int nops2 = view_ops(cv);
        cv[nops2] = nodes[id].enc == GTSC_DELTA ? (int8_t)V_DELTA : (int8_t)V_SCALE;
        cn[nops2] = nodes[id].enc == GTSC_SCALE ? id : -1;
        const uint64_t child_cap = nodes[id].in_cap;
        build_node(t, k, col, id, nodes[id].in_sid, child_cap, depth + 1, cv, cn);
        return;
    }
    for (int j = 0; j < r; j++) build_node(t, k, col, id, nodes[id].out_sid[j + 1], cap[j + 1], depth + 1, nullptr, nullptr);
}

// A node packed by AFL whose min / max its parent's split accumulates while it writes the child's
// input stream, so that the child needs no min/max pass of its own (one read of that stream less):
// the patch outputs, the const node's unmatched values and the dictionary's unmatched values.
// Returns the parent's split output (1 = the matches, 2 = the rest) or 0.
int BatchEngine::folded_minmax(int id) const
{
    const HNode &nd = nodes[id];
    if (nd.parent < 0 || nd.virt || view_ops(nd.vop) != 0) return 0;
    if (!(nd.enc == GTSC_AFL || (nd.enc == GTSC_GFC && !is_fp(nd.dt)))) return 0;
    const HNode &par = nodes[nd.parent];
    const int slot = (int)(std::find(par.kids.begin(), par.kids.end(), id) - par.kids.begin()) + 1;
    switch (par.enc) {
    case GTSC_PATCH: case GTSC_PATCH_OUTSIDE: return slot;
    case GTSC_CONST: return slot == 1 ? 1 : 0;
    case GTSC_DICT: return slot == 2 ? 2 : 0;
    default: return 0;
    }
}

void BatchEngine::plan_passes()
{
    // scratch sizes
    for (auto &nd : nodes) {
        const uint64_t n = nd.in_cap / nd.es;
        uint64_t c = 64;
        switch (nd.enc) {
        case GTSC_PATCH: case GTSC_PATCH_OUTSIDE:
            nd.split_tiles = std::max<uint64_t>(1, cdiv(n, kBTile));
            c = 64 + align_up(lookback_bytes(nd.split_tiles), 256);
            break;
        case GTSC_DICT: case GTSC_CONST: {
            nd.split_tiles = std::max<uint64_t>(1, cdiv(n, kBTile));
            nd.hist_tiles = std::max<uint64_t>(1, cdiv(n, tune.hist_tile));
            uint64_t cap = 1024;
            while (cap < 2 * n + 64) cap <<= 1;
            nd.tab_cap = cap;
            nd.tab_off = 64 + align_up(lookback_bytes(nd.split_tiles), 256);
            c = nd.tab_off + align_up(bhist_bytes(cap, nd.hist_tiles), 256);
            break;
        }
        case GTSC_RLE:
            nd.split_tiles = std::max<uint64_t>(1, cdiv(n, kBTile));
            nd.starts_off = 64 + align_up(lookback_bytes(nd.split_tiles), 256);
            c = nd.starts_off + align_up(4 * n + 16, 256);
            break;
        case GTSC_FLOAT_TO_INT: c = 128; break;
        case GTSC_GFC:
            if (is_fp(nd.dt)) {
                const bool dbl = nd.dt == GTSC_DOUBLE;
                nd.gfc_warps = gfc_warps_for(dbl, n);
                const uint64_t scan_tiles = std::max<uint64_t>(1, cdiv(nd.gfc_warps, kBTile));
                nd.g_sizes = 64 + align_up(lookback_bytes(scan_tiles), 256);
                nd.g_incl = nd.g_sizes + align_up(4 * nd.gfc_warps + 16, 256);
                nd.g_layout = nd.g_incl + align_up(8 * nd.gfc_warps + 16, 256);
                c = nd.g_layout + align_up(((n + 31) & ~31ull) / 2 * (dbl ? 17 : 9) + 64, 256);
            }
            break;
        default: break;
        }
        nd.c_bytes = align_up(c, 256);
        // decode scratch (after the compress scratch, which keeps the hash tables clean)
        uint64_t d = 0;
        const uint64_t tiles = std::max<uint64_t>(1, cdiv(n, kBTile));
        switch (nd.enc) {
        case GTSC_DELTA: case GTSC_PATCH: case GTSC_PATCH_OUTSIDE: case GTSC_DICT: case GTSC_CONST:
            nd.dlb_off = nd.c_bytes;
            d = align_up(lookback_bytes(tiles), 256);
            break;
        case GTSC_RLE:
            nd.dlb_off = nd.c_bytes;
            nd.dends_off = nd.dlb_off + align_up(lookback_bytes(tiles), 256);
            nd.druns_off = nd.dends_off + align_up(8 * n + 16, 256);
            nd.dtiles_off = nd.druns_off + 256;  // run holding each expand tile's first element
            d = nd.dtiles_off + align_up(8 * tiles + 16, 256) - nd.c_bytes;
            break;
        case GTSC_GFC:
            if (is_fp(nd.dt)) {
                const uint64_t scan_tiles = std::max<uint64_t>(1, cdiv(nd.gfc_warps, kBTile));
                nd.dlb_off = nd.c_bytes;
                nd.dsizes_off = nd.dlb_off + align_up(lookback_bytes(scan_tiles), 256);
                nd.dincl_off = nd.dsizes_off + align_up(4 * nd.gfc_warps + 16, 256);
                d = nd.dincl_off + align_up(8 * nd.gfc_warps + 16, 256) - nd.c_bytes;
            }
            break;
        default: break;
        }
        nd.d_bytes = align_up(d, 256);
    }

    auto base_item = [](const HNode &nd, int op, uint64_t tiles) {
        BItem it{};
        it.op = (int16_t)op;
        it.es = (int16_t)nd.es;
        it.order = (int16_t)ORD_INT;
        it.dt = nd.dt;
        it.tiles = (uint32_t)std::max<uint64_t>(1, tiles);
        for (int j = 0; j < 3; j++) {
            it.in[j] = -1;
            it.out[j] = nd.out_sid[j];
        }
        it.in[0] = nd.in_sid;
        for (int j = 0; j < kMaxViewOps; j++) it.vop[j] = nd.vop[j];
        return it;
    };
    // a min/max pass with the tuned tile (p[0]) and values per thread (p[1]); its tiles are
    // reserved for the smallest tile the tuner tries, so that both can change without a rebuild
    // (the pass skips tiles past its real extent)
    auto minmax_item = [&](const HNode &nd, uint64_t n) {
        BItem it = base_item(nd, B_MINMAX, cdiv(n, kMinMaxTileMin));
        it.p[0] = tune.minmax_tile;
        it.p[1] = tune.minmax_vpt;
        return it;
    };

    // ---------------- compress passes (parents before children)
    for (size_t id = 0; id < nodes.size(); id++) {
        HNode &nd = nodes[id];
        const int start = nd.parent >= 0 ? nodes[nd.parent].last_c_level + 1 : 0;
        const uint64_t n = nd.in_cap / nd.es;
        const uint64_t t2k = cdiv(n, kBTile);
        std::vector<BItem> ps;
        auto add = [&](BItem it) { ps.push_back(it); };
        const int nops = view_ops(nd.vop);
        const bool scale_view = nops > 0 && nd.vop[nops - 1] == V_SCALE;
        // split items: p[2] / p[3] = 1 + the node whose min/max the matches / the rest feed (0 =
        // none); layout() turns them into that node's scratch address
        auto set_folds = [&](BItem &sp) {
            for (int kid : nd.kids) {
                const int slot = folded_minmax(kid);
                if (slot) sp.p[1 + slot] = (uint64_t)kid + 1;
            }
        };
        if (nd.virt) {
            // delta: metadata only, the child can start at once; scale: min/max, then metadata
            BItem vm = base_item(nd, B_VMETA, 1);
            vm.mode = (int16_t)nd.enc;
            if (nd.enc == GTSC_SCALE) {
                add(minmax_item(nd, n));
                add(vm);
            } else {
                add(vm);
            }
            int lvl = start;
            for (auto &it : ps) pass_c.push_back(Pass{lvl++, it.op, (int)id, it});
            // children start with the last pass (the metadata pass has no consumer)
            nd.last_c_level = start + (int)ps.size() - 2;
            continue;
        }
        switch (nd.enc) {
        case GTSC_NONE: break;
        case GTSC_DELTA: add(base_item(nd, B_DELTA_ENC, t2k)); break;
        case GTSC_SCALE:
            add(minmax_item(nd, n));
            add(base_item(nd, B_SCALE_SUB, t2k));
            break;
        case GTSC_AFL: {
            BItem pk = base_item(nd, B_AFL_PACK, t2k);
            if (scale_view) pk.vflags |= 1;  // width from the scale's min / max: no min/max pass
            else if (!folded_minmax((int)id)) add(minmax_item(nd, n));
            add(pk);
            break;
        }
        case GTSC_PATCH: case GTSC_PATCH_OUTSIDE: {
            BItem mm = minmax_item(nd, n);
            mm.order = (int16_t)native_order(nd.dt);
            add(mm);
            BItem sp = base_item(nd, B_SPLIT, nd.split_tiles);
            sp.order = (int16_t)native_order(nd.dt);
            sp.mode = SPLIT_LOWER;
            sp.p[0] = 64;
            sp.p[1] = nd.enc == GTSC_PATCH_OUTSIDE;  // the outside variant's stencil
            set_folds(sp);
            add(sp);
            break;
        }
        case GTSC_DICT: case GTSC_CONST: {
            const int k = nd.enc == GTSC_DICT ? 4 : 1;
            BItem h = base_item(nd, B_HIST, nd.hist_tiles);
            h.order = (int16_t)native_order(nd.dt);
            h.mode = (int16_t)k;
            h.p[0] = nd.tab_cap;
            h.p[1] = nd.hist_tiles;
            h.p[2] = nd.tab_off;
            h.p[3] = tune.hist_tile;
            add(h);
            BItem tk = h;
            tk.op = B_TOPK;
            tk.tiles = (uint32_t)nd.hist_tiles;  // one block per histogram tile
            add(tk);
            BItem sp = base_item(nd, B_SPLIT, nd.split_tiles);
            sp.order = (int16_t)native_order(nd.dt);
            sp.mode = (int16_t)(nd.enc == GTSC_DICT ? SPLIT_DICT : SPLIT_NOT_CONST);
            sp.p[0] = 64;
            set_folds(sp);
            add(sp);
            break;
        }
        case GTSC_RLE: {
            BItem h = base_item(nd, B_RLE_HEADS, nd.split_tiles);
            h.order = (int16_t)native_order(nd.dt);
            h.p[0] = 64;
            h.p[1] = nd.starts_off;
            add(h);
            BItem l = h;
            l.op = B_RLE_LENGTHS;
            add(l);
            break;
        }
        case GTSC_FLOAT_TO_INT: {
            BItem s1 = base_item(nd, B_F2I_STATS, t2k);
            s1.order = (int16_t)native_order(nd.dt);
            add(s1);
            BItem s2 = s1;
            s2.op = B_F2I_ENC;
            add(s2);
            BItem s3 = s1;
            s3.op = B_F2I_RAW;
            add(s3);
            break;
        }
        case GTSC_GFC:
            if (is_fp(nd.dt)) {
                BItem g = base_item(nd, B_GFC_COMPRESS, cdiv(nd.gfc_warps, kBGfcChunks));
                g.p[0] = 64;
                g.p[1] = nd.g_sizes;
                g.p[2] = nd.g_incl;
                g.p[3] = nd.g_layout;
                add(g);
                BItem sc = g;
                sc.op = B_GFC_SCAN;
                sc.mode = 0;
                sc.tiles = (uint32_t)std::max<uint64_t>(1, cdiv(nd.gfc_warps, kBTile));
                add(sc);
                BItem cp = g;
                cp.op = B_GFC_COMPACT;
                add(cp);
            } else {
                BItem pk = base_item(nd, B_AFL_PACK, t2k);
                if (scale_view) pk.vflags |= 1;
                else if (!folded_minmax((int)id)) add(minmax_item(nd, n));
                add(pk);
            }
            break;
        default: break;
        }
        int lvl = start;
        for (auto &it : ps) pass_c.push_back(Pass{lvl++, it.op, (int)id, it});
        nd.last_c_level = ps.empty() ? start - 1 : lvl - 1;
    }

    // ---------------- decode passes (children before parents)
    std::vector<int> order(nodes.size());
    for (size_t i = 0; i < nodes.size(); i++) order[i] = (int)i;
    // post-order by depth: process nodes with larger ids first works for pre-order trees
    std::reverse(order.begin(), order.end());
    for (int id : order) {
        HNode &nd = nodes[id];
        int start = 0;
        for (int kid : nd.kids) start = std::max(start, nodes[kid].d_ready);
        // how the parent will read this node's decoded output
        nd.dview = DView{};
        nd.dview.data = nd.enc == GTSC_NONE ? nd.dec_data_sid : nd.dec_out_sid;
        if (nd.parent >= 0) {
            const HNode &par = nodes[nd.parent];
            const int slot = (int)(std::find(par.kids.begin(), par.kids.end(), id) - par.kids.begin()) + 1;
            const bool consumer = par.enc == GTSC_DELTA || par.enc == GTSC_SCALE || par.enc == GTSC_PATCH ||
                                  par.enc == GTSC_PATCH_OUTSIDE ||
                                  par.enc == GTSC_CONST || par.enc == GTSC_RLE || par.enc == GTSC_FLOAT_TO_INT ||
                                  (par.enc == GTSC_DICT && slot == 2);
            if (consumer && nd.enc == GTSC_AFL && nd.kids.size() == 1 && nodes[nd.kids[0]].enc == GTSC_NONE) {
                nd.dvirt = true;
                nd.dview.data = nodes[nd.kids[0]].dec_data_sid;
                nd.dview.afl_meta = nd.dec_meta_sid;
            } else if (consumer && nd.enc == GTSC_SCALE && nd.kids.size() == 1 && nodes[nd.kids[0]].dview.add[1] < 0) {
                nd.dvirt = true;
                nd.dview = nodes[nd.kids[0]].dview;
                nd.dview.add[nd.dview.add[0] < 0 ? 0 : 1] = nd.dec_meta_sid;
            }
        }
        if (nd.dvirt) {
            streams[nd.dec_out_sid].cap = 0;  // never written
            nd.d_ready = start;
            nd.last_d_level = start - 1;
            continue;
        }
        const uint64_t n = nd.in_cap / nd.es;
        const uint64_t t2k = std::max<uint64_t>(1, cdiv(n, kBTile));
        auto child_out = [&](int j) {
            const int kid = nd.kids[j];
            return nodes[kid].enc == GTSC_NONE ? nodes[kid].dec_data_sid : nodes[kid].dec_out_sid;
        };
        auto ditem = [&](int op, uint64_t tiles) {
            BItem it{};
            it.op = (int16_t)op;
            it.es = (int16_t)nd.es;
            it.order = (int16_t)native_order(nd.dt);
            it.dt = nd.dt;
            it.tiles = (uint32_t)std::max<uint64_t>(1, tiles);
            for (int j = 0; j < 3; j++) it.in[j] = it.out[j] = -1;
            it.in[0] = nd.dec_meta_sid;
            for (size_t j = 0; j < nd.kids.size() && j < 2; j++) it.in[j + 1] = child_out((int)j);
            it.out[0] = nd.dec_out_sid;
            // the passes that read their children element-wise take them through DViews
            if (op == B_DELTA_DEC || op == B_SCALE_ADD || op == B_MERGE || op == B_RLE_SCAN || op == B_RLE_EXPAND ||
                op == B_F2I_DEC)
                for (size_t j = 0; j < nd.kids.size() && j < 2; j++) it.dv[j] = nodes[nd.kids[j]].dview;
            return it;
        };
        std::vector<BItem> ps;
        switch (nd.enc) {
        case GTSC_NONE:
            if (nd.parent < 0) {  // a lone none root: copy the data out
                BItem it = ditem(B_NONE_COPY, cdiv(nd.in_cap, batch_copy_piece()));
                it.in[0] = nd.dec_data_sid;
                ps.push_back(it);
            }
            break;
        case GTSC_AFL: ps.push_back(ditem(B_AFL_UNPACK, t2k)); break;
        case GTSC_DELTA: { BItem it = ditem(B_DELTA_DEC, t2k); it.p[0] = nd.dlb_off; ps.push_back(it); break; }
        case GTSC_SCALE: ps.push_back(ditem(B_SCALE_ADD, t2k)); break;
        case GTSC_PATCH: case GTSC_PATCH_OUTSIDE: case GTSC_DICT: case GTSC_CONST: {
            BItem it = ditem(B_MERGE, cdiv(t2k, kBMergeSub));
            it.mode = (int16_t)(nd.enc == GTSC_PATCH || nd.enc == GTSC_PATCH_OUTSIDE ? SPLIT_LOWER : nd.enc == GTSC_DICT ? SPLIT_DICT : SPLIT_NOT_CONST);
            it.p[0] = nd.dlb_off;
            it.p[1] = t2k;
            // the stencil counts need only the node's metadata, parsed before the first level: one
            // launch ahead of every level (a merge may itself run at level 0)
            BItem cnt = it;
            cnt.op = B_MERGE_COUNT;
            cnt.tiles = (uint32_t)t2k;
            pass_d.push_back(Pass{-1, B_MERGE_COUNT, id, cnt});
            ps.push_back(it);
            break;
        }
        case GTSC_RLE: {
            BItem it = ditem(B_RLE_SCAN, t2k);
            it.p[0] = nd.dlb_off;
            it.p[1] = nd.dends_off;
            it.p[2] = nd.druns_off;
            it.p[3] = nd.dtiles_off;
            ps.push_back(it);
            BItem ex = it;
            ex.op = B_RLE_EXPAND;
            ps.push_back(ex);
            break;
        }
        case GTSC_FLOAT_TO_INT: ps.push_back(ditem(B_F2I_DEC, t2k)); break;
        case GTSC_GFC:
            if (is_fp(nd.dt)) {
                const uint64_t st = std::max<uint64_t>(1, cdiv(nd.gfc_warps, kBTile));
                BItem a = ditem(B_GFC_SIZES, st);
                a.p[0] = nd.dlb_off;
                a.p[1] = nd.dsizes_off;
                a.p[2] = nd.dincl_off;
                a.p[3] = nd.gfc_warps;
                ps.push_back(a);
                BItem b = a;
                b.op = B_GFC_SCAN;
                b.mode = 1;
                ps.push_back(b);
                BItem c = a;
                c.op = B_GFC_DEC;
                c.tiles = (uint32_t)std::max<uint64_t>(1, cdiv(nd.gfc_warps, kBGfcChunks));
                ps.push_back(c);
            } else {
                ps.push_back(ditem(B_AFL_UNPACK, t2k));
            }
            break;
        default: break;
        }
        int lvl = start;
        for (auto &it : ps) pass_d.push_back(Pass{lvl++, it.op, id, it});
        nd.last_d_level = ps.empty() ? start - 1 : lvl - 1;
        nd.d_ready = nd.enc == GTSC_NONE ? 0 : nd.last_d_level + 1;
    }
}

void BatchEngine::layout(cudaStream_t s)
{
    // arena: node scratch, then streams
    uint64_t off = 0;
    for (auto &nd : nodes) {
        nd.scratch = off;
        off += nd.c_bytes + nd.d_bytes;
    }
    std::vector<uint64_t> sid_off(streams.size(), UINT64_MAX);
    for (size_t i = 0; i < streams.size(); i++) {
        if (streams[i].cap == 0) continue;
        sid_off[i] = off;
        off += align_up(streams[i].cap + 64, 256);
    }
    framed_cap = 8 + 8 * (uint64_t)col_root.size();  // column count and directory
    for (auto &nd : nodes) {
        framed_cap += 16;
        if (nd.enc != GTSC_NONE) framed_cap += streams[nd.out_sid[0]].cap;
        else framed_cap += nd.in_cap;
    }
    const uint64_t framed_off = off;
    off += align_up(framed_cap + 64, 256);
    arena = dev_alloc(off, s);
    GTSC_CUDA(cudaMemsetAsync(arena.get(), 0, off, s));
    uint8_t *A = arena.get();
    d_framed = A + framed_off;
    for (size_t i = 0; i < streams.size(); i++)
        if (sid_off[i] != UINT64_MAX) streams[i].ptr = A + sid_off[i];
    for (size_t c = 0; c < col_root.size(); c++) {
        streams[col_in_sid[c]].len = col_bytes[c];
        streams[col_out_sid[c]].cap = col_bytes[c];
    }
    // hash tables start empty: keys all ones
    for (auto &nd : nodes)
        if (nd.tab_cap) {
            GTSC_CUDA(cudaMemsetAsync(A + nd.scratch + nd.tab_off + 16, 0xff, 8 * nd.tab_cap, s));
        }

    // items: patch scratch offsets into device addresses, group into launches
    auto build = [&](std::vector<Pass> &ps, std::vector<BItem> &items, std::vector<Launch> &launches,
                     std::vector<int> &item_col) {
        std::stable_sort(ps.begin(), ps.end(), [](const Pass &a, const Pass &b) {
            return std::make_tuple(a.level, a.op) < std::make_tuple(b.level, b.op);
        });
        for (size_t i = 0; i < ps.size();) {
            size_t j = i;
            Launch L{ps[i].op, (int)items.size(), 0, 0, 0, ps[i].level};
            while (j < ps.size() && ps[j].level == ps[i].level && ps[j].op == ps[i].op) {
                BItem it = ps[j].item;
                it.scratch = A + nodes[ps[j].node].scratch;
                if (ps[j].op == B_SPLIT)  // the children whose min / max the split accumulates
                    for (int q = 2; q < 4; q++)
                        it.p[q] = it.p[q] ? (uint64_t)(uintptr_t)(A + nodes[it.p[q] - 1].scratch) : 0;
                if (ps[j].op < B_NONE_COPY || ps[j].op == B_VMETA)  // compress passes: the view's scale nodes
                    for (int v = 0; v < kMaxViewOps; v++) {
                        const int sn = nodes[ps[j].node].vnode[v];
                        it.vscr[v] = sn >= 0 ? A + nodes[sn].scratch : nullptr;
                    }
                it.tile_base = L.tiles;
                L.tiles += it.tiles;
                items.push_back(it);
                item_col.push_back(nodes[ps[j].node].col);
                j++;
            }
            L.count = (int)items.size() - L.first;
            L.map_off = item_of.size();
            for (int k = 0; k < L.count; k++) item_of.insert(item_of.end(), items[L.first + k].tiles, (uint32_t)k);
            if (dyn_pass(L.op)) {
                // claim order: tile j of every item before tile j + 1 of any, so the tiles in flight
                // spread over the items' look-back chains instead of queueing on one
                std::vector<int> live(L.count);
                for (int k = 0; k < L.count; k++) live[k] = k;
                for (uint32_t j = 0; !live.empty(); j++) {
                    size_t w = 0;
                    for (int k : live) {
                        const BItem &b = items[L.first + k];
                        if (j < b.tiles) {
                            item_of.push_back((uint32_t)(b.tile_base + j));
                            live[w++] = k;
                        }
                    }
                    live.resize(w);
                }
            }
            launches.push_back(L);
            i = j;
        }
    };
    build(pass_c, items_c, launch_c, item_col_c);
    build(pass_d, items_d, launch_d, item_col_d);
    plan_persistent(launch_c, items_c, item_col_c, punit_c, pitem_c, q_total_c);
    plan_persistent(launch_d, items_d, item_col_d, punit_d, pitem_d, q_total_d);

    // zero ranges per step
    auto zr = [](std::vector<unsigned long long> &z, uint8_t *p, uint64_t bytes) {
        z.push_back((unsigned long long)(uintptr_t)p);
        z.push_back(align_up(bytes, 4));
    };
    for (auto &nd : nodes) {
        uint8_t *sc = A + nd.scratch;
        zr(zero_c, sc, 64);
        if (nd.enc == GTSC_FLOAT_TO_INT) zr(zero_c, sc + 64, 64);
        if (nd.split_tiles) zr(zero_c, sc + 64, lookback_zero_bytes(nd.split_tiles));
        if (nd.gfc_warps) zr(zero_c, sc + 64, lookback_zero_bytes(std::max<uint64_t>(1, cdiv(nd.gfc_warps, kBTile))));
        const uint64_t n = nd.in_cap / nd.es;
        const uint64_t t2k = std::max<uint64_t>(1, cdiv(n, kBTile));
        switch (nd.enc) {
        case GTSC_DELTA: case GTSC_PATCH: case GTSC_PATCH_OUTSIDE: case GTSC_DICT: case GTSC_CONST: case GTSC_RLE:
            zr(zero_d, sc + nd.dlb_off, lookback_zero_bytes(t2k));
            break;
        case GTSC_GFC:
            if (nd.gfc_warps) zr(zero_d, sc + nd.dlb_off, lookback_zero_bytes(std::max<uint64_t>(1, cdiv(nd.gfc_warps, kBTile))));
            break;
        default: break;
        }
    }

    // framing tables
    for (size_t c = 0; c < col_root.size(); c++) {
        BColumnDev cd;
        cd.first = (int)nodes_c.size();
        int cnt = 0;
        for (size_t id = 0; id < nodes.size(); id++) {
            if (nodes[id].col != (int)c) continue;
            const HNode &nd = nodes[id];
            const int henc = nd.enc == GTSC_PATCH_OUTSIDE ? GTSC_PATCH : nd.enc;  // the serialised type
            BNodeDev a{henc, nd.dt, nd.enc == GTSC_NONE ? -1 : nd.out_sid[0], nd.enc == GTSC_NONE ? nd.in_sid : -1, 0, 0};
            BNodeDev b{henc, nd.dt, nd.dec_meta_sid, nd.dec_data_sid, 0, 0};
            nodes_c.push_back(a);
            nodes_d.push_back(b);
            cnt++;
        }
        cd.n_nodes = cnt;
        cols_dev.push_back(cd);
    }
    // copy items: every metadata and every none leaf's data
    for (size_t k = 0; k < nodes_c.size(); k++) {
        const BNodeDev &nd = nodes_c[k];
        for (int which = 0; which < 2; which++) {
            const int sid = which ? nd.data : nd.meta;
            if (sid < 0) continue;
            // a lone none root copies the caller's column: an external stream with no arena capacity
            const uint64_t cap = std::max(streams[sid].cap, streams[sid].len);
            BItem it{};
            it.tiles = (uint32_t)std::max<uint64_t>(1, cdiv(cap, batch_copy_piece()));
            it.tile_base = copy_tiles;
            it.p[0] = k;
            it.p[1] = (uint64_t)which;
            copy_tiles += it.tiles;
            items_copy.push_back(it);
        }
    }
    copy_map_off = item_of.size();
    for (size_t k = 0; k < items_copy.size(); k++) item_of.insert(item_of.end(), items_copy[k].tiles, (uint32_t)k);
    // counters: one per launch
    n_counters = (int)(launch_c.size() + launch_d.size()) + 4;

    // device tables in one allocation
    auto sz = [](size_t n, size_t e) { return align_up(n * e + 16, 256); };
    uint64_t t_off = 0;
    const uint64_t o_streams = t_off; t_off += sz(streams.size(), sizeof(StreamDesc));
    const uint64_t o_ic = t_off; t_off += sz(items_c.size(), sizeof(BItem));
    const uint64_t o_id = t_off; t_off += sz(items_d.size(), sizeof(BItem));
    const uint64_t o_icp = t_off; t_off += sz(items_copy.size(), sizeof(BItem));
    const uint64_t o_cols = t_off; t_off += sz(cols_dev.size(), sizeof(BColumnDev));
    const uint64_t o_nc = t_off; t_off += sz(nodes_c.size(), sizeof(BNodeDev));
    const uint64_t o_nd = t_off; t_off += sz(nodes_d.size(), sizeof(BNodeDev));
    const uint64_t o_coloff = t_off; t_off += sz(col_root.size() + 1, 8);
    const uint64_t o_coloff_d = t_off; t_off += sz(col_root.size() + 1, 8);
    const uint64_t o_total = t_off; t_off += 256;
    const uint64_t o_zc = t_off; t_off += sz(zero_c.size() + 8, 8);
    const uint64_t o_zd = t_off; t_off += sz(zero_d.size() + 8, 8);
    // (pointer, length) pairs: the inputs of compress, then the outputs of decompress
    const uint64_t o_setv = t_off; t_off += sz(4 * col_root.size() + 2, 8);
    const uint64_t o_sets = t_off; t_off += sz(2 * col_root.size() + 2, 4);
    const uint64_t o_frame = t_off; t_off += 256;
    const uint64_t o_status = t_off; t_off += 256;
    const uint64_t o_counters = t_off; t_off += sz(n_counters, 4);
    const uint64_t o_item_of = t_off; t_off += sz(item_of.size(), 4);
    const uint64_t ncol = col_root.size();
    const uint64_t o_plc = t_off; t_off += sz(punit_c.size(), sizeof(PUnit));
    const uint64_t o_pld = t_off; t_off += sz(punit_d.size(), sizeof(PUnit));
    const uint64_t o_pic = t_off; t_off += sz(pitem_c.size(), sizeof(PItem));
    const uint64_t o_pid = t_off; t_off += sz(pitem_d.size(), sizeof(PItem));
    const uint64_t o_done_c = t_off; t_off += sz(ncol, 4);
    const uint64_t o_done_d = t_off; t_off += sz(ncol, 4);
    const uint64_t o_ext_c = t_off; t_off += sz(items_c.size(), 4);
    const uint64_t o_ext_d = t_off; t_off += sz(items_d.size(), 4);
    const uint64_t o_queue = t_off; t_off += 256;
    tables = dev_alloc(t_off, s);
    uint8_t *T = tables.get();
    GTSC_CUDA(cudaMemsetAsync(T, 0, t_off, s));
    d_streams = (StreamDesc *)(T + o_streams);
    d_items_c = (BItem *)(T + o_ic);
    d_items_d = (BItem *)(T + o_id);
    d_items_copy = (BItem *)(T + o_icp);
    d_cols = (BColumnDev *)(T + o_cols);
    d_nodes_c = (BNodeDev *)(T + o_nc);
    d_nodes_d = (BNodeDev *)(T + o_nd);
    d_col_off = (unsigned long long *)(T + o_coloff);
    d_col_off_d = (unsigned long long *)(T + o_coloff_d);
    d_total = (unsigned long long *)(T + o_total);
    d_zero_c = (unsigned long long *)(T + o_zc);
    d_zero_d = (unsigned long long *)(T + o_zd);
    d_set_vals = (unsigned long long *)(T + o_setv);
    d_set_sids = (int *)(T + o_sets);
    d_frame_ptr = (uint8_t **)(T + o_frame);
    d_frame_len = (unsigned long long *)(T + o_frame + 8);
    d_status = (uint32_t *)(T + o_status);
    d_counters = (uint32_t *)(T + o_counters);
    d_item_of = (uint32_t *)(T + o_item_of);
    d_punit_c = (PUnit *)(T + o_plc);
    d_punit_d = (PUnit *)(T + o_pld);
    d_pitem_c = (PItem *)(T + o_pic);
    d_pitem_d = (PItem *)(T + o_pid);
    d_done_c = (uint32_t *)(T + o_done_c);
    d_done_d = (uint32_t *)(T + o_done_d);
    d_ext_c = (uint32_t *)(T + o_ext_c);
    d_ext_d = (uint32_t *)(T + o_ext_d);
    d_queue = (uint32_t *)(T + o_queue);
    // the status word and the counters are zeroed with the other ranges at each step
    zr(zero_c, (uint8_t *)d_status, 8);   // [0] error code, [1] decode: the frames did not parse
    zr(zero_d, (uint8_t *)d_status, 8);
    zr(zero_c, (uint8_t *)d_counters, 4ull * n_counters);
    zr(zero_d, (uint8_t *)d_counters, 4ull * n_counters);
    // the persistent schedule's per-column progress, extent cache and claim counters
    zr(zero_c, (uint8_t *)d_done_c, 4 * ncol);
    zr(zero_d, (uint8_t *)d_done_d, 4 * ncol);
    zr(zero_c, (uint8_t *)d_ext_c, 4 * std::max<uint64_t>(items_c.size(), 1));
    zr(zero_d, (uint8_t *)d_ext_d, 4 * std::max<uint64_t>(items_d.size(), 1));
    zr(zero_c, (uint8_t *)d_queue, 4);
    zr(zero_d, (uint8_t *)(d_queue + 1), 4);
    auto h2d = [&](void *dst, const void *src, size_t bytes) {
        if (bytes) GTSC_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    };
    h2d(d_streams, streams.data(), streams.size() * sizeof(StreamDesc));
    h2d(d_items_c, items_c.data(), items_c.size() * sizeof(BItem));
    h2d(d_items_d, items_d.data(), items_d.size() * sizeof(BItem));
    h2d(d_items_copy, items_copy.data(), items_copy.size() * sizeof(BItem));
    h2d(d_cols, cols_dev.data(), cols_dev.size() * sizeof(BColumnDev));
    h2d(d_nodes_c, nodes_c.data(), nodes_c.size() * sizeof(BNodeDev));
    h2d(d_nodes_d, nodes_d.data(), nodes_d.size() * sizeof(BNodeDev));
    h2d(d_zero_c, zero_c.data(), zero_c.size() * 8);
    h2d(d_zero_d, zero_d.data(), zero_d.size() * 8);
    h2d(d_item_of, item_of.data(), item_of.size() * 4);
    h2d(d_punit_c, punit_c.data(), punit_c.size() * sizeof(PUnit));
    h2d(d_punit_d, punit_d.data(), punit_d.size() * sizeof(PUnit));
    h2d(d_pitem_c, pitem_c.data(), pitem_c.size() * sizeof(PItem));
    h2d(d_pitem_d, pitem_d.data(), pitem_d.size() * sizeof(PItem));
    GTSC_CUDA(cudaStreamSynchronize(s));
}

// The persistent schedule of one phase (batch.hpp, PUnit): the level launches end to end as one
// queue of units, and per item its column and the number of that column's tiles in earlier levels.
void BatchEngine::plan_persistent(const std::vector<Launch> &launches, const std::vector<BItem> &items,
                                  const std::vector<int> &item_col, std::vector<PUnit> &units,
                                  std::vector<PItem> &pi, uint32_t &total)
{
    static_assert(kPersistChunk <= 15, "a unit's tile count has four bits");
    const size_t nc = col_root.size();
    std::vector<uint64_t> tot(nc, 0), before(nc, 0);  // tiles so far / in the earlier levels
    pi.assign(items.size(), PItem{0, 0});
    units.clear();
    int level = INT32_MIN;
    for (const Launch &L : launches) {
        if (L.level != level) {  // launches are sorted by level
            before = tot;
            level = L.level;
        }
        for (int k = L.first; k < L.first + L.count; k++) {
            const int c = item_col[k];
            if (before[c] > 0xffffffffull) fail(GTSC_ERR_CAPACITY, "batch: too many tiles for the persistent schedule");
            pi[k] = PItem{(uint32_t)c, (uint32_t)before[c]};
            tot[c] += items[k].tiles;
        }
        const bool dyn = dyn_pass(L.op);
        const uint32_t per = dyn ? 1u : kPersistChunk;
        for (uint64_t t = 0; t < L.tiles; t += per) {
            // the unit's first tile: look-back passes in the launch's claim order (item_of after its
            // tile table), the others in tile order
            const uint64_t tt = dyn ? item_of[L.map_off + L.tiles + t] : t;
            const int gi = L.first + (int)item_of[L.map_off + tt];
            const uint64_t tile = tt - items[gi].tile_base;
            const uint32_t cnt = (uint32_t)std::min<uint64_t>(per, L.tiles - t);
            if (tile >= (1u << 28)) fail(GTSC_ERR_CAPACITY, "batch: an item has too many tiles for the persistent schedule");
            units.push_back(PUnit{(uint32_t)gi, (uint32_t)tile | (cnt << 28)});
        }
    }
    if (units.size() >= 0xffffffffull) fail(GTSC_ERR_CAPACITY, "batch: too many tiles for the persistent schedule");
    total = (uint32_t)units.size();
}

PersistArgs BatchEngine::persist_args(bool compress) const
{
    PersistArgs a;
    a.units = compress ? d_punit_c : d_punit_d;
    a.total = compress ? q_total_c : q_total_d;
    a.items = compress ? d_items_c : d_items_d;
    a.pitems = compress ? d_pitem_c : d_pitem_d;
    a.done = compress ? d_done_c : d_done_d;
    a.ext = compress ? d_ext_c : d_ext_d;
    a.qcounter = d_queue + (compress ? 0 : 1);
    a.S = d_streams;
    a.status = d_status;
    return a;
}

// Launch-sequence markers: the stage op, or one of these for the fixed kernels of a step.
enum : int { M_SET = -1, M_ZERO = -2, M_FRAME_SIZES = -3, M_FRAME_LAYOUT = -4, M_FRAME_COPY = -5, M_PARSE = -6,
             M_PERSIST = -7 };

void BatchEngine::record_compress(cudaStream_t s, const std::function<void(int)> &mark, bool pers)
{
    const int nc = (int)col_root.size();
    k_set_streams<<<(nc + 127) / 128, 128, 0, s>>>(d_set_vals, d_set_sids, nc, d_streams);
    GTSC_CUDA(cudaGetLastError());
    mark(M_SET);
    launch_zero_ranges(d_zero_c, (int)zero_c.size() / 2, s);
    mark(M_ZERO);
    if (pers) {
        launch_batch_persistent_c(persist_args(true), s);
        mark(M_PERSIST);
    } else {
        int ctr = 0;
        for (auto &L : launch_c) {
            launch_batch_stage(L.op, d_items_c + L.first, d_item_of + L.map_off, L.count, L.tiles, d_streams,
                               d_counters + ctr++, d_status, s);
            mark(L.op);
        }
    }
    launch_frame_sizes(d_cols, nc, d_nodes_c, d_streams, d_col_off, d_total, d_framed, s);
    mark(M_FRAME_SIZES);
    launch_frame_layout(d_cols, nc, d_nodes_c, d_streams, d_col_off, d_framed, s);
    mark(M_FRAME_LAYOUT);
    launch_frame_copy(d_items_copy, d_item_of + copy_map_off, (int)items_copy.size(), copy_tiles, d_nodes_c, d_streams,
                      d_framed, s);
    mark(M_FRAME_COPY);
}

void BatchEngine::record_decompress(cudaStream_t s, const std::function<void(int)> &mark, bool pers)
{
    const int nc = (int)col_root.size();
    k_set_streams<<<(nc + 127) / 128, 128, 0, s>>>(d_set_vals + 2 * nc, d_set_sids + nc, nc, d_streams);
    GTSC_CUDA(cudaGetLastError());
    mark(M_SET);
    launch_zero_ranges(d_zero_d, (int)zero_d.size() / 2, s);
    mark(M_ZERO);
    launch_parse_frames(d_cols, nc, d_nodes_d, d_streams, d_col_off_d, (const uint8_t *const *)d_frame_ptr,
                        d_frame_len, d_status, s);
    mark(M_PARSE);
    if (pers) {
        launch_batch_persistent_d(persist_args(false), s);
        mark(M_PERSIST);
        return;
    }
    int ctr = (int)launch_c.size();
    for (auto &L : launch_d) {
        launch_batch_stage(L.op, d_items_d + L.first, d_item_of + L.map_off, L.count, L.tiles, d_streams,
                           d_counters + ctr++, d_status, s);
        mark(L.op);
    }
}

void BatchEngine::capture(cudaStream_t s)
{
    for (int which = 0; which < 4; which++) {
        const bool comp = which % 2 == 0, pers = which >= 2;
        cudaGraph_t g;
        GTSC_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        try {
            if (comp) record_compress(s, [](int) {}, pers);
            else record_decompress(s, [](int) {}, pers);
        } catch (...) {
            cudaGraph_t junk;
            cudaStreamEndCapture(s, &junk);
            if (junk) cudaGraphDestroy(junk);
            throw;
        }
        GTSC_CUDA(cudaStreamEndCapture(s, &g));
        cudaGraphExec_t ex;
        GTSC_CUDA(cudaGraphInstantiate(&ex, g, 0));
        cudaGraphDestroy(g);
        (comp ? graph_c : graph_d)[pers ? 1 : 0] = ex;
    }
}

// ---------------------------------------------------------------------------------- public

BatchEngine *batch_create(const std::vector<BatchColumn> &cols, const std::vector<Tree> &trees, cudaStream_t s,
                          const BatchTuning &tuning)
{
    if (cols.empty() || cols.size() != trees.size()) fail(GTSC_ERR_ARG, "batch: columns and trees differ in number");
    if (!s) fail(GTSC_ERR_ARG, "batch: needs a non-default stream (steps are captured as CUDA graphs)");
    if (cols.size() >= (1u << 24)) fail(GTSC_ERR_ARG, "batch: at most 2^24 - 1 columns");
    for (const auto &c : cols)
        if (!aligned16(c.data)) fail(GTSC_ERR_ARG, "batch: column pointers must be 16-byte aligned");
    if (tuning.minmax_vpt != 1 && tuning.minmax_vpt != 2 && tuning.minmax_vpt != 4 && tuning.minmax_vpt != 8 &&
        tuning.minmax_vpt != 16)
        fail(GTSC_ERR_ARG, "batch: min/max values per thread must be 1, 2, 4, 8 or 16");
    if (tuning.minmax_tile < kMinMaxTileMin || tuning.minmax_tile % (256 * tuning.minmax_vpt) ||
        tuning.minmax_tile > (1u << 20))
        fail(GTSC_ERR_ARG, "batch: the min/max tile must be a multiple of 256 x its values per thread, 1K .. 1M");
    if (tuning.hist_tile < 256 || tuning.hist_tile % 256 || tuning.hist_tile > kBHistTileMax)
        fail(GTSC_ERR_ARG, "batch: the histogram tile must be a multiple of 256");
    std::unique_ptr<BatchEngine> e(new BatchEngine());
    e->tune = tuning;
    e->src_cols = cols;
    e->src_trees = trees;
    for (size_t c = 0; c < cols.size(); c++) {
        const Tree &t = trees[c];
        if (t.size() == 0 || t.dt[0] != cols[c].dtype) fail(GTSC_ERR_ARG, "batch: tree root type differs from the column");
        const int in_sid = e->new_stream(0);
        const int out_sid = e->new_stream(0);
        e->col_in_sid.push_back(in_sid);
        e->col_out_sid.push_back(out_sid);
        e->col_bytes.push_back(cols[c].bytes);
        e->col_root.push_back((int)e->nodes.size());
        int k = 0;
        e->build_node(t, k, (int)c, -1, in_sid, cols[c].bytes, 0, nullptr, nullptr);
        if (k != t.size()) fail(GTSC_ERR_ARG, "batch: extra nodes in tree");
        e->nodes[e->col_root.back()].dec_out_sid = out_sid;
    }
    e->plan_passes();
    e->layout(s);
    // column inputs
    std::vector<unsigned long long> vals;
    std::vector<int> sids;
    for (size_t c = 0; c < cols.size(); c++) {
        vals.push_back((unsigned long long)(uintptr_t)cols[c].data);
        vals.push_back(cols[c].bytes);
        sids.push_back(e->col_in_sid[c]);
    }
    for (size_t c = 0; c < cols.size(); c++) sids.push_back(e->col_out_sid[c]);
    GTSC_CUDA(cudaMemcpyAsync(e->d_set_vals, vals.data(), vals.size() * 8, cudaMemcpyHostToDevice, s));
    GTSC_CUDA(cudaMemcpyAsync(e->d_set_sids, sids.data(), sids.size() * 4, cudaMemcpyHostToDevice, s));
    GTSC_CUDA(cudaStreamSynchronize(s));
    e->capture(s);
    return e.release();
}

void batch_destroy(BatchEngine *e)
{
    if (!e) return;
    // the arena was allocated on the caller's stream, which may already be gone: finish all work,
    // then release on the legacy stream
    cudaDeviceSynchronize();
    e->arena.release_on_default_stream();
    e->tables.release_on_default_stream();
    for (int k = 0; k < 2; k++) {
        if (e->graph_c[k]) cudaGraphExecDestroy(e->graph_c[k]);
        if (e->graph_d[k]) cudaGraphExecDestroy(e->graph_d[k]);
    }
    delete e;
}

void batch_compress(BatchEngine *e, cudaStream_t s) { GTSC_CUDA(cudaGraphLaunch(e->graph_c[e->tune.persistent_c], s)); }

void batch_set_schedule(BatchEngine *e, bool persistent) { e->tune.persistent_c = e->tune.persistent_d = persistent; }
bool batch_schedule(const BatchEngine *e) { return e->tune.persistent_c && e->tune.persistent_d; }
BatchTuning batch_tuning(const BatchEngine *e) { return e->tune; }

void batch_set_inputs(BatchEngine *e, const std::vector<const void *> &inputs, cudaStream_t s)
{
    const size_t nc = e->col_root.size();
    if (inputs.size() != nc) fail(GTSC_ERR_ARG, "batch: one input per column");
    for (const void *p : inputs)
        if (!aligned16(p)) fail(GTSC_ERR_ARG, "batch: column pointers must be 16-byte aligned");
    std::vector<unsigned long long> vals;
    for (size_t c = 0; c < nc; c++) {
        vals.push_back((unsigned long long)(uintptr_t)inputs[c]);
        vals.push_back(e->col_bytes[c]);
    }
    GTSC_CUDA(cudaMemcpyAsync(e->d_set_vals, vals.data(), vals.size() * 8, cudaMemcpyHostToDevice, s));
    for (size_t c = 0; c < nc; c++) e->src_cols[c].data = inputs[c];
}

uint64_t batch_output_bytes(BatchEngine *e, cudaStream_t s)
{
    unsigned long long t = 0;
    d2h(&t, e->d_total, 8, s);
    return t;
}

const uint8_t *batch_output(BatchEngine *e) { return e->d_framed; }

std::vector<uint64_t> batch_blob_sizes(BatchEngine *e, cudaStream_t s)
{
    const size_t nc = e->col_root.size();
    std::vector<uint64_t> r(nc);
    d2h(r.data(), e->d_framed + 8, 8 * nc, s);  // the directory of the framed output
    return r;
}

void batch_decompress(BatchEngine *e, const uint8_t *framed, uint64_t framed_bytes, const std::vector<void *> &outputs,
                      cudaStream_t s)
{
    const size_t nc = e->col_root.size();
    if (outputs.size() != nc) fail(GTSC_ERR_ARG, "batch: one output per column");
    for (const void *p : outputs)
        if (!aligned16(p)) fail(GTSC_ERR_ARG, "batch: output pointers must be 16-byte aligned");
    std::vector<unsigned long long> vals;
    for (size_t c = 0; c < nc; c++) {
        vals.push_back((unsigned long long)(uintptr_t)outputs[c]);
        vals.push_back(0);
    }
    GTSC_CUDA(cudaMemcpyAsync(e->d_set_vals + 2 * nc, vals.data(), vals.size() * 8, cudaMemcpyHostToDevice, s));
    unsigned long long fr[2] = {(unsigned long long)(uintptr_t)framed, framed_bytes};
    GTSC_CUDA(cudaMemcpyAsync(e->d_frame_ptr, fr, 16, cudaMemcpyHostToDevice, s));
    GTSC_CUDA(cudaGraphLaunch(e->graph_d[e->tune.persistent_d], s));
}

// Bytes a pass must move at least: its inputs read and its outputs written (from the stream table
// after the step).  Scratch, look-back state and hash tables are not counted.
static uint64_t item_bytes(const BItem &it, const std::vector<StreamDesc> &S)
{
    auto L = [&](int sid) -> uint64_t { return sid >= 0 ? S[sid].len : 0; };
    auto D = [&](int slot) -> uint64_t {  // a decode input: its view's source, else the stream
        const DView &d = it.dv[slot - 1];
        return d.data >= 0 ? S[d.data].len : L(it.in[slot]);
    };
    const uint64_t in = L(it.in[0]);
    switch (it.op) {
    case B_MINMAX: case B_HIST: case B_F2I_STATS: return in;
    case B_TOPK: case B_F2I_RAW: case B_GFC_SCAN: return 0;
    case B_DELTA_ENC: case B_SCALE_SUB: case B_AFL_PACK: case B_F2I_ENC: return in + L(it.out[0]) + L(it.out[1]);
    case B_SPLIT: return in + L(it.out[0]) + L(it.out[1]) + L(it.out[2]);
    case B_RLE_HEADS: return in + L(it.out[0]) + L(it.out[2]) + L(it.out[1]);  // values, run starts
    case B_RLE_LENGTHS: return 2 * L(it.out[1]);
    case B_GFC_COMPRESS: return in + L(it.out[1]) + L(it.out[2]);
    case B_GFC_COMPACT: return 2 * L(it.out[2]);
    case B_NONE_COPY: return 2 * in;
    case B_AFL_UNPACK: return L(it.in[1]) + L(it.out[0]);
    case B_DELTA_DEC: case B_SCALE_ADD: case B_F2I_DEC: return D(1) + L(it.out[0]);
    case B_MERGE: return in + (it.mode == SPLIT_DICT ? L(it.in[1]) : D(1)) + D(2) + L(it.out[0]);
    case B_RLE_SCAN: return D(1);
    case B_MERGE_COUNT: return L(it.in[0]);
    case B_RLE_EXPAND: return D(2) + L(it.out[0]);
    case B_GFC_SIZES: return L(it.in[1]);
    case B_GFC_DEC: return L(it.in[2]) + L(it.out[0]);
    default: return 0;
    }
}

std::vector<BatchLaunchProfile> batch_profile(BatchEngine *e, bool compress, cudaStream_t s)
{
    std::vector<int> marks;
    std::vector<cudaEvent_t> ev;
    auto new_event = [&]() {
        cudaEvent_t x;
        GTSC_CUDA(cudaEventCreate(&x));
        ev.push_back(x);
        return x;
    };
    std::vector<BatchLaunchProfile> out;
    try {
        GTSC_CUDA(cudaEventRecord(new_event(), s));
        auto mark = [&](int m) {
            marks.push_back(m);
            GTSC_CUDA(cudaEventRecord(new_event(), s));
        };
        if (compress) e->record_compress(s, mark, e->tune.persistent_c);
        else e->record_decompress(s, mark, e->tune.persistent_d);
        GTSC_CUDA(cudaStreamSynchronize(s));
        std::vector<StreamDesc> S(e->streams.size());
        d2h(S.data(), e->d_streams, S.size() * sizeof(StreamDesc), s);
        unsigned long long total = 0;
        d2h(&total, e->d_total, 8, s);
        int li = 0;
        for (size_t k = 0; k < marks.size(); k++) {
            BatchLaunchProfile p{};
            p.op = marks[k];
            GTSC_CUDA(cudaEventElapsedTime(&p.ms, ev[k], ev[k + 1]));
            if (marks[k] >= 0) {
                const Launch &L = compress ? e->launch_c[li] : e->launch_d[li];
                const BItem *items = compress ? &e->items_c[L.first] : &e->items_d[L.first];
                for (int j = 0; j < L.count; j++) p.bytes += item_bytes(items[j], S);
                p.blocks = L.tiles;
                ++li;
            } else if (marks[k] == M_FRAME_COPY) {
                p.bytes = 2 * total;
                p.blocks = e->copy_tiles;
            } else if (marks[k] == M_PERSIST) {  // every pass of the step in one launch
                for (const BItem &it : compress ? e->items_c : e->items_d) p.bytes += item_bytes(it, S);
                p.blocks = compress ? e->q_total_c : e->q_total_d;
            }
            out.push_back(p);
        }
    } catch (...) {
        for (auto x : ev) cudaEventDestroy(x);
        throw;
    }
    for (auto x : ev) cudaEventDestroy(x);
    return out;
}

// ---------------------------------------------------------------------------------- autotuner

namespace {

using Clock = std::chrono::steady_clock;

// median milliseconds of `reps` steps (after one untimed step), CUDA events on s
float time_step(BatchEngine *e, bool compress, const uint8_t *framed, uint64_t framed_bytes,
                const std::vector<void *> &outs, cudaStream_t s, int reps)
{
    auto one = [&]() {
        if (compress) batch_compress(e, s);
        else batch_decompress(e, framed, framed_bytes, outs, s);
    };
    one();
    std::vector<float> t;
    cudaEvent_t a, b;
    GTSC_CUDA(cudaEventCreate(&a));
    GTSC_CUDA(cudaEventCreate(&b));
    for (int r = 0; r < reps; r++) {
        GTSC_CUDA(cudaEventRecord(a, s));
        one();
        GTSC_CUDA(cudaEventRecord(b, s));
        GTSC_CUDA(cudaEventSynchronize(b));
        float ms = 0;
        GTSC_CUDA(cudaEventElapsedTime(&ms, a, b));
        t.push_back(ms);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    std::sort(t.begin(), t.end());
    return t[t.size() / 2];
}

// the summed time of the compress launches of the given pass kinds (min over `reps` profiles)
float time_passes(BatchEngine *e, std::initializer_list<int> ops, cudaStream_t s, int reps)
{
    float best = 1e30f;
    for (int r = 0; r < reps; r++) {
        float sum = 0;
        for (const auto &p : batch_profile(e, true, s))
            for (int op : ops)
                if (p.op == op) sum += p.ms;
        best = std::min(best, sum);
    }
    return best;
}

}  // namespace

// the min/max tile and values per thread of every min/max item (no rebuild: tiles are reserved for
// the smallest tile)
static void set_minmax_params(BatchEngine *e, uint32_t tile, uint32_t vpt, cudaStream_t s)
{
    for (auto &it : e->items_c)
        if (it.op == B_MINMAX) {
            it.p[0] = tile;
            it.p[1] = vpt;
        }
    GTSC_CUDA(cudaMemcpyAsync(e->d_items_c, e->items_c.data(), e->items_c.size() * sizeof(BItem),
                              cudaMemcpyHostToDevice, s));
    GTSC_CUDA(cudaStreamSynchronize(s));
    e->tune.minmax_tile = tile;
    e->tune.minmax_vpt = vpt;
}

BatchEngine *batch_autotune(BatchEngine *e, cudaStream_t s, TuneReport *report)
{
    const auto t_start = Clock::now();
    TuneReport rep;
    int cands = 0;
    // decode outputs for the timing (one allocation, 256-byte aligned pieces)
    uint64_t out_bytes = 0;
    for (uint64_t b : e->col_bytes) out_bytes += align_up(std::max<uint64_t>(b, 16), 256);
    DevBuf outbuf = dev_alloc(out_bytes, s);
    std::vector<void *> outs;
    uint64_t off = 0;
    for (uint64_t b : e->col_bytes) {
        outs.push_back(outbuf.get() + off);
        off += align_up(std::max<uint64_t>(b, 16), 256);
    }
    auto measure = [&](BatchEngine *x, float ms[2]) {
        batch_compress(x, s);
        const uint64_t fb = batch_output_bytes(x, s);
        ms[0] = time_step(x, true, nullptr, 0, outs, s, 5);
        ms[1] = time_step(x, false, batch_output(x), fb, outs, s, 5);
        if (batch_status(x, s) != GTSC_OK) fail(GTSC_ERR_FORMAT, "autotune: a candidate step failed");
    };
    // 1. the schedule of each step (both recorded in every batch: no rebuild)
    BatchTuning best = e->tune;
    best.persistent_c = best.persistent_d = false;
    e->tune.persistent_c = e->tune.persistent_d = false;
    measure(e, rep.ms_default);
    e->tune.persistent_c = e->tune.persistent_d = true;
    float pers[2];
    measure(e, pers);
    cands += 2;
    best.persistent_c = pers[0] < rep.ms_default[0];
    best.persistent_d = pers[1] < rep.ms_default[1];
    e->tune.persistent_c = best.persistent_c;
    e->tune.persistent_d = best.persistent_d;
    // 2. the min/max tile x values per thread, on the min/max launches of the level schedule
    const bool keep_c = e->tune.persistent_c;
    e->tune.persistent_c = false;
    batch_compress(e, s);
    float best_mm = time_passes(e, {B_MINMAX}, s, 3);
    for (uint32_t tile : {1024u, 2048u, 4096u, 8192u, 16384u})
        for (uint32_t vpt : {1u, 2u, 4u, 8u, 16u}) {
            if (tile % (256 * vpt) || (tile == best.minmax_tile && vpt == best.minmax_vpt)) continue;
            set_minmax_params(e, tile, vpt, s);
            const float t = time_passes(e, {B_MINMAX}, s, 3);
            ++cands;
            if (t < best_mm * 0.98f) {
                best_mm = t;
                best.minmax_tile = tile;
                best.minmax_vpt = vpt;
            }
        }
    set_minmax_params(e, best.minmax_tile, best.minmax_vpt, s);
    e->tune.persistent_c = keep_c;
    // 3. the histogram tile (it sizes the top-k pass's tiles: a rebuild per candidate)
    const bool has_hist = std::any_of(e->items_c.begin(), e->items_c.end(), [](const BItem &it) { return it.op == B_HIST; });
    if (has_hist) {
        e->tune.persistent_c = false;
        float best_h = time_passes(e, {B_HIST, B_TOPK}, s, 3);
        e->tune.persistent_c = keep_c;
        for (uint32_t tile : {8192u, 16384u, 32768u}) {
            if (tile == best.hist_tile) continue;
            BatchTuning cand = best;
            cand.hist_tile = tile;
            cand.persistent_c = false;
            BatchEngine *x = batch_create(e->src_cols, e->src_trees, s, cand);
            float t = 1e30f;
            try {
                batch_compress(x, s);
                t = time_passes(x, {B_HIST, B_TOPK}, s, 3);
            } catch (...) {
                batch_destroy(x);
                throw;
            }
            batch_destroy(x);
            ++cands;
            if (t < best_h * 0.98f) {
                best_h = t;
                best.hist_tile = tile;
            }
        }
    }
    // the tuned batch
    BatchEngine *out = e;
    if (best.hist_tile != e->tune.hist_tile) {
        out = batch_create(e->src_cols, e->src_trees, s, best);
        batch_destroy(e);
    }
    out->tune = best;
    measure(out, rep.ms_tuned);
    rep.best = best;
    rep.candidates = cands;
    rep.seconds = std::chrono::duration<float>(Clock::now() - t_start).count();
    if (report) *report = rep;
    return out;
}

gtsc_status batch_status(BatchEngine *e, cudaStream_t s)
{
    uint32_t w = 0;
    d2h(&w, e->d_status, 4, s);
    return w ? -(gtsc_status)w : GTSC_OK;
}

int batch_launches(BatchEngine *e, bool compress)
{
    // compress: set streams, zero, stages, frame sizes / layout / copy; decompress: set streams,
    // zero, parse directory + frames, stages
    if (compress ? e->tune.persistent_c : e->tune.persistent_d) return compress ? 6 : 4;
    return compress ? (int)e->launch_c.size() + 5 : (int)e->launch_d.size() + 4;
}

}  // namespace gtsc
