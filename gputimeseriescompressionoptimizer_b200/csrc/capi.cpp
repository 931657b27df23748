// capi.cpp -- the extern "C" boundary of libgtsc.  Every entry point converts C++ exceptions into
// gtsc_status codes and records the message for gtsc_last_error().
#include "common.cuh"
#include "encodings.hpp"
#include "kernels.hpp"
#include "batch.hpp"
#include "predict.hpp"
#include "learned.hpp"
#include "optimizer.hpp"
#include "planner.hpp"
#include "tree.hpp"

#include <cstring>
#include <exception>

namespace gtsc {
const std::string &last_error();
}

using namespace gtsc;

namespace {

template <class F>
gtsc_status guard(F &&f)
{
    try {
        set_last_error("");
        f();
        return GTSC_OK;
    } catch (const Error &e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc &) {
        set_last_error("host allocation failed");
        return GTSC_ERR_CAPACITY;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return GTSC_ERR_ARG;
    }
}

inline cudaStream_t S(void *p) { return reinterpret_cast<cudaStream_t>(p); }

// hands a library-owned buffer to the caller, who releases it with gtsc_free
gtsc_buffer release(DevBuf &b)
{
    gtsc_buffer r{b.disown(), b.bytes};
    b.m.reset();
    return r;
}

}  // namespace

extern "C" {

const char *gtsc_last_error(void) { return last_error().c_str(); }

const char *gtsc_version(void) { return "gtsc 0.1 sm_100a"; }

int32_t gtsc_dtype_size(int32_t dtype) { return dtype_size(dtype); }

gtsc_status gtsc_malloc(void **d_ptr, uint64_t bytes, void *stream)
{
    return guard([&] {
        if (!d_ptr) fail(GTSC_ERR_ARG, "null d_ptr");
        *d_ptr = nullptr;
        if (bytes) GTSC_CUDA(cudaMallocAsync(d_ptr, bytes, S(stream)));
    });
}

gtsc_status gtsc_free(void *d_ptr, void *stream)
{
    return guard([&] {
        if (d_ptr) GTSC_CUDA(cudaFreeAsync(d_ptr, S(stream)));
    });
}

gtsc_status gtsc_memcpy(void *dst, const void *src, uint64_t bytes, int32_t kind, void *stream)
{
    return guard([&] {
        if (kind < 1 || kind > 3) fail(GTSC_ERR_ARG, "bad copy kind");
        if (bytes) GTSC_CUDA(cudaMemcpyAsync(dst, src, bytes, (cudaMemcpyKind)kind, S(stream)));
        if (kind == 2) GTSC_CUDA(cudaStreamSynchronize(S(stream)));
    });
}

gtsc_status gtsc_memcpy_async(void *dst, const void *src, uint64_t bytes, int32_t kind, void *stream)
{
    return guard([&] {
        if (kind < 1 || kind > 3) fail(GTSC_ERR_ARG, "bad copy kind");
        if (bytes) GTSC_CUDA(cudaMemcpyAsync(dst, src, bytes, (cudaMemcpyKind)kind, S(stream)));
    });
}

gtsc_status gtsc_stream_synchronize(void *stream)
{
    return guard([&] { GTSC_CUDA(cudaStreamSynchronize(S(stream))); });
}

gtsc_status gtsc_stream_create(void **stream)
{
    return guard([&] {
        if (!stream) fail(GTSC_ERR_ARG, "null argument");
        cudaStream_t s;
        GTSC_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        *stream = (void *)s;
    });
}

gtsc_status gtsc_stream_destroy(void *stream)
{
    return guard([&] {
        if (stream) GTSC_CUDA(cudaStreamDestroy(S(stream)));
    });
}

gtsc_status gtsc_encode(int32_t encoding, int32_t dtype, const void *d_in, uint64_t in_bytes,
                        gtsc_buffer out[3], uint32_t *n_out, void *stream)
{
    return guard([&] {
        if (!out || !n_out) fail(GTSC_ERR_ARG, "null output");
        Parts p = encode(encoding, dtype, View(d_in, in_bytes), S(stream));
        GTSC_CUDA(cudaStreamSynchronize(S(stream)));
        for (int i = 0; i < 3; i++) out[i] = gtsc_buffer{nullptr, 0};
        *n_out = (uint32_t)p.size();
        for (size_t i = 0; i < p.size(); i++) out[i] = release(p[i]);
    });
}

gtsc_status gtsc_decode(int32_t encoding, int32_t dtype, const gtsc_buffer in[3], uint32_t n_in,
                        gtsc_buffer *out, void *stream)
{
    return guard([&] {
        if (!out || (!in && n_in)) fail(GTSC_ERR_ARG, "null argument");
        if (n_in > 3) fail(GTSC_ERR_ARG, "at most 3 inputs");
        std::vector<View> v;
        for (uint32_t i = 0; i < n_in; i++) v.push_back(View(in[i].ptr, in[i].bytes));
        DevBuf r = decode(encoding, dtype, v, S(stream));
        GTSC_CUDA(cudaStreamSynchronize(S(stream)));
        *out = release(r);
    });
}

gtsc_status gtsc_stats(int32_t dtype, const void *d_in, uint64_t in_bytes, gtsc_data_statistics *out,
                       void *stream)
{
    return guard([&] {
        if (!out) fail(GTSC_ERR_ARG, "null output");
        Stats st = column_stats(dtype, View(d_in, in_bytes), S(stream));
        static_assert(sizeof(Stats) == sizeof(gtsc_data_statistics), "layout");
        std::memcpy(out, &st, sizeof(st));
    });
}

static void write_tree(const Tree &t, int16_t *nodes_out, int32_t cap, int32_t *n_nodes)
{
    if (!nodes_out || !n_nodes) fail(GTSC_ERR_ARG, "null output");
    if (t.size() > cap) fail(GTSC_ERR_CAPACITY, "node list longer than cap");
    tree_to_nodes(t, nodes_out);
    *n_nodes = t.size();
}

gtsc_status gtsc_tree_from_path(const int16_t *encodings, int32_t n_encodings, int32_t dtype,
                                int16_t *nodes_out, int32_t cap, int32_t *n_nodes)
{
    return guard([&] {
        if (!encodings || n_encodings <= 0) fail(GTSC_ERR_ARG, "empty path");
        write_tree(tree_from_path(encodings, n_encodings, dtype), nodes_out, cap, n_nodes);
    });
}

gtsc_status gtsc_tree_compress(const int16_t *nodes, int32_t n_nodes, const void *d_in, uint64_t in_bytes,
                               gtsc_buffer *blob, void *stream)
{
    return guard([&] {
        if (!blob) fail(GTSC_ERR_ARG, "null output");
        DevBuf b = tree_compress(tree_from_nodes(nodes, n_nodes), View(d_in, in_bytes), S(stream));
        *blob = release(b);
    });
}

gtsc_status gtsc_tree_decompress(const void *d_blob, uint64_t blob_bytes, gtsc_buffer *out, int32_t *dtype,
                                 void *stream)
{
    return guard([&] {
        if (!out) fail(GTSC_ERR_ARG, "null output");
        int dt = 0;
        DevBuf b = tree_decompress(View(d_blob, blob_bytes), &dt, S(stream));
        if (dtype) *dtype = dt;
        *out = release(b);
    });
}

gtsc_status gtsc_tree_predict_size(const int16_t *nodes, int32_t n_nodes, const void *d_in, uint64_t in_bytes,
                                   uint64_t *size, void *stream)
{
    return guard([&] {
        if (!size) fail(GTSC_ERR_ARG, "null output");
        *size = tree_predict_size(tree_from_nodes(nodes, n_nodes), View(d_in, in_bytes), S(stream));
    });
}

gtsc_status gtsc_plan_exhaustive(int32_t dtype, const void *d_sample, uint64_t sample_bytes_, int16_t *nodes_out,
                                 int32_t cap, int32_t *n_nodes, uint64_t *candidate_size, void *stream)
{
    return guard([&] {
        uint64_t sz = 0;
        Tree t = plan_exhaustive(dtype, View(d_sample, sample_bytes_), &sz, nullptr, S(stream));
        write_tree(t, nodes_out, cap, n_nodes);
        if (candidate_size) *candidate_size = sz;
    });
}

gtsc_status gtsc_optimize_tree(int32_t dtype, const void *d_in, uint64_t in_bytes, int16_t *nodes_out,
                               int32_t cap, int32_t *n_nodes, uint64_t *predicted_size, void *stream)
{
    return guard([&] {
        uint64_t sz = 0;
        Tree t = optimize_tree(dtype, View(d_in, in_bytes), &sz, S(stream));
        write_tree(t, nodes_out, cap, n_nodes);
        if (predicted_size) *predicted_size = sz;
    });
}

uint64_t gtsc_sample_bytes(int32_t dtype, uint64_t in_bytes) { return sample_bytes(dtype, in_bytes); }

struct gtsc_batch {
    BatchEngine *e;
    uint32_t n_cols;
};

static BatchTuning to_tuning(const gtsc_batch_tuning &t)
{
    BatchTuning b;
    b.minmax_tile = t.minmax_tile;
    b.minmax_vpt = t.minmax_values_per_thread;
    b.hist_tile = t.hist_tile;
    b.persistent_c = t.schedule_compress == GTSC_SCHEDULE_PERSISTENT;
    b.persistent_d = t.schedule_decompress == GTSC_SCHEDULE_PERSISTENT;
    return b;
}

static void from_tuning(const BatchTuning &b, gtsc_batch_tuning *t)
{
    t->minmax_tile = b.minmax_tile;
    t->minmax_values_per_thread = b.minmax_vpt;
    t->hist_tile = b.hist_tile;
    t->schedule_compress = b.persistent_c ? GTSC_SCHEDULE_PERSISTENT : GTSC_SCHEDULE_LEVELS;
    t->schedule_decompress = b.persistent_d ? GTSC_SCHEDULE_PERSISTENT : GTSC_SCHEDULE_LEVELS;
}

gtsc_status gtsc_batch_create_tuned(const gtsc_column *cols, uint32_t n_cols, const int16_t *nodes,
                                    const int32_t *node_counts, const gtsc_batch_tuning *tuning, gtsc_batch **out,
                                    void *stream)
{
    return guard([&] {
        if (!cols || !nodes || !node_counts || !out || !n_cols) fail(GTSC_ERR_ARG, "null argument");
        std::vector<BatchColumn> c;
        std::vector<Tree> t;
        const int16_t *p = nodes;
        for (uint32_t i = 0; i < n_cols; i++) {
            c.push_back(BatchColumn{cols[i].d_data, cols[i].bytes, cols[i].dtype});
            t.push_back(tree_from_nodes(p, node_counts[i]));
            p += 2 * node_counts[i];
        }
        BatchEngine *e = batch_create(c, t, S(stream), tuning ? to_tuning(*tuning) : BatchTuning());
        *out = new gtsc_batch{e, n_cols};
    });
}

gtsc_status gtsc_batch_create(const gtsc_column *cols, uint32_t n_cols, const int16_t *nodes,
                              const int32_t *node_counts, gtsc_batch **out, void *stream)
{
    return gtsc_batch_create_tuned(cols, n_cols, nodes, node_counts, nullptr, out, stream);
}

gtsc_status gtsc_batch_get_tuning(gtsc_batch *b, gtsc_batch_tuning *tuning)
{
    return guard([&] {
        if (!b || !tuning) fail(GTSC_ERR_ARG, "null argument");
        *tuning = gtsc_batch_tuning{};
        from_tuning(batch_tuning(b->e), tuning);
    });
}

gtsc_status gtsc_batch_autotune(gtsc_batch *b, gtsc_batch_tuning *report, void *stream)
{
    return guard([&] {
        if (!b) fail(GTSC_ERR_ARG, "null batch");
        TuneReport rep;
        b->e = batch_autotune(b->e, S(stream), &rep);
        if (report) {
            *report = gtsc_batch_tuning{};
            from_tuning(rep.best, report);
            report->ms_default_compress = rep.ms_default[0];
            report->ms_default_decompress = rep.ms_default[1];
            report->ms_tuned_compress = rep.ms_tuned[0];
            report->ms_tuned_decompress = rep.ms_tuned[1];
            report->candidates = rep.candidates;
            report->seconds = rep.seconds;
        }
    });
}

gtsc_status gtsc_batch_set_inputs(gtsc_batch *b, const void *const *d_inputs, void *stream)
{
    return guard([&] {
        if (!b || !d_inputs) fail(GTSC_ERR_ARG, "null argument");
        batch_set_inputs(b->e, std::vector<const void *>(d_inputs, d_inputs + b->n_cols), S(stream));
    });
}

gtsc_status gtsc_batch_compress(gtsc_batch *b, void *stream)
{
    return guard([&] {
        if (!b) fail(GTSC_ERR_ARG, "null batch");
        batch_compress(b->e, S(stream));
    });
}

gtsc_status gtsc_batch_output(gtsc_batch *b, const void **d_framed, uint64_t *bytes, void *stream)
{
    return guard([&] {
        if (!b || !d_framed || !bytes) fail(GTSC_ERR_ARG, "null argument");
        *bytes = batch_output_bytes(b->e, S(stream));
        *d_framed = batch_output(b->e);
    });
}

gtsc_status gtsc_batch_blob_sizes(gtsc_batch *b, uint64_t *sizes, void *stream)
{
    return guard([&] {
        if (!b || !sizes) fail(GTSC_ERR_ARG, "null argument");
        std::vector<uint64_t> v = batch_blob_sizes(b->e, S(stream));
        std::memcpy(sizes, v.data(), 8 * v.size());
    });
}

gtsc_status gtsc_batch_decompress(gtsc_batch *b, const void *d_framed, uint64_t framed_bytes,
                                  void *const *d_outputs, void *stream)
{
    return guard([&] {
        if (!b || !d_framed || !d_outputs) fail(GTSC_ERR_ARG, "null argument");
        batch_decompress(b->e, (const uint8_t *)d_framed, framed_bytes,
                         std::vector<void *>(d_outputs, d_outputs + b->n_cols), S(stream));
    });
}

gtsc_status gtsc_batch_status(gtsc_batch *b, void *stream)
{
    gtsc_status st = GTSC_OK;
    gtsc_status g = guard([&] {
        if (!b) fail(GTSC_ERR_ARG, "null batch");
        st = batch_status(b->e, S(stream));
        if (st) set_last_error("batch: a device-side check failed in a step");
    });
    return g ? g : st;
}

int32_t gtsc_batch_launches(gtsc_batch *b, int32_t compress) { return b ? batch_launches(b->e, compress != 0) : 0; }

gtsc_status gtsc_batch_set_schedule(gtsc_batch *b, int32_t schedule)
{
    return guard([&] {
        if (!b) fail(GTSC_ERR_ARG, "null batch");
        if (schedule != GTSC_SCHEDULE_LEVELS && schedule != GTSC_SCHEDULE_PERSISTENT) fail(GTSC_ERR_ARG, "unknown schedule");
        batch_set_schedule(b->e, schedule == GTSC_SCHEDULE_PERSISTENT);
    });
}

int32_t gtsc_batch_schedule(gtsc_batch *b) { return b && batch_schedule(b->e) ? GTSC_SCHEDULE_PERSISTENT : GTSC_SCHEDULE_LEVELS; }

gtsc_status gtsc_batch_profile(gtsc_batch *b, int32_t compress, int32_t *ops, float *ms, uint64_t *bytes,
                               uint64_t *blocks, int32_t cap, int32_t *n, void *stream)
{
    return guard([&] {
        if (!b || !ops || !ms || !bytes || !blocks || !n) fail(GTSC_ERR_ARG, "null argument");
        const auto p = batch_profile(b->e, compress != 0, S(stream));
        if ((int64_t)p.size() > cap) fail(GTSC_ERR_CAPACITY, "profile: more launches than cap");
        for (size_t i = 0; i < p.size(); i++) {
            ops[i] = p[i].op;
            ms[i] = p[i].ms;
            bytes[i] = p[i].bytes;
            blocks[i] = p[i].blocks;
        }
        *n = (int32_t)p.size();
    });
}

gtsc_status gtsc_batch_destroy(gtsc_batch *b)
{
    return guard([&] {
        if (!b) return;
        batch_destroy(b->e);
        delete b;
    });
}

// ------------------------------------------------------------------------------- pipeline
struct gtsc_pipeline {
    Pipeline *p;
    uint32_t n_cols;
};

gtsc_status gtsc_pipeline_create(const gtsc_column *cols, uint32_t n_cols, const int16_t *nodes,
                                 const int32_t *node_counts, int32_t groups, gtsc_pipeline **out)
{
    return guard([&] {
        if (!cols || !nodes || !node_counts || !out || !n_cols) fail(GTSC_ERR_ARG, "null argument");
        std::vector<uint64_t> bytes;
        std::vector<int> dts;
        std::vector<Tree> t;
        const int16_t *p = nodes;
        for (uint32_t i = 0; i < n_cols; i++) {
            bytes.push_back(cols[i].bytes);
            dts.push_back(cols[i].dtype);
            t.push_back(tree_from_nodes(p, node_counts[i]));
            p += 2 * node_counts[i];
        }
        *out = new gtsc_pipeline{pipeline_create(bytes, dts, t, groups), n_cols};
    });
}

int32_t gtsc_pipeline_groups(gtsc_pipeline *p) { return p ? pipeline_groups(p->p) : 0; }

gtsc_status gtsc_pipeline_group_columns(gtsc_pipeline *p, int32_t g, int32_t *cols, int32_t cap, int32_t *n)
{
    return guard([&] {
        if (!p || !cols || !n || g < 0 || g >= pipeline_groups(p->p)) fail(GTSC_ERR_ARG, "bad argument");
        const auto &m = pipeline_group_columns(p->p, g);
        if ((int64_t)m.size() > cap) fail(GTSC_ERR_CAPACITY, "pipeline_group_columns: cap too small");
        for (size_t i = 0; i < m.size(); i++) cols[i] = m[i];
        *n = (int32_t)m.size();
    });
}

gtsc_status gtsc_pipeline_compress_host(gtsc_pipeline *p, const void *const *host_cols, void *host_framed,
                                        uint64_t cap, uint64_t *group_bytes)
{
    return guard([&] {
        if (!p || !host_cols || !host_framed || !group_bytes) fail(GTSC_ERR_ARG, "null argument");
        pipeline_compress_host(p->p, host_cols, (uint8_t *)host_framed, cap, group_bytes, false);
    });
}

gtsc_status gtsc_pipeline_roundtrip_host(gtsc_pipeline *p, const void *const *host_cols, void *host_framed,
                                         uint64_t cap, uint64_t *group_bytes)
{
    return guard([&] {
        if (!p || !host_cols || !host_framed || !group_bytes) fail(GTSC_ERR_ARG, "null argument");
        pipeline_compress_host(p->p, host_cols, (uint8_t *)host_framed, cap, group_bytes, true);
    });
}

gtsc_status gtsc_pipeline_decompress(gtsc_pipeline *p)
{
    return guard([&] {
        if (!p) fail(GTSC_ERR_ARG, "null argument");
        const gtsc_status st = pipeline_decompress(p->p);
        if (st != GTSC_OK) fail(st, "pipeline: a decode step reported an error");
    });
}

gtsc_status gtsc_pipeline_column(gtsc_pipeline *p, int32_t c, const void **d_input, const void **d_output)
{
    return guard([&] {
        if (!p || c < 0 || (uint32_t)c >= p->n_cols) fail(GTSC_ERR_ARG, "bad column");
        if (d_input) *d_input = pipeline_column_input(p->p, c);
        if (d_output) *d_output = pipeline_column_output(p->p, c);
    });
}

gtsc_status gtsc_pipeline_destroy(gtsc_pipeline *p)
{
    return guard([&] {
        if (!p) return;
        pipeline_destroy(p->p);
        delete p;
    });
}

// ------------------------------------------------------------------------------- learned planner
struct gtsc_planner {
    Planner *p;
};

gtsc_status gtsc_planner_features(const gtsc_column *cols, uint32_t n_cols, float *d_features, void *stream)
{
    return guard([&] {
        if ((!cols && n_cols) || (!d_features && n_cols)) fail(GTSC_ERR_ARG, "null argument");
        std::vector<FeatureColumn> fc(n_cols);
        for (uint32_t c = 0; c < n_cols; c++) {
            const int es = dtype_size(cols[c].dtype);
            if (!es) fail(GTSC_ERR_ARG, "unknown data type");
            fc[c] = FeatureColumn{cols[c].d_data, cols[c].bytes / es, cols[c].dtype};
        }
        compute_features(fc, d_features, S(stream));
    });
}

gtsc_status gtsc_planner_create(const int16_t *class_encs, const int32_t *class_lens, int32_t n_classes,
                                uint64_t seed, gtsc_planner **out)
{
    return guard([&] {
        if (!class_encs || !class_lens || !out || n_classes <= 0) fail(GTSC_ERR_ARG, "null argument");
        std::vector<std::vector<int16_t>> cls(n_classes);
        size_t off = 0;
        for (int c = 0; c < n_classes; c++) {
            if (class_lens[c] <= 0 || class_lens[c] > 1024) fail(GTSC_ERR_ARG, "planner: bad class length");
            cls[c].assign(class_encs + off, class_encs + off + class_lens[c]);
            off += class_lens[c];
        }
        std::unique_ptr<Planner> p(new Planner(cls, seed));
        *out = new gtsc_planner{p.release()};
    });
}

gtsc_status gtsc_planner_load(const void *model, uint64_t bytes, gtsc_planner **out)
{
    return guard([&] {
        if (!model || !out) fail(GTSC_ERR_ARG, "null argument");
        *out = new gtsc_planner{Planner::load(model, bytes)};
    });
}

gtsc_status gtsc_planner_save(gtsc_planner *p, void *buf, uint64_t cap, uint64_t *bytes)
{
    return guard([&] {
        if (!p || !bytes) fail(GTSC_ERR_ARG, "null argument");
        const std::vector<uint8_t> m = p->p->save();
        *bytes = m.size();
        if (buf) {
            if (cap < m.size()) fail(GTSC_ERR_CAPACITY, "planner_save: buffer too small");
            std::memcpy(buf, m.data(), m.size());
        }
    });
}

gtsc_status gtsc_planner_destroy(gtsc_planner *p)
{
    return guard([&] {
        if (!p) return;
        delete p->p;
        delete p;
    });
}

int32_t gtsc_planner_classes(gtsc_planner *p) { return p ? p->p->K : 0; }
uint64_t gtsc_planner_param_count(gtsc_planner *p) { return p ? p->p->n_params() : 0; }

gtsc_status gtsc_planner_get_params(gtsc_planner *p, float *params, float *mu, float *sd)
{
    return guard([&] {
        if (!p) fail(GTSC_ERR_ARG, "null argument");
        if (params) p->p->get_params(params, nullptr);
        if (mu) std::memcpy(mu, p->p->mu.data(), 4 * kFeatures);
        if (sd) std::memcpy(sd, p->p->sd.data(), 4 * kFeatures);
    });
}

gtsc_status gtsc_planner_set_params(gtsc_planner *p, const float *params, const float *mu, const float *sd)
{
    return guard([&] {
        if (!p) fail(GTSC_ERR_ARG, "null argument");
        if (params) p->p->set_params(params, nullptr);
        if (mu) std::memcpy(p->p->mu.data(), mu, 4 * kFeatures);
        if (sd) std::memcpy(p->p->sd.data(), sd, 4 * kFeatures);
    });
}

gtsc_status gtsc_planner_valid(gtsc_planner *p, uint8_t *valid)
{
    return guard([&] {
        if (!p || !valid) fail(GTSC_ERR_ARG, "null argument");
        std::memcpy(valid, p->p->valid.data(), p->p->valid.size());
    });
}

gtsc_status gtsc_planner_gradient(gtsc_planner *p, const float *d_features, const int32_t *labels, uint32_t n_rows,
                                  float *grad, float *loss, void *stream)
{
    return guard([&] {
        if (!p || !d_features || !labels || !loss) fail(GTSC_ERR_ARG, "null argument");
        *loss = p->p->gradient(d_features, labels, n_rows, grad, S(stream));
    });
}

gtsc_status gtsc_planner_train(gtsc_planner *p, const float *d_features, const int32_t *labels, uint32_t n_rows,
                               int32_t epochs, int32_t batch, float lr, uint64_t seed, float *final_loss,
                               void *stream)
{
    return guard([&] {
        if (!p || !d_features || !labels) fail(GTSC_ERR_ARG, "null argument");
        const float l = p->p->train(d_features, labels, n_rows, epochs, batch, lr, seed, S(stream));
        if (final_loss) *final_loss = l;
    });
}

gtsc_status gtsc_planner_predict(gtsc_planner *p, const float *d_features, const int32_t *dtypes, uint32_t n_rows,
                                 int32_t *classes, float *confidence, void *stream)
{
    return guard([&] {
        if (!p || (!d_features && n_rows) || !dtypes || !classes || !confidence) fail(GTSC_ERR_ARG, "null argument");
        p->p->predict(d_features, dtypes, n_rows, classes, confidence, S(stream));
    });
}

gtsc_status gtsc_plan_learned(gtsc_planner *p, const gtsc_column *cols, uint32_t n_cols, float min_confidence,
                              int16_t *nodes_out, int32_t nodes_cap, int32_t *node_counts, int32_t *fallback,
                              void *stream)
{
    return guard([&] {
        if (!p || (!cols && n_cols) || !nodes_out || !node_counts || !fallback) fail(GTSC_ERR_ARG, "null argument");
        cudaStream_t s = S(stream);
        if (!n_cols) return;
        std::vector<FeatureColumn> fc(n_cols);
        std::vector<int32_t> dts(n_cols);
        for (uint32_t c = 0; c < n_cols; c++) {
            const int es = dtype_size(cols[c].dtype);
            if (!es) fail(GTSC_ERR_ARG, "unknown data type");
            fc[c] = FeatureColumn{cols[c].d_data, cols[c].bytes / es, cols[c].dtype};
            dts[c] = cols[c].dtype;
        }
        DevBuf feats = dev_alloc((size_t)n_cols * kFeatures * 4, s);
        compute_features(fc, (float *)feats.get(), s);
        std::vector<int32_t> cls(n_cols);
        std::vector<float> conf(n_cols);
        p->p->predict((const float *)feats.get(), dts.data(), n_cols, cls.data(), conf.data(), s);
        int32_t used = 0;
        for (uint32_t c = 0; c < n_cols; c++) {
            Tree t;
            fallback[c] = !(cls[c] >= 0 && conf[c] >= min_confidence);
            if (!fallback[c]) {
                t = p->p->class_tree(cls[c], dts[c]);
            } else {
                const uint64_t sb = sample_bytes(dts[c], cols[c].bytes);
                uint64_t sz = 0;
                t = plan_exhaustive(dts[c], View{cols[c].d_data, sb}, &sz, nullptr, s);
            }
            if (used + t.size() > nodes_cap) fail(GTSC_ERR_CAPACITY, "plan_learned: nodes_cap too small");
            tree_to_nodes(t, nodes_out + 2 * used);
            node_counts[c] = t.size();
            used += t.size();
        }
    });
}

gtsc_status gtsc_predict_sizes(int32_t encoding, int32_t dtype, const void *d_in, uint64_t in_bytes,
                               uint64_t *metadata_bytes, uint64_t *compressed_bytes, void *stream)
{
    return guard([&] {
        if ((!d_in && in_bytes) || !metadata_bytes || !compressed_bytes) fail(GTSC_ERR_ARG, "null argument");
        const SizePrediction p = predict_sizes(encoding, dtype, View(d_in, in_bytes), S(stream));
        *metadata_bytes = p.meta;
        *compressed_bytes = p.data;
    });
}

static void afl_args(int32_t dtype, uint32_t b)
{
    const int es = dtype_size(dtype);
    if (!es || is_fp(dtype)) fail(GTSC_ERR_TYPE, "afl kernels: integer data types only");
    if (b < 1 || b > 8u * es) fail(GTSC_ERR_ARG, "afl kernels: bit length out of range");
}

uint64_t gtsc_afl32_bytes(int32_t dtype, uint32_t bit_length, uint64_t n)
{
    const int es = dtype_size(dtype);
    return es ? afl32_words(n, (int)bit_length, es) * es : 0;
}

gtsc_status gtsc_afl32_compress_gpu(int32_t dtype, uint32_t bit_length, const void *d_data, uint64_t n, void *d_out,
                                    uint64_t out_bytes, void *stream)
{
    return guard([&] {
        afl_args(dtype, bit_length);
        const int es = dtype_size(dtype);
        if ((!d_data && n) || !d_out) fail(GTSC_ERR_ARG, "null argument");
        if (((uintptr_t)d_data | (uintptr_t)d_out) % es) fail(GTSC_ERR_ARG, "afl32: pointers must be element aligned");
        const uint64_t words = afl32_words(n, (int)bit_length, es);
        if (out_bytes < words * es) fail(GTSC_ERR_CAPACITY, "afl32: output smaller than gtsc_afl32_bytes");
        // the layout has holes only in a last, partial block of 32 x W elements: clear just that block
        const uint64_t full = n / (32ull * 8 * es) * 32ull * bit_length;
        if (words > full) GTSC_CUDA(cudaMemsetAsync((uint8_t *)d_out + full * es, 0, (words - full) * es, S(stream)));
        launch_afl32_pack((const uint8_t *)d_data, n, es, (int)bit_length, (uint8_t *)d_out, words, S(stream));
    });
}

gtsc_status gtsc_afl32_decompress_gpu(int32_t dtype, uint32_t bit_length, const void *d_comp, uint64_t comp_bytes,
                                      void *d_out, uint64_t n, void *stream)
{
    return guard([&] {
        afl_args(dtype, bit_length);
        const int es = dtype_size(dtype);
        if ((!d_comp || !d_out) && n) fail(GTSC_ERR_ARG, "null argument");
        if (((uintptr_t)d_comp | (uintptr_t)d_out) % es) fail(GTSC_ERR_ARG, "afl32: pointers must be element aligned");
        launch_afl32_unpack((const uint8_t *)d_comp, comp_bytes / es, n, es, (int)bit_length, (uint8_t *)d_out, S(stream));
    });
}

gtsc_status gtsc_afl_values_gpu(int32_t dtype, uint32_t bit_length, int32_t omega, const void *d_comp,
                                uint64_t comp_bytes, const uint64_t *d_index, uint64_t n, void *d_out, void *stream)
{
    return guard([&] {
        afl_args(dtype, bit_length);
        const int es = dtype_size(dtype);
        if (omega != 1 && omega != 32) fail(GTSC_ERR_ARG, "afl values: omega is 1 or 32");
        if ((!d_comp || !d_out) && n) fail(GTSC_ERR_ARG, "null argument");
        if (((uintptr_t)d_comp | (uintptr_t)d_out) % es) fail(GTSC_ERR_ARG, "afl values: pointers must be element aligned");
        launch_afl_values((const uint8_t *)d_comp, comp_bytes / es, es, (int)bit_length, omega, d_index, n,
                          (uint8_t *)d_out, S(stream));
    });
}

gtsc_status gtsc_afl_compress_gpu(int32_t dtype, uint32_t bit_length, const void *d_data, uint64_t n,
                                  void *d_out, uint64_t out_bytes, void *stream)
{
    return guard([&] {
        const int es = dtype_size(dtype);
        if (!es || is_fp(dtype)) fail(GTSC_ERR_TYPE, "afl: integer data types only");
        const uint64_t W = 8ull * es;
        if (out_bytes < (bit_length * n + W - 1) / W * es) fail(GTSC_ERR_CAPACITY, "afl: output too small");
        launch_afl_pack((const uint8_t *)d_data, n, es, (int)bit_length, (uint8_t *)d_out, out_bytes, S(stream));
    });
}

gtsc_status gtsc_afl_decompress_gpu(int32_t dtype, uint32_t bit_length, const void *d_comp,
                                    uint64_t comp_bytes, void *d_out, uint64_t n, void *stream)
{
    return guard([&] {
        const int es = dtype_size(dtype);
        if (!es || is_fp(dtype)) fail(GTSC_ERR_TYPE, "afl: integer data types only");
        if (comp_bytes * 8 < n * (uint64_t)bit_length) fail(GTSC_ERR_FORMAT, "afl: stream too short");
        launch_afl_unpack((const uint8_t *)d_comp, comp_bytes, n, es, (int)bit_length, (uint8_t *)d_out, S(stream));
    });
}


struct gtsc_edge_stats {
    std::shared_ptr<EdgeStats> p;
};
struct gtsc_optimal_tree {
    std::unique_ptr<OptimalTree> t;
};
struct gtsc_optimizer {
    Optimizer o;
    gtsc_edge_stats view;
    explicit gtsc_optimizer(int dt) : o(dt) { view.p = o.stats; }
};

static void write_flat(const FlatTree &f, int16_t *nodes_out, double *ratios_out, int32_t cap, int32_t *n_nodes)
{
    if (!n_nodes) fail(GTSC_ERR_ARG, "null output");
    std::vector<double> r;
    const Tree t = f.preorder(&r);
    *n_nodes = t.size();
    if (t.size() > cap) fail(GTSC_ERR_CAPACITY, "node list longer than cap");
    if (nodes_out) tree_to_nodes(t, nodes_out);
    if (ratios_out) std::memcpy(ratios_out, r.data(), sizeof(double) * r.size());
}

static FlatTree flat_of(const int16_t *nodes, const double *ratios, int32_t n_nodes)
{
    const Tree t = tree_from_nodes(nodes, n_nodes);
    std::vector<double> r;
    if (ratios) r.assign(ratios, ratios + n_nodes);
    return FlatTree::from(t, r);
}

gtsc_status gtsc_optimizer_create(int32_t dtype, gtsc_optimizer **out)
{
    return guard([&] {
        if (!out) fail(GTSC_ERR_ARG, "null output");
        if (!dtype_size(dtype)) fail(GTSC_ERR_ARG, "unknown data type");
        *out = new gtsc_optimizer(dtype);
    });
}

gtsc_status gtsc_optimizer_compress(gtsc_optimizer *o, const void *d_in, uint64_t in_bytes, gtsc_buffer *blob,
                                    int32_t *full_update, int32_t *corrected, void *stream)
{
    return guard([&] {
        if (!o || !blob || (!d_in && in_bytes)) fail(GTSC_ERR_ARG, "null argument");
        bool full = false, corr = false;
        DevBuf b = o->o.compress_data(View(d_in, in_bytes), &full, &corr, S(stream));
        if (full_update) *full_update = full;
        if (corrected) *corrected = corr;
        *blob = release(b);
    });
}

gtsc_status gtsc_optimizer_tree(const gtsc_optimizer *o, int16_t *nodes_out, double *ratios_out, int32_t cap,
                                int32_t *n_nodes)
{
    return guard([&] {
        if (!o) fail(GTSC_ERR_ARG, "null optimizer");
        if (!o->o.opt) fail(GTSC_ERR_ARG, "optimizer: no part compressed yet");
        write_flat(o->o.opt->tree, nodes_out, ratios_out, cap, n_nodes);
    });
}

gtsc_status gtsc_optimizer_statistics(gtsc_optimizer *o, gtsc_edge_stats **stats)
{
    return guard([&] {
        if (!o || !stats) fail(GTSC_ERR_ARG, "null argument");
        *stats = &o->view;
    });
}

gtsc_status gtsc_optimizer_destroy(gtsc_optimizer *o)
{
    return guard([&] { delete o; });
}

gtsc_status gtsc_edge_stats_create(int32_t tree_height, gtsc_edge_stats **out)
{
    return guard([&] {
        if (!out) fail(GTSC_ERR_ARG, "null output");
        auto *s = new gtsc_edge_stats();
        try {
            s->p = std::make_shared<EdgeStats>(tree_height);
        } catch (...) {
            delete s;
            throw;
        }
        *out = s;
    });
}

gtsc_status gtsc_edge_stats_destroy(gtsc_edge_stats *s)
{
    return guard([&] { delete s; });
}

gtsc_status gtsc_edge_stats_set(gtsc_edge_stats *s, int32_t edge, int16_t from, int16_t to, double value)
{
    return guard([&] {
        if (!s) fail(GTSC_ERR_ARG, "null statistics");
        s->p->set(edge, EdgeType{from, to}, value);
    });
}

gtsc_status gtsc_edge_stats_update(gtsc_edge_stats *s, int32_t edge, int16_t from, int16_t to, double ratio)
{
    return guard([&] {
        if (!s) fail(GTSC_ERR_ARG, "null statistics");
        if (edge < 0 || edge >= s->p->edges()) fail(GTSC_ERR_ARG, "edge number out of range");
        s->p->update(edge, EdgeType{from, to}, ratio);
    });
}

gtsc_status gtsc_edge_stats_get(const gtsc_edge_stats *s, int32_t edge, int16_t from, int16_t to, double *value)
{
    return guard([&] {
        if (!s || !value) fail(GTSC_ERR_ARG, "null argument");
        *value = s->p->get(edge, EdgeType{from, to});
    });
}

gtsc_status gtsc_edge_stats_best(const gtsc_edge_stats *s, int32_t edge, int16_t from, int16_t to,
                                 int32_t same_beginning, int16_t *best_from, int16_t *best_to, double *value)
{
    return guard([&] {
        if (!s || !best_from || !best_to || !value) fail(GTSC_ERR_ARG, "null argument");
        const EdgeStats::Best b = s->p->best(edge, EdgeType{from, to}, same_beginning != 0);
        *best_from = (int16_t)b.type.first;
        *best_to = (int16_t)b.type.second;
        *value = b.value;
    });
}

gtsc_status gtsc_edge_stats_entries(const gtsc_edge_stats *s, int32_t edge, int16_t *pairs_out, double *values_out,
                                    int32_t cap, int32_t *n)
{
    return guard([&] {
        if (!s || !n) fail(GTSC_ERR_ARG, "null argument");
        if (edge < 0 || edge >= s->p->edges()) fail(GTSC_ERR_ARG, "edge number out of range");
        const auto &m = s->p->e[edge];
        *n = (int32_t)m.size();
        if ((int32_t)m.size() > cap) fail(GTSC_ERR_CAPACITY, "more entries than cap");
        int k = 0;
        for (auto &kv : m) {
            if (pairs_out) {
                pairs_out[2 * k] = (int16_t)kv.first.first;
                pairs_out[2 * k + 1] = (int16_t)kv.first.second;
            }
            if (values_out) values_out[k] = kv.second;
            k++;
        }
    });
}

gtsc_status gtsc_tree_edges(const int16_t *nodes, int32_t n_nodes, int32_t *edge_no, int32_t *from_node,
                            int32_t *to_node, int32_t cap, int32_t *n_edges)
{
    return guard([&] {
        if (!n_edges) fail(GTSC_ERR_ARG, "null output");
        const FlatTree f = flat_of(nodes, nullptr, n_nodes);  // node k of f = pre-order node k
        const std::vector<TreeEdge> ed = tree_edges(f);
        *n_edges = (int32_t)ed.size();
        if ((int32_t)ed.size() > cap) fail(GTSC_ERR_CAPACITY, "more edges than cap");
        for (size_t k = 0; k < ed.size(); k++) {
            if (edge_no) edge_no[k] = ed[k].no;
            if (from_node) from_node[k] = ed[k].from;
            if (to_node) to_node[k] = ed[k].to;
        }
    });
}

gtsc_status gtsc_tree_update_statistics(const int16_t *nodes, const double *ratios, int32_t n_nodes,
                                        gtsc_edge_stats *s)
{
    return guard([&] {
        if (!s || !ratios) fail(GTSC_ERR_ARG, "null argument");
        update_statistics(flat_of(nodes, ratios, n_nodes), *s->p);
    });
}

gtsc_status gtsc_optimal_tree_create(const int16_t *nodes, const double *ratios, int32_t n_nodes,
                                     gtsc_edge_stats *stats, gtsc_optimal_tree **out)
{
    return guard([&] {
        if (!stats || !out || !ratios) fail(GTSC_ERR_ARG, "null argument");
        auto *t = new gtsc_optimal_tree();
        try {
            t->t.reset(new OptimalTree(flat_of(nodes, ratios, n_nodes), stats->p));
        } catch (...) {
            delete t;
            throw;
        }
        *out = t;
    });
}

gtsc_status gtsc_optimal_tree_set_ratio(gtsc_optimal_tree *t, int32_t node, double ratio)
{
    return guard([&] {
        if (!t) fail(GTSC_ERR_ARG, "null tree");
        if (node < 0 || node >= (int32_t)t->t->tree.ratio.size()) fail(GTSC_ERR_ARG, "node out of range");
        t->t->tree.ratio[node] = ratio;  // the tree is kept in pre-order
    });
}

gtsc_status gtsc_optimal_tree_try_correct(gtsc_optimal_tree *t, int32_t *corrected)
{
    return guard([&] {
        if (!t) fail(GTSC_ERR_ARG, "null tree");
        const bool c = t->t->try_correct();
        if (corrected) *corrected = c;
    });
}

gtsc_status gtsc_optimal_tree_get(const gtsc_optimal_tree *t, int16_t *nodes_out, double *ratios_out, int32_t cap,
                                  int32_t *n_nodes)
{
    return guard([&] {
        if (!t) fail(GTSC_ERR_ARG, "null tree");
        write_flat(t->t->tree, nodes_out, ratios_out, cap, n_nodes);
    });
}

gtsc_status gtsc_optimal_tree_destroy(gtsc_optimal_tree *t)
{
    return guard([&] { delete t; });
}

}  // extern "C"
