// pipeline.cu -- column chunks from host memory to framed host output with the batched engine,
// the copies of one column group overlapping the compression of the others.
//
// It replaces the reference's chunk loop (ParallelTSCompressor::Compress, parallel_ts_compressor.cpp
// 39-63: per column chunk a CompressionTask that compresses and writes `size_t len` + blob,
// optimizer/compression_task.cpp:35-77).  The columns are split into groups of about equal bytes;
// each group has its own batch engine (its trees captured as CUDA graphs) and stream.  A chunk:
//   1. the host -> device copies of all groups, group after group, on one upload stream; each
//      group's compress graph waits only for its own group's copies;
//   2. every group in turn: wait for its compress, copy its framed output to the host (async),
// so group 0 compresses while group 1 uploads, and group g's device -> host copy runs while groups
// g+1.. still upload and compress.  (Copies queued on every group's stream at once share the copy
// engines: every group's upload then ends near the end of all of them, and the compression and
// read-back of the early groups no longer hide behind the later uploads.)
#include "batch.hpp"

#include <algorithm>
#include <cstring>
#include <numeric>

namespace gtsc {

struct Pipeline {
    int groups = 0;
    std::vector<std::vector<int>> members;      // columns of each group
    std::vector<uint64_t> bytes;                // per column
    std::vector<int> dtypes;
    std::vector<DevBuf> d_in, d_out;            // per column
    std::vector<BatchEngine *> eng;             // per group
    std::vector<cudaStream_t> st;               // per group
    cudaStream_t up = nullptr;                  // the host -> device copies of every group, in order
    std::vector<cudaEvent_t> uploaded;          // per group: its copies are done
    std::vector<const uint8_t *> framed;        // per group: last compress output (device)
    std::vector<uint64_t> framed_bytes;
    ~Pipeline()
    {
        cudaDeviceSynchronize();
        for (auto &b : d_in) b.release_on_default_stream();
        for (auto &b : d_out) b.release_on_default_stream();
        for (auto *e : eng) batch_destroy(e);
        for (auto s : st)
            if (s) cudaStreamDestroy(s);
        for (auto e : uploaded)
            if (e) cudaEventDestroy(e);
        if (up) cudaStreamDestroy(up);
    }
};

Pipeline *pipeline_create(const std::vector<uint64_t> &bytes, const std::vector<int> &dtypes,
                          const std::vector<Tree> &trees, int groups)
{
    const size_t n = bytes.size();
    if (n == 0 || trees.size() != n || dtypes.size() != n) fail(GTSC_ERR_ARG, "pipeline: one tree per column");
    groups = std::max(1, std::min<int>(groups, (int)n));
    std::unique_ptr<Pipeline> p(new Pipeline());
    p->groups = groups;
    p->bytes = bytes;
    p->dtypes = dtypes;
    // largest columns first, each to the group with the fewest bytes so far
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return bytes[a] > bytes[b]; });
    std::vector<uint64_t> load(groups, 0);
    p->members.assign(groups, {});
    for (int c : order) {
        const int g = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        p->members[g].push_back(c);
        load[g] += bytes[c];
    }
    for (auto &m : p->members) std::sort(m.begin(), m.end());
    p->st.assign(groups, nullptr);
    for (int g = 0; g < groups; g++) GTSC_CUDA(cudaStreamCreateWithFlags(&p->st[g], cudaStreamNonBlocking));
    GTSC_CUDA(cudaStreamCreateWithFlags(&p->up, cudaStreamNonBlocking));
    p->uploaded.assign(groups, nullptr);
    for (int g = 0; g < groups; g++) GTSC_CUDA(cudaEventCreateWithFlags(&p->uploaded[g], cudaEventDisableTiming));
    p->d_in.resize(n);
    p->d_out.resize(n);
    for (size_t c = 0; c < n; c++) {
        p->d_in[c] = dev_alloc(std::max<uint64_t>(bytes[c], 16), p->st[0]);
        p->d_out[c] = dev_alloc(std::max<uint64_t>(bytes[c], 16), p->st[0]);
    }
    GTSC_CUDA(cudaStreamSynchronize(p->st[0]));
    p->eng.assign(groups, nullptr);
    p->framed.assign(groups, nullptr);
    p->framed_bytes.assign(groups, 0);
    for (int g = 0; g < groups; g++) {
        std::vector<BatchColumn> bc;
        std::vector<Tree> bt;
        for (int c : p->members[g]) {
            bc.push_back(BatchColumn{p->d_in[c].get(), bytes[c], dtypes[c]});
            bt.push_back(trees[c]);
        }
        if (!bc.empty()) p->eng[g] = batch_create(bc, bt, p->st[g]);
    }
    return p.release();
}

void pipeline_destroy(Pipeline *p) { delete p; }

int pipeline_groups(const Pipeline *p) { return p->groups; }

const std::vector<int> &pipeline_group_columns(const Pipeline *p, int g) { return p->members.at(g); }

// Compress one chunk (host columns, same sizes as at creation).  host_framed receives, per group
// in order, that group's framed output (column count, blob sizes, blobs), back to back; *sizes
// (groups entries) their bytes.  Host memory should be pinned for the copies to overlap.
void pipeline_compress_host(Pipeline *p, const void *const *host_cols, uint8_t *host_framed, uint64_t cap,
                            uint64_t *sizes, bool decode)
{
    const int G = p->groups;
    // (the previous call ended with every group's stream synchronised, so no step still reads the
    // input buffers that these copies overwrite)
    for (int g = 0; g < G; g++) {
        if (!p->eng[g]) continue;
        for (int c : p->members[g])
            if (p->bytes[c])
                GTSC_CUDA(cudaMemcpyAsync(p->d_in[c].get(), host_cols[c], p->bytes[c], cudaMemcpyHostToDevice, p->up));
        GTSC_CUDA(cudaEventRecord(p->uploaded[g], p->up));
        GTSC_CUDA(cudaStreamWaitEvent(p->st[g], p->uploaded[g], 0));
        batch_compress(p->eng[g], p->st[g]);
    }
    uint64_t off = 0;
    for (int g = 0; g < G; g++) {
        sizes[g] = 0;
        if (!p->eng[g]) continue;
        const uint64_t nb = batch_output_bytes(p->eng[g], p->st[g]);  // waits for this group only
        if (off + nb > cap) {
            // earlier groups' copies into host_framed (and their decodes) are in flight: let them
            // finish so that nothing writes the caller's buffer after the error returns
            cudaStreamSynchronize(p->up);
            for (int h = 0; h < G; h++) cudaStreamSynchronize(p->st[h]);
            fail(GTSC_ERR_CAPACITY, "pipeline: host framed buffer too small");
        }
        p->framed[g] = batch_output(p->eng[g]);
        p->framed_bytes[g] = nb;
        GTSC_CUDA(cudaMemcpyAsync(host_framed + off, p->framed[g], nb, cudaMemcpyDeviceToHost, p->st[g]));
        if (decode) {  // the round trip: this group's device decode runs while later groups copy
            std::vector<void *> outs;
            for (int c : p->members[g]) outs.push_back(p->d_out[c].get());
            batch_decompress(p->eng[g], p->framed[g], nb, outs, p->st[g]);
        }
        sizes[g] = nb;
        off += nb;
    }
    for (int g = 0; g < G; g++) GTSC_CUDA(cudaStreamSynchronize(p->st[g]));
    for (int g = 0; g < G; g++) {
        if (!p->eng[g]) continue;
        const gtsc_status st = batch_status(p->eng[g], p->st[g]);
        if (st != GTSC_OK) fail(st, decode ? "pipeline: a compress or decode step reported an error"
                                           : "pipeline: a compress step reported an error");
    }
}

// Decompress the last compressed chunk from its device framed buffers into the pipeline's device
// column outputs (all groups' steps in flight together); returns the first failing status.
gtsc_status pipeline_decompress(Pipeline *p)
{
    const int G = p->groups;
    for (int g = 0; g < G; g++) {
        if (!p->eng[g] || !p->framed[g]) continue;
        std::vector<void *> outs;
        for (int c : p->members[g]) outs.push_back(p->d_out[c].get());
        batch_decompress(p->eng[g], p->framed[g], p->framed_bytes[g], outs, p->st[g]);
    }
    gtsc_status st = GTSC_OK;
    for (int g = 0; g < G; g++) {
        if (!p->eng[g]) continue;
        const gtsc_status s = batch_status(p->eng[g], p->st[g]);
        if (s != GTSC_OK && st == GTSC_OK) st = s;
    }
    return st;
}

// device buffers of column c: its input (written by the last compress) and its decoded output
const void *pipeline_column_input(Pipeline *p, int c) { return p->d_in.at(c).get(); }
const void *pipeline_column_output(Pipeline *p, int c) { return p->d_out.at(c).get(); }

}  // namespace gtsc
