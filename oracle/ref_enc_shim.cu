/*
 * ref_enc_shim.cu -- exposes the reference's own encoders and compression tree for parity checks.
 *
 * TEST INFRASTRUCTURE ONLY.  This file contains no reference code.  oracle/Makefile (target
 * refenc) compiles the reference's encoder, utility and tree sources where they lie in the
 * reference tree, with the stand-in headers of oracle/refshim/ for boost, log4cplus, gtest and the
 * un-vendored data_type.hpp, and links them with this file into oracle/_ref/libref_enc.so, which
 * is never committed.  The entry points below take host buffers, copy them to the device, run the
 * reference's code path exactly as CompressionNode does (tree/compression_node.cpp:103-161: the
 * factory's Get(data) to encode, Get() to decode) and copy the results back; ref_dev_* keep a
 * column on the device to time the reference's tree compress alone.
 *
 * Encoding and data-type codes are the library's: the encodings follow EncodingType
 * (compression/encoding_type.hpp:17-30), 11 selects PatchEncodingFactory with PatchType::outside
 * (compression/patch/patch_encoding_factory.hpp:47-55), and the data types are CHAR 0, SHORT 1,
 * INT 2, TIME 3, FLOAT 4, DOUBLE 5 (oracle/refshim/data_type.hpp).
 *
 * Not exposed: the GFC encoder (compression/gfc/), whose kernels rely on implicit warp-synchronous
 * shared-memory exchanges that are not guaranteed on sm_70 and later, and the shared-memory
 * histogram CudaHistogram (util/histogram/cuda_histogram.cu), whose legacy vote instructions do not
 * assemble for sm_100a; neither is on a path the encoders below take (dict and const count values
 * with ThrustSparseHistogram).  CudaHistogram is defined here to fail loudly, so that the library
 * links.
 */
#include "compression/default_encoding_factory.hpp"
#include "compression/patch/patch_encoding_factory.hpp"
#include "tree/compression_tree.hpp"
#include "util/histogram/histogram.hpp"

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>

// the reference's exit(1) on a CUDA error (refshim/ref_compat.hpp renames exit to this)
[[noreturn]] void ref_exit(int status)
{
    throw std::runtime_error("the reference stopped on a CUDA error (exit status " + std::to_string(status) + ")");
}

namespace ddj {
template <typename T>
SharedCudaPtr<int> Histogram::CudaHistogram(SharedCudaPtr<T>, int)
{
    throw std::runtime_error("CudaHistogram is not built for sm_100a");
}
template SharedCudaPtr<int> Histogram::CudaHistogram<char>(SharedCudaPtr<char>, int);
template SharedCudaPtr<int> Histogram::CudaHistogram<short>(SharedCudaPtr<short>, int);
template SharedCudaPtr<int> Histogram::CudaHistogram<int>(SharedCudaPtr<int>, int);
template SharedCudaPtr<int> Histogram::CudaHistogram<long>(SharedCudaPtr<long>, int);
template SharedCudaPtr<int> Histogram::CudaHistogram<long long>(SharedCudaPtr<long long>, int);
template SharedCudaPtr<int> Histogram::CudaHistogram<unsigned int>(SharedCudaPtr<unsigned int>, int);
template SharedCudaPtr<int> Histogram::CudaHistogram<float>(SharedCudaPtr<float>, int);
template SharedCudaPtr<int> Histogram::CudaHistogram<double>(SharedCudaPtr<double>, int);
}  // namespace ddj

namespace {

using namespace ddj;

constexpr int kOutsidePatch = 11;
constexpr int kGfc = (int)EncodingType::gfc;

std::string g_error;

DataType data_type(int code)
{
    if (code < 0 || code > 5) throw std::invalid_argument("unknown data type code");
    return (DataType)code;
}

boost::shared_ptr<EncodingFactory> factory(int enc, DataType dt)
{
    if (enc == kGfc) throw std::invalid_argument("the reference's GFC encoder is not exposed");
    if (enc == kOutsidePatch) {
        switch (dt) {
        case DataType::d_char: return boost::make_shared<PatchEncodingFactory<char>>(dt, PatchType::outside);
        case DataType::d_short: return boost::make_shared<PatchEncodingFactory<short>>(dt, PatchType::outside);
        case DataType::d_int: return boost::make_shared<PatchEncodingFactory<int>>(dt, PatchType::outside);
        case DataType::d_time: return boost::make_shared<PatchEncodingFactory<time_t>>(dt, PatchType::outside);
        case DataType::d_float: return boost::make_shared<PatchEncodingFactory<float>>(dt, PatchType::outside);
        case DataType::d_double: return boost::make_shared<PatchEncodingFactory<double>>(dt, PatchType::outside);
        }
    }
    if (enc < 0 || enc >= (int)EncodingType::length) throw std::invalid_argument("unknown encoding code");
    return DefaultEncodingFactory::Get((EncodingType)enc, dt);
}

SharedCudaPtr<char> to_device(const void *p, uint64_t n)
{
    auto d = CudaPtr<char>::make_shared(n);
    if (n) d->fillFromHost((const char *)p, n);
    return d;
}

// a malloc'd host copy of a device buffer (freed with ref_enc_free)
void *to_host(SharedCudaPtr<char> d, uint64_t *n)
{
    *n = d ? d->size() : 0;
    void *h = malloc(*n ? *n : 1);
    if (!h) throw std::bad_alloc();
    if (*n && cudaMemcpy(h, d->get(), *n, cudaMemcpyDeviceToHost) != cudaSuccess) {
        free(h);
        throw std::runtime_error("device to host copy failed");
    }
    return h;
}

// Adds the tree whose nodes are given in pre-order as (encoding, data type) pairs to an empty
// CompressionTree: a node has as many children as its encoding has results (none: zero), added in
// that order, as CompressionTree::AddNode numbers them (tree/compression_tree.cpp:59-79).
void build_tree(CompressionTree &tree, const int16_t *nodes, int n_nodes)
{
    if (n_nodes <= 0) throw std::invalid_argument("empty tree");
    std::vector<std::pair<unsigned, int>> open;  // (parent number, children still to add)
    unsigned next = 0;
    for (int k = 0; k < n_nodes; k++) {
        const int enc = nodes[2 * k];
        const DataType t = data_type(nodes[2 * k + 1]);
        while (!open.empty() && open.back().second == 0) open.pop_back();
        if (k > 0 && open.empty()) throw std::invalid_argument("more nodes than the tree has slots");
        const unsigned parent = k == 0 ? 0 : open.back().first;
        if (k > 0) open.back().second--;
        if (!tree.AddNode(boost::make_shared<CompressionNode>(factory(enc, t)), parent))
            throw std::runtime_error("AddNode failed");
        const int children = enc == (int)EncodingType::none ? 0 : (int)factory(enc, t)->Get()->GetNumberOfResults();
        open.push_back({next, children});
        next++;
    }
    while (!open.empty() && open.back().second == 0) open.pop_back();
    if (!open.empty()) throw std::invalid_argument("the tree has unfilled slots");
}

template <class F>
int guarded(F f)
{
    try {
        f();
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            g_error = cudaGetErrorString(e);
            return -2;
        }
        return 0;
    } catch (const std::exception &x) {
        g_error = x.what();
        return -1;
    } catch (...) {
        g_error = "unknown exception";
        return -1;
    }
}

}  // namespace

extern "C" {

const char *ref_enc_error() { return g_error.c_str(); }

void ref_enc_free(void *p) { free(p); }

// Encoding::Encode (compression/encoding.hpp:27-47) through the factory's Get(data): the result
// streams (metadata first) are copied to malloc'd host buffers outs[0..*nres-1] (at most 4).
int ref_enc_encode(int enc, int dt, const void *in, uint64_t nbytes, int *nres, void **outs, uint64_t *sizes)
{
    *nres = 0;
    return guarded([&] {
        const DataType t = data_type(dt);
        auto data = to_device(in, nbytes);
        auto encoding = factory(enc, t)->Get(data);
        auto result = encoding->Encode(data, t);
        if (result.size() > 4) throw std::runtime_error("more than four result streams");
        for (size_t i = 0; i < result.size(); i++) {
            outs[i] = to_host(result[i], &sizes[i]);
            *nres = (int)i + 1;
        }
    });
}

// Encoding::Decode (compression/encoding.hpp:49-69) through the factory's Get()
int ref_enc_decode(int enc, int dt, int nparts, const void *const *parts, const uint64_t *sizes, void **out,
                   uint64_t *out_bytes)
{
    *out = nullptr;
    *out_bytes = 0;
    return guarded([&] {
        const DataType t = data_type(dt);
        SharedCudaPtrVector<char> data;
        for (int i = 0; i < nparts; i++) data.push_back(to_device(parts[i], sizes[i]));
        auto encoding = factory(enc, t)->Get();
        *out = to_host(encoding->Decode(data, t), out_bytes);
    });
}

// CompressionTree::Compress (tree/compression_tree.cpp) of a pre-order node list (build_tree)
int ref_tree_compress(const int16_t *nodes, int n_nodes, const void *in, uint64_t nbytes, void **out,
                      uint64_t *out_bytes)
{
    *out = nullptr;
    *out_bytes = 0;
    return guarded([&] {
        CompressionTree tree;
        build_tree(tree, nodes, n_nodes);
        *out = to_host(tree.Compress(to_device(in, nbytes)), out_bytes);
    });
}

// A column kept on the device for timing the reference's tree compress without host copies:
// ref_dev_upload returns a handle to a device copy (freed by ref_dev_free).
void *ref_dev_upload(const void *in, uint64_t nbytes)
{
    void *h = nullptr;
    const int rc = guarded([&] { h = new SharedCudaPtr<char>(to_device(in, nbytes)); });
    return rc == 0 ? h : nullptr;
}

void ref_dev_free(void *h) { delete (SharedCudaPtr<char> *)h; }

// CompressionTree::Compress of a resident column; the blob stays on the device and is freed (its
// size is returned).  Synchronous, as the reference's API is.
int ref_dev_tree_compress(void *h, const int16_t *nodes, int n_nodes, uint64_t *out_bytes)
{
    *out_bytes = 0;
    return guarded([&] {
        CompressionTree tree;
        build_tree(tree, nodes, n_nodes);
        auto blob = tree.Compress(*(SharedCudaPtr<char> *)h);
        *out_bytes = blob ? blob->size() : 0;
    });
}

// CompressionTree::Decompress (tree/compression_tree.cpp:148-155)
int ref_tree_decompress(const void *blob, uint64_t nbytes, void **out, uint64_t *out_bytes)
{
    *out = nullptr;
    *out_bytes = 0;
    return guarded([&] {
        CompressionTree tree;
        *out = to_host(tree.Decompress(to_device(blob, nbytes)), out_bytes);
    });
}

}  // extern "C"
