/*
 * gtsc/ddj.hpp -- header-only C++ layer that re-creates the reference's public class names
 * (namespace ddj) over the C ABI of libgtsc (gtsc.h), so code written against the reference's
 * Encoding / CompressionTree / CompressionOptimizer API compiles against the B200 library with an
 * include change.
 *
 *   reference                                               here
 *   core/cuda_ptr.hpp: CudaPtr<T>, SharedCudaPtr<T>          CudaPtr<T> (device buffer freed with
 *     (boost::shared_ptr), CastSharedCudaPtr,                  gtsc_free), std::shared_ptr, the same
 *     MoveSharedCudaPtr (:124-160)                             casts
 *   compression/encoding.hpp: Encoding (:18-113)             Encoding over gtsc_encode / gtsc_decode /
 *                                                              gtsc_predict_sizes
 *   compression/encoding_factory.hpp (:22-40),               EncodingFactory, DefaultEncodingFactory
 *     default_encoding_factory.hpp (:36-82)
 *   tree/compression_tree.hpp (:29-53)                       CompressionTree over gtsc_tree_*
 *   optimizer/path_generator.hpp (:26-31)                    PathGenerator
 *   optimizer/compression_optimizer.hpp (:42-46)             CompressionOptimizer over gtsc_optimizer_*
 *
 * Differences a caller sees: errors are C++ exceptions (ddj::GtscException) instead of exit(1);
 * every call takes an optional CUDA stream (the reference always uses the default stream);
 * CompressionTree holds a node list (pre-order (encoding, data type) pairs, every leaf `none`)
 * instead of node objects.  Data type codes are this library's (GTSC_CHAR .. GTSC_DOUBLE).
 */
#ifndef GTSC_DDJ_HPP_
#define GTSC_DDJ_HPP_

#include "../gtsc.h"

#include <algorithm>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace ddj {

enum class EncodingType : int16_t {
    delta = GTSC_DELTA, afl = GTSC_AFL, scale = GTSC_SCALE, rle = GTSC_RLE, dict = GTSC_DICT,
    unique = GTSC_UNIQUE, patch = GTSC_PATCH, none = GTSC_NONE, floatToInt = GTSC_FLOAT_TO_INT,
    constData = GTSC_CONST, gfc = GTSC_GFC
};

enum class DataType : int16_t {
    d_char = GTSC_CHAR, d_short = GTSC_SHORT, d_int = GTSC_INT, d_time = GTSC_TIME, d_float = GTSC_FLOAT,
    d_double = GTSC_DOUBLE
};

inline size_t GetDataTypeSize(DataType t) { return (size_t)gtsc_dtype_size((int32_t)t); }

struct GtscException : std::runtime_error {
    gtsc_status status;
    GtscException(gtsc_status s, const std::string &what)
        : std::runtime_error(what + ": " + gtsc_last_error()), status(s)
    {
    }
};

inline void Check(gtsc_status s, const char *what)
{
    if (s != GTSC_OK) throw GtscException(s, what);
}

// ------------------------------------------------------------------------------ device buffers

// An owned device array of T (size() counts elements, as in core/cuda_ptr.hpp).
template <typename T>
class CudaPtr {
public:
    CudaPtr() = default;
    explicit CudaPtr(size_t size) : _bytes(size * sizeof(T))
    {
        void *p = nullptr;
        if (_bytes) Check(gtsc_malloc(&p, _bytes, nullptr), "gtsc_malloc");
        _pointer = (T *)p;
    }
    // adopts a library-owned buffer
    CudaPtr(T *pointer, size_t bytes, bool adopt) : _pointer(pointer), _bytes(bytes), _owned(adopt) {}
    ~CudaPtr() { release(); }
    CudaPtr(const CudaPtr &) = delete;
    CudaPtr &operator=(const CudaPtr &) = delete;

    T *get() { return _pointer; }
    size_t size() const { return _bytes / sizeof(T); }
    size_t bytes() const { return _bytes; }

    void fillFromHost(const T *host, size_t size)
    {
        reset(size);
        if (_bytes) Check(gtsc_memcpy(_pointer, host, _bytes, 1, nullptr), "gtsc_memcpy h2d");
    }
    std::vector<T> copyToHost() const
    {
        std::vector<T> out(size());
        if (_bytes) Check(gtsc_memcpy(out.data(), _pointer, _bytes, 2, nullptr), "gtsc_memcpy d2h");
        return out;
    }
    void reset(size_t size)
    {
        release();
        _bytes = size * sizeof(T);
        void *p = nullptr;
        if (_bytes) Check(gtsc_malloc(&p, _bytes, nullptr), "gtsc_malloc");
        _pointer = (T *)p;
        _owned = true;
    }
    // gives the pointer to another CudaPtr (MoveSharedCudaPtr)
    T *disown()
    {
        _owned = false;
        return _pointer;
    }

    static std::shared_ptr<CudaPtr<T>> make_shared() { return std::make_shared<CudaPtr<T>>(); }
    static std::shared_ptr<CudaPtr<T>> make_shared(size_t size) { return std::make_shared<CudaPtr<T>>(size); }

private:
    void release()
    {
        if (_pointer && _owned) gtsc_free(_pointer, nullptr);
        _pointer = nullptr;
        _bytes = 0;
    }
    T *_pointer = nullptr;
    size_t _bytes = 0;
    bool _owned = true;
};

template <typename T> using SharedCudaPtr = std::shared_ptr<CudaPtr<T>>;
template <typename T> using SharedCudaPtrVector = std::vector<SharedCudaPtr<T>>;

// a view of the same device bytes as another element type (shares ownership)
template <typename From, typename To>
SharedCudaPtr<To> CastSharedCudaPtr(SharedCudaPtr<From> data)
{
    return std::reinterpret_pointer_cast<CudaPtr<To>>(data);
}

// takes the bytes over into a new CudaPtr of another element type; `data` is left empty
template <typename From, typename To>
SharedCudaPtr<To> MoveSharedCudaPtr(SharedCudaPtr<From> data)
{
    const size_t bytes = data->bytes();
    return std::make_shared<CudaPtr<To>>((To *)data->disown(), bytes, true);
}

namespace detail {
inline SharedCudaPtr<char> adopt(const gtsc_buffer &b)
{
    return std::make_shared<CudaPtr<char>>((char *)b.ptr, (size_t)b.bytes, true);
}
}  // namespace detail

// ----------------------------------------------------------------------------------- encodings

class Encoding {
public:
    Encoding(EncodingType t) : _type(t), _code((int32_t)t) {}
    // `code`: the library's encoding code when it differs from the type (GTSC_PATCH_OUTSIDE)
    Encoding(EncodingType t, int32_t code) : _type(t), _code(code) {}
    virtual ~Encoding() = default;

    SharedCudaPtrVector<char> Encode(SharedCudaPtr<char> data, DataType type, void *stream = nullptr)
    {
        gtsc_buffer out[3];
        uint32_t n = 0;
        Check(gtsc_encode(_code, (int32_t)type, data ? data->get() : nullptr, data ? data->bytes() : 0, out,
                          &n, stream),
              "Encode");
        SharedCudaPtrVector<char> r;
        for (uint32_t i = 0; i < n; i++) r.push_back(detail::adopt(out[i]));
        return r;
    }

    SharedCudaPtr<char> Decode(SharedCudaPtrVector<char> input, DataType type, void *stream = nullptr)
    {
        gtsc_buffer in[3] = {};
        const uint32_t n = (uint32_t)std::min<size_t>(input.size(), 3);
        for (uint32_t i = 0; i < n; i++) in[i] = gtsc_buffer{input[i]->get(), input[i]->bytes()};
        gtsc_buffer out{};
        Check(gtsc_decode(_code, (int32_t)type, in, n, &out, stream), "Decode");
        return detail::adopt(out);
    }

    unsigned int GetNumberOfResults() const
    {
        switch (_type) {
        case EncodingType::rle: case EncodingType::dict: case EncodingType::patch: case EncodingType::gfc: return 2;
        case EncodingType::none: return 0;
        default: return 1;
        }
    }

    std::vector<DataType> GetReturnTypes(DataType type) const
    {
        if (_type == EncodingType::rle) return {DataType::d_int, type};
        if (_type == EncodingType::floatToInt) return {DataType::d_int};
        std::vector<DataType> r(GetNumberOfResults(), type);
        return r;
    }

    size_t GetMetadataSize(SharedCudaPtr<char> data, DataType type, void *stream = nullptr)
    {
        uint64_t m = 0, d = 0;
        Check(gtsc_predict_sizes(_code, (int32_t)type, data->get(), data->bytes(), &m, &d, stream),
              "GetMetadataSize");
        return m;
    }

    size_t GetCompressedSize(SharedCudaPtr<char> data, DataType type, void *stream = nullptr)
    {
        uint64_t m = 0, d = 0;
        Check(gtsc_predict_sizes(_code, (int32_t)type, data->get(), data->bytes(), &m, &d, stream),
              "GetCompressedSize");
        return d;
    }

    static inline double GetCompressionRatio(size_t inputSize, size_t outputSize)
    {
        if (outputSize == 0 || outputSize > inputSize) return 1.0;
        return (double)inputSize / (double)outputSize;
    }

    EncodingType GetType() const { return _type; }
    // the code this encoding passes to the library (the tree node list entry for it)
    int32_t GetCode() const { return _code; }

private:
    EncodingType _type;
    int32_t _code;
};

using SharedEncodingPtr = std::shared_ptr<Encoding>;

class EncodingFactory {
public:
    EncodingFactory(DataType dt, EncodingType et) : dataType(dt), encodingType(et) {}
    virtual ~EncodingFactory() = default;
    virtual SharedEncodingPtr Get() { return std::make_shared<Encoding>(encodingType); }
    virtual SharedEncodingPtr Get(SharedCudaPtr<char>) { return Get(); }
    DataType dataType;
    EncodingType encodingType;
};

using SharedEncodingFactoryPtr = std::shared_ptr<EncodingFactory>;

// compression/patch/patch_type.hpp
enum class PatchType { outside, lower };

// PatchEncodingFactory<T> (compression/patch/patch_encoding_factory.hpp:20-57).  The encoding's
// bounds come from the data's min / max, which the library computes on the device inside
// gtsc_encode, so Get(data) only picks the variant.  Get() without data is the reference's
// OutsidePatchEncoding(0, 0, 0) placeholder: use it to decode (both variants decode alike).
class PatchEncodingFactory : public EncodingFactory {
public:
    PatchEncodingFactory(DataType dt, PatchType pt) : EncodingFactory(dt, EncodingType::patch), patchType(pt) {}
    SharedEncodingPtr Get() override { return std::make_shared<Encoding>(EncodingType::patch, GTSC_PATCH_OUTSIDE); }
    SharedEncodingPtr Get(SharedCudaPtr<char> data) override
    {
        if (!data || data->bytes() == 0) return Get();
        return std::make_shared<Encoding>(EncodingType::patch,
                                          patchType == PatchType::outside ? GTSC_PATCH_OUTSIDE : GTSC_PATCH);
    }
    PatchType patchType;
};

class DefaultEncodingFactory {
public:
    // default_encoding_factory.hpp:36-82: patch is the lower variant
    static SharedEncodingFactoryPtr Get(EncodingType encodingType, DataType dataType)
    {
        if (encodingType == EncodingType::patch) return std::make_shared<PatchEncodingFactory>(dataType, PatchType::lower);
        return std::make_shared<EncodingFactory>(dataType, encodingType);
    }
};

// -------------------------------------------------------------------------------- trees

using Path = std::vector<EncodingType>;
using PathList = std::vector<Path>;

class CompressionTree {
public:
    CompressionTree() = default;
    // a single-node tree, Fix()ed
    CompressionTree(EncodingType et, DataType dt) { *this = FromPath({et}, dt, true); }

    static CompressionTree FromNodes(std::vector<int16_t> nodes)
    {
        CompressionTree t;
        t._nodes = std::move(nodes);
        return t;
    }

    SharedCudaPtr<char> Compress(SharedCudaPtr<char> data, void *stream = nullptr)
    {
        gtsc_buffer blob{};
        Check(gtsc_tree_compress(_nodes.data(), (int32_t)(_nodes.size() / 2), data->get(), data->bytes(), &blob,
                                 stream),
              "CompressionTree::Compress");
        return detail::adopt(blob);
    }

    SharedCudaPtr<char> Decompress(SharedCudaPtr<char> data, void *stream = nullptr)
    {
        gtsc_buffer out{};
        int32_t dt = 0;
        Check(gtsc_tree_decompress(data->get(), data->bytes(), &out, &dt, stream), "CompressionTree::Decompress");
        return detail::adopt(out);
    }

    size_t GetPredictedSizeAfterCompression(SharedCudaPtr<char> data, DataType, void *stream = nullptr)
    {
        uint64_t sz = 0;
        Check(gtsc_tree_predict_size(_nodes.data(), (int32_t)(_nodes.size() / 2), data->get(), data->bytes(), &sz,
                                     stream),
              "GetPredictedSizeAfterCompression");
        return sz;
    }

    const std::vector<int16_t> &Nodes() const { return _nodes; }
    std::string ToString() const
    {
        static const char *names[] = {"delta", "afl", "scale", "rle", "dict", "unique", "patch", "none",
                                      "floatToInt", "constData", "gfc", "patch"};
        std::string s;
        for (size_t i = 0; i < _nodes.size(); i += 2) s += std::string(names[_nodes[i]]) + ",";
        return s;
    }

    // PathGenerator::GenerateTree; `fix` also gives a bare single node its `none` children
    static CompressionTree FromPath(const Path &path, DataType dt, bool fix = false)
    {
        std::vector<int16_t> p;
        for (auto e : path) p.push_back((int16_t)e);
        if (fix) {
            const unsigned r = Encoding(path.back()).GetNumberOfResults();
            for (unsigned i = 0; i < r; i++) p.push_back((int16_t)EncodingType::none);
        }
        std::vector<int16_t> nodes(2 * 1024);
        int32_t n = 0;
        Check(gtsc_tree_from_path(p.data(), (int32_t)p.size(), (int32_t)dt, nodes.data(), 1024, &n),
              "GenerateTree");
        nodes.resize(2 * (size_t)n);
        return FromNodes(std::move(nodes));
    }

private:
    std::vector<int16_t> _nodes;
};

class PathGenerator {
public:
    // optimizer/path_generator.cpp:20-68: 6 prefixes x 5 terminal shapes
    PathList GeneratePaths() const
    {
        using E = EncodingType;
        const PathList first = {{}, {E::floatToInt}, {E::delta}, {E::scale}, {E::delta, E::floatToInt},
                                {E::scale, E::floatToInt}};
        const PathList second = {{E::dict, E::afl, E::none, E::afl, E::none}, {E::constData, E::afl, E::none},
                                 {E::rle, E::afl, E::none, E::afl, E::none}, {E::afl, E::none},
                                 {E::patch, E::afl, E::none, E::afl, E::none}};
        PathList out;
        for (auto &a : first)
            for (auto &b : second) {
                Path p = a;
                p.insert(p.end(), b.begin(), b.end());
                out.push_back(p);
            }
        return out;
    }
    CompressionTree GenerateTree(const Path &path, DataType type) const { return CompressionTree::FromPath(path, type); }
};

// --------------------------------------------------------------------------------- optimizer

class CompressionOptimizer {
public:
    CompressionOptimizer() = default;
    ~CompressionOptimizer()
    {
        if (_opt) gtsc_optimizer_destroy(_opt);
    }
    CompressionOptimizer(const CompressionOptimizer &) = delete;
    CompressionOptimizer &operator=(const CompressionOptimizer &) = delete;

    // OptimizeTree: the smallest predicted size over the 30 generated paths
    CompressionTree OptimizeTree(SharedCudaPtr<char> data, DataType type, void *stream = nullptr)
    {
        std::vector<int16_t> nodes(2 * 1024);
        int32_t n = 0;
        uint64_t sz = 0;
        Check(gtsc_optimize_tree((int32_t)type, data->get(), data->bytes(), nodes.data(), 1024, &n, &sz, stream),
              "OptimizeTree");
        nodes.resize(2 * (size_t)n);
        return CompressionTree::FromNodes(std::move(nodes));
    }

    // CompressData: one part of a column (all parts of one optimizer share its data type)
    SharedCudaPtr<char> CompressData(SharedCudaPtr<char> dataPart, DataType type, void *stream = nullptr)
    {
        if (!_opt) Check(gtsc_optimizer_create((int32_t)type, &_opt), "CompressionOptimizer");
        gtsc_buffer blob{};
        int32_t full = 0, corrected = 0;
        Check(gtsc_optimizer_compress(_opt, dataPart->get(), dataPart->bytes(), &blob, &full, &corrected, stream),
              "CompressData");
        _parts++;
        return detail::adopt(blob);
    }

    // GetOptimalTree()->GetTree()
    CompressionTree GetOptimalTree() const
    {
        if (!_opt) throw std::runtime_error("CompressionOptimizer: no part compressed yet");
        std::vector<int16_t> nodes(2 * 1024);
        int32_t n = 0;
        Check(gtsc_optimizer_tree(_opt, nodes.data(), nullptr, 1024, &n), "GetOptimalTree");
        nodes.resize(2 * (size_t)n);
        return CompressionTree::FromNodes(std::move(nodes));
    }

    // GetStatistics(): the edge statistics (owned by the optimizer)
    gtsc_edge_stats *GetStatistics()
    {
        if (!_opt) return nullptr;
        gtsc_edge_stats *s = nullptr;
        Check(gtsc_optimizer_statistics(_opt, &s), "GetStatistics");
        return s;
    }

    size_t PartsProcessed() const { return _parts; }

private:
    gtsc_optimizer *_opt = nullptr;
    size_t _parts = 0;
};

}  // namespace ddj

#endif  // GTSC_DDJ_HPP_
