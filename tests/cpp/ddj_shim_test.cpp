// Reference-style client code against include/gtsc/ddj.hpp: the calls and checks mirror the
// reference's own tests (compression/*/ *_unittest.cpp, optimizer/optimizer_unittest.cpp,
// test/compression_unittest_base.hpp), written against the ddj names.  Exit code 0 = all passed.
#include "gtsc/ddj.hpp"

#include <cstdio>
#include <random>

using namespace ddj;

static int failures = 0;
#define EXPECT(c)                                                        \
    do {                                                                 \
        if (!(c)) {                                                      \
            std::fprintf(stderr, "%s:%d: expected %s\n", __FILE__, __LINE__, #c); \
            failures++;                                                  \
        }                                                                \
    } while (0)

template <typename T>
static SharedCudaPtr<T> device(const std::vector<T> &h)
{
    auto p = CudaPtr<T>::make_shared();
    p->fillFromHost(h.data(), h.size());
    return p;
}

template <typename T>
static bool same(SharedCudaPtr<char> a, const std::vector<T> &b)
{
    auto h = CastSharedCudaPtr<char, T>(a)->copyToHost();
    return h == b;
}

static std::vector<int> random_ints(size_t n, int lo, int hi, unsigned seed)
{
    std::mt19937 g(seed);
    std::uniform_int_distribution<int> d(lo, hi);
    std::vector<int> v(n);
    for (auto &x : v) x = d(g);
    return v;
}

int main()
{
    const auto ints = random_ints(10000, 10, 1000, 1);
    std::vector<int> runs;
    for (int i = 0; i < 10000; i++) runs.push_back((i / 37) % 11);
    std::vector<float> floats;
    for (int i = 0; i < 10000; i++) floats.push_back((float)((i % 500) * 0.25));

    // Encode / Decode for each encoding (the per-encoding round-trip tests)
    const EncodingType all[] = {EncodingType::afl, EncodingType::delta, EncodingType::scale, EncodingType::rle,
                                EncodingType::dict, EncodingType::unique, EncodingType::patch, EncodingType::none,
                                EncodingType::floatToInt, EncodingType::constData, EncodingType::gfc};
    for (EncodingType et : all) {
        auto enc = DefaultEncodingFactory::Get(et, DataType::d_int)->Get();
        auto data = CastSharedCudaPtr<int, char>(device(ints));
        auto encoded = enc->Encode(data, DataType::d_int);
        EXPECT(encoded.size() == enc->GetNumberOfResults() + 1 || et == EncodingType::none);
        EXPECT(same(enc->Decode(encoded, DataType::d_int), ints));
    }
    for (EncodingType et : {EncodingType::gfc, EncodingType::floatToInt, EncodingType::afl, EncodingType::dict}) {
        auto enc = DefaultEncodingFactory::Get(et, DataType::d_float)->Get();
        auto data = CastSharedCudaPtr<float, char>(device(floats));
        EXPECT(same(enc->Decode(enc->Encode(data, DataType::d_float), DataType::d_float), floats));
    }

    // PatchEncodingFactory with either patch type (patch_encoding_factory.hpp:40-57): Get(data)
    // encodes, Get() decodes either variant
    for (PatchType pt : {PatchType::outside, PatchType::lower}) {
        PatchEncodingFactory f(DataType::d_int, pt);
        auto data = CastSharedCudaPtr<int, char>(device(ints));
        auto enc = f.Get(data);
        EXPECT(enc->GetType() == EncodingType::patch);
        auto encoded = enc->Encode(data, DataType::d_int);
        EXPECT(encoded.size() == 3);
        EXPECT(same(f.Get()->Decode(encoded, DataType::d_int), ints));
    }

    // TestGetMetadataSize / TestGetCompressedSize (test/compression_unittest_base.hpp:32-54)
    for (EncodingType et : {EncodingType::rle, EncodingType::dict, EncodingType::constData, EncodingType::delta,
                            EncodingType::afl, EncodingType::unique}) {
        auto enc = DefaultEncodingFactory::Get(et, DataType::d_int)->Get();
        auto data = CastSharedCudaPtr<int, char>(device(runs));
        auto encoded = enc->Encode(data, DataType::d_int);
        size_t rest = 0;
        for (size_t i = 1; i < encoded.size(); i++) rest += encoded[i]->bytes();
        EXPECT(enc->GetMetadataSize(data, DataType::d_int) == encoded[0]->bytes());
        EXPECT(enc->GetCompressedSize(data, DataType::d_int) == rest);
    }

    // PathGenerator + CompressionTree (optimizer/optimizer_unittest.cpp:28-81)
    PathGenerator gen;
    auto paths = gen.GeneratePaths();
    EXPECT(paths.size() == 30);
    for (auto &path : paths) {
        auto tree = gen.GenerateTree(path, DataType::d_int);
        auto data = CastSharedCudaPtr<int, char>(device(runs));
        auto compressed = tree.Compress(data);
        EXPECT(tree.GetPredictedSizeAfterCompression(data, DataType::d_int) == compressed->bytes());
        CompressionTree decompression;
        EXPECT(same(decompression.Decompress(compressed), runs));
    }

    // CompressionOptimizer::OptimizeTree and CompressData over parts (optimizer_unittest.cpp:83-352)
    {
        CompressionOptimizer opt;
        auto data = CastSharedCudaPtr<int, char>(device(runs));
        auto tree = opt.OptimizeTree(data, DataType::d_int);
        EXPECT(tree.Compress(data)->bytes() < data->bytes());
    }
    {
        CompressionOptimizer opt;
        std::vector<std::vector<int>> parts;
        std::vector<SharedCudaPtr<char>> blobs;
        for (int p = 0; p < 12; p++) {
            parts.push_back(p % 3 == 2 ? random_ints(20000, 0, 100, 10 + p) : std::vector<int>(runs.begin(), runs.end()));
            blobs.push_back(opt.CompressData(CastSharedCudaPtr<int, char>(device(parts.back())), DataType::d_int));
        }
        EXPECT(opt.PartsProcessed() == 12);
        EXPECT(!opt.GetOptimalTree().Nodes().empty());
        CompressionTree decompression;
        for (size_t p = 0; p < parts.size(); p++) EXPECT(same(decompression.Decompress(blobs[p]), parts[p]));
    }

    // MoveSharedCudaPtr takes the bytes over
    {
        auto a = device(ints);
        auto b = MoveSharedCudaPtr<int, char>(a);
        EXPECT(b->bytes() == ints.size() * sizeof(int));
        EXPECT(same(b, ints));
    }

    if (failures) {
        std::fprintf(stderr, "ddj shim: %d check(s) failed\n", failures);
        return 1;
    }
    std::printf("ddj shim: all checks passed\n");
    return 0;
}
