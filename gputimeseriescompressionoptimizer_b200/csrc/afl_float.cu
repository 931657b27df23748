// afl_float.cu -- the float path of AflEncoding (compression/afl/afl_encoding.cu:116-254): a float
// column is split into its 23-bit mantissas, 8-bit exponents and signs; mantissas and exponents
// are AFL packed as int32 columns, the signs kept as one byte or a packed stencil.
#include "kernels.hpp"
#include "vec.cuh"

namespace gtsc {

namespace {

// one thread = 8 floats = one stencil byte (Stencil::pack: the last element fills the last byte)
__global__ void k_float_split(const uint8_t *__restrict__ in, uint64_t n, int32_t *__restrict__ mant,
                              int32_t *__restrict__ expo, uint8_t *__restrict__ stencil, uint32_t *flags)
{
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t base = 8 * t;
    uint32_t any1 = 0, any0 = 0;
    if (base < n) {
        uint32_t bits = 0;
        for (int j = 0; j < 8; j++) {
            const uint64_t i = base + j < n ? base + j : n - 1;
            const uint32_t u = (uint32_t)ld_unaligned<4>(in + 4 * i);
            const uint32_t sg = u >> 31;
            bits |= sg << j;
            if (base + j < n) {
                mant[i] = (int32_t)(u & 0x7fffffu);
                expo[i] = (int32_t)((u >> 23) & 0xffu);
                any1 |= sg;
                any0 |= sg ^ 1u;
            }
        }
        stencil[1 + t] = (uint8_t)bits;
    }
    if (t == 0) stencil[0] = (uint8_t)(int8_t)(n % 8);
    any1 = __any_sync(0xffffffffu, any1 != 0);
    any0 = __any_sync(0xffffffffu, any0 != 0);
    if ((threadIdx.x & 31) == 0) {
        if (any1) atomicOr(flags, 1u);
        if (any0) atomicOr(flags, 2u);
    }
}

// float i = sign | exponent[i] << 23 | mantissa[i]; sign from the stencil or the constant `fill`
__global__ void k_float_compose(const int32_t *__restrict__ mant, const int32_t *__restrict__ expo,
                                const uint8_t *__restrict__ stencil, int fill, uint64_t n, uint32_t *__restrict__ out)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t sg = stencil ? (stencil[i >> 3] >> (i & 7)) & 1u : (uint32_t)fill;
    out[i] = (sg << 31) | (((uint32_t)expo[i] & 0xffu) << 23) | ((uint32_t)mant[i] & 0x7fffffu);
}

}  // namespace

void launch_float_split(const uint8_t *in, uint64_t n, int32_t *mant, int32_t *expo, uint8_t *stencil,
                        uint32_t *flags, cudaStream_t s)
{
    if (!n) return;
    const uint64_t threads = (n + 7) / 8;
    k_float_split<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(in, n, mant, expo, stencil, flags);
    GTSC_CUDA(cudaGetLastError());
}

void launch_float_compose(const int32_t *mant, const int32_t *expo, const uint8_t *stencil, int fill, uint64_t n,
                          uint32_t *out, cudaStream_t s)
{
    if (!n) return;
    k_float_compose<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(mant, expo, stencil, fill, n, out);
    GTSC_CUDA(cudaGetLastError());
}

}  // namespace gtsc
