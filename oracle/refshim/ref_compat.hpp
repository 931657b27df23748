// Test infrastructure: included before every reference source that oracle/Makefile compiles
// (nvcc -include), for what the reference took from older toolchains:
//  - it calls std::abs<T>(x) with an explicit template argument
//    (compression/scale/scale_encoding.cu:50), which the standard library here does not declare;
//    the template below gives that call the meaning of the integer abs of x's promoted value
//    (std::abs(int) / std::abs(long)), wrapping at the type's minimum as those do on x86: the
//    magnitude for char and short, INT_MIN / LONG_MIN for the minimum of int / long;
//  - util/splitter/splitter.cu:111 calls thrust::count and tree/compression_statistics.cpp:121
//    uses std::stringstream without including their headers, which the headers here no longer
//    bring in through the others;
//  - CUDA_ASSERT_RETURN (core/macros.h:8-14) ends the process with exit(1) on any CUDA error; here
//    exit throws (ref_exit, oracle/ref_enc_shim.cu), so that a failing call of the reference
//    returns an error to the test that made it instead of ending the test run.
#pragma once
#include <cstdlib>
#include <cmath>
#include <sstream>
#ifdef __CUDACC__
#include <thrust/count.h>
#endif
#include <type_traits>
namespace std {
template <class T>
inline auto abs(T v) -> decltype(+v)
{
    using P = decltype(+v);
    if constexpr (std::is_integral<P>::value) {
        using U = typename std::make_unsigned<P>::type;
        return v < T(0) ? (P)(U(0) - U(P(v))) : P(v);
    } else {
        return v < T(0) ? P(-v) : P(v);
    }
}
}  // namespace std

#include <stdlib.h>
[[noreturn]] void ref_exit(int status);
#define exit(status) ref_exit(status)
