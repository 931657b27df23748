/*
 * ref_afl_shim.cu -- exposes the reference's own AFL host implementation for parity checks.
 *
 * TEST INFRASTRUCTURE ONLY.  This file contains no reference code: it includes the reference's
 * src/compression/afl/afl_gpu.cu from the reference tree (the include path is given by
 * oracle/Makefile) and wraps the explicitly instantiated host entry points
 * run_afl_compress_cpu<T,1> / run_afl_decompress_cpu<T,1> (afl_gpu.cu:6-65, 253-269) in
 * extern "C" functions, as well as the aligned layout run_afl_compress_cpu<T,32> /
 * run_afl_decompress_cpu<T,32> and the random-access afl_decompress_base_value_gpu<T,W> (host
 * callable), and the reference's GPU launchers run_afl_compress_gpu / run_afl_decompress_gpu /
 * run_afl_decompress_value_gpu <int, 1|32> (afl_gpu.cu:67-89), compiled for sm_100a, to time the
 * reference's own kernels on the B200.  The output goes to oracle/_ref/, which is never committed.
 *
 * The reference's decompress kernels read the packed word at a lane's first position even when that
 * position is the column length (afl_gpu.cu:172-174), one word past a tight buffer; callers pad the
 * packed buffer so every read stays inside it.
 *
 * The reference host path masks with NBITSTOMASK(n) = (1<<n)-1 (core/cuda_macros.cuh:6), which is
 * undefined for n equal to the word width, so callers only use bit widths below the word width.
 */
#include "compression/afl/afl_gpu.cu"

extern "C" {

void ref_afl_compress_char(unsigned b, char *data, char *out, unsigned long n, unsigned long words)
{ run_afl_compress_cpu<char, 1>(b, data, out, n, words); }
void ref_afl_compress_short(unsigned b, short *data, short *out, unsigned long n, unsigned long words)
{ run_afl_compress_cpu<short, 1>(b, data, out, n, words); }
void ref_afl_compress_int(unsigned b, int *data, int *out, unsigned long n, unsigned long words)
{ run_afl_compress_cpu<int, 1>(b, data, out, n, words); }
void ref_afl_compress_long(unsigned b, long *data, long *out, unsigned long n, unsigned long words)
{ run_afl_compress_cpu<long, 1>(b, data, out, n, words); }

void ref_afl_decompress_char(unsigned b, char *comp, char *out, unsigned long n)
{ run_afl_decompress_cpu<char, 1>(b, comp, out, n); }
void ref_afl_decompress_short(unsigned b, short *comp, short *out, unsigned long n)
{ run_afl_decompress_cpu<short, 1>(b, comp, out, n); }
void ref_afl_decompress_int(unsigned b, int *comp, int *out, unsigned long n)
{ run_afl_decompress_cpu<int, 1>(b, comp, out, n); }
void ref_afl_decompress_long(unsigned b, long *comp, long *out, unsigned long n)
{ run_afl_decompress_cpu<long, 1>(b, comp, out, n); }


void ref_afl32_compress_int(unsigned b, int *data, int *out, unsigned long n, unsigned long words)
{ run_afl_compress_cpu<int, 32>(b, data, out, n, words); }
void ref_afl32_compress_long(unsigned b, long *data, long *out, unsigned long n, unsigned long words)
{ run_afl_compress_cpu<long, 32>(b, data, out, n, words); }
void ref_afl32_compress_short(unsigned b, short *data, short *out, unsigned long n, unsigned long words)
{ run_afl_compress_cpu<short, 32>(b, data, out, n, words); }
void ref_afl32_decompress_int(unsigned b, int *comp, int *out, unsigned long n)
{ run_afl_decompress_cpu<int, 32>(b, comp, out, n); }
void ref_afl32_decompress_long(unsigned b, long *comp, long *out, unsigned long n)
{ run_afl_decompress_cpu<long, 32>(b, comp, out, n); }
void ref_afl32_decompress_short(unsigned b, short *comp, short *out, unsigned long n)
{ run_afl_decompress_cpu<short, 32>(b, comp, out, n); }

// element i of a packed int stream, FL (omega 1) or aligned (omega 32)
int ref_afl_value_int(unsigned b, int omega, int *comp, unsigned long i)
{ return omega == 32 ? afl_decompress_base_value_gpu<int, 32>(b, comp, i) : afl_decompress_base_value_gpu<int, 1>(b, comp, i); }
long ref_afl_value_long(unsigned b, int omega, long *comp, unsigned long i)
{ return omega == 32 ? afl_decompress_base_value_gpu<long, 32>(b, comp, i) : afl_decompress_base_value_gpu<long, 1>(b, comp, i); }


// the reference's GPU kernels (legacy default stream); returns the launch status
int ref_afl_gpu_compress_int(int omega, unsigned b, int *d_in, int *d_out, unsigned long n, unsigned long words)
{
    if (omega == 32) run_afl_compress_gpu<int, 32>(b, d_in, d_out, n, words);
    else run_afl_compress_gpu<int, 1>(b, d_in, d_out, n, words);
    return (int)cudaGetLastError();
}
int ref_afl_gpu_decompress_int(int omega, unsigned b, int *d_comp, int *d_out, unsigned long n)
{
    if (omega == 32) run_afl_decompress_gpu<int, 32>(b, d_comp, d_out, n);
    else run_afl_decompress_gpu<int, 1>(b, d_comp, d_out, n);
    return (int)cudaGetLastError();
}
int ref_afl_gpu_values_int(int omega, unsigned b, int *d_comp, int *d_out, unsigned long n)
{
    if (omega == 32) run_afl_decompress_value_gpu<int, 32>(b, d_comp, d_out, n);
    else run_afl_decompress_value_gpu<int, 1>(b, d_comp, d_out, n);
    return (int)cudaGetLastError();
}

}
