/*
 * ref_afl_shim.cu -- exposes the reference's own AFL host implementation for parity checks.
 *
 * TEST INFRASTRUCTURE ONLY.  This file contains no reference code: it includes the reference's
 * src/compression/afl/afl_gpu.cu from the reference tree (the include path is given by
 * oracle/Makefile) and wraps the explicitly instantiated host entry points
 * run_afl_compress_cpu<T,1> / run_afl_decompress_cpu<T,1> (afl_gpu.cu:6-65, 253-269) in
 * extern "C" functions.  The output goes to oracle/_ref/, which is never committed.
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

}
