/*
 * libzkp_gen.so: seeded synthetic inputs on the device (no counterpart in the reference, whose
 * tests draw from an OS random source).  Byte-identical to the CPU oracle's generator, so
 * benchmark inputs need no host round trip.
 */
#ifndef ZKP_GEN_H
#define ZKP_GEN_H
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

/* out_d[i] = Montgomery form of the (start + i)-th uniform Fr element of `seed`, i < n. */
cudaError_t zkp_gen_fr(unsigned long long seed, unsigned long long start, unsigned long long n,
                       unsigned int *out_d, cudaStream_t stream);

/* out_d[i] = k * G (affine, Montgomery), k the (start + i)-th canonical element of `seed`;
 * table_d is caller scratch of 32 * 256 * 64 bytes for the fixed-base table. */
cudaError_t zkp_gen_points(unsigned long long seed, unsigned long long start, unsigned long long n,
                           unsigned int *table_d, unsigned int *out_d, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif
