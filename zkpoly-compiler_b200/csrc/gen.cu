// libzkp_gen.so: seeded synthetic inputs generated on the device.
//
// Element i of seed s is the i-th output of a counter-based generator: candidate limbs are the
// SplitMix64 finalizer of (mix(s) + ctr * golden) with ctr = (i << 8) | (attempt << 2) | limb,
// the top limb masked to 62 bits, candidates >= r rejected.  Nothing depends on other elements,
// so the device and the CPU oracle produce the same bytes.  Points are P_i = k_i * G with k_i
// drawn from the same generator and G = (1, 2), built from a fixed-base table of
// d * 2^(8w) * G (32 x 256 affine points) with 32 mixed additions per point.
#include <cuda_runtime.h>

#include "../../include/zkp_gen.h"
#include "common.cuh"
#include "curve.cuh"

namespace zk {
namespace gen {

ZK_DI u64 mix64(u64 z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

ZK_DI bool lt_r(const u64 *c) {
    const u64 R[4] = {0x43e1f593f0000001ull, 0x2833e84879b97091ull, 0xb85045b68181585dull, 0x30644e72e131a029ull};
    for (int i = 3; i >= 0; i--)
        if (c[i] != R[i]) return c[i] < R[i];
    return false;
}

// canonical integer k_i (as 8 u32 limbs)
ZK_DI Fr raw(u64 seed, u64 idx) {
    const u64 s = mix64(seed ^ 0x6a09e667f3bcc909ull);
    u64 c[4];
    for (u64 attempt = 0; attempt < 64; attempt++) {
        for (u64 k = 0; k < 4; k++) c[k] = mix64(s + ((idx << 8) | (attempt << 2) | k) * 0x9E3779B97F4A7C15ull);
        c[3] &= 0x3FFFFFFFFFFFFFFFull;
        if (lt_r(c)) {
            Fr r;
            for (int k = 0; k < 4; k++) {
                r.v[2 * k] = (u32)c[k];
                r.v[2 * k + 1] = (u32)(c[k] >> 32);
            }
            return r;
        }
    }
    return Fr::zero();
}

__global__ void __launch_bounds__(256) fr_kernel(u64 seed, u64 start, u64 n, u32 *out) {
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        Fr::to_mont(raw(seed, start + i)).store(out + i * 8);
}

// table[w * 256 + d] = d * 2^(8w) * G (affine); d = 0 slot holds the identity
__global__ void __launch_bounds__(128) table_kernel(u32 *table) {
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 32 * 256) return;
    const u32 w = t / 256, d = t % 256;
    G1A g;
    Fq one_int = Fq::zero(), two_int = Fq::zero();
    one_int.v[0] = 1;
    two_int.v[0] = 2;
    g.x = Fq::to_mont(one_int);
    g.y = Fq::to_mont(two_int);
    G1X base = G1X::from_affine(g);
    for (u32 k = 0; k < 8 * w; k++) base = g1_dbl(base);
    G1X p = g1_mul_u64(base, d);
    g1_to_affine(p).store(table + (u64)t * 16);
}

__global__ void __launch_bounds__(128) points_kernel(u64 seed, u64 start, u64 n, const u32 *table, u32 *out) {
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        Fr k = raw(seed, start + i);
        G1X acc = G1X::identity();
        for (u32 w = 0; w < 32; w++) {
            const u32 d = (k.v[w / 4] >> ((w % 4) * 8)) & 0xffu;
            if (d) acc = g1_madd(acc, G1A::load_nc(table + (u64)(w * 256 + d) * 16));
        }
        g1_to_affine(acc).store(out + i * 16);
    }
}

}  // namespace gen
}  // namespace zk

using namespace zk;

extern "C" cudaError_t zkp_gen_fr(unsigned long long seed, unsigned long long start, unsigned long long n,
                                  unsigned int *out_d, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    ZK_CHECK_ARG(out_d != nullptr);
    const u64 blocks = (n + 255) / 256;
    gen::fr_kernel<<<(u32)(blocks < (u64)num_sms() * 16 ? blocks : (u64)num_sms() * 16), 256, 0, stream>>>(
        seed, start, n, out_d);
    return cudaGetLastError();
}

extern "C" cudaError_t zkp_gen_points(unsigned long long seed, unsigned long long start, unsigned long long n,
                                      unsigned int *table_d, unsigned int *out_d, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    ZK_CHECK_ARG(out_d != nullptr && table_d != nullptr);
    gen::table_kernel<<<(32 * 256 + 127) / 128, 128, 0, stream>>>(table_d);
    ZK_TRY(cudaGetLastError());
    const u64 blocks = (n + 127) / 128;
    gen::points_kernel<<<(u32)(blocks < (u64)num_sms() * 16 ? blocks : (u64)num_sms() * 16), 128, 0, stream>>>(
        seed, start, n, table_d, out_d);
    return cudaGetLastError();
}
