// Env-map preprocessing helpers: bilinear lat-long sampling of directions, and the GGX-lobe blur
// of an env map (prefiltered radiance for a given roughness).
//
// Reference correspondence (zjumsj/diff_envshade, etc.cu):
//   lat-long bilinear lookup             SampleEnvmap (527-583), with config.h's LEFT_TOP_AS_ORIGIN
//                                        (v flipped) and FIX_ENVMAP_SEAM (columns wrap, rows clamp)
//   sample_envmap_forward                SampleEnvmap_Forward (687-705), host 1145-1178
//   blur_envmap_forward                  BlurEnvmap_Forward (603-685), TrowbridgeReitzDistributionSample
//                                        (585-601), host 1103-1143
//
// The blur draws its samples from curand's XORWOW generator with the reference's seed (0) and
// subsequence (the output texel), so both produce the same sample directions; each output texel
// averages N_samples lookups of directions drawn from the GGX (Trowbridge-Reitz) distribution
// around the texel's direction: tan^2(theta) = alpha^2 u / (1 - u), phi = 2 pi v.
// sample_envmap_forward writes C x P outputs for a C-channel map (the reference allocates 3 x P
// whatever C is).
#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <stdint.h>

#include "des_internal.h"
#include "des_math.cuh"
#include "diff_envshade_b200.h"

namespace des {
namespace envtools {

// Bilinear lookup of unit direction (x, y, z); channel c of the sample goes to out[c * stride].
__device__ __forceinline__ void lookup(float x, float y, float z, int H, int W, int C, const float* __restrict__ env,
                                       float* __restrict__ out, int64_t stride) {
  float phi = atan2f(z, x);
  if (phi < 0.f) phi += 2 * kPiF;
  if (y < -1.f)
    y = -1.f;
  else if (y > 1.f)
    y = 1.f;
  const float theta = asinf(y);
  const float u = phi / (2 * kPiF);
  const float v = 1.f - (theta / kPiF + 0.5f);  // row 0 of the map is the top
  const float pu = u * W, pv = v * H;
  int x0 = int(floorf(pu - 0.5f)), y0 = int(floorf(pv - 0.5f));
  int x1 = x0 + 1, y1 = y0 + 1;
  const float kx = pu - float(x0) - 0.5f, ky = pv - float(y0) - 0.5f;
  x0 = x0 < 0 ? x0 + W : (x0 >= W ? x0 - W : x0);  // the longitude seam wraps
  x1 = x1 < 0 ? x1 + W : (x1 >= W ? x1 - W : x1);
  y0 = y0 < 0 ? 0 : (y0 >= H ? H - 1 : y0);  // the poles clamp
  y1 = y1 < 0 ? 0 : (y1 >= H ? H - 1 : y1);
  for (int c = 0; c < C; ++c) {
    const float* m = env + (int64_t)c * H * W;
    const float v00 = m[y0 * W + x0], v01 = m[y0 * W + x1], v10 = m[y1 * W + x0], v11 = m[y1 * W + x1];
    out[c * stride] = (1 - ky) * ((1 - kx) * v00 + kx * v01) + ky * ((1 - kx) * v10 + kx * v11);
  }
}

__global__ void __launch_bounds__(256) sample_kernel(int64_t P, int H, int W, int C, const float* __restrict__ q,
                                                     const float* __restrict__ env, float* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  float x = q[i], y = q[P + i], z = q[2 * P + i];
  const float L = sqrtf(x * x + y * y + z * z);
  lookup(x / L, y / L, z / L, H, W, C, env, out + i, P);
}

__device__ __forceinline__ void normalize3(float& x, float& y, float& z) {
  const float L = sqrtf(x * x + y * y + z * z);
  x /= L;
  y /= L;
  z /= L;
}

template <int C>
__global__ void __launch_bounds__(256) blur_kernel(int H, int W, int tH, int tW, int N_samples, float alpha,
                                                   const float* __restrict__ env, float* __restrict__ out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int P = tH * tW;
  if (idx >= P) return;
  const int ih = idx / tW, iw = idx % tW;
  // direction of the output texel's centre (row 0 = top: theta from +y down)
  const float theta = ((ih + 0.5f) / float(tH)) * kPiF;
  const float phi = ((iw + 0.5f) / float(tW)) * 2 * kPiF;
  float st, ct, sp, cp;
  sincosf(theta, &st, &ct);
  sincosf(phi, &sp, &cp);
  float nx = st * cp, ny = ct, nz = st * sp;
  normalize3(nx, ny, nz);
  // tangent frame (tx, ty, n)
  float tx0, tx1, tx2;
  if (fabsf(nx) > 0.9f) {
    tx0 = nz;
    tx1 = 0.f;
    tx2 = -nx;
  } else {
    tx0 = 0.f;
    tx1 = -nz;
    tx2 = ny;
  }
  normalize3(tx0, tx1, tx2);
  float ty0 = ny * tx2 - nz * tx1, ty1 = nz * tx0 - nx * tx2, ty2 = nx * tx1 - ny * tx0;
  normalize3(ty0, ty1, ty2);

  curandState rng;
  curand_init(0, idx, 0, &rng);
  float acc[C], s[C];
#pragma unroll
  for (int c = 0; c < C; ++c) acc[c] = 0.f;
  for (int i = 0; i < N_samples; ++i) {
    const float u0 = curand_uniform(&rng);
    const float u1 = curand_uniform(&rng);
    // GGX half-vector distribution in the local frame
    const float ph = (2 * kPiF) * u1;
    const float tan2 = alpha * alpha * u0 / (1.0f - u0);
    const float cth = 1 / sqrtf(1 + tan2);
    const float sth = sqrtf(fmaxf(1.f - cth * cth, 0.f));
    const float lx = sth * cosf(ph), ly = sth * sinf(ph), lz = cth;
    float dx = tx0 * lx + ty0 * ly + nx * lz;
    float dy = tx1 * lx + ty1 * ly + ny * lz;
    float dz = tx2 * lx + ty2 * ly + nz * lz;
    normalize3(dx, dy, dz);
    lookup(dx, dy, dz, H, W, C, env, s, 1);
#pragma unroll
    for (int c = 0; c < C; ++c) acc[c] += s[c];
  }
#pragma unroll
  for (int c = 0; c < C; ++c) out[(int64_t)c * P + idx] = acc[c] / float(N_samples);
}

inline unsigned blocks_for(int64_t n) { return (unsigned)((n + 255) / 256); }

}  // namespace envtools
}  // namespace des

using namespace des::envtools;

extern "C" {

int des_sample_envmap_forward(int64_t P, int32_t H, int32_t W, int32_t C, const float* query_point,
                              const float* envmap, float* out, des_stream_t stream) {
  if (P < 0 || H <= 0 || W <= 0 || C <= 0 || (P > 0 && (!query_point || !envmap || !out)))
    return DES_ERR_INVALID_ARGUMENT;
  if (P == 0) return DES_OK;
  sample_kernel<<<blocks_for(P), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(P, H, W, C, query_point, envmap,
                                                                                   out);
  des::count_launches(1);
  return cudaGetLastError() == cudaSuccess ? DES_OK : DES_ERR_CUDA;
}

int des_blur_envmap_forward(int32_t H, int32_t W, int32_t C, int32_t tar_H, int32_t tar_W, int32_t N_samples,
                            float alpha, const float* envmap, float* out, des_stream_t stream) {
  if (H <= 0 || W <= 0 || tar_H < 0 || tar_W < 0 || N_samples <= 0 || !envmap || (!out && tar_H * tar_W > 0))
    return DES_ERR_INVALID_ARGUMENT;
  if (C != 3 && C != 4) return DES_ERR_UNSUPPORTED;
  const int64_t P = (int64_t)tar_H * tar_W;
  if (P == 0) return DES_OK;
  if (P > INT32_MAX) return DES_ERR_UNSUPPORTED;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (C == 3)
    blur_kernel<3><<<blocks_for(P), 256, 0, s>>>(H, W, tar_H, tar_W, N_samples, alpha, envmap, out);
  else
    blur_kernel<4><<<blocks_for(P), 256, 0, s>>>(H, W, tar_H, tar_W, N_samples, alpha, envmap, out);
  des::count_launches(1);
  return cudaGetLastError() == cudaSuccess ? DES_OK : DES_ERR_CUDA;
}

}  // extern "C"
