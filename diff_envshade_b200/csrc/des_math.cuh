// Device math shared by the shading kernels (sm_100a).
//
// Two groups of functions live here:
//  * texel geometry that must stay bit-exact with the reference extension: the same source
//    expressions as bruteforce_shader.cu:124-147 (getDeltaOmega / getLightDir) and the
//    rotation of bruteforce_shader.cu:2194-2197, compiled with nvcc's default -fmad=true and
//    IEEE division (this project never builds with --use_fast_math);
//  * the per-(point, texel) BRDF arithmetic in a form with hoisted per-point constants and
//    approximate reciprocals, whose results agree with the reference to FP32 rounding.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace des {

constexpr float kPiF = 3.141592653589793f;        // M_PIf of the reference
constexpr float kInvPiF = 0.318309886183790672f;  // 1/pi
constexpr float kR0 = 0.04f;                      // F0, bruteforce_shader.cu:30
constexpr float kThres = 1e-9f;                   // NDF floor, bruteforce_shader.cu:31
constexpr float kHalfVecFloor = 1e-30f;           // keeps 1/|l+v| finite when l = -v exactly

// Solid angle of a texel row: (sin(theta1) - sin(theta0)) * 2pi / W, with __sinf.
// Same expressions as bruteforce_shader.cu:124-131 so the FP32 result is identical.
__device__ __forceinline__ float texel_delta_omega(int iy, int W, int H) {
  float delta_phi = (2 * kPiF) / W;
  float delta_theta = kPiF / H;
  float sin_theta1 = __sinf(delta_theta * (iy + 1) - kPiF * 0.5f);
  float sin_theta0 = __sinf(delta_theta * iy - kPiF * 0.5f);
  return (sin_theta1 - sin_theta0) * delta_phi;
}

// Texel centre direction (cos t cos p, sin t, cos t sin p), t = latitude, p = longitude.
// Same expressions as bruteforce_shader.cu:133-147 so the FP32 result is identical.
__device__ __forceinline__ float3 texel_direction(int iy, int ix, int W, int H) {
  float v = (float(iy) + 0.5f) / H;
  float u = (float(ix) + 0.5f) / W;
  float phi = u * kPiF * 2;
  float theta = (v - 0.5f) * kPiF;
  float sin_theta, cos_theta, sin_phi, cos_phi;
  sincosf(theta, &sin_theta, &cos_theta);
  sincosf(phi, &sin_phi, &cos_phi);
  float3 c;
  c.y = sin_theta;
  c.x = cos_theta * cos_phi;
  c.z = cos_theta * sin_phi;
  return c;
}

// l' = R l (bruteforce_shader.cu:2194-2197).  The reference writes each row as
// m0*x + m1*y + m2*z and leaves the FMA contraction to nvcc; its compiled kernels evaluate row 0 as
// fma(m2, z, fma(m1, y, m0*x)) and rows 1 and 2 as fma(m5, z, fma(m3, x, m4*y)).  That order was
// identified from the reference's own outputs (tests/golden/table_probe_*) and is spelled out here
// with explicit round-to-nearest intrinsics, so the table does not depend on contraction choices.
__device__ __forceinline__ float3 rotate3(const float* m, float3 l) {
  float3 r;
  r.x = __fmaf_rn(m[2], l.z, __fmaf_rn(m[1], l.y, __fmul_rn(m[0], l.x)));
  r.y = __fmaf_rn(m[5], l.z, __fmaf_rn(m[3], l.x, __fmul_rn(m[4], l.y)));
  r.z = __fmaf_rn(m[8], l.z, __fmaf_rn(m[6], l.x, __fmul_rn(m[7], l.y)));
  return r;
}

// Hardware approximate reciprocal / reciprocal square root (PTX rcp.approx / rsqrt.approx).
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float rsqrt_approx(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
  return fmaf(az, bz, fmaf(ay, by, ax * bx));
}

// Barycentric visibility of one texel: bit j of the three vertex words, weighted by c0..c2,
// summed in the reference's order ((b0 c0 + b1 c1) + b2 c2) (bruteforce_shader.cu:2186-2189).
__device__ __forceinline__ float vis_weight(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t mask, float c0,
                                            float c1, float c2) {
  float b0 = (w0 & mask) ? c0 : 0.f;
  float b1 = (w1 & mask) ? c1 : 0.f;
  float b2 = (w2 & mask) ? c2 : 0.f;
  return (b0 + b1) + b2;
}

}  // namespace des
