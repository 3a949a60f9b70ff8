// Per-point inputs and per-point constants of the shading sum, shared by every kernel that
// evaluates the BRDF per (point, texel) pair (des_shade.cu, des_multienv.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "des_internal.h"
#include "des_math.cuh"

namespace des {

// Copies texels [base, base + len) of the table into shared memory (len a multiple of 32).
__device__ __forceinline__ void stage_table(float4* __restrict__ s_tab, const float4* __restrict__ g_tab,
                                            int base, int len) {
  for (int i = threadIdx.x; i < 2 * len; i += blockDim.x) s_tab[i] = g_tab[2 * base + i];
}

struct PointGeom {
  float nx, ny, nz;  // normal (zeroed for inactive lanes: then no texel passes n.l > 0)
  float vx, vy, vz;  // view direction
  int v0, v1, v2;    // visibility vertices
  float c0, c1, c2;  // barycentric weights
};

// Loads a lane's normal / view / visibility vertices.  Out-of-range triangle or vertex ids set
// the workspace error bit and make the point inactive (it then shades to zero).
template <bool VIS>
__device__ __forceinline__ PointGeom load_geom(const ShadeParams& p, int64_t pid, bool valid, bool need_view) {
  PointGeom g;
  g.nx = g.ny = g.nz = 0.f;
  g.vx = g.vy = g.vz = 0.f;
  g.v0 = g.v1 = g.v2 = 0;
  g.c0 = g.c1 = g.c2 = 0.f;
  if (!valid) return g;
  g.nx = p.normal[3 * pid];
  g.ny = p.normal[3 * pid + 1];
  g.nz = p.normal[3 * pid + 2];
  if (need_view) {
    g.vx = p.view[3 * pid];
    g.vy = p.view[3 * pid + 1];
    g.vz = p.view[3 * pid + 2];
  }
  if (VIS) {
    const int64_t f = p.tri[pid];
    bool ok = (f >= 0) && (f < p.N_face);
    if (ok) {
      g.v0 = p.faces[f];
      g.v1 = p.faces[f + p.N_face];
      g.v2 = p.faces[f + 2 * (int64_t)p.N_face];
      ok = (g.v0 >= 0) && (g.v0 < p.N_vertex) && (g.v1 >= 0) && (g.v1 < p.N_vertex) && (g.v2 >= 0) &&
           (g.v2 < p.N_vertex);
    }
    if (!ok) {
      atomicOr(&p.ctrl[kCtrlError], 1u);
      g.v0 = g.v1 = g.v2 = 0;
      g.nx = g.ny = g.nz = 0.f;
    }
    g.c0 = p.bary[pid];
    g.c1 = p.bary[pid + p.P];
    g.c2 = p.bary[pid + 2 * p.P];
  }
  // backface clamp (bruteforce_shader.cu:1111): the whole texel loop is skipped when n.v <= 0
  if (p.clamp && !(dot3(g.nx, g.ny, g.nz, g.vx, g.vy, g.vz) > 0.f)) g.nx = g.ny = g.nz = 0.f;
  return g;
}

__device__ __forceinline__ void load_vis_words(const ShadeParams& p, const PointGeom& g, bool valid, int slot,
                                               uint32_t& w0, uint32_t& w1, uint32_t& w2) {
  if (valid) {
    const uint32_t* row = p.vis + (int64_t)slot * p.N_vertex;
    w0 = __ldg(row + g.v0);
    w1 = __ldg(row + g.v1);
    w2 = __ldg(row + g.v2);
  } else {
    w0 = w1 = w2 = 0u;
  }
}

// Per-point GGX constants (bruteforce_shader.cu:1601-1604 and G1_robust's view factor).
struct SpecConst {
  float alpha2, am1;  // alpha^2 = r^4 and alpha^2 - 1
  float k, omk;       // k = (r+1)^2/8 and 1 - k
  float invB;         // 1 / (max(n.v,0) (1-k) + k)
  float nvp;          // max(n.v, 0)
  float omn;          // 1 - |n|^2 (zero for an exactly unit normal)
};

__device__ __forceinline__ SpecConst spec_const(float r, const PointGeom& g) {
  SpecConst s;
  float a0 = r * r;
  s.alpha2 = a0 * a0;
  s.am1 = s.alpha2 - 1.f;
  float a1 = r + 1.f;
  s.k = (a1 * a1) / 8.f;
  s.omk = 1.f - s.k;
  s.nvp = fmaxf(dot3(g.vx, g.vy, g.vz, g.nx, g.ny, g.nz), 0.f);
  s.invB = 1.f / fmaf(s.nvp, s.omk, s.k);
  const double n2 = (double)g.nx * g.nx + (double)g.ny * g.ny + (double)g.nz * g.nz;
  s.omn = (float)(1.0 - n2);
  return s;
}

// GGX denominator t = (n.h)^2 (alpha^2 - 1) + 1 for h = h0 / |h0|, evaluated without cancellation:
// 1 - (n.h)^2 = |n x h0|^2 / |h0|^2 + (1 - |n|^2), so t = |n x h0|^2 ri2 + omn + (n.h)^2 alpha^2.
// Near the specular peak t ~ alpha^2 << 1, where the direct form loses ~log2(1/alpha^2) bits.
__device__ __forceinline__ float ggx_t(const PointGeom& g, float hx, float hy, float hz, float ri, float nh2,
                                       const SpecConst& sc) {
  const float cx = fmaf(g.ny, hz, -g.nz * hy);
  const float cy = fmaf(g.nz, hx, -g.nx * hz);
  const float cz = fmaf(g.nx, hy, -g.ny * hx);
  const float cc = dot3(cx, cy, cz, cx, cy, cz);
  return fmaf(nh2, sc.alpha2, fmaf(cc, ri * ri, sc.omn));
}

// Forward weights of one (point, texel) pair: wd = vis * max(n.l,0) * dw/pi (Lambert) and
// ws = vis * dw * F G D / 4 (GGX), zero where the reference adds nothing (n.l <= 0, FGD/4 <= 0).
// A = (l'x, l'y, l'z, dw) of the texel, dwpi = dw/pi.  bruteforce_shader.cu:2200-2234.
template <bool DIFF, bool SPEC>
__device__ __forceinline__ void pair_fwd_weights(const PointGeom& g, const SpecConst& sc, const float4& A, float dwpi,
                                                 float vis, float& wd, float& ws) {
  const float nl = dot3(g.nx, g.ny, g.nz, A.x, A.y, A.z);
  const bool act = nl > 0.f;
  wd = 0.f;
  ws = 0.f;
  if (DIFF) wd = act ? nl * dwpi * vis : 0.f;
  if (SPEC) {
    const float hx = A.x + g.vx, hy = A.y + g.vy, hz = A.z + g.vz;
    const float hh = fmaxf(dot3(hx, hy, hz, hx, hy, hz), kHalfVecFloor);
    const float ri = rsqrt_approx(hh);
    const float nh = dot3(g.nx, g.ny, g.nz, hx, hy, hz) * ri;
    const float lh = dot3(A.x, A.y, A.z, hx, hy, hz) * ri;
    const float a = 1.f - __saturatef(lh);
    const float a2 = a * a;
    const float F = fmaf(a2 * a2 * a, 1.f - kR0, kR0);
    const float G = nl * rcp_approx(fmaf(nl, sc.omk, sc.k)) * sc.invB;
    const float tt = ggx_t(g, hx, hy, hz, ri, nh * nh, sc);
    const float D = sc.alpha2 * rcp_approx(fmaxf(kPiF * tt * tt, kThres));
    const float tmp = F * G * D * 0.25f;
    ws = (act && tmp > 0.f) ? tmp * A.w * vis : 0.f;
  }
}

}  // namespace des
