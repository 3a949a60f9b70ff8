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

// Point of tile slot `slot` (slot < P: the slot's lane is active).  With a permutation the point
// is perm[slot]; an entry outside [0, P) sets error bit 8 and leaves the lane inactive instead of
// being dereferenced.  Returns whether the lane is active; `pid` receives the point index.
__device__ __forceinline__ bool ordered_point(const int32_t* __restrict__ perm, int64_t slot, int64_t P,
                                              unsigned* ctrl, int64_t& pid) {
  pid = slot;
  if (slot >= P) return false;
  if (perm == nullptr) return true;
  const int32_t q = perm[slot];
  if (q < 0 || (int64_t)q >= P) {
    atomicOr(&ctrl[kCtrlError], 8u);
    pid = 0;
    return false;
  }
  pid = q;
  return true;
}

struct PointGeom {
  float nx, ny, nz;  // normal (zeroed for inactive lanes: then no texel passes n.l > 0)
  float vx, vy, vz;  // view direction
  int v0, v1, v2;    // visibility vertices
  float c0, c1, c2;  // barycentric weights
};

// Loads a lane's normal / view / visibility vertices.  Out-of-range triangle or vertex ids set
// the workspace error bit and make the point inactive (it then shades to zero).
// PP is any parameter struct with the members P, normal, view, tri, faces, N_face, N_vertex, bary,
// clamp and ctrl (ShadeParams, or the serving request descriptor).
template <bool VIS, class PP>
__device__ __forceinline__ PointGeom load_geom(const PP& p, int64_t pid, bool valid, bool need_view) {
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

// Visibility words of one 32-texel slot for a lane: the words of its triangle's three vertices, or
// with ONEV (all three vertices of the lane's triangle are one vertex) that vertex's word alone.
template <bool ONEV = false, class PP>
__device__ __forceinline__ void load_vis_words(const PP& p, const PointGeom& g, bool valid, int slot,
                                               uint32_t& w0, uint32_t& w1, uint32_t& w2) {
  if (valid) {
    const uint32_t* row = p.vis + (int64_t)slot * p.N_vertex;
    w0 = __ldg(row + g.v0);
    if (ONEV) {
      w1 = w0;
      w2 = w0;
    } else {
      w1 = __ldg(row + g.v1);
      w2 = __ldg(row + g.v2);
    }
  } else {
    w0 = w1 = w2 = 0u;
  }
}

// Whether every lane of the warp interpolates its visibility within a single vertex (v0 = v1 = v2:
// one visibility row per point, e.g. per-Gaussian visibility).  Then the three bits of a texel are
// equal and the barycentric sum ((b c0 + b c1) + b c2) is b ? cs : 0 with cs = (c0 + c1) + c2 --
// the same FP32 value -- so one word per slot and one select per texel suffice.  Lanes without a
// point have v0 = v1 = v2 = 0.  Every warp of a CTA that shares one tile sees the same 32 points,
// so the answer is the same for all of them.
__device__ __forceinline__ bool warp_single_vertex(const PointGeom& g) {
  return __all_sync(0xffffffffu, g.v0 == g.v1 && g.v1 == g.v2);
}

// Visibility weight of one (point, texel) pair; mask selects the texel's bit in the slot words.
template <bool VIS, bool ONEV>
__device__ __forceinline__ float pair_vis(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t mask, const PointGeom& g,
                                          float cs) {
  if (!VIS) return 1.f;
  if (ONEV) return (w0 & mask) ? cs : 0.f;
  return vis_weight(w0, w1, w2, mask, g.c0, g.c1, g.c2);
}

// Per-point GGX constants (bruteforce_shader.cu:1601-1604 and G1_robust's view factor).
struct SpecConst {
  float alpha2, am1x2;  // alpha^2 = r^4 and 2 (alpha^2 - 1)
  float k, omk;         // k = (r+1)^2/8 and 1 - k
  float invB;           // 1 / (max(n.v,0) (1-k) + k)
  float nv, nvp;        // n.v and max(n.v, 0)
  float omn;            // 1 - |n|^2 (zero for an exactly unit normal)
  float c;              // alpha^2 invB
};

__device__ __forceinline__ SpecConst spec_const(float r, const PointGeom& g) {
  SpecConst s;
  float a0 = r * r;
  s.alpha2 = a0 * a0;
  s.am1x2 = 2.f * (s.alpha2 - 1.f);
  float a1 = r + 1.f;
  s.k = (a1 * a1) / 8.f;
  s.omk = 1.f - s.k;
  s.nv = dot3(g.vx, g.vy, g.vz, g.nx, g.ny, g.nz);
  s.nvp = fmaxf(s.nv, 0.f);
  s.invB = 1.f / fmaf(s.nvp, s.omk, s.k);
  s.c = s.alpha2 * s.invB;
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
// ws = vis * dw * F G D / 4 (GGX), zero where the reference adds nothing (n.l <= 0, and a FGD/4
// that is not > 0, e.g. NaN).  A = (l'x, l'y, l'z, dw/4) of the texel (the 1/4 of FGD/4 is folded
// into the table, an exact power-of-two scaling), dwpi = dw/pi, nl = n.l.
// G = max(n.l,0) / (max(n.l,0)(1-k) + k) * invB and D = alpha^2 / max(pi t^2, 1e-9) share one
// reciprocal: FGD = F max(n.l,0) (alpha^2 invB) / ((max(n.l,0)(1-k) + k) max(pi t^2, 1e-9)).
// n.h = (n.l + n.v) / |l + v|.  bruteforce_shader.cu:2200-2234.
template <bool DIFF, bool SPEC>
__device__ __forceinline__ void pair_fwd_weights(const PointGeom& g, const SpecConst& sc, const float4& A, float dwpi,
                                                 float nl, float vis, float& wd, float& ws) {
  const float nlp = fmaxf(nl, 0.f);  // also maps a NaN n.l to 0, as the reference's n.l > 0 test does
  wd = 0.f;
  ws = 0.f;
  if (DIFF) wd = nlp * dwpi * vis;
  if (SPEC) {
    const float hx = A.x + g.vx, hy = A.y + g.vy, hz = A.z + g.vz;
    const float hh = fmaxf(dot3(hx, hy, hz, hx, hy, hz), kHalfVecFloor);
    const float ri = rsqrt_approx(hh);
    const float nh = (nl + sc.nv) * ri;
    const float lh = dot3(A.x, A.y, A.z, hx, hy, hz) * ri;
    const float a = 1.f - __saturatef(lh);
    const float a2 = a * a;
    const float F = fmaf(a2 * a2 * a, 1.f - kR0, kR0);
    const float tt = ggx_t(g, hx, hy, hz, ri, nh * nh, sc);
    const float den = fmaf(nlp, sc.omk, sc.k) * fmaxf(kPiF * tt * tt, kThres);
    const float fgd = fmaxf(F * nlp * sc.c * rcp_approx(den), 0.f);
    ws = fgd * A.w * vis;
  }
}


// The k-th 32-texel slot (of nsl) integrated by warp `warp` of NW, or -1 past its last.  The
// slots are taken in the order 0, nsl-1, 1, nsl-2, ... -- mirrored pairs, i.e. rows at opposite
// elevations for the usual map widths -- and dealt to the warps a pair at a time (unit 2), or a
// slot at a time when there are fewer pairs than warps (unit 1).  The horizon skip removes whole
// rows for points that face up or down; mirrored pairs keep the surviving work of the warps of a
// tile even, so they reach the end-of-tile barrier together.
__device__ __forceinline__ int warp_slot(int k, int warp, int NW, int nsl, int ushift) {
  // ushift = log2(unit)
  const int j = (((k >> ushift) * NW + warp) << ushift) + (k & ushift);
  if (j >= nsl) return -1;
  return (j & 1) ? nsl - 1 - (j >> 1) : (j >> 1);
}

// Incoming gradients of one point folded with its albedos (bruteforce_shader.cu:2585-2588):
// gd = g_shading * albedo + g_diffuse_shading, gs = g_shading * specular_albedo.
struct BwdPoint {
  float gd0, gd1, gd2, gs0, gs1, gs2;
};

// Per-point sums of the fused adjoint (one set per lane; layout is relied on as 15 floats):
// Da = sum L w_d (-> g_albedo), Sa = sum L w_s (-> g_specular_albedo), gn/gv = normal/view gradients
// without the Schlick-Smith view factor, ga1 = d/dk, ga2 = d/d alpha^2, gbs = sum of d/dG * Ga over
// the pairs (the gradient with respect to the view-side denominator B is -gbs/B, applied per point).
struct BwdAcc {
  float Da0, Da1, Da2, Sa0, Sa1, Sa2, gnx, gny, gnz, gvx, gvy, gvz, ga1, ga2, gbs;
};

// Adjoint of one (point, texel) pair: accumulates into `acc` and returns the pair's forward
// weights (for the env-map gradient e_c = gd_c wd + gs_c ws).  A = (l', dw/4), B = (L, dw/pi),
// nl = n.l.  The per-point view factor 1/B of G is folded into the pair's weight once (wsv), so
// that G = Ga / B needs no multiply of its own: q = dshading/d(FGD) / B, dL/dF = q Ga D,
// dL/dD = q F Ga, dL/dGa = q F D.  bruteforce_shader.cu:2380-2484.
template <bool DIFF, bool SPEC>
__device__ __forceinline__ void pair_bwd(const PointGeom& g, const SpecConst& sc, const BwdPoint& gp, const float4& A,
                                         const float4& B, float nl, float vis, BwdAcc& acc, float& wd_out,
                                         float& ws_out) {
  const float visa = nl > 0.f ? vis : 0.f;  // visibility of a pair above the horizon, else 0
  wd_out = 0.f;
  ws_out = 0.f;
  if (DIFF) {
    // Lambert adjoint (bruteforce_shader.cu:2413-2426)
    const float wdv = B.w * visa;  // d_omega/pi * vis
    const float wd = nl * wdv;
    acc.Da0 = fmaf(B.x, wd, acc.Da0);
    acc.Da1 = fmaf(B.y, wd, acc.Da1);
    acc.Da2 = fmaf(B.z, wd, acc.Da2);
    const float gdot = dot3(gp.gd0, gp.gd1, gp.gd2, B.x, B.y, B.z) * wdv;
    acc.gnx = fmaf(gdot, A.x, acc.gnx);
    acc.gny = fmaf(gdot, A.y, acc.gny);
    acc.gnz = fmaf(gdot, A.z, acc.gnz);
    wd_out = wd;
  }
  if (SPEC) {
    const float hx = A.x + g.vx, hy = A.y + g.vy, hz = A.z + g.vz;
    const float hh = fmaxf(dot3(hx, hy, hz, hx, hy, hz), kHalfVecFloor);
    const float ri = rsqrt_approx(hh);
    const float nh = (nl + sc.nv) * ri;
    const float lh = dot3(A.x, A.y, A.z, hx, hy, hz) * ri;
    const float a = 1.f - __saturatef(lh);
    const float a2 = a * a;
    const float a4 = a2 * a2;
    const float F = fmaf(a4 * a, 1.f - kR0, kR0);
    // max(n.l, 0) as in G1_robust: equal to n.l on every pair that contributes, and it keeps the
    // denominator >= k on the others, whose products are masked by multiplying with zero
    const float nlp = fmaxf(nl, 0.f);
    const float ia = rcp_approx(fmaf(nlp, sc.omk, sc.k));
    const float Ga = nlp * ia;
    const float nh2 = nh * nh;
    const float tt = ggx_t(g, hx, hy, hz, ri, nh2, sc);
    const float t2 = kPiF * tt * tt;
    const float itm = rcp_approx(fmaxf(t2, kThres));
    const float D = sc.alpha2 * itm;
    const float FGa = F * Ga;
    const float wsv = A.w * visa * sc.invB;  // d_omega/4 * vis / B
    const float ws = FGa * D * wsv;
    acc.Sa0 = fmaf(B.x, ws, acc.Sa0);
    acc.Sa1 = fmaf(B.y, ws, acc.Sa1);
    acc.Sa2 = fmaf(B.z, ws, acc.Sa2);
    ws_out = ws;
    // d shading / d (F G D), over B, then split into F, Ga, D (bruteforce_shader.cu:2436-2445)
    const float q = dot3(gp.gs0, gp.gs1, gp.gs2, B.x, B.y, B.z) * wsv;
    const float gF = q * (Ga * D);
    const float gA = q * (F * D);
    const float gD = q * FGa;
    // Fresnel adjoint (bruteforce_shader.cu:155-159)
    const float gch = (lh >= 0.f && lh <= 1.f) ? (5.f * (kR0 - 1.f)) * gF * a4 : 0.f;
    float ghx = gch * A.x, ghy = gch * A.y, ghz = gch * A.z;
    // Schlick-Smith adjoint, light side (bruteforce_shader.cu:173-201); the view side is
    // linear in a per-point factor and is applied once per point after the loop
    const float gAi = gA * (ia * ia);
    const float gdln = gAi * sc.k;
    acc.gnx = fmaf(gdln, A.x, acc.gnx);
    acc.gny = fmaf(gdln, A.y, acc.gny);
    acc.gnz = fmaf(gdln, A.z, acc.gnz);
    acc.ga1 = fmaf(gAi, fmaf(nl, nl, -nl), acc.ga1);
    acc.gbs = fmaf(gA, Ga, acc.gbs);
    // GGX NDF adjoint (bruteforce_shader.cu:212-227): dD/d alpha^2 = 1/max(pi t^2, eps), and
    // dD/dt = -2 pi alpha^2 t / (pi t^2)^2 = -2 pi t D / (pi t^2) while pi t^2 is above the floor
    const float u = gD * itm;
    acc.ga2 += u;
    const float gt = (t2 > kThres) ? ((-2.f * kPiF) * tt) * u * D : 0.f;
    acc.ga2 = fmaf(nh2, gt, acc.ga2);
    const float gdnh = gt * sc.am1x2 * nh;
    const float hnx = hx * ri, hny = hy * ri, hnz = hz * ri;
    acc.gnx = fmaf(gdnh, hnx, acc.gnx);
    acc.gny = fmaf(gdnh, hny, acc.gny);
    acc.gnz = fmaf(gdnh, hnz, acc.gnz);
    ghx = fmaf(gdnh, g.nx, ghx);
    ghy = fmaf(gdnh, g.ny, ghy);
    ghz = fmaf(gdnh, g.nz, ghz);
    // normalize adjoint (bruteforce_shader.cu:63-71) and h = l + v -> v
    const float hg = dot3(hnx, hny, hnz, ghx, ghy, ghz);
    acc.gvx = fmaf(fmaf(-hnx, hg, ghx), ri, acc.gvx);
    acc.gvy = fmaf(fmaf(-hny, hg, ghy), ri, acc.gvy);
    acc.gvz = fmaf(fmaf(-hnz, hg, ghz), ri, acc.gvz);
  }
}

// Transposing butterfly: e[j] (j = 0..7) per lane -> every lane holds the 32-lane sum of texel
// 4*b4 + 2*b3 + b2 of its lane id (b4 = bit 4, ...), identical in lanes that differ in bits 0-1.
__device__ __forceinline__ float butterfly8(const float (&e)[8], int lane) {
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
  float x[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float keep = b4 ? e[i + 4] : e[i];
    const float send = b4 ? e[i] : e[i + 4];
    x[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
  float y[2];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const float keep = b3 ? x[i + 2] : x[i];
    const float send = b3 ? x[i] : x[i + 2];
    y[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  float z;
  {
    const float keep = b2 ? y[1] : y[0];
    const float send = b2 ? y[0] : y[1];
    z = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
  z += __shfl_xor_sync(0xffffffffu, z, 2);
  z += __shfl_xor_sync(0xffffffffu, z, 1);
  return z;
}


// Forward sums of one 32-texel slot for the lane's point: acc[0..2] += sum L wd, acc[3..5] += sum
// L ws.  rec = the slot's 32 texel records (2 float4 each), w0..w2 = the slot's visibility words,
// cs = (c0 + c1) + c2 (used with ONEV).  Texels are taken two at a time: a pair below the horizon of
// all 32 lanes adds nothing to any of them and is skipped by one warp vote; otherwise both texels are
// evaluated side by side (two independent dependency chains per lane; a texel of the pair that is
// below every horizon yields exact zeros).  Per texel the sums are updated in texel order.
template <bool DIFF, bool SPEC, bool VIS, bool ONEV>
__device__ __forceinline__ void fwd_slot(const PointGeom& g, const SpecConst& sc, float cs, const float4* rec,
                                         uint32_t w0, uint32_t w1, uint32_t w2, float (&acc)[6]) {
#pragma unroll 1
  for (int gq = 0; gq < 4; ++gq) {
#pragma unroll
    for (int j = 0; j < 8; j += 2) {
      const float4 A0 = rec[2 * (gq * 8 + j)];
      const float4 A1 = rec[2 * (gq * 8 + j + 1)];
      const float nl0 = dot3(g.nx, g.ny, g.nz, A0.x, A0.y, A0.z);
      const float nl1 = dot3(g.nx, g.ny, g.nz, A1.x, A1.y, A1.z);
      if (!__any_sync(0xffffffffu, nl0 > 0.f || nl1 > 0.f)) continue;
      const float4 B0 = rec[2 * (gq * 8 + j) + 1];
      const float4 B1 = rec[2 * (gq * 8 + j + 1) + 1];
      const float vis0 = pair_vis<VIS, ONEV>(w0, w1, w2, 1u << j, g, cs);
      const float vis1 = pair_vis<VIS, ONEV>(w0, w1, w2, 2u << j, g, cs);
      float wd0, ws0, wd1, ws1;
      pair_fwd_weights<DIFF, SPEC>(g, sc, A0, B0.w, nl0, vis0, wd0, ws0);
      pair_fwd_weights<DIFF, SPEC>(g, sc, A1, B1.w, nl1, vis1, wd1, ws1);
      if (DIFF) {
        acc[0] = fmaf(B1.x, wd1, fmaf(B0.x, wd0, acc[0]));
        acc[1] = fmaf(B1.y, wd1, fmaf(B0.y, wd0, acc[1]));
        acc[2] = fmaf(B1.z, wd1, fmaf(B0.z, wd0, acc[2]));
      }
      if (SPEC) {
        acc[3] = fmaf(B1.x, ws1, fmaf(B0.x, ws0, acc[3]));
        acc[4] = fmaf(B1.y, ws1, fmaf(B0.y, ws0, acc[4]));
        acc[5] = fmaf(B1.z, ws1, fmaf(B0.z, ws0, acc[5]));
      }
    }
    if (VIS) {
      w0 >>= 8;
      w1 >>= 8;
      w2 >>= 8;
    }
  }
}

// Adjoint of one 32-texel slot for the lane's point (arguments as fwd_slot): accumulates the point's
// sums into acc, and per 8-texel group sums the 32 lanes' env-map gradient contributions
// e_c = gd_c wd + gs_c ws with the transposing butterfly, then calls sink(group, y0, y1, y2) in every
// lane -- lanes with (lane & 3) == 0 hold the sums of texel group * 8 + butterfly_texel(lane), one per
// channel.  Texels are taken in pairs as in fwd_slot; a group whose 8 texels are below every lane's
// horizon skips the butterfly and the sink.
template <bool DIFF, bool SPEC, bool VIS, bool ONEV, class Sink>
__device__ __forceinline__ void bwd_slot(const PointGeom& g, const SpecConst& sc, float cs, const BwdPoint& gp,
                                         const float4* rec, uint32_t w0, uint32_t w1, uint32_t w2, int lane,
                                         BwdAcc& acc, Sink& sink) {
#pragma unroll 1
  for (int gq = 0; gq < 4; ++gq) {
    float wdj[8], wsj[8];
    bool live = false;  // warp-uniform: some texel of the group is above some lane's horizon
#pragma unroll
    for (int j = 0; j < 8; j += 2) {
      wdj[j] = wsj[j] = wdj[j + 1] = wsj[j + 1] = 0.f;
      const float4 A0 = rec[2 * (gq * 8 + j)];
      const float4 A1 = rec[2 * (gq * 8 + j + 1)];
      const float nl0 = dot3(g.nx, g.ny, g.nz, A0.x, A0.y, A0.z);
      const float nl1 = dot3(g.nx, g.ny, g.nz, A1.x, A1.y, A1.z);
      // both texels below the horizon of all 32 points: no contribution to any output
      if (!__any_sync(0xffffffffu, nl0 > 0.f || nl1 > 0.f)) continue;
      live = true;
      const float4 B0 = rec[2 * (gq * 8 + j) + 1];
      const float4 B1 = rec[2 * (gq * 8 + j + 1) + 1];
      const float vis0 = pair_vis<VIS, ONEV>(w0, w1, w2, 1u << j, g, cs);
      const float vis1 = pair_vis<VIS, ONEV>(w0, w1, w2, 2u << j, g, cs);
      pair_bwd<DIFF, SPEC>(g, sc, gp, A0, B0, nl0, vis0, acc, wdj[j], wsj[j]);
      pair_bwd<DIFF, SPEC>(g, sc, gp, A1, B1, nl1, vis1, acc, wdj[j + 1], wsj[j + 1]);
    }
    if (VIS) {
      w0 >>= 8;
      w1 >>= 8;
      w2 >>= 8;
    }
    if (!live) continue;
    float e[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) e[j] = fmaf(gp.gs0, wsj[j], gp.gd0 * wdj[j]);
    const float y0 = butterfly8(e, lane);
#pragma unroll
    for (int j = 0; j < 8; ++j) e[j] = fmaf(gp.gs1, wsj[j], gp.gd1 * wdj[j]);
    const float y1 = butterfly8(e, lane);
#pragma unroll
    for (int j = 0; j < 8; ++j) e[j] = fmaf(gp.gs2, wsj[j], gp.gd2 * wdj[j]);
    const float y2 = butterfly8(e, lane);
    sink(gq, y0, y1, y2);
  }
}

// Texel of an 8-texel group whose env-map gradient sum lane `lane` holds after butterfly8.
__device__ __forceinline__ int butterfly_texel(int lane) {
  return ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
}

// Outputs of the fused adjoint (any of the last four may be null).
struct BwdOutputs {
  float *g_normal, *g_view, *g_albedo, *g_spec, *g_rough;
};

// One point's gradients from its reduced adjoint sums (BwdAcc order): applies the Schlick-Smith
// view factor (bruteforce_shader.cu:194-200) and the roughness chain rule (2501-2502).
// r = roughness, (g0, g1, g2) = the point's incoming shading gradient.
struct BwdGrads {
  float n[3], v[3], a[3], s[3], rough;
};

template <bool DIFF, bool SPEC>
__device__ __forceinline__ BwdGrads bwd_point_grads(const float (&sums)[15], const PointGeom& g, const SpecConst& sc,
                                                    float r, float g0, float g1, float g2) {
  BwdGrads q;
  float n_x = sums[6], n_y = sums[7], n_z = sums[8];
  float v_x = sums[9], v_y = sums[10], v_z = sums[11];
  float g_rough = 0.f;
  if (SPEC) {
    // view side of the Schlick-Smith adjoint (bruteforce_shader.cu:194-200): dL/dB = -gbs / B
    const float gB = -sums[14] * sc.invB;
    const float gdvn = gB * sc.omk;
    if (sc.nvp > 0.f) {
      v_x = fmaf(gdvn, g.nx, v_x);
      v_y = fmaf(gdvn, g.ny, v_y);
      v_z = fmaf(gdvn, g.nz, v_z);
      n_x = fmaf(gdvn, g.vx, n_x);
      n_y = fmaf(gdvn, g.vy, n_y);
      n_z = fmaf(gdvn, g.vz, n_z);
    }
    const float gk = fmaf(gB, 1.f - sc.nvp, sums[12]);
    // roughness chain rule (bruteforce_shader.cu:2501-2502)
    g_rough = sums[13] * 4.f * r * r * r;
    g_rough += gk * (1.f + r) / 4.f;
  }
  q.n[0] = n_x;
  q.n[1] = n_y;
  q.n[2] = n_z;
  q.a[0] = DIFF ? g0 * sums[0] : 0.f;
  q.a[1] = DIFF ? g1 * sums[1] : 0.f;
  q.a[2] = DIFF ? g2 * sums[2] : 0.f;
  q.s[0] = SPEC ? g0 * sums[3] : 0.f;
  q.s[1] = SPEC ? g1 * sums[4] : 0.f;
  q.s[2] = SPEC ? g2 * sums[5] : 0.f;
  q.v[0] = SPEC ? v_x : 0.f;
  q.v[1] = SPEC ? v_y : 0.f;
  q.v[2] = SPEC ? v_z : 0.f;
  q.rough = g_rough;
  return q;
}

// Finishes one point: its gradients (bwd_point_grads) stored at index pid.  g_shading3 = the
// point's incoming shading gradient.
template <bool DIFF, bool SPEC>
__device__ __forceinline__ void finish_bwd_point(const float (&sums)[15], const PointGeom& g, const SpecConst& sc,
                                                 float r, const float* g_shading3, int64_t pid, const BwdOutputs& o) {
  const BwdGrads q = bwd_point_grads<DIFF, SPEC>(sums, g, sc, r, g_shading3[0], g_shading3[1], g_shading3[2]);
#pragma unroll
  for (int c = 0; c < 3; ++c) o.g_normal[3 * pid + c] = q.n[c];
  if (o.g_albedo != nullptr)
#pragma unroll
    for (int c = 0; c < 3; ++c) o.g_albedo[3 * pid + c] = q.a[c];
  if (o.g_spec != nullptr)
#pragma unroll
    for (int c = 0; c < 3; ++c) o.g_spec[3 * pid + c] = q.s[c];
  if (o.g_view != nullptr)
#pragma unroll
    for (int c = 0; c < 3; ++c) o.g_view[3 * pid + c] = q.v[c];
  if (o.g_rough != nullptr) o.g_rough[pid] = q.rough;
}

// Stores the 3-vectors of a tile's 32 consecutive points (lane = point, first point `first`, P
// points in all) as whole 128-byte rows: round k writes floats 32k .. 32k+31 of the tile's 96, each
// lane fetching its value from the owning lane by shuffle.  All 32 lanes take part.
__device__ __forceinline__ void store_rows3(float* dst, int64_t first, int64_t P, float x, float y, float z,
                                            int lane) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int f = 32 * k + lane, p = f / 3, c = f - 3 * p;
    const float a = __shfl_sync(0xffffffffu, x, p), b = __shfl_sync(0xffffffffu, y, p),
                d = __shfl_sync(0xffffffffu, z, p);
    if (first + p < P) dst[3 * first + f] = c == 0 ? a : (c == 1 ? b : d);
  }
}

}  // namespace des
