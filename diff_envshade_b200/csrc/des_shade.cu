// Brute-force environment-map shading on B200 (sm_100a): forward sum and fused adjoint.
//
// Work decomposition (all shading kernels):
//  * a tile is 32 consecutive points, one point per lane of a warp;
//  * a CTA of NW warps processes one tile at a time, warp w integrating the tile over its own
//    share of the 32-texel visibility slots (mirrored pairs, see warp_slot), so the NW warps
//    split the texel axis;
//  * CTAs are persistent: the grid is sized to the resident capacity of the device, and CTAs
//    pull tiles from a device counter (the next tile index is fetched one tile ahead);
//  * the texel table {rotated direction, d_omega, radiance, d_omega/pi} of the whole env map is
//    staged once per CTA in shared memory (in chunks of kChunk texels for very large maps).
// Per-point partial sums of the NW warps are combined through shared memory at the end of a
// tile in a fixed order, so every per-point output is deterministic.
//
// Env-map gradient: per 8-texel group the 32 lanes' contributions are summed by a transposing
// butterfly of warp shuffles (each of 8 lanes ends up holding one texel), added into a per-CTA
// FP64 accumulator in shared memory, written once per CTA, and summed over CTAs in FP64 by
// des_env_reduce_kernel.
//
// Reference correspondence (zjumsj/diff_envshade, bruteforce_shader.cu):
//   forward     = BruteForce{Diffuse,Specular,SpecularClamp}ShaderKernel_Forward (231, 532, 1040),
//                 BruteForceSpecular{,Visibility}ShaderKernel_Forward2 (1554, 2068)
//   backward    = the matching *_Backward / *_Backward2 point-gradient kernels (318, 689, 1197,
//                 1701, 2248) fused with the *_BackwardEnvmap* env-gradient kernels (435, 888,
//                 1396, 1928, 2508) into one pass.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>
#include <utility>

#include "des_internal.h"
#include "des_math.cuh"
#include "des_point.cuh"
#include "diff_envshade_b200.h"

namespace des {



// ------------------------------------------------------------------------------------------
// Texel table
// ------------------------------------------------------------------------------------------

// Texel record t: rec[2t] = (l'x, l'y, l'z, d_omega/4), rec[2t+1] = (L0, L1, L2, d_omega/pi) for
// t < H*W, zeros for the padding up to a multiple of 32.  The 1/4 is the denominator of the GGX
// term F G D / 4, folded into the table (a power of two: every product it enters is unchanged).  `export4` (optional) receives
// (x, y, z, d_omega) per texel for des_texel_table.
__device__ __forceinline__ void table_entry(int t, int H, int W, const float* __restrict__ R,
                                            const float* __restrict__ env, float4* __restrict__ rec,
                                            float* __restrict__ export4) {
  const int HW = H * W;
  if (t < HW) {
    int ix = t % W;
    int iy = t / W;
    iy = H - 1 - iy;  // LEFT_TOP_AS_ORIGIN (reference config.h:11): memory row 0 is the top row
    float m[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) m[i] = R[i];
    const float3 l = rotate3(m, texel_direction(iy, ix, W, H));
    const float dw = texel_delta_omega(iy, W, H);
    if (rec != nullptr) {
      rec[2 * t] = make_float4(l.x, l.y, l.z, dw * 0.25f);
      rec[2 * t + 1] = make_float4(env[t], env[HW + t], env[2 * HW + t], dw * kInvPiF);
    }
    if (export4 != nullptr) {
      export4[4 * t + 0] = l.x;
      export4[4 * t + 1] = l.y;
      export4[4 * t + 2] = l.z;
      export4[4 * t + 3] = dw;
    }
  } else if (rec != nullptr) {
    rec[2 * t] = make_float4(0.f, 0.f, 0.f, 0.f);
    rec[2 * t + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// The texel table of one call (one thread per texel); also resets the control words of the
// workspace (tile counter, error word) for the kernel that follows on the same stream.
__global__ void des_table_kernel(int H, int W, int HWpad, const float* __restrict__ R,
                                 const float* __restrict__ env, float4* __restrict__ rec,
                                 float* __restrict__ export4, unsigned* __restrict__ ctrl) {
  pdl_enter();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0 && ctrl != nullptr) {
    ctrl[kCtrlTileCounter] = 0u;
    ctrl[kCtrlError] = 0u;
    ctrl[kCtrlTileCounterBwd] = 0u;
  }
  if (t < HWpad) table_entry(t, H, W, R, env, rec, export4);
}

// ------------------------------------------------------------------------------------------
// Normal-direction ordering
// ------------------------------------------------------------------------------------------
// A warp shades 32 points against the same texel at the same time.  When the 32 normals point
// the same way, whole texels lie below every lane's horizon (n.l <= 0 for all 32 points: no
// diffuse and no specular contribution) and are skipped by a warp vote.  Points are therefore
// visited in the order of a stable counting sort by the octahedral cell of their normal (y is
// the polar axis; 32 x 32 cells in Morton order so that neighbouring cells stay close).  Each
// point's own arithmetic is unchanged, so per-point results do not depend on the order.

// Morton spread of a 5-bit value: bit i -> bit 2i.
__device__ __forceinline__ unsigned spread5(unsigned v) {
  v = (v | (v << 4)) & 0x0F0Fu;
  v = (v | (v << 2)) & 0x3333u;
  v = (v | (v << 1)) & 0x5555u;
  return v;
}

__device__ __forceinline__ int normal_key(const float* __restrict__ normal, int64_t p) {
  const float x = normal[3 * p], y = normal[3 * p + 1], z = normal[3 * p + 2];
  const float s = fabsf(x) + fabsf(y) + fabsf(z);
  float u = 0.f, v = 0.f;
  if (s > 0.f) {
    const float is = 1.f / s;
    u = x * is;
    v = z * is;
    if (y < 0.f) {  // fold the lower hemisphere onto the outer triangles of the square
      const float fu = (1.f - fabsf(v)) * (u >= 0.f ? 1.f : -1.f);
      const float fv = (1.f - fabsf(u)) * (v >= 0.f ? 1.f : -1.f);
      u = fu;
      v = fv;
    }
  }
  // [-1, 1] -> cell 0..31 (NaN inputs land in cell 0: fmaxf returns the non-NaN operand)
  const unsigned iu = (unsigned)fminf(fmaxf((u + 1.f) * 16.f, 0.f), 31.f);
  const unsigned iv = (unsigned)fminf(fmaxf((v + 1.f) * 16.f, 0.f), 31.f);
  return (int)(spread5(iu) | (spread5(iv) << 1));
}

// Ordering, step 1 (fused with the texel table and the control-word reset of the call).
// CTA c ranks the points of chunk c = [c*chunk, (c+1)*chunk) (chunk a multiple of 1024), 1024
// points at a time: warp w takes 64 consecutive points in 2 rounds of 32, and lanes with equal
// cells rank themselves with __match_any_sync against the warp's own per-cell counters.  An
// exclusive prefix of those counters over the warps then gives every point its rank among the
// chunk's points of its cell (input order when the chunk is one pass of 1024 points; otherwise
// warp by warp -- a fixed order either way, so the permutation is deterministic).  Outputs:
// keys[p] = cell, rank[p] = rank, and the chunk's cell counts in row c of counts[chunk][cell]
// (one coalesced 4 KB row per CTA).
// Threads of every CTA also build the texel records (grid-stride over the table).
__global__ void __launch_bounds__(kSortThreads, 1) des_prep_kernel(int H, int W, int HWpad, const float* __restrict__ R,
                                                                const float* __restrict__ env,
                                                                float4* __restrict__ rec, unsigned* __restrict__ ctrl,
                                                                const float* __restrict__ normal, int64_t P,
                                                                int chunk, unsigned* __restrict__ counts,
                                                                uint16_t* __restrict__ keys,
                                                                uint32_t* __restrict__ rank) {
  pdl_enter();
  constexpr int NW = kSortThreads / 32;
  constexpr int SUB = 2 * kSortThreads;  // points per pass: 2 rounds per warp
  __shared__ uint16_t cnt[NW][kSortBins];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  if (blockIdx.x == 0 && tid == 0 && ctrl != nullptr) {
    ctrl[kCtrlTileCounter] = 0u;
    ctrl[kCtrlError] = 0u;
    ctrl[kCtrlTileCounterBwd] = 0u;
  }
  for (int t = blockIdx.x * kSortThreads + tid; t < HWpad; t += gridDim.x * kSortThreads)
    table_entry(t, H, W, R, env, rec, nullptr);

  for (int i = tid; i < NW * kSortBins / 2; i += kSortThreads) reinterpret_cast<uint32_t*>(&cnt[0][0])[i] = 0u;
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  const int64_t cbase = (int64_t)blockIdx.x * chunk;
  const int nsub = chunk / SUB;
  int key[2] = {0, 0};
  unsigned lr[2] = {0u, 0u};
  for (int sub = 0; sub < nsub; ++sub) {
    const int64_t wbase = cbase + (int64_t)sub * SUB + w * 64;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int64_t p = wbase + r * 32 + lane;
      key[r] = (p < P) ? normal_key(normal, p) : kSortBins + lane;  // invalid lanes match no one
    }
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int64_t p = wbase + r * 32 + lane;
      const bool valid = p < P;
      const unsigned peers = __match_any_sync(0xffffffffu, key[r]);
      lr[r] = valid ? cnt[w][key[r]] + __popc(peers & lt) : 0u;
      __syncwarp();
      if (valid && (peers & lt) == 0u) cnt[w][key[r]] += (uint16_t)__popc(peers);
      __syncwarp();
      if (nsub > 1 && valid) {  // kept in registers when there is a single pass
        keys[p] = (uint16_t)key[r];
        rank[p] = lr[r];
      }
    }
  }
  __syncthreads();
  // exclusive prefix of the per-warp counters over the warps, per cell; chunk totals to global
  for (int k = tid; k < kSortBins; k += kSortThreads) {
    unsigned run = 0;
#pragma unroll
    for (int q = 0; q < NW; ++q) {
      const unsigned c = cnt[q][k];
      cnt[q][k] = (uint16_t)run;
      run += c;
    }
    counts[(size_t)blockIdx.x * kSortBins + k] = run;
  }
  __syncthreads();
  if (nsub == 1) {
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int64_t p = cbase + w * 64 + r * 32 + lane;
      if (p < P) {
        keys[p] = (uint16_t)key[r];
        rank[p] = cnt[w][key[r]] + lr[r];
      }
    }
  } else {
    for (int sub = 0; sub < nsub; ++sub) {
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int64_t p = cbase + (int64_t)sub * SUB + w * 64 + r * 32 + lane;
        if (p < P) rank[p] += cnt[w][keys[p]];  // this thread wrote both in the first pass
      }
    }
  }
}

// Ordering, step 2.  CTA c: thread k reads column k of counts (cell k's count in every chunk; the
// warp's reads of one row are coalesced) and sums it over all chunks (total) and over the chunks
// before c (prefix); a block scan of the totals gives the first position of cell k; then every
// point p of chunk c goes to perm[first(k) + prefix_c(k) + rank[p]]: cells in order, chunks in
// order within a cell.
__global__ void __launch_bounds__(kSortBins) des_place_kernel(int64_t P, int chunk, int nchunks,
                                                              const unsigned* __restrict__ counts,
                                                              const uint16_t* __restrict__ keys,
                                                              const uint32_t* __restrict__ rank,
                                                              int32_t* __restrict__ perm) {
  pdl_enter();
  __shared__ unsigned off[kSortBins];
  __shared__ unsigned warp_tot[kSortBins / 32];
  const int k = threadIdx.x, lane = k & 31, w = k >> 5;
  const int c = blockIdx.x;
  unsigned pre = 0, tot = 0;
  for (int c0 = 0; c0 < nchunks; c0 += 8) {
    unsigned v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = (c0 + j < nchunks) ? counts[(size_t)(c0 + j) * kSortBins + k] : 0u;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      tot += v[j];
      if (c0 + j < c) pre += v[j];
    }
  }
  unsigned incl = tot;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[w] = incl;
  __syncthreads();
  if (w == 0) {
    unsigned x = warp_tot[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += t;
    }
    warp_tot[lane] = x;
  }
  __syncthreads();
  off[k] = (incl - tot) + (w > 0 ? warp_tot[w - 1] : 0u) + pre;
  __syncthreads();
  const int64_t base = (int64_t)c * chunk;
  for (int i0 = 0; i0 < chunk; i0 += 4 * kSortBins) {
    int kk[4];
    unsigned rr[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t p = base + i0 + j * kSortBins + k;
      const bool ok = (i0 + j * kSortBins < chunk) && p < P;
      kk[j] = ok ? (int)keys[p] : -1;
      rr[j] = ok ? rank[p] : 0u;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (kk[j] >= 0) perm[off[kk[j]] + rr[j]] = (int32_t)(base + i0 + j * kSortBins + k);
  }
}

// ------------------------------------------------------------------------------------------
// Forward
// ------------------------------------------------------------------------------------------

// The NW warps of a CTA integrate one tile over their texel slots (mirrored pairs, see warp_slot);
// a warp's visibility words of its next slot are loaded while it integrates the current one, and a
// slot whose words are zero for all 32 lanes is skipped.  Tables with more than p.chunk texels are
// staged chunk by chunk (every warp of the CTA calls this with the same arguments).
template <bool DIFF, bool SPEC, bool VIS, bool ONEV>
__device__ __forceinline__ void fwd_tile_sums(const ShadeParams& p, const PointGeom& g, bool valid, const SpecConst& sc,
                                              float4* s_tab, int nchunks, int warp, int NW, float (&acc)[6]) {
  const float cs = (g.c0 + g.c1) + g.c2;
  for (int c = 0; c < nchunks; ++c) {
    const int cbase = c * p.chunk;
    const int clen = min(p.chunk, p.HWpad - cbase);
    if (nchunks > 1) {
      __syncthreads();
      stage_table(s_tab, p.table, cbase, clen);
      __syncthreads();
    }
    const int nsl = clen >> 5;
    const int ushift = ((nsl + 1) >> 1) >= NW ? 1 : 0;
    const int gslot0 = cbase >> 5;
    uint32_t n0 = 0u, n1 = 0u, n2 = 0u;
    int sl = warp_slot(0, warp, NW, nsl, ushift);
    if (VIS && sl >= 0) load_vis_words<ONEV>(p, g, valid, gslot0 + sl, n0, n1, n2);
    for (int k = 1; sl >= 0; ++k) {
      const int cur = sl;
      sl = warp_slot(k, warp, NW, nsl, ushift);
      const uint32_t w0 = n0, w1 = n1, w2 = n2;
      if (VIS) {
        if (sl >= 0) load_vis_words<ONEV>(p, g, valid, gslot0 + sl, n0, n1, n2);
        // skip a 32-point x 32-texel tile that is fully occluded for every lane
        if (!__any_sync(0xffffffffu, (w0 | w1 | w2) != 0u)) continue;
      }
      fwd_slot<DIFF, SPEC, VIS, ONEV>(g, sc, cs, s_tab + 2 * (cur << 5), w0, w1, w2, acc);
    }
  }
}

template <bool DIFF, bool SPEC, bool VIS>
__global__ void __maxnreg__(64) des_fwd_kernel(const ShadeParams p) {
  pdl_enter();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* s_tab = reinterpret_cast<float4*>(smem_raw);
  float* s_red = reinterpret_cast<float*>(smem_raw + (size_t)p.chunk * 32);
  __shared__ int s_next[2];

  const int NW = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nchunks = (p.HWpad + p.chunk - 1) / p.chunk;
  const bool need_view = SPEC || p.clamp;

  if (nchunks == 1) {
    stage_table(s_tab, p.table, 0, p.HWpad);
    __syncthreads();
  }

  int tile = blockIdx.x;
  int it = 0;
  while (tile < p.ntiles) {
    if (threadIdx.x == 0) s_next[it & 1] = (int)gridDim.x + (int)atomicAdd(&p.ctrl[kCtrlTileCounter], 1u);

    const int64_t slot = (int64_t)tile * 32 + lane;
    int64_t pid = slot;
    const bool valid = ordered_point(p.perm, slot, p.P, p.ctrl, pid);
    const PointGeom g = load_geom<VIS>(p, pid, valid, need_view);
    SpecConst sc;
    if (SPEC) sc = spec_const(valid ? p.rough[pid] : 0.f, g);

    // acc[0..2] = sum L * diffuse weight (white diffuse shading), acc[3..5] = sum L * specular weight
    float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (VIS && warp_single_vertex(g))
      fwd_tile_sums<DIFF, SPEC, VIS, true>(p, g, valid, sc, s_tab, nchunks, warp, NW, acc);
    else
      fwd_tile_sums<DIFF, SPEC, VIS, false>(p, g, valid, sc, s_tab, nchunks, warp, NW, acc);

    // combine the NW texel ranges in warp order
    float* red = s_red + warp * 6 * 32 + lane;
#pragma unroll
    for (int q = 0; q < 6; ++q) red[q * 32] = acc[q];
    __syncthreads();
    if (warp == 0 && valid) {
      float sum[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      for (int w = 0; w < NW; ++w) {
        const float* r = s_red + w * 6 * 32 + lane;
#pragma unroll
        for (int q = 0; q < 6; ++q) sum[q] += r[q * 32];
      }
#pragma unroll
      for (int ch = 0; ch < 3; ++ch) {
        float out = 0.f;
        if (DIFF) out = p.albedo[3 * pid + ch] * sum[ch];
        if (SPEC) out = fmaf(p.spec[3 * pid + ch], sum[3 + ch], out);
        p.shading[3 * pid + ch] = out;
        if (p.white != nullptr) p.white[3 * pid + ch] = sum[ch];
      }
    }
    __syncthreads();
    tile = s_next[it & 1];
    ++it;
  }
}

// ------------------------------------------------------------------------------------------
// Backward (point gradients + env-map gradient in one pass)
// ------------------------------------------------------------------------------------------

// As fwd_tile_sums, for the adjoint: the point's sums go to acc, the env-map gradient of each
// 8-texel group (summed over the 32 lanes) to the CTA's FP64 accumulator env_acc (row stride env_ld;
// indexed by the texel within the staged chunk when the accumulator is in shared memory, by the
// texel of the whole map otherwise).
template <bool DIFF, bool SPEC, bool VIS, bool ONEV>
__device__ __forceinline__ void bwd_tile_sums(const ShadeParams& p, const PointGeom& g, bool valid, const SpecConst& sc,
                                              const BwdPoint& gp, float4* s_tab, double* env_acc, int env_ld,
                                              int nchunks, int warp, int NW, int lane, BwdAcc& acc) {
  const float cs = (g.c0 + g.c1) + g.c2;
  const int jsel = butterfly_texel(lane);
  for (int c = 0; c < nchunks; ++c) {
    const int cbase = c * p.chunk;
    const int clen = min(p.chunk, p.HWpad - cbase);
    if (nchunks > 1) {
      __syncthreads();
      stage_table(s_tab, p.table, cbase, clen);
      __syncthreads();
    }
    const int nsl = clen >> 5;
    const int ushift = ((nsl + 1) >> 1) >= NW ? 1 : 0;
    const int gslot0 = cbase >> 5;
    const int ebase = p.env_in_smem ? 0 : cbase;
    uint32_t n0 = 0u, n1 = 0u, n2 = 0u;
    int sl = warp_slot(0, warp, NW, nsl, ushift);
    if (VIS && sl >= 0) load_vis_words<ONEV>(p, g, valid, gslot0 + sl, n0, n1, n2);
    for (int k = 1; sl >= 0; ++k) {
      const int cur = sl;
      sl = warp_slot(k, warp, NW, nsl, ushift);
      const uint32_t w0 = n0, w1 = n1, w2 = n2;
      if (VIS) {
        if (sl >= 0) load_vis_words<ONEV>(p, g, valid, gslot0 + sl, n0, n1, n2);
        if (!__any_sync(0xffffffffu, (w0 | w1 | w2) != 0u)) continue;
      }
      double* const eslot = env_acc + ebase + (cur << 5) + jsel;
      auto sink = [&](int gq, float y0, float y1, float y2) {
        if ((lane & 3) == 0) {
          double* a = eslot + gq * 8;
          a[0] += (double)y0;
          a[env_ld] += (double)y1;
          a[2 * env_ld] += (double)y2;
        }
      };
      bwd_slot<DIFF, SPEC, VIS, ONEV>(g, sc, cs, gp, s_tab + 2 * (cur << 5), w0, w1, w2, lane, acc, sink);
    }
  }
}

template <bool DIFF, bool SPEC, bool VIS>
__global__ void __launch_bounds__(kMaxThreads, 1) des_bwd_kernel(const ShadeParams p) {
  pdl_enter();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* s_tab = reinterpret_cast<float4*>(smem_raw);
  double* s_env = reinterpret_cast<double*>(smem_raw + (size_t)p.chunk * 32);  // [3][chunk], single chunk
  float* s_red = reinterpret_cast<float*>(smem_raw + (size_t)p.chunk * 32 + (p.env_in_smem ? (size_t)p.chunk * 24 : 0));
  __shared__ int s_next[2];

  constexpr int NACC = 15;
  const int NW = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nchunks = (p.HWpad + p.chunk - 1) / p.chunk;
  const bool need_view = SPEC || p.clamp;
  // env-gradient accumulator of this CTA: [3][HWpad] doubles (shared memory if it fits)
  double* env_acc = p.env_in_smem ? s_env : p.env_partial + (size_t)blockIdx.x * 3 * p.HWpad;
  const int env_ld = p.env_in_smem ? p.chunk : p.HWpad;
  {
    const int n = 3 * env_ld;
    for (int i = threadIdx.x; i < n; i += blockDim.x) env_acc[i] = 0.0;
  }
  if (nchunks == 1) stage_table(s_tab, p.table, 0, p.HWpad);
  __syncthreads();

  int tile = blockIdx.x;
  int it = 0;
  while (tile < p.ntiles) {
    if (threadIdx.x == 0) s_next[it & 1] = (int)gridDim.x + (int)atomicAdd(&p.ctrl[kCtrlTileCounterBwd], 1u);

    const int64_t slot = (int64_t)tile * 32 + lane;
    int64_t pid = slot;
    const bool valid = ordered_point(p.perm, slot, p.P, p.ctrl, pid);
    const PointGeom g = load_geom<VIS>(p, pid, valid, need_view);
    // incoming gradients folded with the albedos (bruteforce_shader.cu:2585-2588)
    float gd0 = 0.f, gd1 = 0.f, gd2 = 0.f, gs0 = 0.f, gs1 = 0.f, gs2 = 0.f;
    SpecConst sc;
    if (valid) {
      const float g0 = p.g_shading[3 * pid], g1 = p.g_shading[3 * pid + 1], g2 = p.g_shading[3 * pid + 2];
      if (DIFF) {
        gd0 = g0 * p.albedo[3 * pid];
        gd1 = g1 * p.albedo[3 * pid + 1];
        gd2 = g2 * p.albedo[3 * pid + 2];
        if (p.g_white != nullptr) {
          gd0 += p.g_white[3 * pid];
          gd1 += p.g_white[3 * pid + 1];
          gd2 += p.g_white[3 * pid + 2];
        }
      }
      if (SPEC) {
        gs0 = g0 * p.spec[3 * pid];
        gs1 = g1 * p.spec[3 * pid + 1];
        gs2 = g2 * p.spec[3 * pid + 2];
      }
    }
    if (SPEC) sc = spec_const(valid ? p.rough[pid] : 0.f, g);

    BwdAcc acc = {};
    const BwdPoint gp{gd0, gd1, gd2, gs0, gs1, gs2};
    if (VIS && warp_single_vertex(g))
      bwd_tile_sums<DIFF, SPEC, VIS, true>(p, g, valid, sc, gp, s_tab, env_acc, env_ld, nchunks, warp, NW, lane, acc);
    else
      bwd_tile_sums<DIFF, SPEC, VIS, false>(p, g, valid, sc, gp, s_tab, env_acc, env_ld, nchunks, warp, NW, lane, acc);

    // combine the NW texel ranges in warp order, then finish the per-point chain rule
    float* red = s_red + warp * NACC * 32 + lane;
    const float* av = &acc.Da0;
#pragma unroll
    for (int q = 0; q < NACC; ++q) red[q * 32] = av[q];
    __syncthreads();
    if (warp == 0 && valid) {
      float sums[NACC];
#pragma unroll
      for (int q = 0; q < NACC; ++q) sums[q] = 0.f;
      for (int w = 0; w < NW; ++w) {
        const float* r = s_red + w * NACC * 32 + lane;
#pragma unroll
        for (int q = 0; q < NACC; ++q) sums[q] += r[q * 32];
      }
      const BwdOutputs o{p.g_normal, p.g_view, p.g_albedo, p.g_spec, p.g_rough};
      finish_bwd_point<DIFF, SPEC>(sums, g, sc, SPEC ? p.rough[pid] : 0.f, p.g_shading + 3 * pid, pid, o);
    }
    __syncthreads();
    tile = s_next[it & 1];
    ++it;
  }

  // publish this CTA's env-gradient partial (FP64)
  if (p.env_in_smem) {
    double* dst = p.env_partial + (size_t)blockIdx.x * 3 * p.HWpad;
    for (int i = threadIdx.x; i < 3 * p.HWpad; i += blockDim.x) dst[i] = s_env[i];
  }
}

// Deterministic FP64 sum of the per-CTA env-gradient partials: g_env[c][t] = sum_b partial[b][c][t].
// Block = kReduceCols columns x kReduceRows rows (192 blocks for a 16x32 map, so every SM takes part):
// row y sums partials y, y + kReduceRows, ... in order, then a fixed-order tree over the rows.
constexpr int kReduceCols = 8, kReduceRows = 128;
__global__ void __launch_bounds__(kReduceCols* kReduceRows) des_env_reduce_kernel(const double* __restrict__ partial,
                                                                                  int nparts, int HW, int HWpad,
                                                                                  float* __restrict__ g_env) {
  pdl_enter();
  __shared__ double s[kReduceRows][kReduceCols + 1];
  const int x = threadIdx.x, y = threadIdx.y;
  const int k = blockIdx.x * kReduceCols + x;  // index into [3][HWpad]
  const int n = 3 * HWpad;
  double acc = 0.0;
  if (k < n) {
    for (int b = y; b < nparts; b += kReduceRows) acc += partial[(size_t)b * n + k];
  }
  s[y][x] = acc;
  __syncthreads();
#pragma unroll
  for (int off = kReduceRows / 2; off > 0; off >>= 1) {
    if (y < off) s[y][x] += s[y + off][x];
    __syncthreads();
  }
  if (y == 0 && k < n) {
    const int c = k / HWpad, t = k - c * HWpad;
    if (t < HW) g_env[(size_t)c * HW + t] = (float)s[0][x];
  }
}

// ------------------------------------------------------------------------------------------
// Host-side launch logic
// ------------------------------------------------------------------------------------------

namespace {

struct DeviceInfo {
  int sms = 0;
  int max_smem_optin = 0;
  int smem_per_sm = 0;
};

DeviceInfo device_info(int dev) {
  static std::mutex mu;
  static DeviceInfo cache[64];
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 0 || dev >= 64) return DeviceInfo{};
  if (cache[dev].sms == 0) {
    cudaDeviceGetAttribute(&cache[dev].sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&cache[dev].max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&cache[dev].smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  }
  return cache[dev];
}

// Resident CTAs per SM of `kernel` at this block size and dynamic shared memory, cached per
// (device, kernel, threads, smem); also opts the kernel in to that much dynamic shared memory on
// the current device (once per raise).  Host-side only; keeps per-call overhead to a map lookup.
template <typename K>
int occupancy(K kernel, int threads, size_t smem) {
  struct Key {
    int dev;
    const void* fn;
    int threads;
    size_t smem;
    bool operator<(const Key& o) const {
      return std::tie(dev, fn, threads, smem) < std::tie(o.dev, o.fn, o.threads, o.smem);
    }
  };
  static std::mutex mu;
  static std::map<Key, int> occ_cache;
  static std::map<std::pair<int, const void*>, size_t> optin;
  int dev = 0;
  cudaGetDevice(&dev);
  const Key key{dev, reinterpret_cast<const void*>(kernel), threads, smem};
  std::lock_guard<std::mutex> lk(mu);
  auto it = occ_cache.find(key);
  if (it != occ_cache.end()) return it->second;
  size_t& granted = optin[{dev, key.fn}];
  if (smem > granted) {
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    granted = smem;
  }
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, smem) != cudaSuccess) return 0;
  occ_cache[key] = nb;
  return nb;
}

using KernelFn = void (*)(const ShadeParams);

template <template <bool, bool, bool> class Sel>
KernelFn pick(bool diff, bool spec, bool vis) {
  if (diff) {
    if (spec) return vis ? Sel<true, true, true>::fn() : Sel<true, true, false>::fn();
    return vis ? Sel<true, false, true>::fn() : Sel<true, false, false>::fn();
  }
  return vis ? Sel<false, true, true>::fn() : Sel<false, true, false>::fn();
}
template <bool D, bool S, bool V>
struct FwdSel {
  static KernelFn fn() { return des_fwd_kernel<D, S, V>; }
};
template <bool D, bool S, bool V>
struct BwdSel {
  static KernelFn fn() { return des_bwd_kernel<D, S, V>; }
};

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
// Rows allocated for the [chunk][cell] count table: the chunks, rounded up to a multiple of 4.
inline int sort_row(const LaunchPlan& lp) { return (lp.sort_chunks + 3) / 4 * 4; }

}  // namespace

LaunchPlan plan_launch(int64_t P, int H, int W, bool backward, int dev, bool compact) {
  LaunchPlan lp{};
  const DeviceInfo di = device_info(dev);
  const int HW = H * W;
  lp.HWpad = (HW + 31) / 32 * 32;
  lp.chunk = std::min(lp.HWpad, kChunk);
  lp.ntiles = (int)((P + 31) / 32);
  lp.env_in_smem = backward && (lp.HWpad <= kChunk);
  // texel-split width (warps per tile).  With few tiles, 16 warps share each tile.  Otherwise the
  // width that keeps the most warps resident per SM, from the register bound of the kernel (128 per
  // thread for the adjoint, 64 for the forward), its shared memory and the thread limit; on a tie
  // the adjoint takes the narrowest CTA (more independent tiles in flight, smaller barrier groups)
  // and the forward 8 warps (measured best at 16x32 maps).
  const int nslots = lp.chunk / 32;
  const int nacc = backward ? 15 : 6;
  const int regs = backward ? 128 : 64;
  auto smem_for = [&](int w) {
    return (size_t)lp.chunk * 32 + (lp.env_in_smem ? (size_t)lp.chunk * 24 : 0) + (size_t)w * nacc * 32 * 4;
  };
  int nw = 16;
  if (!(compact && backward) && lp.ntiles >= 2 * std::max(di.sms, 1) && di.smem_per_sm > 0) {
    int best_warps = -1;
    const int order[3] = {backward ? 4 : 8, backward ? 8 : 4, 16};
    for (int w : order) {
      if (w > nslots) continue;
      const int by_regs = 65536 / (regs * 32 * w);
      const int by_smem = (int)((size_t)di.smem_per_sm / (smem_for(w) + 1024));
      const int by_threads = 2048 / (32 * w);
      const int warps = w * std::min(by_regs, std::min(by_smem, by_threads));
      if (warps > best_warps) {
        best_warps = warps;
        nw = w;
      }
    }
  }
  while (nw > 1 && nw > nslots) nw >>= 1;
  lp.nw = nw;
  lp.smem = smem_for(nw);
  lp.sms = di.sms;
  lp.max_smem = di.max_smem_optin;
  lp.sort = !compact && P >= kSortMinP && P <= kSortMaxP;
  lp.sort_chunk = sort_chunk_for(P);
  lp.sort_chunks = lp.sort ? (int)((P + lp.sort_chunk - 1) / lp.sort_chunk) : 0;
  return lp;
}

// Workspace layout: control words | texel table | ordering (when ordering) | env partials (adjoint).
// The permutation starts at the same offset in the forward's and the adjoint's workspace of a
// problem, so one buffer can carry a forward's ordering into the adjoint (DES_REUSE_ORDER).
size_t sort_area_bytes(const LaunchPlan& lp) {
  if (!lp.sort) return 0;
  return align_up((size_t)lp.ntiles * 32 * sizeof(int32_t), 256) +             // permutation
         align_up((size_t)kSortBins * sort_row(lp) * sizeof(unsigned), 256) +  // cell counts [chunk][cell]
         align_up((size_t)lp.ntiles * 32 * sizeof(uint16_t), 256) +            // cell of each point
         align_up((size_t)lp.ntiles * 32 * sizeof(uint32_t), 256);             // rank of each point
}

size_t workspace_bytes(const LaunchPlan& lp, bool backward, int grid) {
  size_t off = kCtrlBytes;
  off += align_up((size_t)lp.HWpad * 32, 256);  // texel table
  off += sort_area_bytes(lp);
  if (backward) off += align_up((size_t)std::max(grid, 1) * 3 * lp.HWpad * sizeof(double), 256);
  return off;
}

// Persistent grid: every CTA resident at once, never more CTAs than tiles.
int shade_grid(const LaunchPlan& lp, unsigned flags, bool backward, bool vis) {
  const bool diff = flags & DES_DIFFUSE, spec = flags & DES_SPECULAR;
  if (!diff && !spec) return 1;
  KernelFn k = backward ? pick<BwdSel>(diff, spec, vis) : pick<FwdSel>(diff, spec, vis);
  const int occ = occupancy(k, lp.nw * 32, lp.smem);
  if (occ <= 0) return 0;
  return std::max(1, std::min(lp.ntiles, occ * lp.sms));
}

namespace {
std::atomic<cudaEvent_t> g_timing_start{nullptr};
std::atomic<cudaEvent_t> g_timing_stop{nullptr};
}  // namespace

void set_timing_events(cudaEvent_t start, cudaEvent_t stop) {
  g_timing_start.store(start);
  g_timing_stop.store(stop);
}

void timing_events(cudaEvent_t& start, cudaEvent_t& stop) {
  start = g_timing_start.load();
  stop = g_timing_stop.load();
}

namespace {
std::atomic<unsigned long long> g_launches{0};
}  // namespace

void count_launches(int n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }
unsigned long long launches_so_far() { return g_launches.load(std::memory_order_relaxed); }

int launch_shade(const ShadeCall& call, des_stream_t stream_) {
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  const des_shade_args& a = *call.args;
  const bool diff = call.flags & DES_DIFFUSE, spec = call.flags & DES_SPECULAR;
  const bool vis = a.visibility != nullptr;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DES_ERR_CUDA;
  const bool compact = (call.flags & DES_COMPACT) != 0;
  LaunchPlan lp = plan_launch(a.P, a.H, a.W, call.backward, dev, compact);
  if (call.flags & DES_INPUT_ORDER) {
    lp.sort = false;
    lp.sort_chunks = 0;
  }
  if (lp.smem > (size_t)lp.max_smem) return DES_ERR_UNSUPPORTED;
  int grid = shade_grid(lp, call.flags, call.backward, vis);
  if (grid <= 0) return DES_ERR_CUDA;
  size_t need = workspace_bytes(lp, call.backward, grid);
  // A workspace sized for a smaller plan (e.g. the allocation-free entry point's static array):
  // shade in input order, then with the compact plan -- same results, less scratch.
  if (lp.sort && call.workspace_bytes < need) {
    lp.sort = false;
    lp.sort_chunks = 0;
    need = workspace_bytes(lp, call.backward, grid);
  }
  if (!compact && call.workspace_bytes < need) {
    lp = plan_launch(a.P, a.H, a.W, call.backward, dev, true);
    if (lp.smem > (size_t)lp.max_smem) return DES_ERR_UNSUPPORTED;
    grid = shade_grid(lp, call.flags, call.backward, vis);
    if (grid <= 0) return DES_ERR_CUDA;
    need = workspace_bytes(lp, call.backward, grid);
  }
  if (call.workspace == nullptr || call.workspace_bytes < need ||
      (reinterpret_cast<uintptr_t>(call.workspace) & 255u) != 0)
    return DES_ERR_WORKSPACE;

  unsigned char* ws = static_cast<unsigned char*>(call.workspace);
  unsigned* ctrl = reinterpret_cast<unsigned*>(ws);
  float4* table = reinterpret_cast<float4*>(ws + kCtrlBytes);
  unsigned char* sort_area = ws + kCtrlBytes + align_up((size_t)lp.HWpad * 32, 256);
  double* env_partial = reinterpret_cast<double*>(sort_area + sort_area_bytes(lp));
  int32_t* perm = reinterpret_cast<int32_t*>(sort_area);
  unsigned* sort_counts =
      reinterpret_cast<unsigned*>(sort_area + align_up((size_t)lp.ntiles * 32 * sizeof(int32_t), 256));
  uint16_t* sort_keys = reinterpret_cast<uint16_t*>(reinterpret_cast<unsigned char*>(sort_counts) +
                                                    align_up((size_t)kSortBins * sort_row(lp) * sizeof(unsigned), 256));
  uint32_t* sort_rank = reinterpret_cast<uint32_t*>(reinterpret_cast<unsigned char*>(sort_keys) +
                                                    align_up((size_t)lp.ntiles * 32 * sizeof(uint16_t), 256));

  // texel table + control-word reset (+ step 1 of the ordering when ordering, unless the workspace
  // already holds this problem's ordering from the previous call on it)
  const bool sort = lp.sort && a.P > 0 && (diff || spec);
  const bool reuse = sort && (call.flags & DES_REUSE_ORDER) != 0;
  // an adjoint right after its forward on this workspace: the table (and the ordering, when the
  // call orders its points and reuses it) are there already, and its tile counter is still zero
  const bool reuse_table = call.backward && (call.flags & DES_REUSE_TABLE) != 0 && (!sort || reuse);
  if (reuse_table) {
    // nothing to launch before the adjoint
  } else if (sort && !reuse) {
    launch_pdl(des_prep_kernel, dim3(lp.sort_chunks), dim3(kSortThreads), 0, stream, a.H, a.W, lp.HWpad,
               a.light2obj_rotmat, a.envmap, table, ctrl, a.normal, a.P, lp.sort_chunk, sort_counts, sort_keys,
               sort_rank);
  } else {
    const int threads = 256;
    const int blocks = (lp.HWpad + threads - 1) / threads;
    launch_pdl(des_table_kernel, dim3(blocks), dim3(threads), 0, stream, a.H, a.W, lp.HWpad, a.light2obj_rotmat,
               a.envmap, table, nullptr, ctrl);
  }
  if (cudaGetLastError() != cudaSuccess) return DES_ERR_CUDA;
  if (!reuse_table) count_launches(1);
  if (a.P == 0) {
    if (call.backward && call.g_envmap != nullptr)
      if (cudaMemsetAsync(call.g_envmap, 0, sizeof(float) * 3 * (size_t)a.H * a.W, stream) != cudaSuccess)
        return DES_ERR_CUDA;
    return DES_OK;
  }
  if (!diff && !spec) {
    // nothing to integrate: every output is zero (reference allocates zeros for disabled terms)
    const size_t pb = sizeof(float) * 3 * (size_t)a.P;
    cudaError_t e = cudaSuccess;
    if (!call.backward) {
      e = cudaMemsetAsync(call.shading, 0, pb, stream);
      if (e == cudaSuccess && call.white) e = cudaMemsetAsync(call.white, 0, pb, stream);
    } else {
      float* outs[4] = {call.g_normal, call.g_view, call.g_albedo, call.g_spec};
      for (float* o : outs)
        if (o && e == cudaSuccess) e = cudaMemsetAsync(o, 0, pb, stream);
      if (call.g_rough && e == cudaSuccess) e = cudaMemsetAsync(call.g_rough, 0, pb / 3, stream);
      if (call.g_envmap && e == cudaSuccess)
        e = cudaMemsetAsync(call.g_envmap, 0, sizeof(float) * 3 * (size_t)a.H * a.W, stream);
    }
    return e == cudaSuccess ? DES_OK : DES_ERR_CUDA;
  }

  ShadeParams prm{};
  prm.P = a.P;
  prm.HWpad = lp.HWpad;
  prm.chunk = lp.chunk;
  prm.ntiles = lp.ntiles;
  prm.N_face = a.N_face;
  prm.N_vertex = a.N_vertex;
  prm.normal = a.normal;
  prm.view = a.view_dir;
  prm.albedo = a.albedo;
  prm.spec = a.specular_albedo;
  prm.rough = a.roughness;
  prm.faces = a.face_vertex_list;
  prm.tri = a.nearest_triangle_id;
  prm.bary = a.barycentric_coord;
  prm.vis = a.visibility;
  prm.table = table;
  prm.clamp = (call.flags & DES_CLAMP) != 0;
  prm.ctrl = ctrl;
  prm.shading = call.shading;
  prm.white = call.white;
  prm.g_shading = call.g_shading;
  prm.g_white = call.g_white;
  prm.g_normal = call.g_normal;
  prm.g_view = call.g_view;
  prm.g_albedo = call.g_albedo;
  prm.g_spec = call.g_spec;
  prm.g_rough = call.g_rough;
  prm.env_partial = env_partial;
  prm.env_in_smem = lp.env_in_smem;
  prm.perm = nullptr;
  if (sort && !reuse) {
    launch_pdl(des_place_kernel, dim3(lp.sort_chunks), dim3(kSortBins), 0, stream, a.P, lp.sort_chunk,
               lp.sort_chunks, sort_counts, sort_keys, sort_rank, perm);
    if (cudaGetLastError() != cudaSuccess) return DES_ERR_CUDA;
    count_launches(1);
  }
  if (sort) prm.perm = perm;

  KernelFn k = call.backward ? pick<BwdSel>(diff, spec, vis) : pick<FwdSel>(diff, spec, vis);
  cudaEvent_t ev0 = g_timing_start.load(), ev1 = g_timing_stop.load();
  if (ev0 != nullptr && ev1 != nullptr) cudaEventRecord(ev0, stream);
  launch_pdl(k, dim3(grid), dim3(lp.nw * 32), lp.smem, stream, prm);
  if (cudaGetLastError() != cudaSuccess) return DES_ERR_CUDA;
  count_launches(1);
  if (ev0 != nullptr && ev1 != nullptr) cudaEventRecord(ev1, stream);

  if (call.backward && call.g_envmap != nullptr) {
    const dim3 rb(kReduceCols, kReduceRows);
    const int rg = (3 * lp.HWpad + kReduceCols - 1) / kReduceCols;
    launch_pdl(des_env_reduce_kernel, dim3(rg), dim3(rb), 0, stream, env_partial, grid, a.H * a.W, lp.HWpad,
               call.g_envmap);
    if (cudaGetLastError() != cudaSuccess) return DES_ERR_CUDA;
    count_launches(1);
  }
  return DES_OK;
}

size_t point_order_scratch_bytes(int64_t P) {
  const int64_t chunk = sort_chunk_for(P), nchunks = (P + chunk - 1) / chunk, ncp = (nchunks + 3) / 4 * 4;
  return align_up((size_t)kSortBins * ncp * sizeof(unsigned), 256) + align_up((size_t)P * sizeof(uint16_t), 256) +
         align_up((size_t)P * sizeof(uint32_t), 256);
}

int launch_point_order(const float* normal, int64_t P, void* scratch, int32_t* perm, cudaStream_t stream) {
  if (P <= 0 || P > kSortMaxP) return DES_ERR_INVALID_ARGUMENT;
  const int chunk = sort_chunk_for(P);
  const int nchunks = (int)((P + chunk - 1) / chunk), ncp = (nchunks + 3) / 4 * 4;
  unsigned* counts = static_cast<unsigned*>(scratch);
  uint16_t* keys = reinterpret_cast<uint16_t*>(static_cast<unsigned char*>(scratch) +
                                               align_up((size_t)kSortBins * ncp * sizeof(unsigned), 256));
  uint32_t* rank = reinterpret_cast<uint32_t*>(reinterpret_cast<unsigned char*>(keys) +
                                               align_up((size_t)P * sizeof(uint16_t), 256));
  launch_pdl(des_prep_kernel, dim3(nchunks), dim3(kSortThreads), 0, stream, 0, 0, 0, nullptr, nullptr, nullptr, nullptr,
             normal, P, chunk, counts, keys, rank);
  launch_pdl(des_place_kernel, dim3(nchunks), dim3(kSortBins), 0, stream, P, chunk, nchunks, counts, keys, rank, perm);
  count_launches(2);
  return cudaGetLastError() == cudaSuccess ? DES_OK : DES_ERR_CUDA;
}

int launch_table(int H, int W, int HWpad, const float* R, const float* env, float4* rec, unsigned* ctrl,
                 cudaStream_t stream) {
  const int threads = 256;
  launch_pdl(des_table_kernel, dim3((HWpad + threads - 1) / threads), dim3(threads), 0, stream, H, W, HWpad, R, env,
             rec, nullptr, ctrl);
  count_launches(1);
  return cudaGetLastError() == cudaSuccess ? DES_OK : DES_ERR_CUDA;
}

int launch_texel_table(int H, int W, const float* R, float* out, des_stream_t stream_) {
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  const int HWpad = (H * W + 31) / 32 * 32;
  const int threads = 256;
  launch_pdl(des_table_kernel, dim3((HWpad + threads - 1) / threads), dim3(threads), 0, stream, H, W, HWpad, R,
             nullptr, nullptr, out, nullptr);
  count_launches(1);
  return cudaGetLastError() == cudaSuccess ? DES_OK : DES_ERR_CUDA;
}

}  // namespace des
