// Serving: continuous batching of shading requests onto the GPU.
//
// Requests (forward, or forward + adjoint) of any point count arrive asynchronously.  A native
// scheduler thread
//   * admits them in arrival order while a device arena of fixed size (the HBM budget) has room,
//     skipping over requests that do not fit yet, and uploads their point data through a copy lane
//     that sends the lowest-ranked request first, in slices (downloads use a second lane);
//     requests shaded in input order whose buffers the device can reach (its own memory, pinned
//     host memory) skip the copies: the batch kernel reads their inputs and stores their outputs
//     in place;
//   * keeps env maps (their texel tables) and meshes (faces + visibility words) resident, shared by
//     reference between requests;
//   * every tick packs 32-point tiles of the ready requests, lowest rank first (remaining points x
//     texels, or remaining work), up to a time budget, into a work list, copies the list (and the
//     descriptors of requests it names for the first time) to the device and launches it as a CUDA
//     graph (one persistent batch kernel) on its own stream, with up to ticks_in_flight ticks
//     queued so that consecutive ticks overlap;
//   * when every tile of a request has finished, copies its outputs back (unless they were stored
//     in place) and frees its memory.
// Work of different requests therefore shares each launch and each SM; a request that arrives
// while others run joins the next tick.
//
// Requests of at least order_min_points points (off by default) are ordered by normal direction
// after their upload (the plain path's ordering kernels, on a stream of their own); the batch
// kernel skips texels below the horizon of a warp's 32 points, as des_fwd_kernel / des_bwd_kernel
// do, in either order.
// The batch kernel evaluates exactly the per-pair arithmetic of des_fwd_kernel / des_bwd_kernel
// (shared helpers in des_point.cuh); per-point outputs are bit-identical to a solo call of the
// batch path, and the env-map gradient is summed per request in FP64 (global FP64 atomics, then a
// final FP32 conversion by whichever CTA finishes the request's last adjoint tile).  A request with
// gradients runs adjoint tiles only: the adjoint integrates the forward weights too, and its sums
// give the request's shading (equal to a forward tile's within rounding), a third less work than
// running both.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <cstddef>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <unordered_set>
#include <tuple>
#include <thread>
#include <vector>

#include "des_internal.h"
#include "des_math.cuh"
#include "des_point.cuh"
#include "diff_envshade_b200.h"

namespace des {
namespace serve {

constexpr int kNW = 8;               // warps per CTA
constexpr int kMaxHWpad = 2048;      // texel table kept in shared memory per CTA
constexpr int kMaxSlots = 8192;      // concurrently admitted requests
constexpr int kTickItems = 4096;     // work items per tick (upper bound; the whole list is uploaded)
constexpr int kNTicks = 4;           // tick buffers (up to this many ticks in flight)
constexpr int kQueuedTicks = 1;      // launched ticks not yet started by the GPU, at most
constexpr int kCopyEvents = 64;                    // completion events per copy lane
// Default ordering threshold of the server (requests of at least this many points are ordered by
// normal direction): none.  An ordered request must be uploaded (the ordering kernels and the
// permuted tiles read device memory), and on a busy host link those uploads slow the in-place
// reads of every other request; the ordering kernels also wait for SMs behind the queued ticks.
// Measured on the mixed serving workload, shading everything in input order and in place gives
// the 50k-100k-point requests the lowest tail latency, at about a sixth less throughput than
// ordering the requests of 128k points and more.
constexpr int64_t kServeOrderMinP = INT64_MAX;
// Throughput of the batch kernel on a 148-SM B200 in pair units per microsecond (a forward pair is
// one unit, an adjoint pair two), measured on mixed workloads; it converts tick_us into work.  A
// fixed figure: an estimate taken from the ticks themselves feeds back on itself (under-filled
// ticks leave SMs idle, which lowers the estimate, which shrinks the ticks).  (A per-tile cost model
// fitted to single-request ticks made the mixed workload's ticks smaller and lost throughput
// without shortening the tail.)
constexpr double kBatchPairsPerUs = 3.5e5;

// Device-side request descriptor (member names shared with ShadeParams for the point loaders).
struct ReqDesc {
  int64_t P;
  int HW, HWpad;
  int diff, spec, has_vis;
  bool clamp;
  const float* normal;
  const float* view;
  const float* albedo;
  const float* spec_alb;
  const float* rough;
  const float4* table;
  int N_face, N_vertex;
  const int32_t* faces;
  const int64_t* tri;
  const float* bary;
  const uint32_t* vis;
  const float* g_shading;
  const float* g_white;
  float* shading;
  float* white;
  float* g_normal;
  float* g_view;
  float* g_albedo;
  float* g_spec;
  float* g_rough;
  float* g_env;
  const int32_t* perm;       // tile slot -> point (normal-direction order), or null for input order
  double* env_acc;           // [3][HWpad], zero when the request starts (zeroed again by its last tile)
  unsigned bwd_target;       // the slot's adjoint-tile counter after the request's last adjoint tile
  unsigned pad_[3];
  unsigned* ctrl;            // [kCtrlError] = error word
};
static_assert(sizeof(ReqDesc) % 16 == 0, "descriptors are staged in 16-byte words");

struct WorkItem {
  int32_t req, tile, kind, pad;  // kind 0 = forward tile, 1 = adjoint tile
};

// One tick's work, written by the scheduler into pinned host memory and copied to the device ahead of
// the tick's launch, on the tick's stream (n and the first n items), so that the batch kernel reads
// its work items, the first ones included, from device memory.  `started` is the exception: the CTA
// that claims item 0 sets it in the host copy (mapped), where the scheduler reads it.
struct WorkList {
  unsigned n;        // items in the list (written by the scheduler)
  unsigned started;  // set to 1 by the CTA that claims item 0 (the tick is running)
  unsigned pad0, pad1;
  WorkItem items[kTickItems];
};

// Device-side control of one tick buffer: [0] next item, [1] CTAs finished.  The last CTA of a
// launch resets both, so every launch starts from zero without a host-side reset.
struct TickCtl {
  unsigned next, exited, pad0, pad1;
};

// ---------------------------------------------------------------------------------------------
// Batch kernel
// ---------------------------------------------------------------------------------------------

// Dynamic shared memory of the batch kernel: texel table [kMaxHWpad x 32 B], per-warp reduction
// rows [kNW x 15 x 32 floats], then two buffers of prefetched tile points.
constexpr size_t kSmemPts = (size_t)kMaxHWpad * 32 + (size_t)kNW * 15 * 32 * 4;

// Asynchronous copies global -> shared (cp.async): 16 bytes bypassing L1, 4 bytes (zero-filled
// when !ok, nothing read then), and the wait for all of the thread's copies.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(__cvta_generic_to_global(gmem))
               : "memory");
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem, bool ok) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(__cvta_generic_to_global(gmem)),
               "r"(ok ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// The inputs of one tile's 32 consecutive points (a request in input order), copied into shared
// memory with cp.async while the CTA computes the tile before it, so that the tile starts with its
// points on chip (for inputs read in place from host memory, without a round trip over the host
// link).  Entries past the request's last point are zero.
struct TilePoints {
  float normal[96], view[96], albedo[96], spec[96], gsh[96], gwh[96], bary[96], rough[32];
  int64_t tri[32];
};

// A staged tile in the shape the point loader expects (index = lane, barycentric rows 32 apart).
struct TileView {
  const float* normal;
  const float* view;
  const int64_t* tri;
  const float* bary;
  int64_t P;
  int N_face, N_vertex;
  const int32_t* faces;
  unsigned* ctrl;
  bool clamp;
};

__device__ __forceinline__ TileView tile_view(const ReqDesc& r, const TilePoints* t) {
  return TileView{t->normal, t->view, t->tri, t->bary, 32, r.N_face, r.N_vertex, r.faces, r.ctrl, r.clamp};
}

// Issues the copies of tile `tile` of request r (input order) into t: threads 0..127 copy 4-byte
// words (a warp's copies cover whole 128-byte rows).  Completed by cp_async_wait_all.
__device__ __forceinline__ void prefetch_points(const ReqDesc& r, int tile, bool adjoint, TilePoints* t) {
  const int64_t first = (int64_t)tile * 32;
  const int n = (int)min((int64_t)32, r.P - first);
  const int i = threadIdx.x;
  if (i < 96) {
    const bool ok = i < 3 * n;
    const int64_t o = ok ? 3 * first + i : 0;
    cp_async4(&t->normal[i], r.normal + o, ok);
    cp_async4(&t->view[i], r.view + o, ok);
    cp_async4(&t->albedo[i], r.albedo + o, ok);
    cp_async4(&t->spec[i], r.spec_alb + o, ok);
    if (adjoint) {
      cp_async4(&t->gsh[i], r.g_shading + o, ok);
      if (r.g_white != nullptr) cp_async4(&t->gwh[i], r.g_white + o, ok);
    }
  } else if (i < 128) {
    const int l = i - 96;
    const bool ok = l < n;
    const int64_t pid = ok ? first + l : 0;
    cp_async4(&t->rough[l], r.rough + pid, ok);
    if (r.has_vis) {
      const float* tw = reinterpret_cast<const float*>(r.tri + pid);
      float* td = reinterpret_cast<float*>(&t->tri[l]);
      cp_async4(td, tw, ok);
      cp_async4(td + 1, tw + 1, ok);
      cp_async4(&t->bary[l], r.bary + pid, ok);
      cp_async4(&t->bary[32 + l], r.bary + (ok ? pid + r.P : 0), ok);
      cp_async4(&t->bary[64 + l], r.bary + (ok ? pid + 2 * r.P : 0), ok);
    }
  }
}

// The tiles run the shading kernels' per-pair arithmetic with the same point ordering, horizon
// skip and mirrored texel split (des_shade.cu), so per-point results equal the plain path's
// arithmetic for the same point and texel, whatever else shares the launch.

// The kNW warps' share of a tile's texel slots (mirrored pairs); a slot whose visibility words are
// zero for all 32 lanes is skipped.
template <bool DIFF, bool SPEC, bool VIS, bool ONEV>
__device__ __forceinline__ void fwd_tile_slots(const ReqDesc& r, const PointGeom& g, bool valid, const SpecConst& sc,
                                               const float4* s_tab, float (&acc)[6]) {
  const int warp = threadIdx.x >> 5;
  const float cs = (g.c0 + g.c1) + g.c2;
  const int nsl = r.HWpad >> 5;
  const int ushift = ((nsl + 1) >> 1) >= kNW ? 1 : 0;
  // the visibility words of a warp's next slot are loaded while it integrates the current one
  uint32_t n0 = 0u, n1 = 0u, n2 = 0u;
  int sl = warp_slot(0, warp, kNW, nsl, ushift);
  if (VIS && sl >= 0) load_vis_words<ONEV>(r, g, valid, sl, n0, n1, n2);
  for (int k = 1; sl >= 0; ++k) {
    const int cur = sl;
    sl = warp_slot(k, warp, kNW, nsl, ushift);
    const uint32_t w0 = n0, w1 = n1, w2 = n2;
    if (VIS) {
      if (sl >= 0) load_vis_words<ONEV>(r, g, valid, sl, n0, n1, n2);
      if (!__any_sync(0xffffffffu, (w0 | w1 | w2) != 0u)) continue;
    }
    fwd_slot<DIFF, SPEC, VIS, ONEV>(g, sc, cs, s_tab + 2 * (cur << 5), w0, w1, w2, acc);
  }
}

// As fwd_tile_slots for the adjoint; each 8-texel group's env-map gradient is added to the
// request's FP64 accumulator.
template <bool DIFF, bool SPEC, bool VIS, bool ONEV>
__device__ __forceinline__ void bwd_tile_slots(const ReqDesc& r, const PointGeom& g, bool valid, const SpecConst& sc,
                                               const BwdPoint& gp, const float4* s_tab, BwdAcc& acc) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const float cs = (g.c0 + g.c1) + g.c2;
  const int nsl = r.HWpad >> 5;
  const int ushift = ((nsl + 1) >> 1) >= kNW ? 1 : 0;
  const int jsel = butterfly_texel(lane);
  uint32_t n0 = 0u, n1 = 0u, n2 = 0u;
  int sl = warp_slot(0, warp, kNW, nsl, ushift);
  if (VIS && sl >= 0) load_vis_words<ONEV>(r, g, valid, sl, n0, n1, n2);
  for (int k = 1; sl >= 0; ++k) {
    const int cur = sl;
    sl = warp_slot(k, warp, kNW, nsl, ushift);
    const uint32_t w0 = n0, w1 = n1, w2 = n2;
    if (VIS) {
      if (sl >= 0) load_vis_words<ONEV>(r, g, valid, sl, n0, n1, n2);
      if (!__any_sync(0xffffffffu, (w0 | w1 | w2) != 0u)) continue;
    }
    const int t0 = (cur << 5) + jsel;
    auto sink = [&](int gq, float y0, float y1, float y2) {
      if ((lane & 3) == 0) {
        const int t = t0 + gq * 8;
        atomicAdd(r.env_acc + t, (double)y0);
        atomicAdd(r.env_acc + r.HWpad + t, (double)y1);
        atomicAdd(r.env_acc + 2 * r.HWpad + t, (double)y2);
      }
    };
    bwd_slot<DIFF, SPEC, VIS, ONEV>(g, sc, cs, gp, s_tab + 2 * (cur << 5), w0, w1, w2, lane, acc, sink);
  }
}

template <bool DIFF, bool SPEC, bool VIS>
// pts: the tile's points already in shared memory (input order), or null to read them from r.
__device__ void fwd_tile(const ReqDesc& r, int tile, const float4* s_tab, float* s_red, const TilePoints* pts) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t slot = (int64_t)tile * 32 + lane;
  int64_t pid = slot;
  const bool valid = ordered_point(r.perm, slot, r.P, r.ctrl, pid);
  const PointGeom g = pts ? load_geom<VIS>(tile_view(r, pts), lane, valid, SPEC || r.clamp)
                          : load_geom<VIS>(r, pid, valid, SPEC || r.clamp);
  SpecConst sc;
  if (SPEC) sc = spec_const(valid ? (pts ? pts->rough[lane] : r.rough[pid]) : 0.f, g);
  // the epilogue's albedos, fetched with the point
  float alb[3] = {0.f, 0.f, 0.f}, spa[3] = {0.f, 0.f, 0.f};
  if (warp == 0 && valid) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (DIFF) alb[c] = pts ? pts->albedo[3 * lane + c] : r.albedo[3 * pid + c];
      if (SPEC) spa[c] = pts ? pts->spec[3 * lane + c] : r.spec_alb[3 * pid + c];
    }
  }
  float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (VIS && warp_single_vertex(g))
    fwd_tile_slots<DIFF, SPEC, VIS, true>(r, g, valid, sc, s_tab, acc);
  else
    fwd_tile_slots<DIFF, SPEC, VIS, false>(r, g, valid, sc, s_tab, acc);
  float* red = s_red + warp * 6 * 32 + lane;
#pragma unroll
  for (int q = 0; q < 6; ++q) red[q * 32] = acc[q];
  __syncthreads();
  if (warp == 0) {
    float s[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int w = 0; w < kNW; ++w)
#pragma unroll
      for (int q = 0; q < 6; ++q) s[q] += s_red[w * 6 * 32 + q * 32 + lane];
    float out[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      out[c] = 0.f;
      if (DIFF) out[c] = alb[c] * s[c];
      if (SPEC) out[c] = fmaf(spa[c], s[3 + c], out[c]);
    }
    if (r.perm == nullptr) {  // consecutive points: whole-row stores (outputs may be in host memory)
      const int64_t first = (int64_t)tile * 32;
      store_rows3(r.shading, first, r.P, out[0], out[1], out[2], lane);
      if (r.white != nullptr) store_rows3(r.white, first, r.P, s[0], s[1], s[2], lane);
    } else if (valid) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        r.shading[3 * pid + c] = out[c];
        if (r.white != nullptr) r.white[3 * pid + c] = s[c];
      }
    }
  }
}

// A point's forward outputs from the adjoint's sums: sums[0..2] = sum of wd L_c (the diffuse
// shading), sums[3..5] = sum of ws L_c, the forward tile's accumulators integrated over the same
// texels in the same order (the pair weights are rounded in another association, so the outputs
// equal a forward tile's within rounding).
template <bool DIFF, bool SPEC>
__device__ __forceinline__ void fwd_outputs(const float* alb, const float* spa, bool valid, const float (&sums)[15],
                                            float (&out)[3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    out[c] = 0.f;
    if (DIFF) out[c] = (valid ? alb[c] : 0.f) * sums[c];
    if (SPEC) out[c] = fmaf(valid ? spa[c] : 0.f, sums[3 + c], out[c]);
  }
}

template <bool DIFF, bool SPEC, bool VIS>
// pts: the tile's points already in shared memory (input order), or null to read them from r.
__device__ void bwd_tile(const ReqDesc& r, int tile, const float4* s_tab, float* s_red, const TilePoints* pts) {
  constexpr int NACC = 15;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t slot = (int64_t)tile * 32 + lane;
  int64_t pid = slot;
  const bool valid = ordered_point(r.perm, slot, r.P, r.ctrl, pid);
  const PointGeom g = pts ? load_geom<VIS>(tile_view(r, pts), lane, valid, SPEC || r.clamp)
                          : load_geom<VIS>(r, pid, valid, SPEC || r.clamp);
  // the point's own inputs: staged (index lane) or the request's arrays (index pid)
  const int64_t ix = pts ? lane : pid;
  const float* in_gsh = pts ? pts->gsh : r.g_shading;
  const float* in_gwh = pts ? pts->gwh : r.g_white;
  const float* in_alb = pts ? pts->albedo : r.albedo;
  const float* in_spa = pts ? pts->spec : r.spec_alb;
  float gd0 = 0.f, gd1 = 0.f, gd2 = 0.f, gs0 = 0.f, gs1 = 0.f, gs2 = 0.f;
  if (valid) {
    const float g0 = in_gsh[3 * ix], g1 = in_gsh[3 * ix + 1], g2 = in_gsh[3 * ix + 2];
    if (DIFF) {
      gd0 = g0 * in_alb[3 * ix];
      gd1 = g1 * in_alb[3 * ix + 1];
      gd2 = g2 * in_alb[3 * ix + 2];
      if (r.g_white != nullptr) {
        gd0 += in_gwh[3 * ix];
        gd1 += in_gwh[3 * ix + 1];
        gd2 += in_gwh[3 * ix + 2];
      }
    }
    if (SPEC) {
      gs0 = g0 * in_spa[3 * ix];
      gs1 = g1 * in_spa[3 * ix + 1];
      gs2 = g2 * in_spa[3 * ix + 2];
    }
  }
  SpecConst sc;
  if (SPEC) sc = spec_const(valid ? (pts ? pts->rough[lane] : r.rough[pid]) : 0.f, g);
  const BwdPoint gp{gd0, gd1, gd2, gs0, gs1, gs2};
  BwdAcc acc = {};
  if (VIS && warp_single_vertex(g))
    bwd_tile_slots<DIFF, SPEC, VIS, true>(r, g, valid, sc, gp, s_tab, acc);
  else
    bwd_tile_slots<DIFF, SPEC, VIS, false>(r, g, valid, sc, gp, s_tab, acc);
  float* red = s_red + warp * NACC * 32 + lane;
  const float* av = &acc.Da0;
#pragma unroll
  for (int q = 0; q < NACC; ++q) red[q * 32] = av[q];
  __syncthreads();
  if (warp == 0) {
    float sums[NACC];
#pragma unroll
    for (int q = 0; q < NACC; ++q) sums[q] = 0.f;
    for (int w = 0; w < kNW; ++w)
#pragma unroll
      for (int q = 0; q < NACC; ++q) sums[q] += s_red[w * NACC * 32 + q * 32 + lane];
    if (r.perm == nullptr) {  // consecutive points: whole-row stores (outputs may be in host memory)
      const float rough = (SPEC && valid) ? (pts ? pts->rough[lane] : r.rough[pid]) : 0.f;
      const float g0 = valid ? in_gsh[3 * ix] : 0.f, g1 = valid ? in_gsh[3 * ix + 1] : 0.f,
                  g2 = valid ? in_gsh[3 * ix + 2] : 0.f;
      const BwdGrads q = bwd_point_grads<DIFF, SPEC>(sums, g, sc, rough, g0, g1, g2);
      const int64_t first = (int64_t)tile * 32;
      float out[3];
      fwd_outputs<DIFF, SPEC>(in_alb + 3 * ix, in_spa + 3 * ix, valid, sums, out);
      store_rows3(r.shading, first, r.P, out[0], out[1], out[2], lane);
      if (r.white != nullptr) store_rows3(r.white, first, r.P, sums[0], sums[1], sums[2], lane);
      store_rows3(r.g_normal, first, r.P, q.n[0], q.n[1], q.n[2], lane);
      if (r.g_albedo != nullptr) store_rows3(r.g_albedo, first, r.P, q.a[0], q.a[1], q.a[2], lane);
      if (r.g_spec != nullptr) store_rows3(r.g_spec, first, r.P, q.s[0], q.s[1], q.s[2], lane);
      if (r.g_view != nullptr) store_rows3(r.g_view, first, r.P, q.v[0], q.v[1], q.v[2], lane);
      if (r.g_rough != nullptr && valid) r.g_rough[pid] = q.rough;
    } else if (valid) {
      float out[3];
      fwd_outputs<DIFF, SPEC>(in_alb + 3 * ix, in_spa + 3 * ix, valid, sums, out);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        r.shading[3 * pid + c] = out[c];
        if (r.white != nullptr) r.white[3 * pid + c] = sums[c];
      }
      const BwdOutputs o{r.g_normal, r.g_view, r.g_albedo, r.g_spec, r.g_rough};
      finish_bwd_point<DIFF, SPEC>(sums, g, sc, SPEC ? r.rough[pid] : 0.f, r.g_shading + 3 * pid, pid, o);
    }
  }
}

template <bool FWD>
__device__ __forceinline__ void dispatch_tile(const ReqDesc& r, int tile, const float4* s_tab, float* s_red,
                                              const TilePoints* pts) {
  const int key = (r.diff ? 4 : 0) | (r.spec ? 2 : 0) | (r.has_vis ? 1 : 0);
  switch (key) {
#define DES_TILE_CASE(K, D, S, V)                                       \
  case K:                                                               \
    if (FWD) fwd_tile<D, S, V>(r, tile, s_tab, s_red, pts);             \
    else bwd_tile<D, S, V>(r, tile, s_tab, s_red, pts);                 \
    break;
    DES_TILE_CASE(7, true, true, true)
    DES_TILE_CASE(6, true, true, false)
    DES_TILE_CASE(5, true, false, true)
    DES_TILE_CASE(4, true, false, false)
    DES_TILE_CASE(3, false, true, true)
    DES_TILE_CASE(2, false, true, false)
#undef DES_TILE_CASE
    default:
      break;
  }
}

// reqs: the slots' descriptors in device memory, copied there by the scheduler on the stream of the
// first tick that names the slot, before its launch; a CTA copies the descriptor of the request it
// works on into shared memory (once per change of request).  wl: the tick's work list (device copy).
// started: the work list's flag that the CTA claiming item 0 sets (mapped host memory; the
// scheduler reads it).  slot_tiles: per slot, the adjoint tiles finished so far over all of the
// slot's requests (never reset).
__global__ void __launch_bounds__(kNW * 32, 2) batch_kernel(const ReqDesc* __restrict__ reqs,
                                                            const WorkList* __restrict__ wl,
                                                            unsigned* started, TickCtl* ctl,
                                                            unsigned* __restrict__ slot_tiles,
                                                            unsigned* __restrict__ ctrl) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* s_tab = reinterpret_cast<float4*>(smem_raw);
  float* s_red = reinterpret_cast<float*>(smem_raw + (size_t)kMaxHWpad * 32);
  TilePoints* s_pts = reinterpret_cast<TilePoints*>(smem_raw + kSmemPts);  // two buffers
  __shared__ __align__(16) ReqDesc s_desc;
  __shared__ int s_idx[3];
  __shared__ __align__(16) WorkItem s_item[3];
  __shared__ int s_pf_req[2], s_pf_tile[2], s_pf_kind[2];  // what each point buffer holds (req -1: nothing)
  __shared__ int s_last;
  const unsigned n = wl->n;
  int staged_req = -1;
  const float4* staged_table = nullptr;
  // Work items go through a ring of three: while the CTA computes item `it`, item it+1 is already
  // in shared memory (its points are being prefetched), and thread 0 copies item it+2 in from the
  // device copy of the work list with cp.async and claims the index after it.  Every thread
  // waits for its own copies just before the barrier that ends the iteration.
  int claimed = 0;
  if (threadIdx.x == 0) {
    for (int j = 0; j < 2; ++j) {
      const int i0 = (int)atomicAdd(&ctl->next, 1u);
      s_idx[j] = i0;
      if (i0 == 0) *reinterpret_cast<volatile unsigned*>(started) = 1u;  // tells the scheduler
      if (i0 < (int)n) s_item[j] = wl->items[i0];
      s_pf_req[j] = -1;
    }
    claimed = (int)atomicAdd(&ctl->next, 1u);
  }
  __syncthreads();
  for (int it = 0;; ++it) {
    const int idx = s_idx[it % 3];
    if (idx >= (int)n) break;
    const WorkItem item = s_item[it % 3];
    const bool has_next = s_idx[(it + 1) % 3] < (int)n;
    const WorkItem next = s_item[(it + 1) % 3];
    const int pb = it & 1;  // point buffer of this item; the next item's is pb ^ 1
    const bool pre = s_pf_req[pb] == item.req && s_pf_tile[pb] == item.tile && s_pf_kind[pb] == item.kind;
    __syncthreads();  // everyone has read the ring and the buffer tags before thread 0 rewrites them
    if (threadIdx.x == 0) {
      s_idx[(it + 2) % 3] = claimed;
      if (claimed < (int)n) cp_async16(&s_item[(it + 2) % 3], &wl->items[claimed]);
      claimed = (int)atomicAdd(&ctl->next, 1u);
      s_pf_req[pb ^ 1] = -1;
    }
    // a malformed work item is reported and skipped, never dereferenced
    if (item.req < 0 || item.req >= kMaxSlots || (item.kind != 0 && item.kind != 1) || item.tile < 0) {
      if (threadIdx.x == 0) atomicOr(&ctrl[kCtrlError], 4u);
      cp_async_wait_all();
      __syncthreads();
      continue;
    }
    if (item.req != staged_req) {
      // plain loads: the descriptor reached device memory before the launch of the first tick that
      // names the slot (stream order), and stays unchanged while any tick names the slot
      constexpr int kWords = (int)(sizeof(ReqDesc) / 16);
      const uint4* src = reinterpret_cast<const uint4*>(reqs + item.req);
      uint4* dst = reinterpret_cast<uint4*>(&s_desc);
      if (threadIdx.x < kWords) dst[threadIdx.x] = src[threadIdx.x];
      __syncthreads();
      staged_req = item.req;
      if (s_desc.table != staged_table) {
        stage_table(s_tab, s_desc.table, 0, s_desc.HWpad);
        staged_table = s_desc.table;
      }
      __syncthreads();
    }
    const ReqDesc& r = s_desc;
    if ((int64_t)item.tile * 32 >= r.P) {
      if (threadIdx.x == 0) atomicOr(&ctrl[kCtrlError], 4u);
      cp_async_wait_all();
      __syncthreads();
      continue;
    }
    // the next item continues this request in input order: copy its points in while this one runs
    if (has_next && next.req == item.req && r.perm == nullptr && (next.kind == 0 || next.kind == 1) &&
        next.tile >= 0 && (int64_t)next.tile * 32 < r.P) {
      prefetch_points(r, next.tile, next.kind == 1, &s_pts[pb ^ 1]);
      if (threadIdx.x == 0) {
        s_pf_req[pb ^ 1] = next.req;
        s_pf_tile[pb ^ 1] = next.tile;
        s_pf_kind[pb ^ 1] = next.kind;
      }
    }
    // a tile in input order whose points were not prefetched (the CTA's first item of the tick, or
    // the first after a change of request): the same copies into this item's buffer, completed
    // before the tile starts, so that the warps read the 32 points from shared memory instead of
    // each warp fetching all of them itself (over the host link for inputs read in place)
    bool staged = pre;
    if (!pre && r.perm == nullptr) {
      prefetch_points(r, item.tile, item.kind == 1, &s_pts[pb]);
      cp_async_wait_all();
      __syncthreads();
      staged = true;
    }
    const TilePoints* pts = staged ? &s_pts[pb] : nullptr;
    if (item.kind == 0) {
      dispatch_tile<true>(r, item.tile, s_tab, s_red, pts);
    } else {
      dispatch_tile<false>(r, item.tile, s_tab, s_red, pts);
      // the CTA that finishes a request's last adjoint tile converts its FP64 env gradient and
      // leaves the accumulator zeroed for its next user
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        s_last = (atomicAdd(slot_tiles + item.req, 1u) + 1u == r.bwd_target) ? 1 : 0;
      }
      __syncthreads();
      if (s_last) {
        __threadfence();
        for (int i = threadIdx.x; i < 3 * r.HWpad; i += blockDim.x) {
          const int c = i / r.HWpad, t = i - c * r.HWpad;
          if (t < r.HW) r.g_env[c * r.HW + t] = (float)__ldcg(r.env_acc + i);
          r.env_acc[i] = 0.0;
        }
      }
    }
    cp_async_wait_all();
    __syncthreads();
  }
  // every CTA has made its last claim before it counts itself out; the last one resets the tick
  if (threadIdx.x == 0) __threadfence();
  if (threadIdx.x == 0 && atomicAdd(&ctl->exited, 1u) == gridDim.x - 1) {
    ctl->next = 0u;
    ctl->exited = 0u;
    __threadfence();
  }
}

// ---------------------------------------------------------------------------------------------
// Host: arena allocator, server
// ---------------------------------------------------------------------------------------------

// First-fit allocator over one device arena (offsets only; nothing is allocated per request).
class Arena {
 public:
  void init(size_t bytes) {
    free_.clear();
    free_[0] = bytes;
    total_ = bytes;
  }
  bool alloc(size_t bytes, size_t* off) {
    bytes = (bytes + 255) / 256 * 256;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *off = it->first;
        const size_t rest = it->second - bytes, start = it->first + bytes;
        free_.erase(it);
        if (rest) free_[start] = rest;
        used_ += bytes;
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    bytes = (bytes + 255) / 256 * 256;
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t used() const { return used_; }
  size_t total() const { return total_; }

 private:
  std::map<size_t, size_t> free_;
  size_t total_ = 0, used_ = 0;
};

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

enum class State { Pending, Uploading, Ordering, Ready, Downloading };

struct Req {
  int64_t ticket;
  des_serve_request in;
  State state = State::Pending;
  int64_t t_submit = 0, t_admit = 0, t_uploaded = 0, t_ready = 0, t_computed = 0;
  size_t off = 0, bytes = 0;
  int slot = -1;
  int n_tiles = 0;
  int fwd_issued = 0, bwd_issued = 0, fwd_done = 0, bwd_done = 0;
  double cost_fwd_tile = 0, cost_bwd_tile = 0;  // pair units per tile
  double tile_pairs = 0;                         // point x texel pairs per tile
  ReqDesc desc{};
  int32_t* d_perm = nullptr;         // normal-direction order (see orders()), else null
  int64_t order_min_p = 0;           // the server's ordering threshold when the request was admitted
  double* env_acc = nullptr;         // FP64 env-gradient accumulator from the server's pool (backward)
  void* d_order_scratch = nullptr;
  // device pointers of outputs (for the download)
  float *d_shading = nullptr, *d_white = nullptr, *d_gn = nullptr, *d_gv = nullptr, *d_ga = nullptr,
        *d_gs = nullptr, *d_gr = nullptr, *d_genv = nullptr;
  // Outputs written in place: every output the caller gave is device memory of the server's
  // device or pinned host memory, and the batch kernel stores into those addresses (as seen from
  // the device) instead of into the arena, so the request needs no download.
  bool direct = false;
  float *o_shading = nullptr, *o_white = nullptr, *o_gn = nullptr, *o_gv = nullptr, *o_ga = nullptr,
        *o_gs = nullptr, *o_gr = nullptr, *o_genv = nullptr;
  // Inputs read in place (device addresses of normal, view, albedo, specular, roughness, triangle
  // ids, barycentrics, shading gradient, diffuse gradient), when inplace_in.
  bool inplace_in = false;
  const void* i[9] = {};
  bool desc_sent = false;  // the descriptor has been queued for the device (with the first tick naming it)
  double remaining() const {
    return (n_tiles - fwd_issued) * cost_fwd_tile + (in.backward ? (n_tiles - bwd_issued) * cost_bwd_tile : 0.0);
  }
  // Scheduling key (lower goes first): with rank_by_size (the server's default) the remaining
  // points x texels, which ranks a request asking for gradients like the same request without;
  // otherwise the remaining work (an adjoint pair counts twice).
  bool rank_by_size = true;
  double rank() const {
    if (!rank_by_size) return remaining();
    const int left = in.backward ? n_tiles - std::min(fwd_issued, bwd_issued) : n_tiles - fwd_issued;
    return left * tile_pairs;
  }
};

// Host<->device copies of the requests go through two copy lanes (one stream per direction, so
// uploads and downloads overlap).  A request's copies form a job of segments; a lane issues its jobs
// in slices, always from the job with the lowest priority value (the request's rank for uploads,
// fewest bytes for downloads), and keeps a bounded number of bytes queued on its stream.  A small
// request therefore waits for at most about one queue's worth of a large one's transfer instead
// of all of it.  (Copies of one direction share a copy engine in submission order, so a short
// queue is the only way to let a later, smaller request go first.)
struct CopySeg {
  void* dst;
  const void* src;
  size_t bytes;
};

struct CopyJob {
  Req* r = nullptr;
  std::vector<CopySeg> segs;
  size_t seg = 0, seg_off = 0;  // next byte to issue
  int outstanding = 0;          // issued slices not yet complete
  double prio = 0;              // lower goes first: the request's rank (uploads), bytes (downloads)
  bool issued_all() const { return seg >= segs.size(); }
  void add(void* dst, const void* src, size_t bytes) {
    if (bytes) segs.push_back(CopySeg{dst, src, bytes});
  }
};

struct CopyLane {
  struct Flight {
    cudaEvent_t ev;
    CopyJob* job;
    size_t bytes;
  };
  cudaStream_t stream = nullptr;
  cudaMemcpyKind kind = cudaMemcpyHostToDevice;
  size_t slice = size_t(1) << 20;   // bytes per issued copy
  size_t window = size_t(2) << 20;  // bytes queued on the stream at most
  std::vector<CopyJob*> queue;  // jobs with slices left to issue, in arrival order
  std::deque<Flight> flight;
  std::vector<cudaEvent_t> free_ev;
  size_t in_flight = 0;

  bool init(cudaMemcpyKind k, size_t slice_bytes, size_t window_bytes) {
    kind = k;
    slice = slice_bytes;
    window = window_bytes;
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) return false;
    for (int i = 0; i < kCopyEvents; ++i) {
      cudaEvent_t e = nullptr;
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return false;
      free_ev.push_back(e);
    }
    return true;
  }
  void destroy() {
    for (CopyJob* j : queue) delete j;
    queue.clear();
    for (auto& f : flight) {
      free_ev.push_back(f.ev);
      if (--f.job->outstanding == 0 && f.job->issued_all()) delete f.job;
    }
    flight.clear();
    for (cudaEvent_t e : free_ev) cudaEventDestroy(e);
    free_ev.clear();
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
  }
  bool idle() const { return queue.empty() && flight.empty(); }
  void pump();
  // retires finished slices; appends jobs whose every slice has completed
  // returns false when the stream reported an error (the server then fails its requests)
  bool poll(std::vector<CopyJob*>& finished) {
    while (!flight.empty()) {
      const cudaError_t e = cudaEventQuery(flight.front().ev);
      if (e == cudaErrorNotReady) break;
      if (e != cudaSuccess) return false;
      const Flight f = flight.front();
      flight.pop_front();
      free_ev.push_back(f.ev);
      in_flight -= f.bytes;
      if (--f.job->outstanding == 0 && f.job->issued_all()) finished.push_back(f.job);
    }
    return true;
  }
};

// Normal-direction ordering of uploaded requests (the plain path's ordering kernels), on a stream
// of its own so that it neither waits behind copies nor holds them up.
struct OrderLane {
  cudaStream_t stream = nullptr;
  std::vector<cudaEvent_t> free_ev;
  std::deque<std::pair<cudaEvent_t, Req*>> flight;
  bool init() {
    // highest priority: its few short CTAs take the first SMs that the persistent batch kernels free
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (cudaStreamCreateWithPriority(&stream, cudaStreamNonBlocking, greatest) != cudaSuccess) return false;
    for (int i = 0; i < kCopyEvents; ++i) {
      cudaEvent_t e = nullptr;
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return false;
      free_ev.push_back(e);
    }
    return true;
  }
  void destroy() {
    for (auto& f : flight) free_ev.push_back(f.first);
    flight.clear();
    for (cudaEvent_t e : free_ev) cudaEventDestroy(e);
    free_ev.clear();
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
  }
};

struct Env {
  int H, W, HWpad;
  float4* table;
};
struct Mesh {
  int N_face, N_vertex, N_slot;
  int32_t* faces;
  uint32_t* vis;
};

struct Tick {
  WorkList* h = nullptr;    // pinned, mapped: the scheduler writes the list here
  WorkList* d = nullptr;    // the device's address of h (the kernel sets d->started)
  WorkList* dev = nullptr;  // device copy of the list, which the kernel reads
  TickCtl* ctl = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  bool busy = false;
  std::vector<std::pair<Req*, std::pair<int, int>>> counts;  // request, (fwd tiles, bwd tiles)
};

}  // namespace serve
}  // namespace des

struct des_server {
  int device = 0;
  int tick_us = 50;
  std::atomic<int> ticks_in_flight{4};  // tick buffers in use at once (<= kNTicks)
  double pairs_per_us = 0;              // the batch kernel's throughput, which sizes the ticks
  std::atomic<int64_t> order_min_p{des::serve::kServeOrderMinP};  // requests with fewer points are shaded in input order
  des::serve::CopyLane up, down;
  des::serve::OrderLane order;
  unsigned char* arena_base = nullptr;
  des::serve::Arena arena;
  unsigned* d_ctrl = nullptr;
  des::serve::ReqDesc* h_desc = nullptr;  // per slot, pinned host memory (written at admission)
  des::serve::ReqDesc* d_desc = nullptr;  // per slot, device copy (sent with the slot's first tick)
  unsigned* d_slot_tiles = nullptr;       // per slot, adjoint tiles finished (device, never reset)
  std::vector<unsigned> slot_tiles_base;  // per slot, the counter's value once its requests are done
  std::vector<double*> acc_pool;          // zeroed FP64 env-gradient accumulators, 3 x kMaxHWpad each
  std::vector<void*> acc_chunks;
  std::vector<int> free_slots;
  std::vector<des::serve::Env> envs;
  std::vector<des::serve::Mesh> meshes;
  des::serve::Tick ticks[des::serve::kNTicks];
  // Ranking by size rather than by work: on the mixed serving workload (Poisson 5k/s, ten runs over
  // five arrival seeds) it gave the 50k-100k-point class a p99 of 0.97 ms on average instead of
  // 1.07 ms at the same throughput -- that class's slowest requests are the ones with gradients,
  // which ranking by work puts behind forward requests of up to twice their size.
  std::atomic<bool> rank_by_size{true};
  int sms = 0, grid = 0;
  size_t smem = 0;

  std::mutex mu;
  std::condition_variable cv;
  std::deque<des::serve::Req*> incoming;
  std::deque<des::serve::Req*> pending;
  std::unordered_set<des::serve::Req*> active;  // admitted, not yet reported done
  // Ready requests with tiles left to issue, by (rank, ticket): the scheduling order
  std::set<std::tuple<double, int64_t, des::serve::Req*>> ready;
  std::vector<des_serve_done> completed;
  int64_t next_ticket = 1;
  int64_t n_submitted = 0, n_done = 0;
  int error = DES_OK;
  std::atomic<bool> stop{false};
  std::atomic<bool> failed{false};  // a CUDA error was seen: outstanding requests fail, submits are refused
  std::thread worker;
  int64_t t0 = 0;
  des_serve_stats stats{};
};

namespace des {
namespace serve {

// Issues slices, job with the lowest priority value first, while the lane has room.
void CopyLane::pump() {
  while (in_flight < window && !queue.empty() && !free_ev.empty()) {
    auto best = queue.begin();
    for (auto it = queue.begin(); it != queue.end(); ++it)
      if ((*it)->prio < (*best)->prio) best = it;
    CopyJob* j = *best;
    const CopySeg& sg = j->segs[j->seg];
    const size_t n = std::min(slice, sg.bytes - j->seg_off);
    cudaMemcpyAsync(static_cast<char*>(sg.dst) + j->seg_off, static_cast<const char*>(sg.src) + j->seg_off, n, kind,
                    stream);
    j->seg_off += n;
    if (j->seg_off == sg.bytes) {
      ++j->seg;
      j->seg_off = 0;
    }
    cudaEvent_t ev = free_ev.back();
    free_ev.pop_back();
    cudaEventRecord(ev, stream);
    flight.push_back(Flight{ev, j, n});
    ++j->outstanding;
    in_flight += n;
    if (j->issued_all()) queue.erase(best);
  }
}

namespace {

// Device buffers of one request inside its arena range.  request_layout() both sizes the range
// (base == nullptr) and hands out the pointers (base = the range's start), from one sequence of
// 256-byte-aligned takes, so the two can never disagree.
struct ReqLayout {
  float *normal, *view, *albedo, *spec, *rough, *bary, *shading, *white, *gsh, *gwh, *grads, *genv;
  int64_t* tri;
  int32_t* perm;
  void* order_scratch;
  size_t bytes;
};

// Whether the server orders a request's points by normal direction before shading it.
inline bool orders(const des_serve_request& q, int64_t order_min_p) {
  return q.P >= std::max(order_min_p, kSortMinP) && q.P <= kSortMaxP;
}

// inplace_in: the inputs are read where the caller keeps them (no arena copies).
ReqLayout request_layout(const des_serve_request& q, const Env& E, int64_t order_min_p, bool inplace_in,
                         unsigned char* base) {
  ReqLayout L{};
  size_t off = 0;
  auto take = [&](size_t n) -> unsigned char* {
    unsigned char* p = base ? base + off : nullptr;
    off += (n + 255) / 256 * 256;
    return p;
  };
  const size_t P = (size_t)q.P;
  if (!inplace_in) {
    L.normal = (float*)take(P * 12);
    L.view = (float*)take(P * 12);
    L.albedo = (float*)take(P * 12);
    L.spec = (float*)take(P * 12);
    L.rough = (float*)take(P * 4);
    if (q.mesh_id >= 0) {
      L.tri = (int64_t*)take(P * 8);
      L.bary = (float*)take(P * 12);
    }
  }
  L.shading = (float*)take(P * 12);
  L.white = (float*)take(P * 12);
  if (orders(q, order_min_p)) {
    L.perm = (int32_t*)take(P * 4);
    L.order_scratch = take(point_order_scratch_bytes(q.P));
  }
  if (q.backward) {
    if (!inplace_in) {
      L.gsh = (float*)take(P * 12);
      L.gwh = (float*)take(P * 12);
    }
    L.grads = (float*)take(P * 12 * 4 + P * 4);
    L.genv = (float*)take((size_t)3 * E.H * E.W * 4);
  }
  L.bytes = off;
  return L;
}

// The address under which the server's device reaches p: p for memory of that device, the
// mapped alias for pinned host memory (*host set); null where the device cannot reach it.
float* device_alias(const void* p, int device, bool* host) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  if (a.type == cudaMemoryTypeDevice && a.device == device) return static_cast<float*>(a.devicePointer);
  if (a.type == cudaMemoryTypeHost && a.devicePointer != nullptr) {
    *host = true;
    return static_cast<float*>(a.devicePointer);
  }
  return nullptr;
}

// Resolves where the batch kernel reads and writes the request's data.  Outputs are stored in place
// when every output it names is reachable from the device (pinned host memory only for requests
// shaded in input order, whose tiles store whole rows).  Inputs are read in place when the request
// is shaded in input order and every input is reachable: its tiles then fetch their points over
// the host link themselves, and the request needs no upload.
void resolve_request(des_server* s, Req* r) {
  const des_serve_request& q = r->in;
  const bool in_order = !orders(q, r->order_min_p);
  bool host = false, ok = true;
  auto take = [&](float* p, float** o) {
    if (p == nullptr) return;
    *o = device_alias(p, s->device, &host);
    ok = ok && *o != nullptr;
  };
  take(q.shading, &r->o_shading);
  take(q.diffuse_shading, &r->o_white);
  if (q.backward) {
    take(q.g_normal, &r->o_gn);
    take(q.g_view_dir, &r->o_gv);
    take(q.g_albedo, &r->o_ga);
    take(q.g_specular_albedo, &r->o_gs);
    take(q.g_roughness, &r->o_gr);
    take(q.g_envmap, &r->o_genv);
  }
  r->direct = ok && (in_order || !host);
  bool in_ok = in_order, in_host = false;
  auto in = [&](const void* p, const void** o) {
    if (p == nullptr || !in_ok) return;
    *o = device_alias(p, s->device, &in_host);
    in_ok = *o != nullptr;
  };
  in(q.normal, &r->i[0]);
  in(q.view_dir, &r->i[1]);
  in(q.albedo, &r->i[2]);
  in(q.specular_albedo, &r->i[3]);
  in(q.roughness, &r->i[4]);
  if (q.mesh_id >= 0) {
    in(q.nearest_triangle_id, &r->i[5]);
    in(q.barycentric_coord, &r->i[6]);
  }
  if (q.backward) {
    in(q.grad_shading, &r->i[7]);
    in(q.grad_diffuse_shading, &r->i[8]);
  }
  r->inplace_in = in_ok;
}

// Lays out the request's buffers in its arena range, writes its descriptor (pinned host memory; it
// reaches the device with the first tick that names the slot) and queues its point data on the
// upload lane in prioritised slices.
// Returns false when the request has nothing to upload (it is ready right away).
bool upload(des_server* s, Req* r) {
  const des_serve_request& q = r->in;
  const Env& E = s->envs[q.env_id];
  const ReqLayout L = request_layout(q, E, r->order_min_p, r->inplace_in, s->arena_base + r->off);
  CopyLane& lane = s->up;
  auto* job = new CopyJob();
  job->r = r;
  const size_t P = (size_t)q.P;
  ReqDesc& d = r->desc;
  d = ReqDesc{};
  d.P = q.P;
  d.HW = E.H * E.W;
  d.HWpad = E.HWpad;
  d.diff = (q.flags & DES_DIFFUSE) ? 1 : 0;
  d.spec = (q.flags & DES_SPECULAR) ? 1 : 0;
  d.clamp = (q.flags & DES_CLAMP) != 0;
  d.table = E.table;
  d.ctrl = s->d_ctrl;
  if (r->inplace_in) {
    d.normal = static_cast<const float*>(r->i[0]);
    d.view = static_cast<const float*>(r->i[1]);
    d.albedo = static_cast<const float*>(r->i[2]);
    d.spec_alb = static_cast<const float*>(r->i[3]);
    d.rough = static_cast<const float*>(r->i[4]);
  } else {
    job->add(L.normal, q.normal, P * 12);
    job->add(L.view, q.view_dir, P * 12);
    job->add(L.albedo, q.albedo, P * 12);
    job->add(L.spec, q.specular_albedo, P * 12);
    job->add(L.rough, q.roughness, P * 4);
    d.normal = L.normal;
    d.view = L.view;
    d.albedo = L.albedo;
    d.spec_alb = L.spec;
    d.rough = L.rough;
  }
  if (q.mesh_id >= 0) {
    const Mesh& M = s->meshes[q.mesh_id];
    d.has_vis = 1;
    d.N_face = M.N_face;
    d.N_vertex = M.N_vertex;
    d.faces = M.faces;
    d.vis = M.vis;
    if (r->inplace_in) {
      d.tri = static_cast<const int64_t*>(r->i[5]);
      d.bary = static_cast<const float*>(r->i[6]);
    } else {
      job->add(L.tri, q.nearest_triangle_id, P * 8);
      job->add(L.bary, q.barycentric_coord, P * 12);
      d.tri = L.tri;
      d.bary = L.bary;
    }
  }
  r->d_shading = L.shading;
  r->d_white = L.white;
  d.shading = L.shading;
  d.white = L.white;
  if (r->direct) {
    d.shading = r->o_shading;
    d.white = r->o_white;  // may be null: the kernel skips it
  }
  if (L.perm != nullptr) {
    r->d_perm = L.perm;
    r->d_order_scratch = L.order_scratch;
    d.perm = L.perm;  // read only once the request is Ready, i.e. after its ordering
  }
  if (q.backward) {
    if (r->inplace_in) {
      d.g_shading = static_cast<const float*>(r->i[7]);
      d.g_white = static_cast<const float*>(r->i[8]);
    } else {
      job->add(L.gsh, q.grad_shading, P * 12);
      if (q.grad_diffuse_shading) job->add(L.gwh, q.grad_diffuse_shading, P * 12);
      d.g_shading = L.gsh;
      d.g_white = q.grad_diffuse_shading ? L.gwh : nullptr;
    }
    r->d_gn = L.grads;
    r->d_gv = r->d_gn + 3 * P;
    r->d_ga = r->d_gv + 3 * P;
    r->d_gs = r->d_ga + 3 * P;
    r->d_gr = r->d_gs + 3 * P;
    d.g_normal = r->d_gn;
    d.g_view = r->d_gv;
    d.g_albedo = r->d_ga;
    d.g_spec = r->d_gs;
    d.g_rough = r->d_gr;
    d.env_acc = r->env_acc;
    r->d_genv = L.genv;
    d.g_env = L.genv;
    if (r->direct) {  // a null output is not written (g_normal and g_env fall back to the arena)
      if (r->o_gn) d.g_normal = r->o_gn;
      d.g_view = r->o_gv;
      d.g_albedo = r->o_ga;
      d.g_spec = r->o_gs;
      d.g_rough = r->o_gr;
      if (r->o_genv) d.g_env = r->o_genv;
    }
    s->slot_tiles_base[r->slot] += (unsigned)r->n_tiles;  // wraps like the device counter
    d.bwd_target = s->slot_tiles_base[r->slot];
  }
  // the descriptor goes to the device with the first tick that names the slot (launch_tick)
  s->h_desc[r->slot] = d;
  if (job->segs.empty()) {  // inputs read in place: nothing to copy
    delete job;
    return false;
  }
  job->prio = r->rank();
  lane.queue.push_back(job);
  return true;
}

// Queues the request's outputs on the download lane.
void download(des_server* s, Req* r) {
  const des_serve_request& q = r->in;
  const size_t P = (size_t)q.P;
  const Env& E = s->envs[q.env_id];
  auto* job = new CopyJob();
  job->r = r;
  if (q.shading) job->add(q.shading, r->d_shading, P * 12);
  if (q.diffuse_shading) job->add(q.diffuse_shading, r->d_white, P * 12);
  if (q.backward) {
    if (q.g_normal) job->add(q.g_normal, r->d_gn, P * 12);
    if (q.g_view_dir) job->add(q.g_view_dir, r->d_gv, P * 12);
    if (q.g_albedo) job->add(q.g_albedo, r->d_ga, P * 12);
    if (q.g_specular_albedo) job->add(q.g_specular_albedo, r->d_gs, P * 12);
    if (q.g_roughness) job->add(q.g_roughness, r->d_gr, P * 4);
    if (q.g_envmap) job->add(q.g_envmap, r->d_genv, (size_t)3 * E.H * E.W * 4);
  }
  for (const CopySeg& sg : job->segs) job->prio += (double)sg.bytes;
  s->down.queue.push_back(job);
}

// Adds a chunk of zeroed env-gradient accumulators to the pool (at creation, then whenever more
// backward requests are admitted at once than the pool holds).
bool grow_acc_pool(des_server* s) {
  constexpr int kPerChunk = 1024;
  constexpr size_t kAcc = (size_t)3 * kMaxHWpad;  // doubles per accumulator
  void* chunk = nullptr;
  if (cudaMalloc(&chunk, kPerChunk * kAcc * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  // zeroed (and finished) before any request can use it
  if (cudaMemsetAsync(chunk, 0, kPerChunk * kAcc * sizeof(double), s->order.stream) != cudaSuccess ||
      cudaStreamSynchronize(s->order.stream) != cudaSuccess) {
    cudaFree(chunk);
    return false;
  }
  s->acc_chunks.push_back(chunk);
  for (int i = kPerChunk - 1; i >= 0; --i) s->acc_pool.push_back(static_cast<double*>(chunk) + i * kAcc);
  return true;
}

// Reports a request whose outputs are in the caller's memory and frees its arena range and slot.
void finish_request(des_server* s, Req* r, int64_t t_done) {
  des_serve_done d{};
  d.ticket = r->ticket;
  d.t_submit_ns = r->t_submit - s->t0;
  d.t_admit_ns = r->t_admit - s->t0;
  d.t_uploaded_ns = r->t_uploaded - s->t0;
  d.t_ready_ns = r->t_ready - s->t0;
  d.t_computed_ns = r->t_computed - s->t0;
  d.t_done_ns = t_done - s->t0;
  d.status = DES_OK;
  s->arena.release(r->off, r->bytes);
  s->free_slots.push_back(r->slot);
  if (r->env_acc != nullptr) s->acc_pool.push_back(r->env_acc);  // zeroed again by the last tile
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->completed.push_back(d);
    s->n_done += 1;
  }
  s->cv.notify_all();
  s->active.erase(r);
  delete r;
}

// Reports a request that was never admitted (no slot, arena range or accumulator) as finished with
// the given error status.
void reject_request(des_server* s, Req* r, int status) {
  des_serve_done d{};
  d.ticket = r->ticket;
  d.t_submit_ns = r->t_submit - s->t0;
  d.t_done_ns = now_ns() - s->t0;
  d.status = status;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->completed.push_back(d);
    s->n_done += 1;
  }
  s->cv.notify_all();
  delete r;
}

// Builds and launches one tick if a tick buffer is free.  Returns true when work was launched.
bool launch_tick(des_server* s) {
  if (s->ready.empty()) return false;
  Tick* t = nullptr;
  int busy = 0;
  for (auto& k : s->ticks) {
    if (k.busy)
      ++busy;
    else if (t == nullptr)
      t = &k;
  }
  if (t == nullptr || busy >= s->ticks_in_flight) return false;
  // at most kQueuedTicks launched ticks that no CTA has started yet: the next one is launched as
  // soon as the GPU begins the last queued one, which keeps the SMs fed across tick boundaries
  // while a request that becomes ready waits behind little queued work
  int queued = 0;
  for (auto& k : s->ticks)
    if (k.busy && *reinterpret_cast<volatile unsigned*>(&k.h->started) == 0u) ++queued;
  if (queued >= kQueuedTicks) return false;
  const double budget = s->pairs_per_us * s->tick_us;
  // lowest rank first, ties by arrival (the set's order); at least one item per
  // resident CTA while there is work, so that no SM idles for want of items
  double used = 0;
  unsigned n = 0;
  const unsigned min_items = std::min<unsigned>((unsigned)s->grid, (unsigned)kTickItems);
  auto room = [&] { return (used < budget || n < min_items) && n < (unsigned)kTickItems; };
  t->counts.clear();
  while (!s->ready.empty() && room()) {
    Req* r = std::get<2>(*s->ready.begin());
    s->ready.erase(s->ready.begin());
    int nf = 0, nb = 0;
    while (room() && (r->fwd_issued < r->n_tiles || (r->in.backward && r->bwd_issued < r->n_tiles))) {
      // interleave forward and adjoint tiles of the same request
      if (r->fwd_issued < r->n_tiles && (!r->in.backward || r->fwd_issued <= r->bwd_issued || r->bwd_issued >= r->n_tiles)) {
        t->h->items[n++] = WorkItem{r->slot, r->fwd_issued++, 0, 0};
        used += r->cost_fwd_tile;
        ++nf;
      } else {
        t->h->items[n++] = WorkItem{r->slot, r->bwd_issued++, 1, 0};
        used += r->cost_bwd_tile;
        ++nb;
      }
    }
    t->counts.push_back({r, {nf, nb}});
    if (r->remaining() > 0) s->ready.insert({r->rank(), r->ticket, r});  // budget is used up
  }
  t->h->n = n;
  t->h->started = 0u;
  std::atomic_thread_fence(std::memory_order_seq_cst);  // items are in host memory before the copies
  // ahead of the kernel on the tick's stream: the descriptors of the slots this tick names for the
  // first time, then the list.  A later tick is launched only once this one has started, i.e. after
  // these copies completed, so every tick finds the descriptors of all the slots it names.
  bool copied = true;
  for (auto& c : t->counts) {
    Req* r = c.first;
    if (r->desc_sent) continue;
    copied = copied && cudaMemcpyAsync(s->d_desc + r->slot, s->h_desc + r->slot, sizeof(ReqDesc),
                                       cudaMemcpyHostToDevice, t->stream) == cudaSuccess;
    r->desc_sent = true;
  }
  copied = copied && cudaMemcpyAsync(t->dev, t->h, offsetof(WorkList, items) + (size_t)n * sizeof(WorkItem),
                                     cudaMemcpyHostToDevice, t->stream) == cudaSuccess;
  if (!copied) {  // nothing launched; the worker fails the outstanding requests
    s->failed = true;
    return false;
  }
  if (cudaGraphLaunch(t->exec, t->stream) != cudaSuccess) {
    // launch the same work without the graph
    cudaGetLastError();
    batch_kernel<<<s->grid, kNW * 32, s->smem, t->stream>>>(s->d_desc, t->dev, &t->d->started, t->ctl,
                                                            s->d_slot_tiles, s->d_ctrl);
    s->stats.device_error |= 16;
  }
  count_launches(1);
  cudaEventRecord(t->done, t->stream);
  t->busy = true;
  s->stats.ticks += 1;
  s->stats.items += n;
  return true;
}

void worker_loop(des_server* s) {
  cudaSetDevice(s->device);
  while (true) {
    bool progressed = false;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      if (s->stop && s->incoming.empty() && s->pending.empty() && s->active.empty()) break;
      while (!s->incoming.empty()) {
        s->pending.push_back(s->incoming.front());
        s->incoming.pop_front();
      }
    }
    // 0. after a CUDA error nothing more can complete: fail every outstanding request at once
    if (s->failed) {
      std::vector<Req*> all(s->active.begin(), s->active.end());
      all.insert(all.end(), s->pending.begin(), s->pending.end());
      s->active.clear();
      s->pending.clear();
      s->ready.clear();
      {
        std::lock_guard<std::mutex> lk(s->mu);
        for (Req* r : all) {
          des_serve_done d{};
          d.ticket = r->ticket;
          d.t_submit_ns = r->t_submit - s->t0;
          d.t_done_ns = now_ns() - s->t0;
          d.status = DES_ERR_CUDA;
          s->completed.push_back(d);
          s->n_done += 1;
          delete r;
        }
        s->error = DES_ERR_CUDA;
      }
      s->cv.notify_all();
      if (s->stop) break;
      std::this_thread::sleep_for(std::chrono::microseconds(200));
      continue;
    }
    // 1. admission (arrival order; requests that do not fit yet are skipped, not blocking others)
    for (auto it = s->pending.begin(); it != s->pending.end();) {
      Req* r = *it;
      const Env& E = s->envs[r->in.env_id];
      r->order_min_p = s->order_min_p.load();
      r->rank_by_size = s->rank_by_size.load();
      resolve_request(s, r);
      r->bytes = request_layout(r->in, E, r->order_min_p, r->inplace_in, nullptr).bytes;
      if ((r->bytes + 255) / 256 * 256 > s->arena.total()) {
        // can never fit: finish it now with an error instead of letting it wait for memory forever
        reject_request(s, r, DES_ERR_WORKSPACE);
        it = s->pending.erase(it);
        progressed = true;
        continue;
      }
      size_t off = 0;
      if (r->in.backward && s->acc_pool.empty() && !grow_acc_pool(s)) {
        ++it;
        continue;
      }
      if (s->free_slots.empty() || !s->arena.alloc(r->bytes, &off)) {
        ++it;
        continue;
      }
      r->off = off;
      r->slot = s->free_slots.back();
      s->free_slots.pop_back();
      if (r->in.backward) {
        r->env_acc = s->acc_pool.back();
        s->acc_pool.pop_back();
      }
      r->t_admit = now_ns();
      r->n_tiles = (int)((r->in.P + 31) / 32);
      // a request with gradients runs adjoint tiles only: they store its forward outputs too
      if (r->in.backward) r->fwd_issued = r->fwd_done = r->n_tiles;
      r->tile_pairs = 32.0 * E.HWpad;
      r->cost_fwd_tile = r->tile_pairs;
      r->cost_bwd_tile = 2.0 * r->tile_pairs;
      s->active.insert(r);
      if (upload(s, r)) {
        r->state = State::Uploading;
      } else {
        r->t_uploaded = r->t_ready = r->t_admit;
        r->state = State::Ready;
        s->ready.insert({r->rank(), r->ticket, r});
      }
      it = s->pending.erase(it);
      progressed = true;
      s->stats.peak_arena_bytes = std::max<int64_t>(s->stats.peak_arena_bytes, (int64_t)s->arena.used());
    }
    // 2. finished ticks
    for (auto& t : s->ticks) {
      if (!t.busy) continue;
      const cudaError_t te = cudaEventQuery(t.done);
      if (te != cudaSuccess && te != cudaErrorNotReady) s->failed = true;
      if (te == cudaSuccess) {
        const int64_t tnow = now_ns();
        for (auto& c : t.counts) {
          Req* r = c.first;
          r->fwd_done += c.second.first;
          r->bwd_done += c.second.second;
          if (r->state == State::Ready && r->fwd_done == r->n_tiles && (!r->in.backward || r->bwd_done == r->n_tiles)) {
            r->t_computed = tnow;
            if (r->direct) {  // outputs are already in place
              finish_request(s, r, tnow);
            } else {
              download(s, r);
              r->state = State::Downloading;
            }
          }
        }
        t.counts.clear();
        t.busy = false;
        progressed = true;
      }
    }
    // 3. copies: retire finished slices, then issue more
    std::vector<CopyJob*> fin;
    if (!s->up.poll(fin)) s->failed = true;
    for (CopyJob* j : fin) {
      Req* r = j->r;
      delete j;
      progressed = true;
      r->t_uploaded = now_ns();
      if (r->d_perm != nullptr && !s->order.free_ev.empty() &&
          launch_point_order(r->desc.normal, r->in.P, r->d_order_scratch, r->d_perm, s->order.stream) == DES_OK) {
        cudaEvent_t ev = s->order.free_ev.back();
        s->order.free_ev.pop_back();
        cudaEventRecord(ev, s->order.stream);
        s->order.flight.push_back({ev, r});
        r->state = State::Ordering;
      } else {
        if (r->d_perm != nullptr) {  // no ordering after all: shade in input order
          r->desc.perm = nullptr;
          s->h_desc[r->slot].perm = nullptr;  // no tick has read the descriptor yet
        }
        r->state = State::Ready;
        r->t_ready = now_ns();
        s->ready.insert({r->rank(), r->ticket, r});
      }
    }
    while (!s->order.flight.empty()) {
      const cudaError_t oe = cudaEventQuery(s->order.flight.front().first);
      if (oe == cudaErrorNotReady) break;
      if (oe != cudaSuccess) {
        s->failed = true;
        break;
      }
      Req* r = s->order.flight.front().second;
      s->order.free_ev.push_back(s->order.flight.front().first);
      s->order.flight.pop_front();
      r->state = State::Ready;
      r->t_ready = now_ns();
      s->ready.insert({r->rank(), r->ticket, r});
      progressed = true;
    }
    fin.clear();
    if (!s->down.poll(fin)) s->failed = true;
    for (CopyJob* j : fin) {
      Req* r = j->r;
      delete j;
      progressed = true;
      finish_request(s, r, now_ns());
    }
    // 4. new ticks, new copies
    while (launch_tick(s)) progressed = true;
    s->up.pump();
    s->down.pump();
    if (!progressed) {
      // poll without sleeping while the GPU or a copy lane has work (a sleep costs ~50 us of
      // reaction time); sleep only when everything is idle
      bool busy = !s->up.idle() || !s->down.idle() || !s->order.flight.empty();
      for (auto& t : s->ticks) busy = busy || t.busy;
      if (busy)
        std::this_thread::yield();
      else
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
  }
}

}  // namespace
}  // namespace serve
}  // namespace des

// ---------------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------------

using des::serve::Req;

extern "C" {

int des_server_create(int device, size_t hbm_budget_bytes, int tick_us, des_server** out) {
  if (out == nullptr || hbm_budget_bytes < (1u << 20) || tick_us <= 0) return DES_ERR_INVALID_ARGUMENT;
  auto* s = new des_server();
  s->device = device;
  s->tick_us = tick_us;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete s;
    return DES_ERR_CUDA;
  }
  cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, device);
  s->pairs_per_us = des::serve::kBatchPairsPerUs * s->sms / 148.0;
  bool ok = s->up.init(cudaMemcpyHostToDevice, size_t(1) << 20, size_t(4) << 20) &&
            s->down.init(cudaMemcpyDeviceToHost, size_t(1) << 20, size_t(4) << 20) && s->order.init() &&
            cudaMalloc(&s->arena_base, hbm_budget_bytes) == cudaSuccess &&
            cudaMalloc(&s->d_ctrl, 256) == cudaSuccess &&
            cudaHostAlloc(&s->h_desc, sizeof(des::serve::ReqDesc) * des::serve::kMaxSlots, cudaHostAllocDefault) ==
                cudaSuccess &&
            cudaMalloc(&s->d_desc, sizeof(des::serve::ReqDesc) * des::serve::kMaxSlots) == cudaSuccess &&
            cudaMalloc(&s->d_slot_tiles, sizeof(unsigned) * des::serve::kMaxSlots) == cudaSuccess &&
            cudaMemset(s->d_slot_tiles, 0, sizeof(unsigned) * des::serve::kMaxSlots) == cudaSuccess &&
            cudaMemset(s->d_ctrl, 0, 256) == cudaSuccess;
  if (!ok) {
    des_server_destroy(s);
    return DES_ERR_CUDA;
  }
  s->arena.init(hbm_budget_bytes);
  s->slot_tiles_base.assign(des::serve::kMaxSlots, 0u);
  if (!des::serve::grow_acc_pool(s)) {
    des_server_destroy(s);
    return DES_ERR_CUDA;
  }
  for (int i = des::serve::kMaxSlots - 1; i >= 0; --i) s->free_slots.push_back(i);
  s->smem = des::serve::kSmemPts + 2 * sizeof(des::serve::TilePoints);
  if (cudaFuncSetAttribute(des::serve::batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s->smem) !=
      cudaSuccess) {
    des_server_destroy(s);
    return DES_ERR_CUDA;
  }
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, des::serve::batch_kernel, des::serve::kNW * 32, s->smem);
  s->grid = std::max(1, occ) * s->sms;
  // one captured graph per tick buffer: the persistent batch kernel over that buffer's work list
  for (auto& t : s->ticks) {
    ok = cudaHostAlloc(&t.h, sizeof(des::serve::WorkList), cudaHostAllocMapped) == cudaSuccess &&
         cudaHostGetDevicePointer(reinterpret_cast<void**>(&t.d), t.h, 0) == cudaSuccess &&
         cudaMalloc(&t.dev, sizeof(des::serve::WorkList)) == cudaSuccess &&
         cudaMalloc(&t.ctl, sizeof(des::serve::TickCtl)) == cudaSuccess &&
         cudaMemset(t.ctl, 0, sizeof(des::serve::TickCtl)) == cudaSuccess &&
         cudaStreamCreateWithFlags(&t.stream, cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&t.done, cudaEventDisableTiming) == cudaSuccess &&
         cudaDeviceSynchronize() == cudaSuccess;
    if (!ok) {
      des_server_destroy(s);
      return DES_ERR_CUDA;
    }
    std::memset(t.h, 0, sizeof(des::serve::WorkList));
    cudaGraph_t g = nullptr;
    ok = cudaStreamBeginCapture(t.stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    des::serve::batch_kernel<<<s->grid, des::serve::kNW * 32, s->smem, t.stream>>>(
        s->d_desc, t.dev, &t.d->started, t.ctl, s->d_slot_tiles, s->d_ctrl);
    ok = ok && cudaStreamEndCapture(t.stream, &g) == cudaSuccess;
    ok = ok && cudaGraphInstantiate(&t.exec, g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
    if (!ok) {
      des_server_destroy(s);
      return DES_ERR_CUDA;
    }
  }
  s->t0 = des::serve::now_ns();
  s->worker = std::thread(des::serve::worker_loop, s);
  *out = s;
  return DES_OK;
}

int des_server_add_envmap(des_server* s, int32_t H, int32_t W, const float* envmap, const float* light2obj_rotmat,
                          int32_t* env_id) {
  if (s == nullptr || envmap == nullptr || light2obj_rotmat == nullptr || env_id == nullptr || H <= 0 || W <= 0)
    return DES_ERR_INVALID_ARGUMENT;
  const int HWpad = (H * W + 31) / 32 * 32;
  if (HWpad > des::serve::kMaxHWpad) return DES_ERR_UNSUPPORTED;
  cudaSetDevice(s->device);
  float *d_env = nullptr, *d_R = nullptr;
  des::serve::Env e{H, W, HWpad, nullptr};
  unsigned* ctrl = nullptr;
  bool ok = cudaMalloc(&d_env, sizeof(float) * 3 * H * W) == cudaSuccess && cudaMalloc(&d_R, 9 * 4) == cudaSuccess &&
            cudaMalloc(&e.table, (size_t)HWpad * 32) == cudaSuccess && cudaMalloc(&ctrl, 256) == cudaSuccess &&
            cudaMemcpy(d_env, envmap, sizeof(float) * 3 * H * W, cudaMemcpyDefault) == cudaSuccess &&
            cudaMemcpy(d_R, light2obj_rotmat, 36, cudaMemcpyDefault) == cudaSuccess &&
            des::launch_table(H, W, HWpad, d_R, d_env, e.table, ctrl, nullptr) == DES_OK &&
            cudaDeviceSynchronize() == cudaSuccess;
  cudaFree(d_env);
  cudaFree(d_R);
  cudaFree(ctrl);
  if (!ok) return DES_ERR_CUDA;
  std::lock_guard<std::mutex> lk(s->mu);
  s->envs.push_back(e);
  *env_id = (int32_t)s->envs.size() - 1;
  return DES_OK;
}

int des_server_add_mesh(des_server* s, int32_t N_face, int32_t N_vertex, int32_t N_slot,
                        const int32_t* face_vertex_list, const int32_t* visibility, int32_t* mesh_id) {
  if (s == nullptr || face_vertex_list == nullptr || visibility == nullptr || mesh_id == nullptr || N_face <= 0 ||
      N_vertex <= 0 || N_slot <= 0)
    return DES_ERR_INVALID_ARGUMENT;
  cudaSetDevice(s->device);
  des::serve::Mesh m{N_face, N_vertex, N_slot, nullptr, nullptr};
  bool ok = cudaMalloc(&m.faces, (size_t)3 * N_face * 4) == cudaSuccess &&
            cudaMalloc(&m.vis, (size_t)N_slot * N_vertex * 4) == cudaSuccess &&
            cudaMemcpy(m.faces, face_vertex_list, (size_t)3 * N_face * 4, cudaMemcpyDefault) == cudaSuccess &&
            cudaMemcpy(m.vis, visibility, (size_t)N_slot * N_vertex * 4, cudaMemcpyDefault) == cudaSuccess;
  if (!ok) {
    cudaFree(m.faces);
    cudaFree(m.vis);
    return DES_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  s->meshes.push_back(m);
  *mesh_id = (int32_t)s->meshes.size() - 1;
  return DES_OK;
}

int des_server_submit(des_server* s, const des_serve_request* req, int64_t* ticket) {
  if (s == nullptr || req == nullptr || ticket == nullptr || req->P <= 0) return DES_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(s->mu);
  if (req->env_id < 0 || req->env_id >= (int)s->envs.size()) return DES_ERR_INVALID_ARGUMENT;
  if (req->mesh_id >= (int)s->meshes.size()) return DES_ERR_INVALID_ARGUMENT;
  if (req->mesh_id >= 0) {
    const auto& m = s->meshes[req->mesh_id];
    const auto& e = s->envs[req->env_id];
    if ((int64_t)m.N_slot * 32 < (int64_t)e.H * e.W || !req->nearest_triangle_id || !req->barycentric_coord)
      return DES_ERR_INVALID_ARGUMENT;
  }
  if (!req->normal || !req->view_dir || !req->albedo || !req->specular_albedo || !req->roughness || !req->shading)
    return DES_ERR_INVALID_ARGUMENT;
  if (req->backward && !req->grad_shading) return DES_ERR_INVALID_ARGUMENT;
  if (!(req->flags & (DES_DIFFUSE | DES_SPECULAR)) || (req->flags & ~(unsigned)(DES_DIFFUSE | DES_SPECULAR | DES_CLAMP)))
    return DES_ERR_INVALID_ARGUMENT;
  if (s->failed) return DES_ERR_CUDA;
  auto* r = new Req();
  r->ticket = s->next_ticket++;
  r->in = *req;
  r->t_submit = des::serve::now_ns();
  s->incoming.push_back(r);
  s->n_submitted += 1;
  *ticket = r->ticket;
  return DES_OK;
}

int des_server_poll(des_server* s, des_serve_done* out, int max_items, int* count) {
  if (s == nullptr || count == nullptr || (max_items > 0 && out == nullptr)) return DES_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(s->mu);
  const int n = std::min<int>(max_items, (int)s->completed.size());
  for (int i = 0; i < n; ++i) out[i] = s->completed[i];
  s->completed.erase(s->completed.begin(), s->completed.begin() + n);
  *count = n;
  return DES_OK;
}

int des_server_drain(des_server* s, int timeout_ms) {
  if (s == nullptr) return DES_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(s->mu);
  const bool done = s->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms),
                                   [&] { return s->n_done == s->n_submitted; });
  return done ? DES_OK : DES_ERR_TIMEOUT;
}

int des_server_set_ticks_in_flight(des_server* s, int n) {
  if (s == nullptr || n < 1 || n > des::serve::kNTicks) return DES_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(s->mu);
  s->ticks_in_flight = n;
  return DES_OK;
}

int des_server_set_rank_by_size(des_server* s, int enable) {
  if (s == nullptr) return DES_ERR_INVALID_ARGUMENT;
  s->rank_by_size = enable != 0;
  return DES_OK;
}

int des_server_set_order_min_points(des_server* s, int64_t n) {
  if (s == nullptr || n < 0) return DES_ERR_INVALID_ARGUMENT;
  s->order_min_p = n;
  return DES_OK;
}

int des_server_stats(des_server* s, des_serve_stats* out) {
  if (s == nullptr || out == nullptr) return DES_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  out->submitted = s->n_submitted;
  out->completed = s->n_done;
  unsigned err = 0;
  cudaMemcpy(&err, s->d_ctrl + des::kCtrlError, 4, cudaMemcpyDeviceToHost);
  out->device_error = (int)err | s->stats.device_error;
  return DES_OK;
}

int des_server_destroy(des_server* s) {
  if (s == nullptr) return DES_ERR_INVALID_ARGUMENT;
  if (s->worker.joinable()) {
    s->stop = true;
    s->worker.join();
  }
  cudaSetDevice(s->device);
  cudaDeviceSynchronize();
  for (auto& t : s->ticks) {
    if (t.exec) cudaGraphExecDestroy(t.exec);
    if (t.h) cudaFreeHost(t.h);
    if (t.dev) cudaFree(t.dev);
    if (t.ctl) cudaFree(t.ctl);
    if (t.done) cudaEventDestroy(t.done);
    if (t.stream) cudaStreamDestroy(t.stream);
  }
  for (auto& e : s->envs) cudaFree(e.table);
  for (auto& m : s->meshes) {
    cudaFree(m.faces);
    cudaFree(m.vis);
  }
  for (Req* r : s->pending) delete r;
  for (Req* r : s->incoming) delete r;
  if (s->h_desc) cudaFreeHost(s->h_desc);
  if (s->d_desc) cudaFree(s->d_desc);
  if (s->d_slot_tiles) cudaFree(s->d_slot_tiles);
  for (void* c : s->acc_chunks) cudaFree(c);
  if (s->d_ctrl) cudaFree(s->d_ctrl);
  if (s->arena_base) cudaFree(s->arena_base);
  s->up.destroy();
  s->down.destroy();
  s->order.destroy();
  delete s;
  return DES_OK;
}

}  // extern "C"
