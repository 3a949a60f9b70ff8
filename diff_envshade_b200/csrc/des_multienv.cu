// Multi-env-map relighting on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// out[p, k, c] = albedo_c[p] sum_t w_d[p, t] L_k[c, t] + specular_c[p] sum_t w_s[p, t] L_k[c, t],
// where w_d = vis * max(n.l, 0) * dw / pi and w_s = vis * dw * F G D / 4 are the per-(point, texel)
// weights of the reference's forward sum (bruteforce_shader.cu:2171-2236).  For one env map this is
// the shading output of bruteforce_specularvisibility_shader_forward2; for K env maps the two sums
// are [points x texels] x [texels x 3K] products (the weights do not depend on the colour channel,
// so one weight matrix per term serves all three channels), which run on the tensor cores; the
// albedos are applied per point when the accumulators are read out.
//
// Precision: the weights are computed in FP32 and split into BF16 hi + lo parts, the radiance too;
// each tile accumulates hi*hi + lo*hi + hi*lo in FP32 (error ~2^-16 relative).  DES_RELIGHT_BF16
// keeps only hi*hi (plain BF16 inputs, error ~2^-8 relative per term).
//
// Kernel structure (one persistent CTA per SM, 22 warps):
//   warps 0-15  builders: per 32-texel stage, the weights of 128 points x 32 texels (W_d and W_s,
//               hi and lo) written to shared memory in the UMMA K-major no-swizzle canonical layout
//               (8-row x 16-byte core matrices, 128 B each); four threads per point row, one 8-texel
//               chunk each;
//   warp 16     allocates 512 TMEM columns; lane 0 issues tcgen05.mma (M=128, N=3K padded, K=16)
//               and tcgen05.commit to the stage-empty / accumulator-full mbarriers;
//   warps 17-20 epilogue: tcgen05.ld of the finished tile (32 TMEM lanes per warp), albedos applied,
//               -> global;
//   warp 21     lane 0 streams the prepared BF16 radiance tiles of each stage with cp.async.bulk
//               (a plain bulk copy from this GPU's memory; no multicast).
// A ring of three shared-memory stages (two for the largest maps) lets each builder warp run up to
// two stages ahead of the slowest one -- their per-stage work differs with the horizon skip -- while
// the MMAs of earlier stages run; two TMEM accumulator sets overlap a tile's epilogue with the next
// tile's MMAs when their columns fit.  Every mbarrier wait is bounded (2 s of %globaltimer): on
// timeout the CTA sets the workspace error word, stops issuing work, waits (bounded) for its own
// bulk copies and MMAs in flight, frees its TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>

#include "des_internal.h"
#include "des_math.cuh"
#include "des_point.cuh"
#include "diff_envshade_b200.h"

namespace des {
namespace relight {

constexpr int kTileM = 128;                  // points per tile (UMMA M)
constexpr int kStageT = 32;                  // texels per stage (one visibility slot)
constexpr int kMaxStages = 3;                // shared-memory ring depth (3 when it fits, else 2)
constexpr int kEnvBlock = 64;                // env maps per pass
constexpr int kBuilderThreads = 512;         // warps 0-15
constexpr int kCtrlWarp = 16;
constexpr int kEpiWarp0 = 17;                // warps 17-20
constexpr int kProdWarp = 21;
constexpr int kThreads = 22 * 32;
constexpr uint32_t kTmemCols = 512;
constexpr int kATile = kTileM * kStageT * 2;  // bytes of one BF16 [128 x 32] operand tile
constexpr long long kWaitNs = 2000000000LL;
constexpr unsigned kErrTimeout = 2u;

struct Params {
  ShadeParams pt;         // point inputs, texel table, control words
  const uint8_t* bprep;   // [nst][hl][ncols x 32] BF16 radiance tiles (canonical layout), row = c * kpad + k
  float* out;             // [P][ldo]; this pass writes columns 3*kbase .. 3*(kbase + kblock) - 1
  int64_t ldo;
  int kbase, kblock, kpad, nst, ntiles;
  int ncols;              // 3 * kpad: the MMA's N (colour channel major, env map minor)
  int nmat;               // weight matrices per stage: Lambert and/or GGX (1 or 2)
  int nstage;             // ring depth (2 or 3)
  int nacc;               // TMEM accumulator sets (2 when 2 * nmat * ncols columns fit, else 1)
  bool split;
  int vec;                // output row chunks stored as 32-byte (2), 16-byte (1) or scalar (0) writes
};

struct Smem {  // byte offsets into dynamic shared memory
  uint32_t tab, a, b, bar, misc, total;
};

__host__ __device__ inline uint32_t align_to(uint32_t x, uint32_t a) { return (x + a - 1) / a * a; }

// Bytes of one stage of radiance tiles: hi and lo, ncols x 32 texels of BF16.
__host__ __device__ inline uint32_t bprep_stage_bytes(int kpad) { return 2u * 3u * (uint32_t)kpad * kStageT * 2u; }
// Bytes of one stage of weight tiles: nmat matrices, hi and lo.
__host__ __device__ inline uint32_t a_stage_bytes(int nmat) { return (uint32_t)nmat * 2u * kATile; }

__host__ __device__ inline Smem smem_layout(int HWpad, int kpad, int nmat, int nstage) {
  Smem s;
  s.tab = 0;
  s.a = align_to((uint32_t)HWpad * 32, 1024);
  s.b = s.a + (uint32_t)nstage * a_stage_bytes(nmat);
  s.bar = align_to(s.b + (uint32_t)nstage * bprep_stage_bytes(kpad), 64);
  s.misc = s.bar + 16 * 8;
  s.total = s.misc + 64;
  return s;
}

// ---- PTX helpers --------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ long long global_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Tests the phase with the given parity; while it is incomplete the thread is suspended in hardware
// until it completes or kSuspendNs pass (the suspend-time hint), so a waiting warp takes no issue
// slots from the warps that share its SM sub-partition (a plain polling loop here took about half
// of the kernel's issue slots).
constexpr uint32_t kSuspendNs = 1000000;
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(kSuspendNs)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase with the given parity.  Returns false when this or another role of
// the CTA gave up (shared abort flag); a timeout sets the workspace error word.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag, unsigned* err) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = global_ns();
  for (;;) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*abort_flag) return false;
    if (global_ns() - t0 > kWaitNs) {
      *abort_flag = 1;
      atomicOr(err, kErrTimeout);
      return false;
    }
  }
}

__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// UMMA shared-memory descriptor, K-major, no swizzle: start, leading (K) and stride (M/N) byte offsets.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor: BF16 x BF16 -> F32, both operands K-major, M x N.
__host__ __device__ inline uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
// 32-byte global store (sm_100: st.global.v8.f32); the address is 32-byte aligned.
__device__ __forceinline__ void st_global_v8(float* ptr, const float (&x)[8]) {
  asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(ptr), "f"(x[0]), "f"(x[1]), "f"(x[2]),
               "f"(x[3]), "f"(x[4]), "f"(x[5]), "f"(x[6]), "f"(x[7])
               : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Byte offset of element (row r, texel j) in a K-major canonical [rows x 32] BF16 tile.
__host__ __device__ inline uint32_t canon_off(int r, int j) {
  return (uint32_t)(((r >> 3) * 4 + (j >> 3)) * 128 + (r & 7) * 16 + (j & 7) * 2);
}

// BF16 hi/lo split of two floats packed as bf16x2 (element 0 in the low half).
__device__ __forceinline__ void split2(float x0, float x1, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
  memcpy(&hi, &h, sizeof(hi));  // bit copies, kept in registers
  memcpy(&lo, &l, sizeof(lo));
}

// ---- radiance preparation ------------------------------------------------------------------

// bprep[st][hl][canon(c * kpad + k, j)] = hi/lo BF16 of L[kbase + k][c][st*32 + j] (zero outside the map
// and the block): per stage one [3 kpad x 32] B operand, rows ordered by colour channel, then env map.
__global__ void prep_kernel(const float* __restrict__ env, int HW, int nst, int kbase, int kblock, int kpad,
                            uint8_t* __restrict__ bprep) {
  pdl_enter();
  const int ncols = 3 * kpad;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;  // over nst * ncols * 32
  const int total = nst * ncols * kStageT;
  if (idx >= total) return;
  const int j = idx % kStageT;
  const int row = (idx / kStageT) % ncols;
  const int st = idx / (kStageT * ncols);
  const int c = row / kpad, k = row - c * kpad;
  const int t = st * kStageT + j;
  float L = 0.f;
  if (k < kblock && t < HW) L = env[((size_t)(kbase + k) * 3 + c) * HW + t];
  const __nv_bfloat16 hi = __float2bfloat16_rn(L);
  const __nv_bfloat16 lo = __float2bfloat16_rn(L - __bfloat162float(hi));
  uint8_t* base = bprep + (size_t)st * bprep_stage_bytes(kpad);
  *reinterpret_cast<__nv_bfloat16*>(base + canon_off(row, j)) = hi;
  *reinterpret_cast<__nv_bfloat16*>(base + (size_t)ncols * kStageT * 2 + canon_off(row, j)) = lo;
}

// ---- weight builders -----------------------------------------------------------------------

// One builder thread's share of one tile: for every 32-texel stage, the 8-texel chunk `quarter` of
// point row `row` of the weight matrices -- W_d = the Lambert weight wd and W_s = the GGX weight ws
// (whichever of the two terms is on), as BF16 hi and lo parts -- into the stage's shared-memory A
// tiles (K-major canonical layout).  The albedos are applied per point in the epilogue, so one pair
// of matrices serves all three colour channels.  Texels are taken in fours: four texels below the
// horizon of the warp's 32 (ordered) points get zero weights after one vote, otherwise all four are
// evaluated side by side.  The visibility words of the next stage are loaded while this one is built.  q counts
// the stages this thread has filled (ring position).  Returns false when the CTA gave up waiting (the
// whole warp leaves together).
template <bool DIFF, bool SPEC, bool VIS, bool ONEV>
__device__ __forceinline__ bool build_tile(const Params& p, const float4* s_tab, const PointGeom& g, bool valid,
                                           const SpecConst& sc, int row, int quarter, uint32_t& q, uint32_t a_base,
                                           uint64_t* full_a, uint64_t* empty, volatile int* s_abort, unsigned* err) {
  constexpr int NMAT = (DIFF ? 1 : 0) + (SPEC ? 1 : 0);
  const float cs = (g.c0 + g.c1) + g.c2;
  const uint32_t nstage = (uint32_t)p.nstage;
  uint32_t n0 = 0u, n1 = 0u, n2 = 0u;
  if (VIS) load_vis_words<ONEV>(p.pt, g, valid, 0, n0, n1, n2);
  for (int st = 0; st < p.nst; ++st, ++q) {
    const uint32_t b = q % nstage, u = q / nstage;
    uint32_t w0 = 0u, w1 = 0u, w2 = 0u;
    if (VIS) {
      w0 = n0 >> (8 * quarter);
      w1 = n1 >> (8 * quarter);
      w2 = n2 >> (8 * quarter);
      if (st + 1 < p.nst) load_vis_words<ONEV>(p.pt, g, valid, st + 1, n0, n1, n2);
    }
    // the whole warp leaves together (the texel votes below need all 32 lanes)
    if (u > 0 && !__all_sync(0xffffffffu, mbar_wait(&empty[b], (u - 1) & 1u, s_abort, err))) return false;
    const uint32_t abuf = a_base + b * a_stage_bytes(NMAT);
    const uint32_t off = abuf + (uint32_t)(((row >> 3) * 4 + quarter) * 128 + (row & 7) * 16);
    // the chunk's 8 texels go out as two 8-byte halves of four texels each: one horizon vote per
    // half (four texels below every lane's horizon get zero weights), then the four texels' weights
    // side by side -- four independent chains, the builders being latency-bound
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      uint32_t hi[NMAT][2], lo[NMAT][2];
      const int tq = st * kStageT + quarter * 8 + half * 4;
      float4 Aq[4];
      float nlq[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        Aq[i] = s_tab[2 * (tq + i)];
        nlq[i] = dot3(g.nx, g.ny, g.nz, Aq[i].x, Aq[i].y, Aq[i].z);
      }
      if (!__any_sync(0xffffffffu, nlq[0] > 0.f || nlq[1] > 0.f || nlq[2] > 0.f || nlq[3] > 0.f)) {
#pragma unroll
        for (int m = 0; m < NMAT; ++m) hi[m][0] = lo[m][0] = hi[m][1] = lo[m][1] = 0u;
      } else {
        float wdq[4], wsq[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const float dwpi = s_tab[2 * (tq + i) + 1].w;
          const float vq = pair_vis<VIS, ONEV>(w0, w1, w2, 1u << (half * 4 + i), g, cs);
          pair_fwd_weights<DIFF, SPEC>(g, sc, Aq[i], dwpi, nlq[i], vq, wdq[i], wsq[i]);
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          if (DIFF) split2(wdq[2 * h], wdq[2 * h + 1], hi[0][h], lo[0][h]);
          if (SPEC) split2(wsq[2 * h], wsq[2 * h + 1], hi[NMAT - 1][h], lo[NMAT - 1][h]);
        }
      }
#pragma unroll
      for (int m = 0; m < NMAT; ++m) {
        const uint32_t ahi = off + (uint32_t)(m * 2) * kATile + half * 8;
        asm volatile("st.shared.v2.b32 [%0], {%1, %2};" ::"r"(ahi), "r"(hi[m][0]), "r"(hi[m][1]) : "memory");
        if (p.split)
          asm volatile("st.shared.v2.b32 [%0], {%1, %2};" ::"r"(ahi + kATile), "r"(lo[m][0]), "r"(lo[m][1])
                       : "memory");
      }
    }
    fence_proxy_async_smem();
    mbar_arrive(&full_a[b]);
  }
  return true;
}

// ---- main kernel ---------------------------------------------------------------------------

template <bool DIFF, bool SPEC, bool VIS>
__global__ void __launch_bounds__(kThreads, 1) relight_kernel(const Params p) {
  pdl_enter();
  constexpr int NMAT = (DIFF ? 1 : 0) + (SPEC ? 1 : 0);
  extern __shared__ __align__(1024) uint8_t smem[];
  const int HWpad = p.pt.HWpad;
  const Smem L = smem_layout(HWpad, p.kpad, NMAT, p.nstage);
  float4* s_tab = reinterpret_cast<float4*>(smem + L.tab);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.bar);
  uint64_t* full_a = bars;          // [nstage] builders -> MMA
  uint64_t* full_b = bars + 3;      // [nstage] copy warp (tx bytes) -> MMA
  uint64_t* empty = bars + 6;       // [nstage] MMA commit -> builders, copy warp
  uint64_t* acc_full = bars + 9;    // [nacc] MMA commit -> epilogue
  uint64_t* acc_empty = bars + 11;  // [nacc] epilogue -> MMA
  uint64_t* drain = bars + 13;      // final MMA drain
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + L.misc);
  volatile int* s_abort = reinterpret_cast<volatile int*>(smem + L.misc + 8);
  unsigned* err = &p.pt.ctrl[kCtrlError];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t nstage = (uint32_t)p.nstage, nacc = (uint32_t)p.nacc;
  const uint32_t a_base = smem_u32(smem + L.a);
  const uint32_t b_base = smem_u32(smem + L.b);
  const uint32_t b_tile = (uint32_t)p.ncols * kStageT * 2;  // one [ncols x 32] BF16 tile (hi or lo)
  const uint32_t b_stage = bprep_stage_bytes(p.kpad);
  const uint32_t acc_cols = (uint32_t)(NMAT * p.ncols);     // TMEM columns of one accumulator set

  stage_table(s_tab, p.pt.table, 0, HWpad);
  if (threadIdx.x == 0) {
    for (uint32_t i = 0; i < nstage; ++i) {
      mbar_init(&full_a[i], kBuilderThreads);
      mbar_init(&full_b[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (uint32_t i = 0; i < nacc; ++i) {
      mbar_init(&acc_full[i], 1);
      mbar_init(&acc_empty[i], 128);
    }
    mbar_init(drain, 1);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kCtrlWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(s_tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;

  if (threadIdx.x < kBuilderThreads) {
    // ------------------------------------------------------------------ weight builders
    // four builder threads per point row, each building one 8-texel chunk of every stage
    const int row = threadIdx.x & 127, quarter = threadIdx.x >> 7;
    const bool need_view = SPEC || p.pt.clamp;
    uint32_t q = 0;
    for (int tile = blockIdx.x; tile < p.ntiles; tile += gridDim.x) {
      int64_t pid = (int64_t)tile * kTileM + row;
      const bool valid = ordered_point(p.pt.perm, (int64_t)tile * kTileM + row, p.pt.P, p.pt.ctrl, pid);
      const PointGeom g = load_geom<VIS>(p.pt, pid, valid, need_view);
      SpecConst sc;
      if (SPEC) sc = spec_const(valid ? p.pt.rough[pid] : 0.f, g);
      const bool onev = VIS && warp_single_vertex(g);
      const bool ok = onev ? build_tile<DIFF, SPEC, VIS, true>(p, s_tab, g, valid, sc, row, quarter, q, a_base, full_a,
                                                               empty, s_abort, err)
                           : build_tile<DIFF, SPEC, VIS, false>(p, s_tab, g, valid, sc, row, quarter, q, a_base,
                                                                full_a, empty, s_abort, err);
      if (!ok) break;
    }
  } else if (warp == kCtrlWarp) {
    // ------------------------------------------------------------------ MMA issue (one thread)
    if (lane == 0) {
      const uint32_t idesc = umma_idesc_bf16(kTileM, p.ncols);
      uint32_t q = 0;
      int i = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < p.ntiles && ok; tile += gridDim.x, ++i) {
        const uint32_t abuf = (uint32_t)i % nacc, au = (uint32_t)i / nacc;
        if (au > 0 && !mbar_wait(&acc_empty[abuf], (au - 1) & 1u, s_abort, err)) break;
        tc_fence_after();
        for (int st = 0; st < p.nst; ++st, ++q) {
          const uint32_t b = q % nstage, u = q / nstage;
          if (!mbar_wait(&full_a[b], u & 1u, s_abort, err) || !mbar_wait(&full_b[b], u & 1u, s_abort, err)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t bh = b_base + b * b_stage;
#pragma unroll
          for (int m = 0; m < NMAT; ++m) {
            // D_m[128 x ncols] += W_m[128 x 16] . B[ncols x 16]^T, per 16-texel half of the stage
            const uint32_t d = tmem + abuf * acc_cols + (uint32_t)m * (uint32_t)p.ncols;
            const uint32_t ah = a_base + b * a_stage_bytes(NMAT) + (uint32_t)(m * 2) * kATile;
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
              const uint64_t da = umma_desc(ah + ks * 256, 128, 512);
              const uint64_t db = umma_desc(bh + ks * 256, 128, 512);
              umma_bf16(d, da, db, idesc, (st | ks) != 0 ? 1u : 0u);
              if (p.split) {
                umma_bf16(d, umma_desc(ah + kATile + ks * 256, 128, 512), db, idesc, 1u);
                umma_bf16(d, da, umma_desc(bh + b_tile + ks * 256, 128, 512), idesc, 1u);
              }
            }
          }
          umma_commit(&empty[b]);
        }
        if (ok) umma_commit(&acc_full[abuf]);
      }
    }
    __syncwarp();
  } else if (warp >= kEpiWarp0 && warp < kEpiWarp0 + 4) {
    // ------------------------------------------------------------------ epilogue
    // out[p, k, c] = albedo_c D_d[c kpad + k] + specular_c D_s[c kpad + k]
    const uint32_t quarter = (uint32_t)warp & 3u;  // TMEM lanes this warp may access
    const int row = (int)quarter * 32 + lane;
    const uint32_t lanes = (quarter * 32u) << 16;
    int i = 0;
    for (int tile = blockIdx.x; tile < p.ntiles; tile += gridDim.x, ++i) {
      const uint32_t abuf = (uint32_t)i % nacc, au = (uint32_t)i / nacc;
      int64_t pid = 0;
      const bool live = ordered_point(p.pt.perm, (int64_t)tile * kTileM + row, p.pt.P, p.pt.ctrl, pid);
      float alb[3] = {0.f, 0.f, 0.f}, spc[3] = {0.f, 0.f, 0.f};
      if (live) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (DIFF) alb[c] = p.pt.albedo[3 * pid + c];
          if (SPEC) spc[c] = p.pt.spec[3 * pid + c];
        }
      }
      if (!mbar_wait(&acc_full[abuf], au & 1u, s_abort, err)) break;
      tc_fence_after();
      float* orow = p.out + pid * p.ldo + (int64_t)p.kbase * 3;
      const uint32_t t0 = tmem + lanes + abuf * acc_cols;
      for (int kb = 0; kb < p.kpad / 8; ++kb) {
        // all six 8-column loads of the chunk (both terms, three channels) in flight before one wait
        float o[3][8], v[3][8];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const uint32_t col = (uint32_t)(c * p.kpad + kb * 8);
          if (DIFF) tmem_ld8(t0 + col, o[c]);
          if (SPEC) tmem_ld8(t0 + (uint32_t)(NMAT - 1) * (uint32_t)p.ncols + col, v[c]);
        }
        tmem_wait_ld();
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int e = 0; e < 8; ++e)
            o[c][e] = DIFF ? (SPEC ? fmaf(spc[c], v[c][e], alb[c] * o[c][e]) : alb[c] * o[c][e]) : spc[c] * v[c][e];
        if (live) {
          const int k0 = kb * 8;
          if (p.vec == 2 && k0 + 8 <= p.kblock) {
            // a chunk's 24 outputs (8 maps x 3 channels, contiguous in the row) as three 32-byte
            // stores: each writes whole 32-byte sectors, half the store instructions of float4s
            float* o8 = orow + k0 * 3;
#pragma unroll
            for (int i8 = 0; i8 < 3; ++i8) {
              float x[8];
#pragma unroll
              for (int e = 0; e < 8; ++e) {
                const int f = i8 * 8 + e;
                x[e] = o[f % 3][f / 3];
              }
              st_global_v8(o8 + i8 * 8, x);
            }
          } else if (p.vec == 1 && k0 + 8 <= p.kblock) {
            float4* o4 = reinterpret_cast<float4*>(orow + k0 * 3);
#pragma unroll
            for (int i4 = 0; i4 < 6; ++i4) {
              float x[4];
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                const int f = i4 * 4 + e;
                x[e] = o[f % 3][f / 3];
              }
              o4[i4] = make_float4(x[0], x[1], x[2], x[3]);
            }
          } else {
#pragma unroll
            for (int kk = 0; kk < 8; ++kk)
              if (k0 + kk < p.kblock) {
#pragma unroll
                for (int c = 0; c < 3; ++c) orow[(k0 + kk) * 3 + c] = o[c][kk];
              }
          }
        }
      }
      tc_fence_before();
      mbar_arrive(&acc_empty[abuf]);
    }
  } else if (warp == kProdWarp) {
    // ------------------------------------------------------------------ radiance bulk copies
    if (lane == 0) {
      uint32_t q = 0;  // copies issued
      for (int tile = blockIdx.x; tile < p.ntiles; tile += gridDim.x) {
        bool ok = true;
        for (int st = 0; st < p.nst; ++st) {
          const uint32_t b = q % nstage, u = q / nstage;
          if (u > 0 && !mbar_wait(&empty[b], (u - 1) & 1u, s_abort, err)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&full_b[b], b_stage);
          bulk_g2s(b_base + b * b_stage, p.bprep + (size_t)st * b_stage, b_stage, &full_b[b]);
          ++q;
        }
        if (!ok) break;
      }
      // never leave a bulk copy in flight: wait (bounded) for the last one into each buffer
      for (uint32_t b = 0; b < nstage; ++b) {
        if (q <= b) continue;
        const uint32_t n_b = (q - b + nstage - 1) / nstage;  // copies into buffer b
        const long long t0 = global_ns();
        while (!mbar_try_wait(&full_b[b], (n_b - 1u) & 1u)) {
          if (global_ns() - t0 > kWaitNs) {
            atomicOr(err, kErrTimeout);
            break;
          }
        }
      }
    }
    __syncwarp();
  }

  // ------------------------------------------------------------------ teardown
  tc_fence_before();
  __syncthreads();
  if (warp == kCtrlWarp) {
    tc_fence_after();
    if (lane == 0) {
      // all MMAs this thread issued have completed before TMEM is freed
      umma_commit(drain);
      const long long t0 = global_ns();
      while (!mbar_try_wait(drain, 0u)) {
        if (global_ns() - t0 > kWaitNs) {
          atomicOr(err, kErrTimeout);
          break;
        }
      }
    }
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

}  // namespace relight

// ---- host side -----------------------------------------------------------------------------

namespace {

inline size_t align256(size_t x) { return (x + 255) / 256 * 256; }

using RelightFn = void (*)(const relight::Params);

RelightFn pick_relight(bool diff, bool spec, bool vis) {
  using namespace relight;
  if (diff) {
    if (spec) return vis ? relight_kernel<true, true, true> : relight_kernel<true, true, false>;
    return vis ? relight_kernel<true, false, true> : relight_kernel<true, false, false>;
  }
  return vis ? relight_kernel<false, true, true> : relight_kernel<false, true, false>;
}

int kpad_of(int kblock) { return std::max(16, (kblock + 15) / 16 * 16); }

}  // namespace

size_t relight_workspace_bytes(int64_t P, int H, int W, int K) {
  if (P < 0 || H <= 0 || W <= 0 || K <= 0) return 0;
  const int HWpad = (H * W + 31) / 32 * 32;
  const int kpad = kpad_of(std::min(K, relight::kEnvBlock));
  size_t b = kCtrlBytes + align256((size_t)HWpad * 32) + align256((size_t)(HWpad / 32) * relight::bprep_stage_bytes(kpad));
  if (P >= kSortMinP && P <= kSortMaxP)  // normal-direction ordering: permutation + its scratch
    b += align256((size_t)P * 4) + align256(point_order_scratch_bytes(P));
  return b;
}

int launch_relight(const des_shade_args& a, const float* envmaps, int K, unsigned flags, float* out, void* ws,
                   size_t ws_bytes, cudaStream_t stream) {
  const bool diff = flags & DES_DIFFUSE, spec = flags & DES_SPECULAR;
  const bool vis = a.visibility != nullptr;
  const int HW = a.H * a.W;
  const int HWpad = (HW + 31) / 32 * 32;
  if (HWpad > 2048) return DES_ERR_UNSUPPORTED;  // the texel table must fit in shared memory
  if (ws == nullptr || ws_bytes < relight_workspace_bytes(a.P, a.H, a.W, K) ||
      (reinterpret_cast<uintptr_t>(ws) & 255u) != 0)
    return DES_ERR_WORKSPACE;
  int dev = 0, sms = 0, max_smem = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DES_ERR_CUDA;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);

  uint8_t* w = static_cast<uint8_t*>(ws);
  unsigned* ctrl = reinterpret_cast<unsigned*>(w);
  float4* table = reinterpret_cast<float4*>(w + kCtrlBytes);
  uint8_t* bprep = w + kCtrlBytes + align256((size_t)HWpad * 32);
  const int kpad_max = kpad_of(std::min(K, relight::kEnvBlock));
  uint8_t* order_area = bprep + align256((size_t)(HWpad / 32) * relight::bprep_stage_bytes(kpad_max));

  int st = launch_table(a.H, a.W, HWpad, a.light2obj_rotmat, envmaps, table, ctrl, stream);
  if (st != DES_OK) return st;
  if (a.P == 0) return DES_OK;
  if (!diff && !spec) {
    return cudaMemsetAsync(out, 0, sizeof(float) * 3 * (size_t)K * a.P, stream) == cudaSuccess ? DES_OK : DES_ERR_CUDA;
  }

  relight::Params prm{};
  ShadeParams& pt = prm.pt;
  pt.P = a.P;
  pt.HWpad = HWpad;
  pt.chunk = HWpad;
  pt.N_face = a.N_face;
  pt.N_vertex = a.N_vertex;
  pt.normal = a.normal;
  pt.view = a.view_dir;
  pt.albedo = a.albedo;
  pt.spec = a.specular_albedo;
  pt.rough = a.roughness;
  pt.faces = a.face_vertex_list;
  pt.tri = a.nearest_triangle_id;
  pt.bary = a.barycentric_coord;
  pt.vis = a.visibility;
  pt.table = table;
  pt.clamp = (flags & DES_CLAMP) != 0;
  pt.ctrl = ctrl;
  prm.bprep = bprep;
  prm.out = out;
  prm.ldo = 3 * (int64_t)K;
  prm.nst = HWpad / relight::kStageT;
  prm.ntiles = (int)((a.P + relight::kTileM - 1) / relight::kTileM);
  prm.split = !(flags & DES_RELIGHT_BF16);
  pt.perm = nullptr;
  if (a.P >= kSortMinP && a.P <= kSortMaxP) {
    // order the points by normal direction: each builder warp's 32 points then face the same way
    // and texels below all of their horizons are skipped (per-point results unchanged)
    int32_t* perm = reinterpret_cast<int32_t*>(order_area);
    st = launch_point_order(a.normal, a.P, order_area + align256((size_t)a.P * 4), perm, stream);
    if (st != DES_OK) return st;
    pt.perm = perm;
  }

  RelightFn k = pick_relight(diff, spec, vis);
  const int grid = std::max(1, std::min(prm.ntiles, sms));
  prm.nmat = (diff ? 1 : 0) + (spec ? 1 : 0);
  for (int kbase = 0; kbase < K; kbase += relight::kEnvBlock) {
    prm.kbase = kbase;
    prm.kblock = std::min(relight::kEnvBlock, K - kbase);
    prm.kpad = kpad_of(prm.kblock);
    prm.ncols = 3 * prm.kpad;
    // two accumulator sets (the epilogue of one tile overlaps the MMAs of the next) when they fit
    // in the 512 TMEM columns, else one
    prm.nacc = 2 * prm.nmat * prm.ncols <= (int)relight::kTmemCols ? 2 : 1;
    const uintptr_t oa = reinterpret_cast<uintptr_t>(out);
    prm.vec = ((oa & 31u) == 0 && prm.ldo % 8 == 0 && (kbase * 3) % 8 == 0)   ? 2
              : ((oa & 15u) == 0 && prm.ldo % 4 == 0 && (kbase * 3) % 4 == 0) ? 1
                                                                               : 0;
    // the deepest ring that fits in shared memory
    prm.nstage = relight::kMaxStages;
    while (prm.nstage > 2 && (int)relight::smem_layout(HWpad, prm.kpad, prm.nmat, prm.nstage).total > max_smem)
      --prm.nstage;
    const relight::Smem L = relight::smem_layout(HWpad, prm.kpad, prm.nmat, prm.nstage);
    if ((int)L.total > max_smem) return DES_ERR_UNSUPPORTED;
    const int total = prm.nst * prm.ncols * relight::kStageT;
    launch_pdl(relight::prep_kernel, dim3((total + 255) / 256), dim3(256), 0, stream, envmaps, HW, prm.nst, kbase,
               prm.kblock, prm.kpad, bprep);
    if (cudaGetLastError() != cudaSuccess) return DES_ERR_CUDA;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total) != cudaSuccess)
      return DES_ERR_CUDA;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    timing_events(ev0, ev1);
    const bool timed = ev0 != nullptr && ev1 != nullptr && kbase == 0;  // the first pass of K
    if (timed) cudaEventRecord(ev0, stream);
    launch_pdl(k, dim3(grid), dim3(relight::kThreads), L.total, stream, prm);
    if (cudaGetLastError() != cudaSuccess) return DES_ERR_CUDA;
    if (timed) cudaEventRecord(ev1, stream);
    count_launches(2);
  }
  return DES_OK;
}

}  // namespace des
