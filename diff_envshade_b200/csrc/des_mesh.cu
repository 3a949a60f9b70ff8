// Mesh-side helpers of the visibility path: the inputs of the shading kernels' visibility gather
// (nearest triangle and barycentric coordinates of each point) and the bit-to-float view of the
// packed visibility words.
//
// Reference correspondence (zjumsj/diff_envshade, etc.cu):
//   closest point on a triangle + its adjoint        closestPointOnTriangle{,_backward} (205-380)
//   get_uv_of_triangle_{forward,backward}             GetUVofTriangle_{Forward,Backward} (707-777)
//   get_nearest_mesh_points_{forward,backward}        GetNearestMeshPoints_{Forward,Backward} (780-935)
//   extract_bitfield_forward                          ExtractBitfield_Forward (1021-1040)
//
// Differences kept on purpose:
//  * nearest mesh points: the candidate faces are visited in the reference's order (the K nearest
//    vertices in order, each vertex's adjacency list in order) and the strictly closest one is kept,
//    so the selection is the reference's; repeated faces are simply evaluated again (a repeat can
//    never beat its own first occurrence), which removes the reference's 128-entry per-thread
//    de-duplication array and its overflow trap.  Out-of-range vertex / face ids are skipped; a
//    query with no candidate face gets triangle id -1 and zero coordinates and sets bit 0 of the
//    optional error word (the reference traps);
//  * nearest mesh points, backward: the incoming gradient is grad_barycentric_coord (the reference
//    kernel reads its own uninitialised output buffer there, etc.cu:884-888).
#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

#include "des_internal.h"
#include "diff_envshade_b200.h"

namespace des {
namespace mesh {

// The arithmetic below is spelled with explicit roundings (__fmaf_rn / __fmul_rn) in the order the
// reference's compiled kernels evaluate their expressions, identified from the reference's outputs
// (its fixtures tests/golden/etc_*.npz are reproduced bit for bit): a dot product
// x.x*y.x + x.y*y.y + x.z*y.z is fma(z, z', fma(x, x', y*y')), and a*b - c*d is fma(a, b, -(c*d)).
// Exact agreement matters for the selected triangle, an index, where two faces are equally close.
struct V3 {
  float x, y, z;
};
__device__ __forceinline__ V3 sub3(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ float dot3v(V3 a, V3 b) {
  return __fmaf_rn(a.z, b.z, __fmaf_rn(a.x, b.x, __fmul_rn(a.y, b.y)));
}
// a*b - c*d
__device__ __forceinline__ float dif2(float a, float b, float c, float d) { return __fmaf_rn(a, b, -__fmul_rn(c, d)); }
__device__ __forceinline__ float clamp01(float v) { return v < 0.f ? 0.f : (v > 1.f ? 1.f : v); }

// Region of the closest point in the triangle's (s, t) parameter plane, for
// P(s, t) = x0 + s (x1 - x0) + t (x2 - x0): 0 interior, 1 on the edge t = 0, 2 on the edge s = 0,
// 3 on the edge s + t = 1 (the classification of the reference's closestPointOnTriangle).
struct TriQuery {
  V3 e0, e1;
  float a, b, c, d, e, det, s, t;
  int region;
};

__device__ __forceinline__ TriQuery tri_query(V3 x0, V3 x1, V3 x2, V3 q) {
  TriQuery r;
  r.e0 = sub3(x1, x0);
  r.e1 = sub3(x2, x0);
  const V3 v0 = sub3(x0, q);
  r.a = dot3v(r.e0, r.e0);
  r.b = dot3v(r.e0, r.e1);
  r.c = dot3v(r.e1, r.e1);
  r.d = dot3v(r.e0, v0);
  r.e = dot3v(r.e1, v0);
  r.det = dif2(r.a, r.c, r.b, r.b);
  r.s = dif2(r.b, r.e, r.c, r.d);
  r.t = dif2(r.b, r.d, r.a, r.e);
  if (r.s + r.t < r.det) {
    if (r.s < 0.f)
      r.region = (r.t < 0.f && r.d < 0.f) ? 1 : 2;
    else
      r.region = (r.t < 0.f) ? 1 : 0;
  } else {
    if (r.s < 0.f)
      r.region = (r.c + r.e > r.b + r.d) ? 3 : 2;
    else if (r.t < 0.f)
      r.region = (r.a + r.d > r.b + r.e) ? 3 : 1;
    else
      r.region = 3;
  }
  return r;
}

// Closest point parameters (s, t) of q on the triangle; returns the point.
__device__ __forceinline__ V3 closest_point(V3 x0, V3 x1, V3 x2, V3 q, float& s, float& t) {
  const TriQuery r = tri_query(x0, x1, x2, q);
  if (r.region == 0) {
    const float inv = 1.f / r.det;
    s = r.s * inv;
    t = r.t * inv;
  } else if (r.region == 1) {
    s = clamp01(-r.d / r.a);
    t = 0.f;
  } else if (r.region == 2) {
    s = 0.f;
    t = clamp01(-r.e / r.c);
  } else {
    s = clamp01((r.c + r.e - r.b - r.d) / (__fmaf_rn(-2.f, r.b, r.a) + r.c));
    t = 1.f - s;
  }
  return V3{__fmaf_rn(t, r.e1.x, __fmaf_rn(s, r.e0.x, x0.x)), __fmaf_rn(t, r.e1.y, __fmaf_rn(s, r.e0.y, x0.y)),
            __fmaf_rn(t, r.e1.z, __fmaf_rn(s, r.e0.z, x0.z))};
}

// d(loss)/dq of the closest point parameters, given gs = dL/ds and gt = dL/dt (zero where a
// parameter is clamped).
__device__ __forceinline__ V3 closest_point_adjoint(V3 x0, V3 x1, V3 x2, V3 q, float gs, float gt) {
  const TriQuery r = tri_query(x0, x1, x2, q);
  V3 g{0.f, 0.f, 0.f};
  if (r.region == 0) {  // s, t = their plane solution: gradient k0 e0 + k1 e1
    const float inv = 1.f / r.det;
    const float k0 = __fmul_rn(dif2(gs, r.c, gt, r.b), inv), k1 = __fmul_rn(dif2(gt, r.a, gs, r.b), inv);
    g = V3{__fmaf_rn(r.e0.x, k0, __fmul_rn(r.e1.x, k1)), __fmaf_rn(r.e0.y, k0, __fmul_rn(r.e1.y, k1)),
           __fmaf_rn(r.e0.z, k0, __fmul_rn(r.e1.z, k1))};
  } else if (r.region == 1) {  // s = -d/a on the edge t = 0 (zero where clamped)
    const float u = -r.d / r.a;
    if (u >= 0.f && u <= 1.f) {
      const float k = gs / r.a;
      g = V3{__fmul_rn(r.e0.x, k), __fmul_rn(r.e0.y, k), __fmul_rn(r.e0.z, k)};
    }
  } else if (r.region == 2) {  // t = -e/c on the edge s = 0
    const float u = -r.e / r.c;
    if (u >= 0.f && u <= 1.f) {
      const float k = gt / r.c;
      g = V3{__fmul_rn(r.e1.x, k), __fmul_rn(r.e1.y, k), __fmul_rn(r.e1.z, k)};
    }
  } else {  // s on the edge s + t = 1, t = 1 - s
    const float den = __fmaf_rn(-2.f, r.b, r.a) + r.c;
    const float u = (r.c + r.e - r.b - r.d) / den;
    if (u >= 0.f && u <= 1.f) {
      const float k = (gs - gt) / den;
      g = V3{__fmul_rn(r.e0.x - r.e1.x, k), __fmul_rn(r.e0.y - r.e1.y, k), __fmul_rn(r.e0.z - r.e1.z, k)};
    }
  }
  return g;
}

// ---------------------------------------------------------------------------------------------
// UV of a triangle (one triangle per point, AoS): barycentric (1 - s - t, s, t) of the closest point
// ---------------------------------------------------------------------------------------------

__global__ void __launch_bounds__(256) uv_fwd_kernel(int64_t P, const float* __restrict__ tri,
                                                     const float* __restrict__ q, float* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const float* T = tri + 9 * i;
  const V3 x0{T[0], T[1], T[2]}, x1{T[3], T[4], T[5]}, x2{T[6], T[7], T[8]};
  const V3 p{q[3 * i], q[3 * i + 1], q[3 * i + 2]};
  float s, t;
  closest_point(x0, x1, x2, p, s, t);
  out[3 * i] = 1.f - s - t;
  out[3 * i + 1] = s;
  out[3 * i + 2] = t;
}

__global__ void __launch_bounds__(256) uv_bwd_kernel(int64_t P, const float* __restrict__ tri,
                                                     const float* __restrict__ q, const float* __restrict__ g,
                                                     float* __restrict__ gq) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const float* T = tri + 9 * i;
  const V3 x0{T[0], T[1], T[2]}, x1{T[3], T[4], T[5]}, x2{T[6], T[7], T[8]};
  const V3 p{q[3 * i], q[3 * i + 1], q[3 * i + 2]};
  const float g0 = g[3 * i], g1 = g[3 * i + 1], g2 = g[3 * i + 2];
  const V3 r = closest_point_adjoint(x0, x1, x2, p, g1 - g0, g2 - g0);
  gq[3 * i] = r.x;
  gq[3 * i + 1] = r.y;
  gq[3 * i + 2] = r.z;
}

// ---------------------------------------------------------------------------------------------
// Nearest mesh point among the faces adjacent to each query's K nearest vertices
// ---------------------------------------------------------------------------------------------

__device__ __forceinline__ V3 vertex(const float* __restrict__ pos, int N_vertex, int v) {
  return V3{pos[v], pos[N_vertex + v], pos[2 * (int64_t)N_vertex + v]};
}

__global__ void __launch_bounds__(256) nearest_fwd_kernel(int N_vertex, int N_face, int64_t P, int K, int64_t N_adj,
                                                          const int32_t* __restrict__ adj_head,
                                                          const int32_t* __restrict__ adj_list,
                                                          const int32_t* __restrict__ faces,
                                                          const float* __restrict__ vpos, const float* __restrict__ q,
                                                          const int64_t* __restrict__ idxs, int64_t* __restrict__ tri_out,
                                                          float* __restrict__ bary_out, unsigned* __restrict__ err) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const V3 p{q[i], q[P + i], q[2 * P + i]};
  float best = FLT_MAX, bs = 0.f, bt = 0.f;
  int best_face = -1;
  for (int k = 0; k < K; ++k) {
    const int64_t v = idxs[i * K + k];
    if (v < 0 || v >= N_vertex) continue;
    const int n = adj_head[v];                   // faces adjacent to v
    const int64_t end = adj_head[N_vertex + v];  // inclusive prefix sum of the counts
    const int64_t begin = end - n;
    if (n <= 0 || begin < 0 || end > N_adj) continue;
    for (int64_t j = begin; j < end; ++j) {
      const int f = adj_list[j];
      if (f < 0 || f >= N_face) continue;
      const int a = faces[f], b = faces[N_face + f], c = faces[2 * (int64_t)N_face + f];
      if (a < 0 || a >= N_vertex || b < 0 || b >= N_vertex || c < 0 || c >= N_vertex) continue;
      float s, t;
      const V3 cp = closest_point(vertex(vpos, N_vertex, a), vertex(vpos, N_vertex, b), vertex(vpos, N_vertex, c), p, s, t);
      const V3 dv = sub3(cp, p);
      const float d2 = dot3v(dv, dv);
      if (d2 < best) {  // strict: the first of equally close faces stays
        best = d2;
        best_face = f;
        bs = s;
        bt = t;
      }
    }
  }
  if (best_face < 0 && err != nullptr) atomicOr(err, 1u);
  tri_out[i] = best_face;
  bary_out[i] = best_face < 0 ? 0.f : 1.f - bs - bt;
  bary_out[P + i] = bs;
  bary_out[2 * P + i] = bt;
}

__global__ void __launch_bounds__(256) nearest_bwd_kernel(int N_vertex, int N_face, int64_t P,
                                                          const int32_t* __restrict__ faces,
                                                          const float* __restrict__ vpos, const float* __restrict__ q,
                                                          const int64_t* __restrict__ tri, const float* __restrict__ g,
                                                          float* __restrict__ gq, unsigned* __restrict__ err) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  V3 r{0.f, 0.f, 0.f};
  const int64_t f = tri[i];
  if (f >= 0 && f < N_face) {
    const int a = faces[f], b = faces[N_face + f], c = faces[2 * (int64_t)N_face + f];
    if (a >= 0 && a < N_vertex && b >= 0 && b < N_vertex && c >= 0 && c < N_vertex) {
      const V3 p{q[i], q[P + i], q[2 * P + i]};
      const float g0 = g[i], g1 = g[P + i], g2 = g[2 * P + i];
      r = closest_point_adjoint(vertex(vpos, N_vertex, a), vertex(vpos, N_vertex, b), vertex(vpos, N_vertex, c), p,
                                g1 - g0, g2 - g0);
    } else if (err != nullptr) {
      atomicOr(err, 1u);
    }
  } else if (err != nullptr) {
    atomicOr(err, 1u);
  }
  gq[i] = r.x;
  gq[P + i] = r.y;
  gq[2 * P + i] = r.z;
}

// ---------------------------------------------------------------------------------------------
// Packed visibility words -> floats: out[b][k] = bit k of point i_start + b (1.0 / 0.0)
// ---------------------------------------------------------------------------------------------

// Four bits per thread, one float4 store (rows of N_bit floats, N_bit % 4 == 0).
__global__ void __launch_bounds__(256) bits4_kernel(int N, int N_bit, int i_start, int n_rows,
                                                    const uint32_t* __restrict__ words, float4* __restrict__ out) {
  const int q4 = N_bit >> 2;
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n_rows * q4) return;
  const int row = (int)(idx / q4), k = (int)(idx - (int64_t)row * q4) * 4;
  const uint32_t w = words[(int64_t)(k >> 5) * N + i_start + row] >> (k & 31);
  out[idx] = make_float4((float)(w & 1u), (float)((w >> 1) & 1u), (float)((w >> 2) & 1u), (float)((w >> 3) & 1u));
}

__global__ void __launch_bounds__(256) bits1_kernel(int N, int N_bit, int i_start, int n_rows,
                                                    const uint32_t* __restrict__ words, float* __restrict__ out) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n_rows * N_bit) return;
  const int row = (int)(idx / N_bit), k = (int)(idx - (int64_t)row * N_bit);
  out[idx] = (float)((words[(int64_t)(k >> 5) * N + i_start + row] >> (k & 31)) & 1u);
}

inline unsigned blocks_for(int64_t n) { return (unsigned)((n + 255) / 256); }

}  // namespace mesh
}  // namespace des

using namespace des::mesh;

extern "C" {

int des_get_uv_of_triangle_forward(int64_t P, const float* triangles, const float* query_pos,
                                   float* barycentric_coord, des_stream_t stream) {
  if (P < 0 || (P > 0 && (!triangles || !query_pos || !barycentric_coord))) return DES_ERR_INVALID_ARGUMENT;
  if (P == 0) return DES_OK;
  uv_fwd_kernel<<<blocks_for(P), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(P, triangles, query_pos,
                                                                                   barycentric_coord);
  des::count_launches(1);
  return cudaGetLastError() == cudaSuccess ? DES_OK : DES_ERR_CUDA;
}

int des_get_uv_of_triangle_backward(int64_t P, const float* triangles, const float* query_pos,
                                    const float* grad_barycentric_coord, float* grad_query_pos, des_stream_t stream) {
  if (P < 0 || (P > 0 && (!triangles || !query_pos || !grad_barycentric_coord || !grad_query_pos)))
    return DES_ERR_INVALID_ARGUMENT;
  if (P == 0) return DES_OK;
  uv_bwd_kernel<<<blocks_for(P), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(P, triangles, query_pos,
                                                                                   grad_barycentric_coord,
                                                                                   grad_query_pos);
  des::count_launches(1);
  return cudaGetLastError() == cudaSuccess ? DES_OK : DES_ERR_CUDA;
}

int des_get_nearest_mesh_points_forward(int32_t N_vertex, int32_t N_face, int64_t P, int32_t K, int64_t N_adj,
                                        const int32_t* adjacency_head, const int32_t* adjacency_list,
                                        const int32_t* face_vertex_list, const float* vertex_pos,
                                        const float* query_pos, const int64_t* idxs, int64_t* nearest_triangle_id,
                                        float* barycentric_coord, unsigned* error_word, des_stream_t stream) {
  if (P < 0 || K < 0 || N_vertex < 0 || N_face < 0 || N_adj < 0) return DES_ERR_INVALID_ARGUMENT;
  if (P == 0) return DES_OK;
  if (!adjacency_head || (N_adj > 0 && !adjacency_list) || !face_vertex_list || !vertex_pos || !query_pos ||
      (K > 0 && !idxs) || !nearest_triangle_id || !barycentric_coord)
    return DES_ERR_INVALID_ARGUMENT;
  nearest_fwd_kernel<<<blocks_for(P), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      N_vertex, N_face, P, K, N_adj, adjacency_head, adjacency_list, face_vertex_list, vertex_pos, query_pos, idxs,
      nearest_triangle_id, barycentric_coord, error_word);
  des::count_launches(1);
  return cudaGetLastError() == cudaSuccess ? DES_OK : DES_ERR_CUDA;
}

int des_get_nearest_mesh_points_backward(int32_t N_vertex, int32_t N_face, int64_t P, const int32_t* face_vertex_list,
                                         const float* vertex_pos, const float* query_pos,
                                         const int64_t* nearest_triangle_id, const float* grad_barycentric_coord,
                                         float* grad_query_pos, unsigned* error_word, des_stream_t stream) {
  if (P < 0 || N_vertex < 0 || N_face < 0) return DES_ERR_INVALID_ARGUMENT;
  if (P == 0) return DES_OK;
  if (!face_vertex_list || !vertex_pos || !query_pos || !nearest_triangle_id || !grad_barycentric_coord ||
      !grad_query_pos)
    return DES_ERR_INVALID_ARGUMENT;
  nearest_bwd_kernel<<<blocks_for(P), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      N_vertex, N_face, P, face_vertex_list, vertex_pos, query_pos, nearest_triangle_id, grad_barycentric_coord,
      grad_query_pos, error_word);
  des::count_launches(1);
  return cudaGetLastError() == cudaSuccess ? DES_OK : DES_ERR_CUDA;
}

int des_extract_bitfield_forward(int32_t N_slot, int32_t N, int32_t N_bit, int32_t i_start, int32_t i_end,
                                 const int32_t* bitfield, float* out, des_stream_t stream) {
  if (N_slot <= 0 || N <= 0 || N_bit < 0 || (int64_t)N_bit > (int64_t)N_slot * 32 || i_start < 0 || i_end > N ||
      i_end < i_start || !bitfield || (!out && i_end > i_start && N_bit > 0))
    return DES_ERR_INVALID_ARGUMENT;
  const int rows = i_end - i_start;
  if (rows == 0 || N_bit == 0) return DES_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const uint32_t* w = reinterpret_cast<const uint32_t*>(bitfield);
  if (N_bit % 4 == 0 && (reinterpret_cast<uintptr_t>(out) & 15u) == 0)
    bits4_kernel<<<blocks_for((int64_t)rows * (N_bit / 4)), 256, 0, s>>>(N, N_bit, i_start, rows, w,
                                                                         reinterpret_cast<float4*>(out));
  else
    bits1_kernel<<<blocks_for((int64_t)rows * N_bit), 256, 0, s>>>(N, N_bit, i_start, rows, w, out);
  des::count_launches(1);
  return cudaGetLastError() == cudaSuccess ? DES_OK : DES_ERR_CUDA;
}

}  // extern "C"
