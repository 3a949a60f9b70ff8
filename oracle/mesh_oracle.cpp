// CPU oracle for the mesh-side helpers of the visibility path and for the env-map sampling helper.
//
// TEST INFRASTRUCTURE ONLY.  Restates on the host, in FP64 (the checker) and FP32, what the
// reference extension zjumsj/diff_envshade computes in etc.cu; the product package never links or
// calls it.  Each function names the reference lines it follows.
//
//   closest point on a triangle and its adjoint          etc.cu:205-380
//   get_uv_of_triangle_{forward,backward}                 etc.cu:707-777, 1218-1275
//   get_nearest_mesh_points_{forward,backward}            etc.cu:780-935, 1277-1373
//   extract_bitfield_forward                              etc.cu:1021-1071
//   sample_envmap_forward (bilinear lat-long lookup)      etc.cu:527-583, 687-705, 1145-1178
//
// The nearest-point backward uses grad_barycentric_coord as its incoming gradient (the
// reference kernel reads its own uninitialised output there, etc.cu:884-888).

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <limits>

namespace {

template <typename T> struct P3 { T x, y, z; };
template <typename T> inline P3<T> sub(P3<T> a, P3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T> inline T dot(P3<T> a, P3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> inline T clamp01(T v) { return v < T(0) ? T(0) : (v > T(1) ? T(1) : v); }

// Region classification of the closest point, etc.cu:205-265 (the same decision tree in the
// forward and the adjoint): 0 interior, 1 edge t = 0, 2 edge s = 0, 3 edge s + t = 1.
template <typename T> struct Tri {
  P3<T> e0, e1;
  T a, b, c, d, e, det, s, t;
  int region;
};

template <typename T> Tri<T> classify(P3<T> x0, P3<T> x1, P3<T> x2, P3<T> q) {
  Tri<T> r;
  r.e0 = sub(x1, x0);
  r.e1 = sub(x2, x0);
  const P3<T> v0 = sub(x0, q);
  r.a = dot(r.e0, r.e0);
  r.b = dot(r.e0, r.e1);
  r.c = dot(r.e1, r.e1);
  r.d = dot(r.e0, v0);
  r.e = dot(r.e1, v0);
  r.det = r.a * r.c - r.b * r.b;
  r.s = r.b * r.e - r.c * r.d;
  r.t = r.b * r.d - r.a * r.e;
  int type = 0;
  if (r.s + r.t < r.det) {
    if (r.s < 0) {
      if (r.t < 0) type = (r.d < 0) ? 1 : 2;
      else type = 2;
    } else if (r.t < 0) {
      type = 1;
    }
  } else {
    if (r.s < 0) type = (r.c + r.e > r.b + r.d) ? 3 : 2;
    else if (r.t < 0) type = (r.a + r.d > r.b + r.e) ? 3 : 1;
    else type = 3;
  }
  r.region = type;
  return r;
}

// etc.cu:302-380
template <typename T> P3<T> closest(P3<T> x0, P3<T> x1, P3<T> x2, P3<T> q, T& s, T& t) {
  const Tri<T> r = classify(x0, x1, x2, q);
  if (r.region == 0) {
    const T inv = T(1) / r.det;
    s = r.s * inv;
    t = r.t * inv;
  } else if (r.region == 1) {
    s = clamp01(-r.d / r.a);
    t = 0;
  } else if (r.region == 2) {
    s = 0;
    t = clamp01(-r.e / r.c);
  } else {
    s = clamp01((r.c + r.e - r.b - r.d) / (r.a - T(2) * r.b + r.c));
    t = T(1) - s;
  }
  return {x0.x + s * r.e0.x + t * r.e1.x, x0.y + s * r.e0.y + t * r.e1.y, x0.z + s * r.e0.z + t * r.e1.z};
}

// etc.cu:266-300
template <typename T> P3<T> closest_adjoint(P3<T> x0, P3<T> x1, P3<T> x2, P3<T> q, T gs, T gt) {
  const Tri<T> r = classify(x0, x1, x2, q);
  T k0 = 0, k1 = 0;
  if (r.region == 0) {
    const T inv = T(1) / r.det;
    k0 = (gs * r.c - gt * r.b) * inv;
    k1 = (gt * r.a - gs * r.b) * inv;
  } else if (r.region == 1) {
    const T u = -r.d / r.a;
    if (u >= 0 && u <= 1) k0 = gs / r.a;
  } else if (r.region == 2) {
    const T u = -r.e / r.c;
    if (u >= 0 && u <= 1) k1 = gt / r.c;
  } else {
    const T den = r.a - T(2) * r.b + r.c;
    const T u = (r.c + r.e - r.b - r.d) / den;
    if (u >= 0 && u <= 1) {
      k0 = (gs - gt) / den;
      k1 = -k0;
    }
  }
  return {k0 * r.e0.x + k1 * r.e1.x, k0 * r.e0.y + k1 * r.e1.y, k0 * r.e0.z + k1 * r.e1.z};
}

template <typename T> P3<T> vert(const T* pos, int64_t N, int64_t v) { return {pos[v], pos[N + v], pos[2 * N + v]}; }

// etc.cu:780-862: candidate faces from the adjacency of the K nearest vertices, in order; the
// strictly closest is kept (the reference's de-duplication keeps first occurrences, which gives
// the same choice).  Returns the number of queries with no candidate face (id -1).
template <typename T>
int64_t nearest(int64_t N_vertex, int64_t N_face, int64_t P, int64_t K, int64_t N_adj, const int32_t* head,
                const int32_t* list, const int32_t* faces, const T* vpos, const T* q, const int64_t* idxs,
                int64_t* tri_out, T* bary_out) {
  int64_t missing = 0;
  for (int64_t i = 0; i < P; ++i) {
    const P3<T> p{q[i], q[P + i], q[2 * P + i]};
    T best = std::numeric_limits<T>::max(), bs = 0, bt = 0;
    int64_t bf = -1;
    for (int64_t k = 0; k < K; ++k) {
      const int64_t v = idxs[i * K + k];
      if (v < 0 || v >= N_vertex) continue;
      const int64_t n = head[v], end = head[N_vertex + v], begin = end - n;
      if (n <= 0 || begin < 0 || end > N_adj) continue;
      for (int64_t j = begin; j < end; ++j) {
        const int64_t f = list[j];
        if (f < 0 || f >= N_face) continue;
        const int64_t a = faces[f], b = faces[N_face + f], c = faces[2 * N_face + f];
        if (a < 0 || a >= N_vertex || b < 0 || b >= N_vertex || c < 0 || c >= N_vertex) continue;
        T s, t;
        const P3<T> cp = closest(vert(vpos, N_vertex, a), vert(vpos, N_vertex, b), vert(vpos, N_vertex, c), p, s, t);
        const P3<T> dv = sub(cp, p);
        const T d2 = dot(dv, dv);
        if (d2 < best) {
          best = d2;
          bf = f;
          bs = s;
          bt = t;
        }
      }
    }
    missing += bf < 0;
    tri_out[i] = bf;
    bary_out[i] = bf < 0 ? T(0) : T(1) - bs - bt;  // etc.cu:858-860 (coordinate order after the fix)
    bary_out[P + i] = bs;
    bary_out[2 * P + i] = bt;
  }
  return missing;
}

// Lat-long bilinear lookup of a unit direction, etc.cu:527-583 with the reference's config.h
// switches: LEFT_TOP_AS_ORIGIN (v flipped) and FIX_ENVMAP_SEAM (columns wrap, rows clamp); writes
// channel c of the sample to out[c * stride].
template <typename T> void sample_dir(T x, T y, T z, int H, int W, int C, const T* env, T* out, int64_t stride) {
  const T pi = T(3.141592653589793238462643383279502884L);
  T phi = std::atan2(z, x);
  if (phi < 0) phi += 2 * pi;
  if (y < -1) y = -1;
  else if (y > 1) y = 1;
  const T theta = std::asin(y);
  const T u = phi / (2 * pi);
  const T v = T(1) - (theta / pi + T(0.5));
  const T pu = u * W, pv = v * H;
  int x0 = (int)std::floor(pu - T(0.5)), y0 = (int)std::floor(pv - T(0.5));
  int x1 = x0 + 1, y1 = y0 + 1;
  const T kx = pu - T(x0) - T(0.5), ky = pv - T(y0) - T(0.5);
  auto cl = [](int a, int n) { return a < 0 ? 0 : (a >= n ? n - 1 : a); };
  auto wrap = [](int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); };
  x0 = wrap(x0, W);
  x1 = wrap(x1, W);
  y0 = cl(y0, H);
  y1 = cl(y1, H);
  for (int c = 0; c < C; ++c) {
    const T v00 = env[((int64_t)c * H + y0) * W + x0], v01 = env[((int64_t)c * H + y0) * W + x1];
    const T v10 = env[((int64_t)c * H + y1) * W + x0], v11 = env[((int64_t)c * H + y1) * W + x1];
    out[c * stride] = (1 - ky) * ((1 - kx) * v00 + kx * v01) + ky * ((1 - kx) * v10 + kx * v11);
  }
}

}  // namespace

extern "C" {

// etc.cu:707-738
void des_oracle_uv_of_triangle_f64(int64_t P, const double* tri, const double* q, double* out) {
  for (int64_t i = 0; i < P; ++i) {
    const double* T = tri + 9 * i;
    double s, t;
    closest<double>({T[0], T[1], T[2]}, {T[3], T[4], T[5]}, {T[6], T[7], T[8]}, {q[3 * i], q[3 * i + 1], q[3 * i + 2]}, s,
                    t);
    out[3 * i] = 1 - s - t;
    out[3 * i + 1] = s;
    out[3 * i + 2] = t;
  }
}

// etc.cu:741-777
void des_oracle_uv_of_triangle_backward_f64(int64_t P, const double* tri, const double* q, const double* g,
                                            double* gq) {
  for (int64_t i = 0; i < P; ++i) {
    const double* T = tri + 9 * i;
    const P3<double> r = closest_adjoint<double>({T[0], T[1], T[2]}, {T[3], T[4], T[5]}, {T[6], T[7], T[8]},
                                                 {q[3 * i], q[3 * i + 1], q[3 * i + 2]}, g[3 * i + 1] - g[3 * i],
                                                 g[3 * i + 2] - g[3 * i]);
    gq[3 * i] = r.x;
    gq[3 * i + 1] = r.y;
    gq[3 * i + 2] = r.z;
  }
}

int64_t des_oracle_nearest_mesh_points_f64(int64_t N_vertex, int64_t N_face, int64_t P, int64_t K, int64_t N_adj,
                                           const int32_t* head, const int32_t* list, const int32_t* faces,
                                           const double* vpos, const double* q, const int64_t* idxs, int64_t* tri,
                                           double* bary) {
  return nearest<double>(N_vertex, N_face, P, K, N_adj, head, list, faces, vpos, q, idxs, tri, bary);
}

int64_t des_oracle_nearest_mesh_points_f32(int64_t N_vertex, int64_t N_face, int64_t P, int64_t K, int64_t N_adj,
                                           const int32_t* head, const int32_t* list, const int32_t* faces,
                                           const float* vpos, const float* q, const int64_t* idxs, int64_t* tri,
                                           float* bary) {
  return nearest<float>(N_vertex, N_face, P, K, N_adj, head, list, faces, vpos, q, idxs, tri, bary);
}

// etc.cu:867-935, with grad_barycentric_coord as the incoming gradient
void des_oracle_nearest_mesh_points_backward_f64(int64_t N_vertex, int64_t N_face, int64_t P, const int32_t* faces,
                                                 const double* vpos, const double* q, const int64_t* tri,
                                                 const double* g, double* gq) {
  for (int64_t i = 0; i < P; ++i) {
    P3<double> r{0, 0, 0};
    const int64_t f = tri[i];
    if (f >= 0 && f < N_face) {
      const int64_t a = faces[f], b = faces[N_face + f], c = faces[2 * N_face + f];
      r = closest_adjoint<double>(vert(vpos, N_vertex, a), vert(vpos, N_vertex, b), vert(vpos, N_vertex, c),
                                  {q[i], q[P + i], q[2 * P + i]}, g[P + i] - g[i], g[2 * P + i] - g[i]);
    }
    gq[i] = r.x;
    gq[P + i] = r.y;
    gq[2 * P + i] = r.z;
  }
}

// etc.cu:1021-1040
void des_oracle_extract_bitfield(int64_t N, int64_t N_bit, int64_t i_start, int64_t i_end, const uint32_t* words,
                                 float* out) {
  for (int64_t i = i_start; i < i_end; ++i)
    for (int64_t k = 0; k < N_bit; ++k)
      out[(i - i_start) * N_bit + k] = ((words[(k / 32) * N + i] >> (k % 32)) & 1u) ? 1.f : 0.f;
}

// etc.cu:687-705: query directions [3 x P] (normalised here), env [C x H x W] -> out [C x P]
void des_oracle_sample_envmap_f64(int64_t P, int H, int W, int C, const double* q, const double* env, double* out) {
  for (int64_t i = 0; i < P; ++i) {
    double x = q[i], y = q[P + i], z = q[2 * P + i];
    const double L = std::sqrt(x * x + y * y + z * z);
    sample_dir<double>(x / L, y / L, z / L, H, W, C, env, out + i, P);
  }
}

}  // extern "C"
