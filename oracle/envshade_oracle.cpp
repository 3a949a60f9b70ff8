// CPU oracle for the brute-force environment-map shading sum and its adjoint.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, in plain C++ on the host, the
// arithmetic of the reference extension zjumsj/diff_envshade (bruteforce_shader.cu).
// It is the checker for the CUDA product path and the timed CPU baseline; the
// product package never links or calls it.
//
// Every function names the reference lines it follows.  The per-(point, texel)
// expressions keep the reference's operation order so that the FP32 instantiation
// is a faithful transcription; the FP64 instantiation is the high-precision oracle.
//
// Texel geometry: the reference evaluates the texel direction with CUDA's sincosf
// and the solid angle with the __sinf intrinsic (bruteforce_shader.cu:124-147).
// Those are not reproducible bit-for-bit on a host, so every entry point takes the
// rotated texel table (x, y, z, d_omega per texel) as an input: tests pass the table
// the GPU built with the reference's own expressions, or the FP64 table made by
// des_oracle_texel_table_f64 below (exact trigonometry).
//
// Threading: std::thread over contiguous point blocks.  The env-map gradient is
// accumulated per thread and summed in thread order, so results are deterministic
// for a fixed thread count.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>
#include <algorithm>

namespace {

enum : unsigned {
  kDiffuse = 1u,   // Lambert term on
  kSpecular = 2u,  // GGX term on
  kClamp = 4u,     // backface clamp: n.v <= 0 -> point contributes nothing (bruteforce_shader.cu:1111)
  kWhite = 8u,     // "2" entry points: white diffuse output + its incoming gradient (bruteforce_shader.cu:1554)
  kV1Order = 16u,  // v1/clamp/diffuse-only entry points: v1 operation order of the diffuse term
};

template <typename T> struct V3 { T x, y, z; };
template <typename T> inline T dot3(const V3<T>& a, const V3<T>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> inline V3<T> add3(const V3<T>& a, const V3<T>& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }

template <typename T> constexpr T kPi() { return T(3.141592653589793238462643383279502884L); }
template <typename T> constexpr T kF0() { return T(0.04); }    // bruteforce_shader.cu:30
template <typename T> constexpr T kThres() { return T(1e-9f); } // bruteforce_shader.cu:31 (a float constant)

// __saturatef semantics: clamp to [0,1], NaN -> 0.
template <typename T> inline T saturate(T x) { return (x > T(0)) ? ((x < T(1)) ? x : T(1)) : T(0); }
// fmaxf semantics: a NaN operand yields the other operand.
template <typename T> inline T fmax_(T a, T b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a > b ? a : b)); }

// bruteforce_shader.cu:53-61
template <typename T> inline V3<T> normalize3(const V3<T>& a) {
  T L = std::sqrt(dot3(a, a));
  return {a.x / L, a.y / L, a.z / L};
}
// bruteforce_shader.cu:63-71
template <typename T> inline V3<T> grad_normalize3(const V3<T>& v, const V3<T>& g) {
  T v2 = dot3(v, v);
  T v15 = std::sqrt(v2) * v2;
  T gx = g.x * (v.y * v.y + v.z * v.z) - g.y * (v.x * v.y) - g.z * (v.x * v.z);
  T gy = -g.x * (v.x * v.y) + g.y * (v.x * v.x + v.z * v.z) - g.z * (v.y * v.z);
  T gz = -g.x * (v.x * v.z) - g.y * (v.y * v.z) + g.z * (v.x * v.x + v.y * v.y);
  return {gx / v15, gy / v15, gz / v15};
}
// bruteforce_shader.cu:49-51
template <typename T> inline T grad_saturate(T x) { return (x >= T(0) && x <= T(1)) ? T(1) : T(0); }
// bruteforce_shader.cu:149-153
template <typename T> inline T fresnel(T R0, T c) {
  T a = T(1) - saturate(c);
  T a2 = a * a;
  return (a2 * a2 * a) * (T(1) - R0) + R0;
}
// bruteforce_shader.cu:155-159
template <typename T> inline T grad_fresnel(T R0, T c, T g) {
  T a = T(1) - saturate(c);
  T a2 = a * a;
  return T(5) * (R0 - T(1)) * g * (a2 * a2) * grad_saturate(c);
}
// bruteforce_shader.cu:161-171 (Schlick-Smith with the n.l cosine folded in)
template <typename T> inline T g1_robust(const V3<T>& l, const V3<T>& v, const V3<T>& n, T alpha) {
  T dvn = std::max(dot3(v, n), T(0));
  T dln = std::max(dot3(l, n), T(0));
  T a = dln / (dln * (T(1) - alpha) + alpha);
  return a / (dvn * (T(1) - alpha) + alpha);
}
// bruteforce_shader.cu:173-201 (the gradient w.r.t. l is not needed: l carries no gradient)
template <typename T> inline void grad_g1_robust(const V3<T>& l, const V3<T>& v, const V3<T>& n, T alpha, T grad,
                                                 V3<T>& gv, V3<T>& gn, T& galpha) {
  T dvn = std::max(dot3(v, n), T(0));
  T dln = std::max(dot3(l, n), T(0));
  T a_det = dln * (T(1) - alpha) + alpha;
  T a = dln / a_det;
  T b = dvn * (T(1) - alpha) + alpha;
  T grad_a = grad / b;
  T grad_b = -grad * a / (b * b);
  T gdln = grad_a * alpha / (a_det * a_det);
  if (dln > T(0)) { gn.x += gdln * l.x; gn.y += gdln * l.y; gn.z += gdln * l.z; }
  galpha += grad_a * dln * (dln - T(1)) / (a_det * a_det);
  T gdvn = grad_b * (T(1) - alpha);
  if (dvn > T(0)) {
    gv.x += gdvn * n.x; gv.y += gdvn * n.y; gv.z += gdvn * n.z;
    gn.x += gdvn * v.x; gn.y += gdvn * v.y; gn.z += gdvn * v.z;
  }
  galpha += grad_b * (T(1) - dvn);
}
// bruteforce_shader.cu:203-210 (GGX NDF with the 1e-9 floor)
template <typename T> inline T ndf1(const V3<T>& n, const V3<T>& h, T alpha2) {
  T nh = dot3(n, h);
  T t = nh * nh * (alpha2 - T(1)) + T(1);
  return alpha2 / fmax_(kPi<T>() * t * t, kThres<T>());
}
// bruteforce_shader.cu:212-227
template <typename T> inline void grad_ndf1(const V3<T>& n, const V3<T>& h, T alpha2, T grad,
                                            V3<T>& gn, V3<T>& gh, T& galpha2) {
  T nh = dot3(n, h);
  T t = nh * nh * (alpha2 - T(1)) + T(1);
  T t2 = kPi<T>() * t * t;
  galpha2 += grad / fmax_(t2, kThres<T>());
  if (t2 > kThres<T>()) {
    T gt = (T(-2) * alpha2 * grad) / (t2 * t);
    galpha2 += nh * nh * gt;
    T gnh = T(2) * gt * (alpha2 - T(1)) * nh;
    gn.x += gnh * h.x; gn.y += gnh * h.y; gn.z += gnh * h.z;
    gh.x += gnh * n.x; gh.y += gnh * n.y; gh.z += gnh * n.z;
  }
}

template <typename T> struct Args {
  int64_t P; int H, W;
  const T *normal, *view, *albedo, *spec, *rough, *env, *table;
  int N_face, N_vertex;
  const int32_t* faces; const int64_t* tri; const T* bary; const uint32_t* vis;
  unsigned flags;
};

template <typename T> struct PointCtx {
  V3<T> n, v; T a[3], s[3]; T r, alpha0, alpha1;
  bool has_vis; int v0, v1, v2; T c0, c1, c2; bool active;
};

template <typename T> inline PointCtx<T> load_point(const Args<T>& A, int64_t p) {
  PointCtx<T> q{};
  q.n = {A.normal[3 * p], A.normal[3 * p + 1], A.normal[3 * p + 2]};
  const bool spec = A.flags & kSpecular, clamp = A.flags & kClamp;
  if ((spec || clamp) && A.view) q.v = {A.view[3 * p], A.view[3 * p + 1], A.view[3 * p + 2]};
  for (int c = 0; c < 3; ++c) {
    q.a[c] = A.albedo ? A.albedo[3 * p + c] : T(0);
    q.s[c] = (spec && A.spec) ? A.spec[3 * p + c] : T(0);
  }
  if (spec) {
    q.r = A.rough[p];
    // bruteforce_shader.cu:1601-1604
    q.alpha0 = q.r * q.r; q.alpha0 = q.alpha0 * q.alpha0;
    q.alpha1 = q.r + T(1); q.alpha1 = (q.alpha1 * q.alpha1) / T(8);
  }
  q.has_vis = A.vis != nullptr;
  if (q.has_vis) {
    // bruteforce_shader.cu:2145-2151
    int64_t f = A.tri[p];
    q.v0 = A.faces[f]; q.v1 = A.faces[f + A.N_face]; q.v2 = A.faces[f + 2 * (int64_t)A.N_face];
    q.c0 = A.bary[p]; q.c1 = A.bary[p + A.P]; q.c2 = A.bary[p + 2 * A.P];
  }
  // bruteforce_shader.cu:1111 (clamp kernels skip the whole texel loop when n.v <= 0)
  q.active = clamp ? (dot3(q.n, q.v) > T(0)) : true;
  return q;
}

// bruteforce_shader.cu:2180-2189: bit (t % 32) of visibility[t / 32][vertex], interpolated barycentrically.
template <typename T> inline T vis_of(const Args<T>& A, const PointCtx<T>& q, int t) {
  if (!q.has_vis) return T(1);
  int slot = t >> 5; uint32_t bit = 1u << (t & 31);
  uint32_t p0 = A.vis[(int64_t)slot * A.N_vertex + q.v0];
  uint32_t p1 = A.vis[(int64_t)slot * A.N_vertex + q.v1];
  uint32_t p2 = A.vis[(int64_t)slot * A.N_vertex + q.v2];
  T b0 = (p0 & bit) ? T(1) : T(0), b1 = (p1 & bit) ? T(1) : T(0), b2 = (p2 & bit) ? T(1) : T(0);
  return b0 * q.c0 + b1 * q.c1 + b2 * q.c2;
}

// Forward sum for one point.
// v1 order:      bruteforce_shader.cu:638-663 (specular v1), 1111-1160 (clamp), 289-309 (diffuse-only)
// "2" order:     bruteforce_shader.cu:1639-1690 (no visibility), 2171-2236 (visibility)
template <typename T> void forward_point(const Args<T>& A, int64_t p, T* shading, T* white) {
  PointCtx<T> q = load_point(A, p);
  T sh[3] = {0, 0, 0}, wh[3] = {0, 0, 0};
  const int HW = A.H * A.W;
  const bool diff = A.flags & kDiffuse, spec = A.flags & kSpecular, v1 = A.flags & kV1Order;
  if (q.active) {
    for (int t = 0; t < HW; ++t) {
      T vis = vis_of(A, q, t);
      V3<T> l = {A.table[4 * t], A.table[4 * t + 1], A.table[4 * t + 2]};
      T dw = A.table[4 * t + 3];
      T L[3] = {A.env[t], A.env[HW + t], A.env[2 * HW + t]};
      if (diff) {
        T cs = dot3(l, q.n);
        if (cs > T(0)) {
          for (int c = 0; c < 3; ++c) {
            if (v1) {
              sh[c] += L[c] * q.a[c] * (cs / kPi<T>()) * dw;
            } else {
              T tmp = L[c] * (cs / kPi<T>()) * dw;
              if (q.has_vis) tmp *= vis;
              wh[c] += tmp;
              sh[c] += tmp * q.a[c];
            }
          }
        }
      }
      if (spec) {
        V3<T> h = normalize3(add3(l, q.v));
        T ch = dot3(l, h);
        T F = fresnel(kF0<T>(), ch);
        T G = g1_robust(l, q.v, q.n, q.alpha1);
        T D = ndf1(q.n, h, q.alpha0);
        T tmp = (F * G * D) / T(4);
        if (tmp > T(0)) {
          for (int c = 0; c < 3; ++c) {
            if (q.has_vis) sh[c] += L[c] * q.s[c] * (tmp * dw * vis);
            else sh[c] += L[c] * q.s[c] * (tmp * dw);
          }
        }
      }
    }
  }
  for (int c = 0; c < 3; ++c) {
    shading[3 * p + c] = sh[c];
    if (white) white[3 * p + c] = wh[c];
  }
}

// Point gradients for one point.
// v1:   bruteforce_shader.cu:770-887 (Backward), 1294 (clamp gate)
// "2":  bruteforce_shader.cu:1851-1925 (Backward2), 2380-2505 (visibility)
// Env-map gradient contributions are accumulated into genv (3*HW, planar):
// v1:   bruteforce_shader.cu:958-1036;  "2": 2000-2064, 2596-2681.
template <typename T> void backward_point(const Args<T>& A, int64_t p, const T* gsh, const T* gwh,
                                          T* gn_out, T* gv_out, T* ga_out, T* gs_out, T* gr_out, T* genv) {
  PointCtx<T> q = load_point(A, p);
  const int HW = A.H * A.W;
  const bool diff = A.flags & kDiffuse, spec = A.flags & kSpecular, v1 = A.flags & kV1Order;
  T g[3] = {gsh[3 * p], gsh[3 * p + 1], gsh[3 * p + 2]};
  T gw[3] = {0, 0, 0};
  if (gwh) for (int c = 0; c < 3; ++c) gw[c] = gwh[3 * p + c];
  V3<T> gn = {0, 0, 0}, gv = {0, 0, 0};
  T ga[3] = {0, 0, 0}, gs[3] = {0, 0, 0};
  T galpha0 = 0, galpha1 = 0;
  // env-gradient weights, bruteforce_shader.cu:2585-2588 ("2") and 958-966 (v1)
  T dgrad[3], sgrad[3];
  for (int c = 0; c < 3; ++c) {
    dgrad[c] = v1 ? g[c] * q.a[c] : g[c] * q.a[c] + gw[c];
    sgrad[c] = g[c] * q.s[c];
  }
  if (q.active) {
    for (int t = 0; t < HW; ++t) {
      T vis = vis_of(A, q, t);
      V3<T> l = {A.table[4 * t], A.table[4 * t + 1], A.table[4 * t + 2]};
      T dw = A.table[4 * t + 3];
      T L[3] = {A.env[t], A.env[HW + t], A.env[2 * HW + t]};
      T e[3] = {0, 0, 0};
      if (diff) {
        T cs = dot3(l, q.n);
        T gdotn = 0;
        if (cs > T(0)) {
          for (int c = 0; c < 3; ++c) {
            T I = L[c];
            if (q.has_vis) I *= vis;
            ga[c] += g[c] * I * (cs / kPi<T>()) * dw;
            if (v1) gdotn += g[c] * I * q.a[c] * dw / kPi<T>();
            else gdotn += (g[c] * q.a[c] + gw[c]) * I * dw / kPi<T>();
            T ev = v1 ? g[c] * q.a[c] * (cs / kPi<T>()) * dw : dgrad[c] * (cs / kPi<T>()) * dw;
            if (q.has_vis) ev *= vis;
            e[c] += ev;
          }
          gn.x += gdotn * l.x; gn.y += gdotn * l.y; gn.z += gdotn * l.z;
        }
      }
      if (spec) {
        V3<T> hb = add3(l, q.v);
        V3<T> h = normalize3(hb);
        T ch = dot3(l, h);
        T F = fresnel(kF0<T>(), ch);
        T G = g1_robust(l, q.v, q.n, q.alpha1);
        T D = ndf1(q.n, h, q.alpha0);
        T tmp = (F * G * D) / T(4);
        if (tmp > T(0)) {
          T gtmp = 0;
          for (int c = 0; c < 3; ++c) {
            T I = L[c];
            if (q.has_vis) I *= vis;
            gs[c] += g[c] * I * (tmp * dw);
            gtmp += g[c] * I * q.s[c] * dw;
            T ev = sgrad[c] * tmp * dw;
            if (q.has_vis) ev *= vis;
            e[c] += ev;
          }
          T gF = gtmp * (G * D) / T(4);
          T gG = gtmp * (F * D) / T(4);
          T gD = gtmp * (F * G) / T(4);
          T gch = grad_fresnel(kF0<T>(), ch, gF);
          V3<T> gh = {gch * l.x, gch * l.y, gch * l.z};
          V3<T> gvv = {0, 0, 0}, gnn = {0, 0, 0};
          grad_g1_robust(l, q.v, q.n, q.alpha1, gG, gvv, gnn, galpha1);
          grad_ndf1(q.n, h, q.alpha0, gD, gnn, gh, galpha0);
          gh = grad_normalize3(hb, gh);
          gvv = add3(gvv, gh);
          gv = add3(gv, gvv);
          gn = add3(gn, gnn);
        }
      }
      if (genv) for (int c = 0; c < 3; ++c) genv[c * HW + t] += e[c];
    }
  }
  gn_out[3 * p] = gn.x; gn_out[3 * p + 1] = gn.y; gn_out[3 * p + 2] = gn.z;
  for (int c = 0; c < 3; ++c) {
    if (ga_out) ga_out[3 * p + c] = diff ? ga[c] : T(0);
    if (gs_out) gs_out[3 * p + c] = spec ? gs[c] : T(0);
  }
  if (gv_out) { gv_out[3 * p] = spec ? gv.x : T(0); gv_out[3 * p + 1] = spec ? gv.y : T(0); gv_out[3 * p + 2] = spec ? gv.z : T(0); }
  if (gr_out) {
    // bruteforce_shader.cu:2501-2502
    T gr = galpha0 * T(4) * q.r * q.r * q.r;
    gr += galpha1 * (T(1) + q.r) / T(4);
    gr_out[p] = spec ? gr : T(0);
  }
}

template <typename F> void parallel_points(int64_t P, int nthreads, F&& fn) {
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  nthreads = (int)std::max<int64_t>(1, std::min<int64_t>(nthreads, P));
  std::vector<std::thread> th;
  int64_t chunk = (P + nthreads - 1) / nthreads;
  for (int i = 0; i < nthreads; ++i) {
    int64_t b = i * chunk, e = std::min(P, b + chunk);
    if (b >= e) break;
    th.emplace_back([=, &fn]() { fn(i, b, e); });
  }
  for (auto& x : th) x.join();
}

template <typename T> Args<T> make_args(int64_t P, int H, int W, const T* normal, const T* view, const T* albedo,
                                        const T* spec, const T* rough, const T* env, const T* table, int N_face,
                                        int N_vertex, const int32_t* faces, const int64_t* tri, const T* bary,
                                        const uint32_t* vis, unsigned flags) {
  Args<T> A;
  A.P = P; A.H = H; A.W = W; A.normal = normal; A.view = view; A.albedo = albedo; A.spec = spec; A.rough = rough;
  A.env = env; A.table = table; A.N_face = N_face; A.N_vertex = N_vertex; A.faces = faces; A.tri = tri;
  A.bary = bary; A.vis = vis; A.flags = flags;
  return A;
}

template <typename T> int forward_impl(const Args<T>& A, T* shading, T* white, int nthreads) {
  if (A.P < 0 || A.H <= 0 || A.W <= 0) return 1;
  parallel_points(A.P, nthreads, [&](int, int64_t b, int64_t e) {
    for (int64_t p = b; p < e; ++p) forward_point(A, p, shading, white);
  });
  return 0;
}

template <typename T> int backward_impl(const Args<T>& A, const T* gsh, const T* gwh, T* gn, T* gv, T* ga, T* gs,
                                        T* gr, T* genv, int nthreads) {
  if (A.P < 0 || A.H <= 0 || A.W <= 0) return 1;
  const int HW = A.H * A.W;
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  int nt = (int)std::max<int64_t>(1, std::min<int64_t>(nthreads, A.P));
  std::vector<std::vector<T>> part(nt, std::vector<T>(genv ? 3 * HW : 0, T(0)));
  parallel_points(A.P, nt, [&](int i, int64_t b, int64_t e) {
    T* ge = genv ? part[i].data() : nullptr;
    for (int64_t p = b; p < e; ++p) backward_point(A, p, gsh, gwh, gn, gv, ga, gs, gr, ge);
  });
  if (genv) {
    for (int k = 0; k < 3 * HW; ++k) {
      T acc = 0;
      for (int i = 0; i < nt; ++i) acc += part[i][k];
      genv[k] = acc;
    }
  }
  return 0;
}

}  // namespace

extern "C" {

// FP64 texel table, bruteforce_shader.cu:124-147 with the LEFT_TOP_AS_ORIGIN row flip
// (config.h:11, bruteforce_shader.cu:2176-2178) and the rotation l' = R l (2194-2197).
// out: H*W*4 doubles (x, y, z, d_omega) in memory (row-major, row 0 = top) texel order.
void des_oracle_texel_table_f64(int H, int W, const double* R, double* out) {
  const double pi = kPi<double>();
  for (int t = 0; t < H * W; ++t) {
    int ix = t % W, iy = H - 1 - t / W;
    double v = (iy + 0.5) / H, u = (ix + 0.5) / W;
    double phi = u * pi * 2, theta = (v - 0.5) * pi;
    double lx = std::cos(theta) * std::cos(phi), ly = std::sin(theta), lz = std::cos(theta) * std::sin(phi);
    double dphi = 2 * pi / W, dth = pi / H;
    double dw = (std::sin(dth * (iy + 1) - pi * 0.5) - std::sin(dth * iy - pi * 0.5)) * dphi;
    out[4 * t + 0] = R[0] * lx + R[1] * ly + R[2] * lz;
    out[4 * t + 1] = R[3] * lx + R[4] * ly + R[5] * lz;
    out[4 * t + 2] = R[6] * lx + R[7] * ly + R[8] * lz;
    out[4 * t + 3] = dw;
  }
}

#define DES_ORACLE_API(T, SUF)                                                                                     \
  int des_oracle_forward_##SUF(int64_t P, int H, int W, const T* normal, const T* view, const T* albedo,          \
                               const T* spec, const T* rough, const T* env, const T* table, int N_face,            \
                               int N_vertex, const int32_t* faces, const int64_t* tri, const T* bary,              \
                               const uint32_t* vis, unsigned flags, T* shading, T* white, int nthreads) {          \
    Args<T> A = make_args<T>(P, H, W, normal, view, albedo, spec, rough, env, table, N_face, N_vertex, faces, tri, \
                             bary, vis, flags);                                                                    \
    return forward_impl(A, shading, white, nthreads);                                                              \
  }                                                                                                                \
  int des_oracle_backward_##SUF(int64_t P, int H, int W, const T* normal, const T* view, const T* albedo,         \
                                const T* spec, const T* rough, const T* env, const T* table, int N_face,           \
                                int N_vertex, const int32_t* faces, const int64_t* tri, const T* bary,             \
                                const uint32_t* vis, unsigned flags, const T* grad_shading, const T* grad_white,   \
                                T* g_normal, T* g_view, T* g_albedo, T* g_spec, T* g_rough, T* g_env,              \
                                int nthreads) {                                                                    \
    Args<T> A = make_args<T>(P, H, W, normal, view, albedo, spec, rough, env, table, N_face, N_vertex, faces, tri, \
                             bary, vis, flags);                                                                    \
    return backward_impl(A, grad_shading, grad_white, g_normal, g_view, g_albedo, g_spec, g_rough, g_env,          \
                         nthreads);                                                                                \
  }

DES_ORACLE_API(double, f64)
DES_ORACLE_API(float, f32)

int des_oracle_abi_version(void) { return 1; }

}  // extern "C"
