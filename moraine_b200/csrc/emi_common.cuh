// Device building blocks shared by the EMI kernels: complex arithmetic over a real type
// T (float or double), block reductions, the Sturm count, the pivoted tridiagonal solve,
// and the common tail of EMI (real tridiagonal scaling, smallest eigenvalue by
// multisection, inverse iteration, back-transformation, normalisation to the reference
// image, temporal coherence).
#pragma once

#include <cfloat>

#include "common.cuh"

namespace mr {
namespace emi {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

template <typename T> struct C2;
template <> struct C2<float> { using type = float2; };
template <> struct C2<double> { using type = double2; };

template <typename T> struct Lim;
template <> struct Lim<float> {
  static __device__ __forceinline__ float eps() { return FLT_EPSILON; }
  static __device__ __forceinline__ float tiny() { return FLT_MIN; }
  static __device__ __forceinline__ float huge() { return FLT_MAX; }
};
template <> struct Lim<double> {
  static __device__ __forceinline__ double eps() { return DBL_EPSILON; }
  static __device__ __forceinline__ double tiny() { return DBL_MIN; }
  static __device__ __forceinline__ double huge() { return DBL_MAX; }
};

template <typename T> __device__ __forceinline__ typename C2<T>::type mk(T x, T y) {
  typename C2<T>::type c; c.x = x; c.y = y; return c;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }
// a * b
template <typename C> __device__ __forceinline__ C cmul_t(C a, C b) {
  C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc_t(C a, C b) {
  C r; r.x = a.x * b.x + a.y * b.y; r.y = a.y * b.x - a.x * b.y; return r;
}

struct Red {
  double v[kWarps];
  double w[kWarps];
  int i[kWarps];
  double lam;
  int flag;
};

__device__ __forceinline__ double block_sum(double x, Red& r) {
  x = warp_sum(x);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) r.v[threadIdx.x >> 5] = x;
  __syncthreads();
  double t = 0;
#pragma unroll
  for (int k = 0; k < kWarps; ++k) t += r.v[k];
  return t;
}

__device__ __forceinline__ double2 block_sum2(double2 x, Red& r) {
  x.x = warp_sum(x.x);
  x.y = warp_sum(x.y);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) { r.v[threadIdx.x >> 5] = x.x; r.w[threadIdx.x >> 5] = x.y; }
  __syncthreads();
  double2 t = make_double2(0, 0);
#pragma unroll
  for (int k = 0; k < kWarps; ++k) { t.x += r.v[k]; t.y += r.w[k]; }
  return t;
}

__device__ __forceinline__ float sturm_div(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double sturm_div(double a, double b) { return a / b; }

// Number of eigenvalues of the real symmetric tridiagonal (d, b^2) below sigma. In FP32
// the quotient is the fast approximate division (a few ulp): the count then belongs to a
// tridiagonal perturbed at that level, which the bisection tolerates.
template <typename T>
__device__ __forceinline__ int sturm_count(const T* d, const T* b2, int n, T sigma, T pivmin) {
  int c = 0;
  T q = d[0] - sigma;
  if (fabs(q) < pivmin) q = -pivmin;
  c += (q < 0);
  for (int i = 1; i < n; ++i) {
    q = (d[i] - sigma) - sturm_div(b2[i - 1], q);
    if (fabs(q) < pivmin) q = -pivmin;
    c += (q < 0);
  }
  return c;
}

// Solve (R - lambda I) y = y in place by elimination with row interchanges; R has
// diagonal d and off-diagonal b. dd, du, dl: work arrays of length n.
template <typename T>
__device__ inline void tridiag_solve(const T* d, const T* b, int n, T lambda, T tiny, T* y, T* dd, T* du, T* dl) {
  for (int i = 0; i < n; ++i) {
    dd[i] = d[i] - lambda;
    if (i < n - 1) { du[i] = b[i]; dl[i] = b[i]; }
  }
  // dl[i] on exit holds the second super-diagonal of row i (0 when no interchange)
  for (int i = 0; i < n - 1; ++i) {
    const T sub = dl[i];
    if (fabs(dd[i]) >= fabs(sub)) {
      if (dd[i] == T(0)) dd[i] = tiny;
      const T f = sub / dd[i];
      dd[i + 1] -= f * du[i];
      y[i + 1] -= f * y[i];
      dl[i] = T(0);
    } else {
      const T f = dd[i] / sub;
      dd[i] = sub;
      const T t = dd[i + 1];
      dd[i + 1] = du[i] - f * t;
      if (i < n - 2) {
        dl[i] = du[i + 1];
        du[i + 1] = -f * dl[i];
      } else {
        dl[i] = T(0);
      }
      du[i] = t;
      const T ty = y[i];
      y[i] = y[i + 1];
      y[i + 1] = ty - f * y[i + 1];
    }
  }
  if (dd[n - 1] == T(0)) dd[n - 1] = tiny;
  y[n - 1] /= dd[n - 1];
  if (n > 1) y[n - 2] = (y[n - 2] - du[n - 2] * y[n - 1]) / dd[n - 2];
  for (int i = n - 3; i >= 0; --i) y[i] = (y[i] - du[i] * y[i + 1] - dl[i] * y[i + 2]) / dd[i];
}

// Vectors of the EMI tail (each of length >= n).
template <typename T>
struct TailVecs {
  using C = typename C2<T>::type;
  const T* d;    // diagonal of T
  const C* e;    // sub-diagonal of T (complex)
  const T* tau;  // reflector scalars (0: identity)
  T* b;
  T* b2;
  T* y;
  T* w1;
  T* w2;
  T* w3;
  C* z;
  double2* phs;
};

// Tail of EMI for one point, executed by the whole CTA. T = Q^H M Q is Hermitian
// tridiagonal (d, e); reflector k is H_k = I - tau_k u_k u_k^H acting on indices k+1..n-1
// with u_k[i] = uk(k, i), i = 0..n-k-2. The eigenvalue search and the back-transformation
// run on warp 0.
template <typename T, class UK>
__device__ void tail(int n, int ref, const TailVecs<T>& v, UK uk, Red& red, bool singular, float2* __restrict__ ph,
                     float* __restrict__ quality, float* __restrict__ tcoh, const float2* __restrict__ c,
                     int64_t npairs) {
  using C = typename C2<T>::type;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
  if (tid < 32) {
    // real tridiagonal R = D^H T D (phases delta in z), by lane 0
    if (lane == 0) {
      C dl = mk<T>(1, 0);
      v.z[0] = dl;
      for (int k = 0; k + 1 < n; ++k) {
        const C ek = v.e[k];
        const T a = sqrt(ek.x * ek.x + ek.y * ek.y);
        v.b[k] = a;
        v.b2[k] = a * a;
        if (a > T(0)) dl = cmul_t(dl, mk<T>(ek.x / a, ek.y / a));
        v.z[k + 1] = dl;
      }
    }
    __syncwarp();
    // lambda_min by multisection (33 points per round)
    T lo = Lim<T>::huge(), hi = -Lim<T>::huge(), tnorm = 0;
    for (int i = 0; i < n; ++i) {
      const T r = (i > 0 ? v.b[i - 1] : T(0)) + (i + 1 < n ? v.b[i] : T(0));
      lo = fmin(lo, v.d[i] - r);
      hi = fmax(hi, v.d[i] + r);
      tnorm = fmax(tnorm, fabs(v.d[i]) + r);
    }
    const T eps = Lim<T>::eps();
    const T pivmin = fmax(Lim<T>::tiny(), eps * eps * tnorm * tnorm) + Lim<T>::tiny();
    const T pad = T(2) * eps * fmax(tnorm, Lim<T>::tiny()) + T(2) * pivmin;
    lo -= pad;
    hi += pad;
    for (int it = 0; it < 64; ++it) {
      const T width = hi - lo;
      if (!(width > T(2) * eps * fmax(fabs(lo), fabs(hi)) + T(4) * pivmin)) break;
      const T sg = lo + width * (T)(lane + 1) / T(33);
      const int cnt = sturm_count(v.d, v.b2, n, sg, pivmin);
      const unsigned ball = __ballot_sync(0xffffffffu, cnt >= 1);
      const int first = ball ? __ffs(ball) - 1 : 32;
      const T nlo = (first == 0) ? lo : lo + width * (T)first / T(33);
      const T nhi = (first == 32) ? hi : lo + width * (T)(first + 1) / T(33);
      lo = nlo;
      hi = nhi;
    }
    const T lam = T(0.5) * (lo + hi);
    if (lane == 0) {
      red.lam = (double)lam;
      for (int i = 0; i < n; ++i) v.y[i] = T(1) + T(0.5) * sin(T(1) + T(3.7) * i);
      const T tiny = eps * fmax(tnorm, Lim<T>::tiny());
      for (int it = 0; it < 3; ++it) {
        tridiag_solve(v.d, v.b, n, lam, tiny, v.y, v.w1, v.w2, v.w3);
        T s = 0;
        for (int i = 0; i < n; ++i) s = fmax(s, fabs(v.y[i]));
        if (!(s > T(0)) || !isfinite(s)) break;
        for (int i = 0; i < n; ++i) v.y[i] /= s;
      }
    }
    __syncwarp();
    // v = Q D y
    for (int i = lane; i < n; i += 32) {
      const C dl = v.z[i];
      const T yi = v.y[i];
      v.z[i] = mk<T>(dl.x * yi, dl.y * yi);
    }
    __syncwarp();
    for (int k = n - 3; k >= 0; --k) {
      const T tau = v.tau[k];
      if (tau == T(0)) continue;
      const int m = n - k - 1;
      C s = mk<T>(0, 0);
      for (int i = lane; i < m; i += 32) {  // u^H z
        const C ui = uk(k, i), zi = v.z[k + 1 + i];
        s.x += ui.x * zi.x + ui.y * zi.y;
        s.y += ui.x * zi.y - ui.y * zi.x;
      }
      s.x = warp_sum(s.x);
      s.y = warp_sum(s.y);
      for (int i = lane; i < m; i += 32) {
        const C t = cmul_t(uk(k, i), s);
        v.z[k + 1 + i].x -= tau * t.x;
        v.z[k + 1 + i].y -= tau * t.y;
      }
      __syncwarp();
    }
  }
  __syncthreads();
  // normalise to the reference image
  const C zr = v.z[ref];
  const float fnan = __int_as_float(0x7fffffff);
  for (int i = tid; i < n; i += nt) {
    const C w = cmulc_t(v.z[i], zr);
    const double wx = w.x, wy = w.y;
    const double a = sqrt(wx * wx + wy * wy);
    float2 o = make_float2((float)(wx / a), (float)(wy / a));
    if (singular) o = make_float2(fnan, fnan);
    ph[i] = o;
    v.phs[i] = make_double2(o.x, o.y);
  }
  if (tid == 0) *quality = singular ? fnan : (float)red.lam;
  __syncthreads();
  if (tcoh) {
    double2 t = make_double2(0, 0);
    // pair q = tid + nt * s walks the upper triangle row-major: (mm, jj) advanced by nt
    int mm = 0, jj = 1 + tid;
    while (jj >= n && mm < n - 1) { mm += 1; jj = jj - n + mm + 1; }
    for (int64_t q = tid; q < npairs; q += nt) {
      const int m0 = mm, j0 = jj;
      jj += nt;
      while (jj >= n && mm < n - 1) { mm += 1; jj = jj - n + mm + 1; }
      const float2 g = c[q];
      const double ga = sqrt((double)g.x * g.x + (double)g.y * g.y);
      const double2 gm = make_double2(g.x / ga, g.y / ga);
      const double2 w = cmul(gm, cmulc(v.phs[j0], v.phs[m0]));  // coh/|coh| conj(ph_m) ph_j
      t.x += w.x;
      t.y += w.y;
    }
    t = block_sum2(t, red);
    if (tid == 0) *tcoh = (float)(sqrt(t.x * t.x + t.y * t.y) / (double)npairs);
  }
  __syncthreads();
}

}  // namespace emi
}  // namespace mr
