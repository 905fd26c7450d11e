// EMI for N <= 128 (moraine/pl.py:46-77: M = inv(|Gamma|) o Gamma, its smallest eigenpair,
// phases referred to image `ref`, fused temporal coherence), in sub-batches of points.
//
// Kernels, each at its own occupancy (the register-bound inverse is not held back by the
// shared memory of the reduction, and the serial O(N) tails of many points overlap on an SM):
//   inverse_kernel<T, NB>  inv(|Gamma|) by Gauss-Jordan with partial pivoting in registers
//                          (gj_tile): the padded 16NB x 16NB matrix on a 16 x 16 thread grid,
//                          rows never swapped, one barrier per step; the result stored
//                          upper-packed in the workspace. FP32 and FP64 EMI, and the FP64
//                          recomputation of routed points.
//   sweep_kernel<NB>       inv(|Gamma|) in FP64 for the refined EMI: the symmetric sweep, two
//                          pivots per barrier, only the lower triangle held.
//   reduce_kernel<T, TA>   M in shared memory as a packed lower triangle, Householder
//                          reduction to a real tridiagonal (tridiag_packed) -> workspace (d, e,
//                          tau, reflectors).
//   tail_kernel<T, TA>     one warp per point: smallest eigenvalue by Sturm multisection,
//                          inverse iteration, back-transformation, normalisation, temporal
//                          coherence.
//   tail_refine_kernel     the refined EMI's tail: FP32 eigenpair of the tridiagonal, one FP64
//                          Newton correction and an FP64 error bound that routes the points
//                          it does not certify to FP64.
//   route_kernel           collects the points to recompute in FP64 over all sub-batches.
#include <algorithm>
#include <atomic>

#include "emi_common.cuh"

namespace mr {
namespace emi {

// Largest sub-batch a caller asked for (mr_set_emi_sub_batch); 0: the default.
std::atomic<int64_t> g_sub_batch_cap{0};

namespace {

constexpr int kMaxFastN = 128;

// Gauss-Jordan thread grid: 16 row lanes (ty) x CX column groups (tx), thread tid = 16 tx + ty;
// thread (tx, ty) holds rows ty + 16 ib (ib < NB) and columns tx + CX jb (jb < NC).
template <int NB, int CX>
struct GjGrid {
  static constexpr int NC = (16 * NB + CX - 1) / CX;
  static constexpr int kThreads = 16 * CX;
  static constexpr int kWarps = kThreads / 32;
};

template <typename T, int NB, int CX>
struct GjShared {
  T col[2][16 * NB];
  int piv[2];
  int piv_of_step[16 * NB];
  int step_of_row[16 * NB];
  T part[GjGrid<NB, CX>::kWarps][16 * NB];  // row sums of |a| per warp (norm estimate)
  T wmax[GjGrid<NB, CX>::kWarps];
};

// max_i sum_j |a_ij| over the n x n block of the register tile (the padding excluded);
// deterministic: fixed reduction order. Whole CTA.
template <typename T, int NB, int CX>
__device__ T max_abs_row_sum(const T (&a)[NB][GjGrid<NB, CX>::NC], int n, int tx, int ty, GjShared<T, NB, CX>& s) {
  constexpr int NC = GjGrid<NB, CX>::NC, W = GjGrid<NB, CX>::kWarps;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
#pragma unroll
  for (int ib = 0; ib < NB; ++ib) {
    T r = 0;
#pragma unroll
    for (int jb = 0; jb < NC; ++jb)
      if (tx + CX * jb < n) r += fabs(a[ib][jb]);
    r += __shfl_xor_sync(0xffffffffu, r, 16);  // the two column groups tx = 2w, 2w + 1 of this warp
    if (lane < 16) s.part[w][ty + 16 * ib] = r;
  }
  __syncthreads();
  T m = 0;
  for (int i = tid; i < n; i += blockDim.x) {
    T r = 0;
#pragma unroll
    for (int q = 0; q < W; ++q) r += s.part[q][i];
    m = fmax(m, r);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) s.wmax[w] = m;
  __syncthreads();
  T r = s.wmax[0];
#pragma unroll
  for (int q = 1; q < W; ++q) r = fmax(r, s.wmax[q]);
  __syncthreads();
  return r;
}

// |Gamma| of point c into the register tile (identity on the padding).
template <typename T, int NB, int CX>
__device__ __forceinline__ void load_abs_gamma(T (&a)[NB][GjGrid<NB, CX>::NC], unsigned& used,
                                               const float2* __restrict__ c, int n, int tx, int ty) {
  constexpr int NC = GjGrid<NB, CX>::NC;
  used = 0;
#pragma unroll
  for (int ib = 0; ib < NB; ++ib) {
    const int i = ty + 16 * ib;
    if (i >= n) used |= 1u << ib;  // padding rows never pivot
#pragma unroll
    for (int jb = 0; jb < NC; ++jb) {
      const int j = tx + CX * jb;
      T v = (i == j) ? T(1) : T(0);
      if (i < n && j < n && i != j) {
        const float2 g = c[i < j ? triu_index(i, j, n) : triu_index(j, i, n)];
        v = (T)sqrt((double)g.x * g.x + (double)g.y * g.y);
      }
      a[ib][jb] = v;
    }
  }
}

__device__ __forceinline__ float recip(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double recip(double x) { return __drcp_rn(x); }  // = 1.0 / x, IEEE round-to-nearest

// One Gauss-Jordan step k = CX KB + kt on the register tile; KB is a compile-time column
// slot, so the pivot column is read and rewritten without dynamic register indexing.
template <typename T, int NB, int CX, int KB>
__device__ __forceinline__ void gj_step(T (&a)[NB][GjGrid<NB, CX>::NC], unsigned& used, int k, int tx, int ty,
                                        bool& singular, GjShared<T, NB, CX>& s) {
  constexpr int NC = GjGrid<NB, CX>::NC;
  const int tid = threadIdx.x;
  const int buf = k & 1;
  const bool owner = tx == (k % CX);
  if (owner) {  // the half-warp owning column k: publish it, find the pivot
    const unsigned half = (tx & 1) ? 0xFFFF0000u : 0x0000FFFFu;
    T best = T(-1);
    int bi = -1;
#pragma unroll
    for (int ib = 0; ib < NB; ++ib) {
      const T v = a[ib][KB];
      s.col[buf][ty + 16 * ib] = v;
      const T av = fabs(v) == fabs(v) ? fabs(v) : T(-0.5);  // NaN ranks last but is taken
      if (!(used & (1u << ib)) && av > best) { best = av; bi = ty + 16 * ib; }
    }
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) {
      const T ob = __shfl_xor_sync(half, best, o, 16);
      const int oi = __shfl_xor_sync(half, bi, o, 16);
      if (ob > best || (ob == best && oi >= 0 && (bi < 0 || oi < bi))) { best = ob; bi = oi; }
    }
    if (ty == 0) s.piv[buf] = bi;
  }
  __syncthreads();
  const int p = s.piv[buf];
  T pv = s.col[buf][p];
  if (pv == T(0)) { singular = true; pv = T(1); }
  const T rp = recip(pv);
  if (ty == (p & 15)) used |= 1u << (p >> 4);
  if (tid == 0) { s.piv_of_step[k] = p; s.step_of_row[p] = k; }
  const int pl = p & 15;
  // pivot row (scaled) from row lane pl of this column group; p >> 4 is CTA-uniform
  T r[NC];
  switch (p >> 4) {
#define MR_GJ_ROW(PB)                                                                  \
  case PB:                                                                             \
    if (PB < NB) {                                                                     \
      _Pragma("unroll") for (int jb = 0; jb < NC; ++jb) r[jb] =                        \
          __shfl_sync(0xffffffffu, a[PB < NB ? PB : 0][jb], pl, 16) * rp;              \
    }                                                                                  \
    break;
    MR_GJ_ROW(0) MR_GJ_ROW(1) MR_GJ_ROW(2) MR_GJ_ROW(3) MR_GJ_ROW(4) MR_GJ_ROW(5) MR_GJ_ROW(6)
    default: MR_GJ_ROW(7)
#undef MR_GJ_ROW
  }
  // a -= f_i r_j everywhere, with f_p = pv - 1 so that the pivot row becomes r; then
  // column k becomes delta_ip / pv - f_i / pv
#pragma unroll
  for (int ib = 0; ib < NB; ++ib) {
    const int i = ty + 16 * ib;
    const T fi = s.col[buf][i];
    const T f = (i == p) ? pv - T(1) : fi;
#pragma unroll
    for (int jb = 0; jb < NC; ++jb) a[ib][jb] -= f * r[jb];
    if (owner) a[ib][KB] = (i == p) ? rp : -fi * rp;
  }
}

// In-place Gauss-Jordan inverse with partial pivoting on the register tile. Returns true
// when a zero pivot was met (the matrix is singular).
template <typename T, int NB, int CX>
__device__ bool gj_tile(T (&a)[NB][GjGrid<NB, CX>::NC], unsigned used, int n, int tx, int ty,
                        GjShared<T, NB, CX>& s) {
  constexpr int NC = GjGrid<NB, CX>::NC;
  bool singular = false;
#pragma unroll
  for (int kb = 0; kb < NC; ++kb) {
    for (int kt = 0; kt < CX; ++kt) {
      const int k = CX * kb + kt;
      if (k >= n) break;
      switch (kb) {  // compile-time slot (the loop over kb is unrolled)
        case 0: gj_step<T, NB, CX, 0>(a, used, k, tx, ty, singular, s); break;
        case 1: if (NC > 1) gj_step<T, NB, CX, (1 < NC ? 1 : 0)>(a, used, k, tx, ty, singular, s); break;
        case 2: if (NC > 2) gj_step<T, NB, CX, (2 < NC ? 2 : 0)>(a, used, k, tx, ty, singular, s); break;
        case 3: if (NC > 3) gj_step<T, NB, CX, (3 < NC ? 3 : 0)>(a, used, k, tx, ty, singular, s); break;
        case 4: if (NC > 4) gj_step<T, NB, CX, (4 < NC ? 4 : 0)>(a, used, k, tx, ty, singular, s); break;
        case 5: if (NC > 5) gj_step<T, NB, CX, (5 < NC ? 5 : 0)>(a, used, k, tx, ty, singular, s); break;
        case 6: if (NC > 6) gj_step<T, NB, CX, (6 < NC ? 6 : 0)>(a, used, k, tx, ty, singular, s); break;
        case 7: if (NC > 7) gj_step<T, NB, CX, (7 < NC ? 7 : 0)>(a, used, k, tx, ty, singular, s); break;
        case 8: if (NC > 8) gj_step<T, NB, CX, (8 < NC ? 8 : 0)>(a, used, k, tx, ty, singular, s); break;
        case 9: if (NC > 9) gj_step<T, NB, CX, (9 < NC ? 9 : 0)>(a, used, k, tx, ty, singular, s); break;
        case 10: if (NC > 10) gj_step<T, NB, CX, (10 < NC ? 10 : 0)>(a, used, k, tx, ty, singular, s); break;
        case 11: if (NC > 11) gj_step<T, NB, CX, (11 < NC ? 11 : 0)>(a, used, k, tx, ty, singular, s); break;
        case 12: if (NC > 12) gj_step<T, NB, CX, (12 < NC ? 12 : 0)>(a, used, k, tx, ty, singular, s); break;
        case 13: if (NC > 13) gj_step<T, NB, CX, (13 < NC ? 13 : 0)>(a, used, k, tx, ty, singular, s); break;
        case 14: if (NC > 14) gj_step<T, NB, CX, (14 < NC ? 14 : 0)>(a, used, k, tx, ty, singular, s); break;
        default: if (NC > 15) gj_step<T, NB, CX, (15 < NC ? 15 : 0)>(a, used, k, tx, ty, singular, s); break;
      }
    }
  }
  __syncthreads();
  return singular;
}

// ----------------------------------------------------------------- packed reduction
template <typename T>
struct TriShared {
  using C = typename C2<T>::type;
  C* L;       // lower triangle by rows: (i, j <= i) at roff[i] + j
  C* pv;      // [2][n] products of the last two steps
  C* vec;     // [3][n]: u_k and u_{k-1} (by step parity), w_{k-1}
  C* e;
  T* d;
  T* tau;
  int* roff;  // row starts, n + 1 entries
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }
__host__ __device__ __forceinline__ int tri(int i) { return i * (i + 1) / 2; }

// Row i of the FP32 triangle starts at roff_of(i) elements: row strides are the smallest
// values >= i + 1 that are 4 mod 16, so that the row segments of mirrored pairs (phase 1) and
// the column walks (phase 2) of a warp fall on distinct 8-byte bank pairs (the reduction
// measured 5 % faster than with packed rows). The FP64 triangle stays packed (tri): there the
// padding measured 3 % slower.
__host__ __device__ __forceinline__ int roff_of(int i) {
  const int a = (i + 12) >> 4, b = (i + 12) & 15;
  return 4 * i + 128 * a * (a - 1) + 16 * a * b;
}
template <typename T> __host__ __device__ __forceinline__ int tri_elems(int n) {
  return sizeof(T) == 4 ? roff_of(n) : n * (n + 1) / 2;
}
template <typename T> __device__ __forceinline__ int rstart(const TriShared<T>& s, int i) {
  if constexpr (sizeof(T) == 4) return s.roff[i];
  else return tri(i);
}

template <typename T>
__host__ __device__ inline size_t tri_bytes(int n) {
  using C = typename C2<T>::type;
  size_t o = align16((size_t)tri_elems<T>(n) * sizeof(C));
  o = align16(o + 2 * (size_t)n * sizeof(C));
  o = align16(o + 3 * (size_t)n * sizeof(C));
  o = align16(o + (size_t)n * sizeof(C));
  o = align16(o + 2 * (size_t)n * sizeof(T));
  return o + (size_t)(n + 1) * sizeof(int);
}

template <typename T>
__device__ inline TriShared<T> tri_layout(unsigned char* base, int n) {
  using C = typename C2<T>::type;
  TriShared<T> s;
  size_t o = 0;
  s.L = reinterpret_cast<C*>(base + o);
  o = align16(o + (size_t)tri_elems<T>(n) * sizeof(C));
  s.pv = reinterpret_cast<C*>(base + o);
  o = align16(o + 2 * (size_t)n * sizeof(C));
  s.vec = reinterpret_cast<C*>(base + o);
  o = align16(o + 3 * (size_t)n * sizeof(C));
  s.e = reinterpret_cast<C*>(base + o);
  o = align16(o + (size_t)n * sizeof(C));
  s.d = reinterpret_cast<T*>(base + o);
  s.tau = s.d + n;
  o = align16(o + 2 * (size_t)n * sizeof(T));
  s.roff = reinterpret_cast<int*>(base + o);
  return s;
}

// a -= ui conj(wj) + wi conj(uj)
template <typename C> __device__ __forceinline__ void rank2(C& a, C ui, C wj, C wi, C uj) {
  // one FMA per product (no separate multiply and add)
  a.x -= ui.x * wj.x; a.x -= ui.y * wj.y; a.x -= wi.x * uj.x; a.x -= wi.y * uj.y;
  a.y -= ui.y * wj.x; a.y += ui.x * wj.y; a.y -= wi.y * uj.x; a.y += wi.x * uj.y;
}

// Householder reduction of the Hermitian M (lower triangle, packed in s.L) to tridiagonal
// (s.d, s.e); reflector k stored in column k (rows k+1..n-1) with scalar s.tau[k]. Whole
// CTA, three barriers per step:
//   1. warp 0 finishes step k-1 (w = p - K u, K = tau/2 u^H p) and forms reflector k from
//      column k brought up to date, x_i = A_i + K B_i, with A_i and B_i computed in the same
//      pass as the dot product (one load pass, two warp reductions);
//   2. phase 1: step k-1's rank-2 update on the lower triangle of rows >= k+1 and the row
//      part of (M u_k)_i = sum_{j<=i} M_ij u_j;
//   3. phase 2: the column part sum_{j>i} conj(M_ji) u_j, then p_k = tau_k M u_k.
// Rows are handled in mirrored pairs (i, n+k-i) by groups of 4 threads, which gives every
// thread of a step the same number of elements in both phases. The packed triangle halves the
// shared memory of full storage, so twice as many points are in flight per SM.
template <typename T>
__device__ void tridiag_packed(const TriShared<T>& s, int n) {
  using C = typename C2<T>::type;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  C* L = s.L;
  C* wp = s.vec + 2 * n;  // w_{k-1}
  for (int k = 0; k + 2 < n; ++k) {
    C* up = s.vec + ((k + 1) & 1) * n;  // u_{k-1}
    C* uc = s.vec + (k & 1) * n;        // u_k
    // ---- warp 0: finish step k-1 and form reflector k
    if (wid == 0) {
      const T tau_prev = k > 0 ? s.tau[k - 1] : T(0);
      const bool pending = tau_prev != T(0);
      const C* p = s.pv + ((k + 1) & 1) * n;
      C A[4], B[4], pp[4], uu[4];
      T dot = 0;
      C pk = mk<T>(0, 0), ukk = mk<T>(0, 0);
      if (pending) { pk = p[k]; ukk = up[k]; }
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int i = k + lane + 32 * t;
        A[t] = B[t] = pp[t] = uu[t] = mk<T>(0, 0);
        if (i < n) {
          const int base = rstart(s, i);
          A[t] = L[base + k];
          if (pending) {
            pp[t] = p[i];
            uu[t] = up[i];
            dot += uu[t].x * pp[t].x + uu[t].y * pp[t].y;
            // x_i = a_ik - u_i conj(w_k) - w_i conj(u_k) = A_i + K B_i, w = p - K u
            rank2(A[t], uu[t], pk, pp[t], ukk);
            B[t] = mk<T>(2 * (uu[t].x * ukk.x + uu[t].y * ukk.y), 2 * (uu[t].y * ukk.x - uu[t].x * ukk.y));
            L[base + k - 1] = uu[t];  // reflector k-1 (rows >= k) kept in column k-1
          }
        }
      }
      const T K = pending ? T(0.5) * tau_prev * warp_sum(dot) : T(0);
      T xn2 = 0;
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int i = k + lane + 32 * t;
        if (i < n) {
          const C x = mk<T>(A[t].x + K * B[t].x, A[t].y + K * B[t].y);
          if (pending) wp[i] = mk<T>(pp[t].x - K * uu[t].x, pp[t].y - K * uu[t].y);
          uc[i] = x;
          if (i >= k + 2) xn2 += x.x * x.x + x.y * x.y;
        }
      }
      xn2 = warp_sum(xn2);
      __syncwarp();
      const C alpha = uc[k + 1];
      T tau_k = 0;
      C ek = alpha;
      if (xn2 != T(0)) {
        const T aa = sqrt(alpha.x * alpha.x + alpha.y * alpha.y);
        const T nrm = sqrt(aa * aa + xn2);
        const C ph1 = aa > T(0) ? mk<T>(alpha.x / aa, alpha.y / aa) : mk<T>(1, 0);
        tau_k = T(2) / ((aa + nrm) * (aa + nrm) + xn2);
        ek = mk<T>(-ph1.x * nrm, -ph1.y * nrm);
        if (lane == 0) uc[k + 1] = mk<T>(ph1.x * (aa + nrm), ph1.y * (aa + nrm));
      }
      if (lane == 0) { s.d[k] = uc[k].x; s.e[k] = ek; s.tau[k] = tau_k; }
    }
    __syncthreads();
    const bool pending = k > 0 && s.tau[k - 1] != T(0);
    const T tau_k = s.tau[k];
    const int m = n - k - 1;         // rows k+1..n-1
    const int npair = (m + 1) >> 1;  // mirrored pairs (the middle row of an odd m alone)
    // G = 4 threads per pair. Widening the groups to keep every thread busy as the trailing
    // matrix shrinks measured 3 % slower: the short rows of late steps then cost more loop
    // set-up than they save, while idle warps leave the issue slots to the other CTAs.
    const int G = 4;
    const int pq = tid / G, sub = tid & (G - 1);
    const unsigned gmask = G == 32 ? 0xffffffffu : ((1u << G) - 1u) << (lane & ~(G - 1));
    const bool active = (pending || tau_k != T(0)) && pq < npair;
    const int i1 = k + 1 + pq, i2 = n - 1 - pq;
    const bool two = i2 != i1;
    // ---- phase 1: update the lower rows, row part of M u
    C rs1 = mk<T>(0, 0), rs2 = mk<T>(0, 0);
    if (active) {
#pragma unroll 1
      for (int r = 0; r < 2; ++r) {
        if (r && !two) break;
        const int i = r ? i2 : i1;
        C* row = L + rstart(s, i);
        C upi = mk<T>(0, 0), wpi = mk<T>(0, 0);
        if (pending) { upi = up[i]; wpi = wp[i]; }
        C acc = mk<T>(0, 0);
#pragma unroll 2  // measured: 5 % faster than the compiler's default, 4 gave less
        for (int j = k + 1 + sub; j <= i; j += G) {
          C a = row[j];
          if (pending) { rank2(a, upi, wp[j], wpi, up[j]); row[j] = a; }
          const C u = uc[j];
          acc.x += a.x * u.x; acc.x -= a.y * u.y;
          acc.y += a.x * u.y; acc.y += a.y * u.x;
        }
        if (r) rs2 = acc; else rs1 = acc;
      }
    }
    __syncthreads();
    // ---- phase 2: column part, then p_k
    if (active && tau_k != T(0)) {
#pragma unroll 1
      for (int r = 0; r < 2; ++r) {
        if (r && !two) break;
        const int i = r ? i2 : i1;
        C acc = r ? rs2 : rs1;
#pragma unroll 2
        for (int j = i + 1 + sub; j < n; j += G) {
          const C a = L[rstart(s, j) + i];  // M_ji, lower triangle
          const C u = uc[j];
          acc.x += a.x * u.x; acc.x += a.y * u.y;  // conj(M_ji) u_j
          acc.y += a.x * u.y; acc.y -= a.y * u.x;
        }
        for (int o = 1; o < G; o <<= 1) {
          acc.x += __shfl_xor_sync(gmask, acc.x, o);
          acc.y += __shfl_xor_sync(gmask, acc.y, o);
        }
        if (sub == 0) s.pv[(k & 1) * n + i] = mk<T>(tau_k * acc.x, tau_k * acc.y);
      }
    }
    __syncthreads();
  }
  // last pending update (step n-3) on the trailing 2 x 2 block; reflector n-3 stored
  if (wid == 0) {
    if (n >= 3 && s.tau[n - 3] != T(0)) {
      const T tau_prev = s.tau[n - 3];
      const C* up = s.vec + ((n - 3) & 1) * n;
      const C* p = s.pv + ((n - 3) & 1) * n;
      T dot = 0;
      for (int i = n - 2 + lane; i < n; i += 32) {
        const C pi = p[i], ui = up[i];
        wp[i] = pi;
        dot += ui.x * pi.x + ui.y * pi.y;
      }
      const T K = T(0.5) * tau_prev * warp_sum(dot);
      for (int i = n - 2 + lane; i < n; i += 32) { wp[i].x -= K * up[i].x; wp[i].y -= K * up[i].y; }
      __syncwarp();
      if (lane < 3) {
        const int i = (lane == 0) ? n - 2 : n - 1, j = (lane == 2) ? n - 1 : n - 2;
        rank2(L[rstart(s, i) + j], up[i], wp[j], wp[i], up[j]);
      }
      for (int i = n - 2 + lane; i < n; i += 32) L[rstart(s, i) + n - 3] = up[i];
      __syncwarp();
    }
    if (lane == 0) {
      s.d[n - 2] = L[rstart(s, n - 2) + n - 2].x;
      s.d[n - 1] = L[rstart(s, n - 1) + n - 1].x;
      s.e[n - 2] = L[rstart(s, n - 1) + n - 2];
    }
  }
  __syncthreads();
}


// acc += a b (one FMA per product)
template <typename C> __device__ __forceinline__ void cmac(C& acc, C a, C b) {
  acc.x += a.x * b.x;
  acc.x -= a.y * b.y;
  acc.y += a.x * b.y;
  acc.y += a.y * b.x;
}
// acc += conj(a) b
template <typename C> __device__ __forceinline__ void cmacc(C& acc, C a, C b) {
  acc.x += a.x * b.x;
  acc.x += a.y * b.y;
  acc.y += a.x * b.y;
  acc.y -= a.y * b.x;
}
template <typename C> __device__ __forceinline__ C shfl_xor_c(C v, int o) {
  v.x = __shfl_xor_sync(0xffffffffu, v.x, o);
  v.y = __shfl_xor_sync(0xffffffffu, v.y, o);
  return v;
}

// Sum over the 32 lanes of four per-lane values r[0..3] (reduce-scatter): afterwards lane l
// holds the total of value (l >> 3) & 3 (lanes 0, 8, 16, 24 hold values 0, 1, 2, 3).
template <typename C> __device__ __forceinline__ C warp_sum4(const C (&r)[4]) {
  const int lane = threadIdx.x & 31;
  const bool hi4 = lane & 16, hi3 = lane & 8;
  C k0 = hi4 ? r[2] : r[0], k1 = hi4 ? r[3] : r[1];
  const C s0 = hi4 ? r[0] : r[2], s1 = hi4 ? r[1] : r[3];
  k0 = cadd(k0, shfl_xor_c(s0, 16));
  k1 = cadd(k1, shfl_xor_c(s1, 16));
  C k = hi3 ? k1 : k0;
  k = cadd(k, shfl_xor_c(hi3 ? k0 : k1, 8));
  k = cadd(k, shfl_xor_c(k, 4));
  k = cadd(k, shfl_xor_c(k, 2));
  k = cadd(k, shfl_xor_c(k, 1));
  return k;
}

// ----------------------------------------------------------------- workspace layout
// Per point: inv(|Gamma|) in the arithmetic TA of the inverse, packed upper triangle by
// rows like the compressed coherence ((m, j >= m) at tri_up(m, j)); then, in the arithmetic
// T of the reduction, the reflectors (column k rows k+1..n-1, packed by column, nq complex
// T), d and tau (n T each), e (n complex T).
__host__ __device__ __forceinline__ int64_t tri_up(int m, int j, int n) {
  return (int64_t)m * n - ((int64_t)m * (m - 1)) / 2 + (j - m);
}

template <typename T, typename TA = T>
struct PointWs {
  size_t np, nq, bytes;
  __host__ __device__ explicit PointWs(int n) {
    using C = typename C2<T>::type;
    np = (size_t)n * (n + 1) / 2;
    nq = (size_t)n * (n - 1) / 2;
    bytes = align16(np * sizeof(TA)) + align16(nq * sizeof(C)) + align16(2 * (size_t)n * sizeof(T)) +
            align16((size_t)n * sizeof(C));
  }
};

template <typename T, typename TA = T>
struct PointPtr {
  using C = typename C2<T>::type;
  TA* ainv;
  C* refl;
  T* d;
  T* tau;
  C* e;
  __device__ PointPtr(unsigned char* ws, int64_t pt, int n) {
    const PointWs<T, TA> w(n);
    unsigned char* b = ws + (size_t)pt * w.bytes;
    ainv = reinterpret_cast<TA*>(b);
    b += align16(w.np * sizeof(TA));
    refl = reinterpret_cast<C*>(b);
    b += align16(w.nq * sizeof(C));
    d = reinterpret_cast<T*>(b);
    tau = d + n;
    b += align16(2 * (size_t)n * sizeof(T));
    e = reinterpret_cast<C*>(b);
  }
};

__host__ __device__ __forceinline__ size_t refl_off(int k, int n) { return (size_t)k * (n - 1) - (size_t)k * (k - 1) / 2; }

// ----------------------------------------------------------------- kernel 1: inverse
// Route flags of a point (sing[] in the workspace, route[] on output).
constexpr uint8_t kRouteCond = 1;      // cond_1(|Gamma|) estimate above the threshold
constexpr uint8_t kRouteSingular = 2;  // a zero pivot: |Gamma| singular at this precision

// Points of a pass: all n_pc of the sub-batch; or, with a list, list[off + i] for
// i < min(*count - off, n_pc), a window of at most n_pc entries of a list that may be longer.
struct PointSet {
  const int32_t* list;
  const int32_t* count;
  int64_t n_pc;
  const int64_t* dcount;  // without a list: the points are dcount[0] - off, at most n_pc
  int64_t off;
  __device__ __forceinline__ int64_t size() const {
    if (list || dcount) {
      const int64_t c = (list ? (int64_t)*count : *dcount) - off;
      return c < 0 ? 0 : (c < n_pc ? c : n_pc);
    }
    return n_pc;
  }
  __device__ __forceinline__ int64_t operator[](int64_t i) const { return list ? (int64_t)list[off + i] : i; }
};

// TW: arithmetic of the reduction that reads the workspace (the point stride depends on it).
template <typename T, int NB, int CX, typename TW>
__global__ void __launch_bounds__(16 * CX, 1) inverse_kernel(const float2* __restrict__ coh, PointSet pts, int n,
                                                          unsigned char* __restrict__ ws, uint8_t* __restrict__ sing,
                                                          float cond_max) {
  constexpr int NC = GjGrid<NB, CX>::NC;
  __shared__ GjShared<T, NB, CX> gs;
  const int tid = threadIdx.x, tx = tid >> 4, ty = tid & 15;
  const int64_t npairs = (int64_t)n * (n - 1) / 2;
  const int64_t npt = pts.size();
  for (int64_t pt = blockIdx.x; pt < npt; pt += gridDim.x) {
    const int64_t gp = pts[pt];
    T a[NB][NC];
    unsigned used;
    load_abs_gamma<T, NB, CX>(a, used, coh + gp * npairs, n, tx, ty);
    const T anorm = cond_max > 0.f ? max_abs_row_sum<T, NB, CX>(a, n, tx, ty, gs) : T(0);
    const bool singular = gj_tile<T, NB, CX>(a, used, n, tx, ty, gs);
    uint8_t flag = singular ? kRouteSingular : 0;
    if (cond_max > 0.f && !singular) {
      // cond_1 = ||A||_1 ||inv(A)||_1 (A symmetric: row sums); the register rows of the
      // result are the rows of inv(A) in pivot order
      const T cond = anorm * max_abs_row_sum<T, NB, CX>(a, n, tx, ty, gs);
      if (!(cond <= (T)cond_max)) flag = kRouteCond;
    }
    T* out = PointPtr<TW, T>(ws, pt, n).ainv;
#pragma unroll
    for (int ib = 0; ib < NB; ++ib) {
      const int r0 = ty + 16 * ib;
      if (r0 >= n) continue;
      const int kr = gs.step_of_row[r0];
#pragma unroll
      for (int jb = 0; jb < NC; ++jb) {
        const int c0 = tx + CX * jb;
        if (c0 >= n) continue;
        const int pc = gs.piv_of_step[c0];
        if (kr >= pc) out[tri_up(pc, kr, n)] = a[ib][jb];  // inv[kr][pc], kept once
      }
    }
    if (tid == 0) sing[pt] = flag;
    __syncthreads();
  }
}

// ----------------------------------------------------------------- kernel 1b: symmetric sweep
// inv(|Gamma|) for the refined mixed precision, FP64: Gauss-Jordan on the symmetric matrix
// with diagonal pivots in natural order (the sweep operator), which keeps the matrix
// symmetric, so only its lower triangle is held and updated: half the registers of the
// pivoted kernel (two CTAs per SM) and half its FMAs, with no pivot search on the serial
// chain of a step. Step k with column c = A[:, k] (c_k = d):
//   A_ij -= c_i c_j / d (i, j != k);  A_ik = c_i / d (i != k);  A_kk = -1 / d,
// and after all n steps A holds -inv(A). Without interchanges a pivot can become small on
// an indefinite |Gamma|; the kernel flags the point (kRouteCond) when a pivot falls below
// kSweepMinPivot in magnitude, and the refined pass recomputes flagged
// points with the pivoted FP64 kernels. On the c2 scene model the natural order stays
// within about 30 eps cond(|Gamma|) of the pivoted inverse (3.7e-9 relative at worst over
// 1,500 points, 41 % of them indefinite), far below what the refinement needs.
constexpr double kSweepMinPivot = 1e-9;

template <int NB>
struct SweepShared {
  double2 col[2][16 * NB];  // columns k and k + 1 of a pivot pair, (A_ik, A_i,k+1), by pair parity
};

__host__ __device__ constexpr int lt(int ib, int jb) { return ib * (ib + 1) / 2 + jb; }  // jb <= ib

// Thread (tx, ty) of the 16 x 16 grid holds A[i][j] for i = ty + 16 ib, j = tx + 16 jb,
// jb <= ib (NB (NB + 1) / 2 values); in a diagonal block only ty >= tx is the lower triangle
// (the rest is updated like it but never read).
//
// Pivots go in pairs K = {k, k + 1} (k even; with n odd the last pair takes the identity row
// of the padding): with P = A_KK, the two sweeps at once are
//   A_ij -= A_iK inv(P) A_Kj (i, j not in K);  A_iK = A_iK inv(P);  A_KK = -inv(P),
// one barrier per pair, evaluated as the two single sweeps in sequence (sweep_pair). The
// owners of columns k, k + 1 (two lanes of every half-warp) write A_iK, the owners of rows
// k, k + 1 (one whole warp, as ty = k, k + 1 share a warp) write A_Kj and -inv(P). The
// point is flagged when a natural-order pivot (P_00, then P_11 - P_10^2 / P_00) falls below
// kSweepMinPivot.

// Columns k2, k2 + 1 of the matrix into `out`: the lower parts (rows >= k2, >= k2 + 1) from
// the owners of those columns, the upper parts from the owners of rows k2, k2 + 1 (symmetry).
// KBX = k2 >> 4 at compile time.
template <int NB, int KBX>
__device__ __forceinline__ void sweep_publish(const double (&a)[NB * (NB + 1) / 2], int k2, int tx, int ty,
                                              double2* out) {
  const int kt2 = k2 & 15;
  if (tx == kt2 || tx == kt2 + 1) {
    const int c = tx - kt2;
#pragma unroll
    for (int ib = KBX; ib < NB; ++ib) {
      const int i = ty + 16 * ib;
      if (i >= k2 + c) (c ? out[i].y : out[i].x) = a[lt(ib, KBX)];
    }
  }
  if (ty == kt2 || ty == kt2 + 1) {
    const int r = ty - kt2;
#pragma unroll
    for (int jb = 0; jb <= KBX; ++jb) {
      const int j = tx + 16 * jb;
      if (j < k2 + r) (r ? out[j].y : out[j].x) = a[lt(KBX, jb)];
    }
  }
}

template <int NB, int KB>
__device__ __forceinline__ void sweep_pair(double (&a)[NB * (NB + 1) / 2], int k, int n, int tx, int ty,
                                           bool& small, SweepShared<NB>& s) {
  const int buf = (k >> 1) & 1;
  const double2* col = s.col[buf];
  const int kt = k & 15;
  const double2 pk = col[k], pk1 = col[k + 1];
  // the two sweeps in sequence, fused: sweep k turns column k + 1 into c1' = c1 - t c0
  // (t = P_10 / P_00) and its pivot into d1 = P_11 - t P_10; then
  //   A_ij -= g0_i c0_j + g1_i c1'_j,  g0 = c0 / P_00, g1 = c1' / d1,
  // the same two roundings per element as two single sweeps (the product form
  // c_i inv(P) c_j^T instead loses accuracy to cancellation when d1 is small)
  const double r0 = recip(pk.x == 0.0 ? 1.0 : pk.x);
  const double t = pk.y * r0;
  const double d1 = pk1.y - t * pk.y;
  const double r1 = recip(d1 == 0.0 ? 1.0 : d1);
  // natural-order pivots P_00 and d1; NaN compares false and is flagged too
  small |= !(fabs(pk.x) >= kSweepMinPivot && fabs(d1) >= kSweepMinPivot);
  double2 cj[NB];  // (c0_j, c1'_j)
#pragma unroll
  for (int jb = 0; jb < NB; ++jb) {
    const double2 c = col[tx + 16 * jb];
    cj[jb] = make_double2(c.x, c.y - t * c.x);
  }
  const bool colk = tx == kt || tx == kt + 1;  // this lane owns column k or k + 1 (block KB)
#pragma unroll
  for (int ib = 0; ib < NB; ++ib) {
    const double2 ci = col[ty + 16 * ib];
    const double g0 = ci.x * r0, g1 = (ci.y - t * ci.x) * r1;
#pragma unroll
    for (int jb = 0; jb <= ib; ++jb) {
      double& v = a[lt(ib, jb)];
      v -= g0 * cj[jb].x;
      v -= g1 * cj[jb].y;
      if (jb == KB && colk) v = tx == kt ? g0 - t * g1 : g1;  // A_iK = c_i inv(P)
    }
  }
  if (ty == kt || ty == kt + 1) {  // rows k, k + 1: warp-uniform
    const bool row1 = ty != kt;
#pragma unroll
    for (int jb = 0; jb <= KB; ++jb) {
      const double g0 = cj[jb].x * r0, g1 = cj[jb].y * r1;
      double w = row1 ? g1 : g0 - t * g1;  // A_Kj = inv(P) c_j^T
      if (jb == KB && colk)                // -inv(P)
        w = row1 ? (tx == kt ? t * r1 : -r1) : (tx == kt ? -(r0 + t * t * r1) : t * r1);
      a[lt(KB, jb)] = w;
    }
  }
  const int k2 = k + 2;
  if (k2 < n) {
    double2* out = s.col[buf ^ 1];
    if (kt + 2 < 16) sweep_publish<NB, KB>(a, k2, tx, ty, out);
    else if (KB + 1 < NB) sweep_publish<NB, (KB + 1 < NB ? KB + 1 : 0)>(a, k2, tx, ty, out);
  }
  __syncthreads();
}

// TW: arithmetic of the reduction that reads the workspace (the point stride depends on it).
template <int NB, typename TW>
__global__ void __launch_bounds__(256, 2) sweep_kernel(const float2* __restrict__ coh, PointSet pts, int n,
                                                       unsigned char* __restrict__ ws, uint8_t* __restrict__ sing) {
  constexpr int NP = NB * (NB + 1) / 2;
  __shared__ SweepShared<NB> ss;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int64_t npairs = (int64_t)n * (n - 1) / 2;
  const int64_t npt = pts.size();
  for (int64_t pt = blockIdx.x; pt < npt; pt += gridDim.x) {
    const float2* c = coh + pts[pt] * npairs;
    if (tid == 0 && pt + gridDim.x < npt) {  // the next point's coherence into L2 (the part
      // between its first and last 16-byte boundaries; 2 % faster than without)
      const uintptr_t a0 = reinterpret_cast<uintptr_t>(coh + pts[pt + gridDim.x] * npairs);
      const uintptr_t lo = (a0 + 15) & ~uintptr_t(15), hi = (a0 + npairs * 8) & ~uintptr_t(15);
      if (hi > lo) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lo), "r"((unsigned)(hi - lo)) : "memory");
    }
    double a[NP];
    // |Gamma| (identity on the padding), lower triangle; a block row's loads are issued
    // together, then converted (7 % faster than loading and converting value by value, which
    // left one L2 round trip per value on the thread's path)
#pragma unroll
    for (int ib = 0; ib < NB; ++ib) {
      const int i = ty + 16 * ib;
      float2 g[NB];
#pragma unroll
      for (int jb = 0; jb <= ib; ++jb) {
        const int j = tx + 16 * jb;
        g[jb] = (i < n && j < n && i > j) ? c[triu_index(j, i, n)] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int jb = 0; jb <= ib; ++jb) {
        const int j = tx + 16 * jb;
        a[lt(ib, jb)] = (i == j) ? 1.0 : sqrt((double)g[jb].x * g[jb].x + (double)g[jb].y * g[jb].y);
      }
    }
    sweep_publish<NB, 0>(a, 0, tx, ty, ss.col[0]);
    __syncthreads();
    bool small = false;
#pragma unroll 1
    for (int kb = 0; kb < NB; ++kb) {
      for (int kt = 0; kt < 16; kt += 2) {
        const int k = 16 * kb + kt;
        if (k >= n) break;
        switch (kb) {  // compile-time block for each kb
          case 0: sweep_pair<NB, 0>(a, k, n, tx, ty, small, ss); break;
          case 1: if (NB > 1) sweep_pair<NB, (1 < NB ? 1 : 0)>(a, k, n, tx, ty, small, ss); break;
          case 2: if (NB > 2) sweep_pair<NB, (2 < NB ? 2 : 0)>(a, k, n, tx, ty, small, ss); break;
          case 3: if (NB > 3) sweep_pair<NB, (3 < NB ? 3 : 0)>(a, k, n, tx, ty, small, ss); break;
          case 4: if (NB > 4) sweep_pair<NB, (4 < NB ? 4 : 0)>(a, k, n, tx, ty, small, ss); break;
          case 5: if (NB > 5) sweep_pair<NB, (5 < NB ? 5 : 0)>(a, k, n, tx, ty, small, ss); break;
          case 6: if (NB > 6) sweep_pair<NB, (6 < NB ? 6 : 0)>(a, k, n, tx, ty, small, ss); break;
          default: if (NB > 7) sweep_pair<NB, (7 < NB ? 7 : 0)>(a, k, n, tx, ty, small, ss); break;
        }
      }
    }
    // every thread saw the same pivots: `small` is uniform
    double* out = PointPtr<TW, double>(ws, pt, n).ainv;
#pragma unroll
    for (int ib = 0; ib < NB; ++ib) {
      const int i = ty + 16 * ib;
#pragma unroll
      for (int jb = 0; jb <= ib; ++jb) {
        const int j = tx + 16 * jb;
        if (i < n && j <= i) out[tri_up(j, i, n)] = -a[lt(ib, jb)];  // inv = -A after the sweep
      }
    }
    if (tid == 0) sing[pt] = small ? kRouteCond : 0;
    __syncthreads();
  }
}

// ----------------------------------------------------------------- kernel 2: reduction
template <typename T, typename TA>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? 4 : 2) reduce_kernel(const float2* __restrict__ coh, PointSet pts, int n,
                                                         unsigned char* __restrict__ ws) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const TriShared<T> s = tri_layout<T>(smem_raw, n);
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = tid; i <= n; i += nt) s.roff[i] = roff_of(i);
  __syncthreads();
  const int64_t npairs = (int64_t)n * (n - 1) / 2;
  const int np = n * (n + 1) / 2;
  const int64_t npt = pts.size();
  for (int64_t pt = blockIdx.x; pt < npt; pt += gridDim.x) {
    const float2* c = coh + pts[pt] * npairs;
    PointPtr<T, TA> w(ws, pt, n);
    // M = inv(|Gamma|) o Gamma: read along the upper triangle (inverse and coherence both
    // contiguous), written to the packed lower triangle as M_jm = conj(M_mj)
    // row m of element q: rows start at tri_up(m, m, n), which grows only up to m = n, so the
    // walk stops at the last row
    int m = 0;
    while (m + 1 < n && tri_up(m + 1, m + 1, n) <= tid) ++m;
    for (int q = tid; q < np; q += nt) {
      while (m + 1 < n && tri_up(m + 1, m + 1, n) <= q) ++m;
      const int j = m + (q - (int)tri_up(m, m, n));
      const TA sc = w.ainv[q];
      T gx = 1, gy = 0;
      if (j != m) {
        const float2 g = c[(int64_t)q - (m + 1)];  // pair (m, j): triu_index(m, j) = tri_up(m, j) - m - 1
        gx = g.x;
        gy = -g.y;
      }
      s.L[rstart(s, j) + m] = mk<T>((T)(sc * gx), (T)(sc * gy));
    }
    __syncthreads();
    tridiag_packed<T>(s, n);
    for (int k = tid; k < n; k += nt) {
      w.d[k] = s.d[k];
      w.tau[k] = (k + 2 < n) ? s.tau[k] : T(0);
      if (k + 1 < n) w.e[k] = s.e[k];
    }
    for (int k = 0; k + 2 < n; ++k)  // reflector k: column k, rows k+1..n-1
      for (int r = tid; r < n - k - 1; r += nt) w.refl[refl_off(k, n) + r] = s.L[rstart(s, k + 1 + r) + k];
    __syncthreads();
  }
}

// Reflector k of a point (its scalar and the lane's four entries, zero past its end) into
// registers.
template <typename T, typename TA>
__device__ __forceinline__ void load_refl(const PointPtr<T, TA>& w, int n, int k, int lane,
                                          typename C2<T>::type (&u)[4], T& tau) {
  tau = w.tau[k];
  const typename C2<T>::type* src = w.refl + refl_off(k, n);
  const int m = n - k - 1;
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int i = lane + 32 * t;
    u[t] = i < m ? src[i] : mk<T>(0, 0);
  }
}

// ----------------------------------------------------------------- kernel 3: tail, one warp per point
constexpr int kTailWarps = 8;

template <typename T>
__host__ __device__ inline size_t tail_warp_bytes(int n) {
  using C = typename C2<T>::type;
  return align16(6 * (size_t)n * sizeof(T)) + align16((size_t)n * sizeof(C)) + align16((size_t)n * sizeof(double2));
}

template <typename T, typename TA>
__global__ void __launch_bounds__(32 * kTailWarps, 3) tail_kernel(const float2* __restrict__ coh, PointSet pts, int n,
                                                              int ref, const unsigned char* __restrict__ ws,
                                                              const uint8_t* __restrict__ sing,
                                                              float2* __restrict__ ph, float* __restrict__ quality,
                                                              float* __restrict__ tcoh) {
  using C = typename C2<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned char* mine = smem_raw + (size_t)wid * tail_warp_bytes<T>(n);
  T* d = reinterpret_cast<T*>(mine);
  T* b = d + n;
  T* b2 = b + n;
  T* y = b2 + n;
  T* w1 = y + n;
  T* w2 = w1 + n;
  C* z = reinterpret_cast<C*>(mine + align16(6 * (size_t)n * sizeof(T)));
  double2* phs = reinterpret_cast<double2*>(mine + align16(6 * (size_t)n * sizeof(T)) + align16((size_t)n * sizeof(C)));
  const int64_t npairs = (int64_t)n * (n - 1) / 2;
  const float fnan = __int_as_float(0x7fffffff);
  const int64_t npt = pts.size();
  for (int64_t pt = (int64_t)blockIdx.x * kTailWarps + wid; pt < npt; pt += (int64_t)gridDim.x * kTailWarps) {
    const int64_t gp = pts[pt];
    const PointPtr<T, TA> w(const_cast<unsigned char*>(ws), pt, n);
    // real tridiagonal: b = |e|, phases delta_{k+1} = delta_k e_k/|e_k| (warp prefix product)
    C carry = mk<T>(1, 0);
    for (int k0 = 0; k0 < n; k0 += 32) {
      const int k = k0 + lane;
      if (k < n) d[k] = w.d[k];
      C f = mk<T>(1, 0);
      if (k + 1 < n) {
        const C ek = w.e[k];
        const T a = sqrt(ek.x * ek.x + ek.y * ek.y);
        b[k] = a;
        b2[k] = a * a;
        if (a > T(0)) f = mk<T>(ek.x / a, ek.y / a);
      }
      // inclusive scan of the factors f over the lanes
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const T ox = __shfl_up_sync(0xffffffffu, f.x, o), oy = __shfl_up_sync(0xffffffffu, f.y, o);
        if (lane >= o) f = cmul_t(mk<T>(ox, oy), f);
      }
      const C dl = cmul_t(carry, f);  // delta_{k+1}
      if (k0 == 0 && lane == 0) z[0] = mk<T>(1, 0);
      if (k + 1 < n) z[k + 1] = dl;
      carry = mk<T>(__shfl_sync(0xffffffffu, dl.x, 31), __shfl_sync(0xffffffffu, dl.y, 31));
    }
    __syncwarp();
    // lambda_min by multisection
    T lo = Lim<T>::huge(), hi = -Lim<T>::huge(), tnorm = 0;
    for (int i = lane; i < n; i += 32) {
      const T r = (i > 0 ? b[i - 1] : T(0)) + (i + 1 < n ? b[i] : T(0));
      lo = fmin(lo, d[i] - r);
      hi = fmax(hi, d[i] + r);
      tnorm = fmax(tnorm, fabs(d[i]) + r);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
      tnorm = fmax(tnorm, __shfl_xor_sync(0xffffffffu, tnorm, o));
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
      const int cnt = sturm_count(d, b2, n, sg, pivmin);
      const unsigned ball = __ballot_sync(0xffffffffu, cnt >= 1);
      const int first = ball ? __ffs(ball) - 1 : 32;
      const T nlo = (first == 0) ? lo : lo + width * (T)first / T(33);
      const T nhi = (first == 32) ? hi : lo + width * (T)(first + 1) / T(33);
      lo = nlo;
      hi = nhi;
    }
    const T lam = T(0.5) * (lo + hi);
    // eigenvector of the real tridiagonal by inverse iteration (lane 0)
    for (int i = lane; i < n; i += 32) y[i] = T(1) + T(0.25) * (T)((i * 37) % 11) / T(11);
    __syncwarp();
    if (lane == 0) {
      const T tiny = eps * fmax(tnorm, Lim<T>::tiny());
      for (int it = 0; it < 2; ++it) {
        tridiag_solve(d, b, n, lam, tiny, y, w1, w2, b2);  // b2 is free after the bisection
        T sc = 0;
        for (int i = 0; i < n; ++i) sc = fmax(sc, fabs(y[i]));
        if (!(sc > T(0)) || !isfinite(sc)) break;
        const T r = T(1) / sc;
        for (int i = 0; i < n; ++i) y[i] *= r;
      }
    }
    __syncwarp();
    // v = Q D y
    for (int i = lane; i < n; i += 32) { const C dl = z[i]; z[i] = mk<T>(dl.x * y[i], dl.y * y[i]); }
    __syncwarp();
    // reflectors applied from the last; the next one's values are loaded while the current
    // one is applied, so the serial chain does not wait on memory
    {
      C uu[4], nu[4];
      T tau = 0, ntau = 0;
      if (n >= 3) load_refl(w, n, n - 3, lane, uu, tau);
      for (int k = n - 3; k >= 0; --k) {
        if (k > 0) load_refl(w, n, k - 1, lane, nu, ntau);
        if (tau != T(0)) {
          const int m = n - k - 1;
          C sacc = mk<T>(0, 0);
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const int i = lane + 32 * t;
            if (i < m) {
              const C zi = z[k + 1 + i];
              sacc.x += uu[t].x * zi.x + uu[t].y * zi.y;
              sacc.y += uu[t].x * zi.y - uu[t].y * zi.x;
            }
          }
          sacc.x = warp_sum(sacc.x);
          sacc.y = warp_sum(sacc.y);
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const int i = lane + 32 * t;
            if (i < m) {
              const C tt = cmul_t(uu[t], sacc);
              z[k + 1 + i].x -= tau * tt.x;
              z[k + 1 + i].y -= tau * tt.y;
            }
          }
          __syncwarp();
        }
#pragma unroll
        for (int t = 0; t < 4; ++t) uu[t] = nu[t];
        tau = ntau;
      }
    }
    // normalise to the reference image
    const bool singular = (sing[pt] & kRouteSingular) != 0;
    const C zr = z[ref];
    for (int i = lane; i < n; i += 32) {
      const C v = cmulc_t(z[i], zr);
      const double vx = v.x, vy = v.y, a = sqrt(vx * vx + vy * vy);
      float2 o = make_float2((float)(vx / a), (float)(vy / a));
      if (singular) o = make_float2(fnan, fnan);
      ph[gp * n + i] = o;
      phs[i] = make_double2(o.x, o.y);
    }
    if (lane == 0) quality[gp] = singular ? fnan : (float)lam;
    __syncwarp();
    if (tcoh) {  // |sum_q coh_q/|coh_q| conj(ph_m) ph_j| / n_pairs
      const float2* c = coh + gp * npairs;
      double tx = 0, ty = 0;
      int mm = 0, jj = 1 + lane;
      while (jj >= n && mm < n - 1) { mm += 1; jj = jj - n + mm + 1; }
      for (int64_t q = lane; q < npairs; q += 32) {
        const int m0 = mm, j0 = jj;
        jj += 32;
        while (jj >= n && mm < n - 1) { mm += 1; jj = jj - n + mm + 1; }
        const float2 g = c[q];
        const double ga = sqrt((double)g.x * g.x + (double)g.y * g.y);
        const double2 v = cmul(make_double2(g.x / ga, g.y / ga), cmulc(phs[j0], phs[m0]));
        tx += v.x;
        ty += v.y;
      }
      tx = warp_sum(tx);
      ty = warp_sum(ty);
      if (lane == 0) tcoh[gp] = (float)(sqrt(tx * tx + ty * ty) / (double)npairs);
    }
    __syncwarp();
  }
}


// ----------------------------------------------------------------- kernel 3b: refined tail
// For the refined mixed precision (FP64 inverse, FP32 reduction): the FP32 eigenvector is
// improved by one step of a Newton (Jacobi-Davidson) correction in FP64,
//   r = M v - lambda v (lambda = v^H M v, M = inv(|Gamma|) o Gamma from the FP64 inverse),
//   (M - lambda I) dv = r solved approximately through the FP32 factors M ~ Q D R D^H Q^H,
//   dv = Q D P (R - lambda I)^-1 P D^H Q^H r, P the projector orthogonal to R's eigenvector,
// which divides the error by about eps32 ||M|| / gap. Then the refined pair is checked in
// FP64: with residual r', gap g = lambda_2(R) - lambda and smallest component |v_i|, the
// phase error of every date is at most |r'| / (g min|v_i|); points above `tol` are flagged
// for an FP64 recomputation. One warp per point.
constexpr int kRefineWarps = 4;

__host__ __device__ inline size_t refine_warp_bytes(int n) {
  return align16(6 * (size_t)n * sizeof(float)) + align16(6 * (size_t)n * sizeof(double)) +
         3 * align16((size_t)n * sizeof(double2));
}

// Solve (R - lambda I) x = y in place, R real symmetric tridiagonal (d, b), by elimination
// with row interchanges, for a real (V = T) or complex (V = C2<T>) right-hand side. Each
// row's final pivot is inverted once and kept in dd, so the back substitution multiplies:
// one reciprocal per row on the serial chain instead of a division per row and component.
// dd, du, dl: work arrays of length n; dl ends as the second super-diagonal of each row.
template <typename T> __device__ __forceinline__ void axpy_r(T& y, T f, const T& x) { y -= f * x; }
template <typename T> __device__ __forceinline__ void axpy_r(typename C2<T>::type& y, T f,
                                                              const typename C2<T>::type& x) {
  y.x -= f * x.x;
  y.y -= f * x.y;
}
template <typename T> __device__ __forceinline__ void scale_r(T& y, T f) { y *= f; }
template <typename T> __device__ __forceinline__ void scale_r(typename C2<T>::type& y, T f) {
  y.x *= f;
  y.y *= f;
}

template <typename T, typename V>
__device__ inline void tridiag_solve_rcp(const T* d, const T* b, int n, T lambda, T tiny, V* y, T* dd, T* du,
                                         T* dl) {
  for (int i = 0; i < n; ++i) {
    dd[i] = d[i] - lambda;
    if (i < n - 1) { du[i] = b[i]; dl[i] = b[i]; }
  }
  for (int i = 0; i < n - 1; ++i) {
    const T sub = dl[i];
    if (fabs(dd[i]) >= fabs(sub)) {
      if (dd[i] == T(0)) dd[i] = tiny;
      const T r = recip(dd[i]);
      const T f = sub * r;
      dd[i + 1] -= f * du[i];
      axpy_r<T>(y[i + 1], f, y[i]);
      dl[i] = T(0);
      dd[i] = r;
    } else {
      const T r = recip(sub);
      const T f = dd[i] * r;
      const T t = dd[i + 1];
      dd[i + 1] = du[i] - f * t;
      if (i < n - 2) {
        dl[i] = du[i + 1];
        du[i + 1] = -f * dl[i];
      } else {
        dl[i] = T(0);
      }
      du[i] = t;
      const V ty = y[i];
      y[i] = y[i + 1];
      y[i + 1] = ty;
      axpy_r<T>(y[i + 1], f, y[i]);
      dd[i] = r;
    }
  }
  if (dd[n - 1] == T(0)) dd[n - 1] = tiny;
  scale_r<T>(y[n - 1], recip(dd[n - 1]));
  if (n > 1) {
    axpy_r<T>(y[n - 2], du[n - 2], y[n - 1]);
    scale_r<T>(y[n - 2], dd[n - 2]);
  }
  for (int i = n - 3; i >= 0; --i) {
    axpy_r<T>(y[i], du[i], y[i + 1]);
    axpy_r<T>(y[i], dl[i], y[i + 2]);
    scale_r<T>(y[i], dd[i]);
  }
}

// out = M v for M = inv(|Gamma|) o Gamma (Hermitian), read along the upper triangle: the
// element (m, j > m) adds M_mj v_j to row m and conj(M_mj) v_m to row j. Lanes own columns
// j = lane + 32 c; rows go four at a time through warp_sum4. One warp.
__device__ void herm_matvec(const double* __restrict__ ainv, const float2* __restrict__ c, int n,
                            const double2* v, double2* out) {
  constexpr int NC = (kMaxFastN + 31) / 32;
  const int lane = threadIdx.x & 31;
  double2 vj[NC], cacc[NC];
#pragma unroll
  for (int t = 0; t < NC; ++t) {
    const int j = lane + 32 * t;
    vj[t] = j < n ? v[j] : make_double2(0, 0);
    cacc[t] = make_double2(0, 0);
  }
  for (int m0 = 0; m0 < n; m0 += 4) {
    double2 racc[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      racc[r] = make_double2(0, 0);
      const int m = m0 + r;
      if (m >= n) continue;  // warp-uniform
      const double2 vm = v[m];
      const int64_t um = tri_up(m, m, n), qm = um - (m + 1);
#pragma unroll
      for (int t = 0; t < NC; ++t) {
        const int j = lane + 32 * t;
        if (j < m || j >= n) continue;
        const double s = ainv[um + (j - m)];
        if (j == m) {
          racc[r].x += s * vm.x;
          racc[r].y += s * vm.y;
        } else {
          const float2 g = c[qm + (j - m)];
          const double2 a = make_double2(s * (double)g.x, s * (double)g.y);  // M_mj
          cmac(racc[r], a, vj[t]);
          cmacc(cacc[t], a, vm);
        }
      }
    }
    const double2 tot = warp_sum4(racc);
    const int r = lane >> 3;
    if ((lane & 7) == 0 && m0 + r < n) out[m0 + r] = tot;
  }
  __syncwarp();
#pragma unroll
  for (int t = 0; t < NC; ++t) {
    const int j = lane + 32 * t;
    if (j < n) out[j] = cadd(out[j], cacc[t]);
  }
  __syncwarp();
}

// z <- H_k z for the reflectors of the workspace, k ascending (forward, Q^H z) or
// descending (back, Q z), in the arithmetic V of z (float2 or double2); the reflectors'
// stored values are used exactly. One warp.
template <typename V, typename T, typename TA>
__device__ void apply_q(const PointPtr<T, TA>& w, int n, typename C2<V>::type* z, bool forward) {
  using C = typename C2<T>::type;
  using CV = typename C2<V>::type;
  const int lane = threadIdx.x & 31;
  if (n < 3) return;
  C cu[4], nu[4];
  T ct = 0, nt = 0;
  load_refl(w, n, forward ? 0 : n - 3, lane, cu, ct);
  for (int s = 0; s + 2 < n; ++s) {
    const int k = forward ? s : n - 3 - s;
    if (s + 3 < n) load_refl(w, n, forward ? s + 1 : n - 4 - s, lane, nu, nt);  // the next one, early
    const V tau = (V)ct;
    if (tau != V(0)) {
      const int m = n - k - 1;
      CV acc = mk<V>(0, 0), uu[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int i = lane + 32 * t;
        uu[t] = mk<V>((V)cu[t].x, (V)cu[t].y);
        if (i < m) cmacc(acc, uu[t], z[k + 1 + i]);  // u^H z
      }
      acc.x = warp_sum(acc.x);
      acc.y = warp_sum(acc.y);
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int i = lane + 32 * t;
        if (i < m) {
          const CV tt = cmul(uu[t], acc);
          z[k + 1 + i].x -= tau * tt.x;
          z[k + 1 + i].y -= tau * tt.y;
        }
      }
      __syncwarp();
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) cu[t] = nu[t];
    ct = nt;
  }
}

// Smallest sigma (to the bisection's resolution) with at least `target` eigenvalues of the
// real tridiagonal (d, b2) at or below it, by multisection over the warp from [lo, hi].
template <typename T>
__device__ T multisect(const T* d, const T* b2, int n, T lo, T hi, int target, T pivmin, int rounds) {
  const int lane = threadIdx.x & 31;
  const T eps = Lim<T>::eps();
  for (int it = 0; it < rounds; ++it) {
    const T width = hi - lo;
    if (!(width > T(2) * eps * fmax(fabs(lo), fabs(hi)) + T(4) * pivmin)) break;
    const T sg = lo + width * (T)(lane + 1) / T(33);
    const int cnt = sturm_count(d, b2, n, sg, pivmin);
    const unsigned ball = __ballot_sync(0xffffffffu, cnt >= target);
    const int first = ball ? __ffs(ball) - 1 : 32;
    const T nlo = (first == 0) ? lo : lo + width * (T)first / T(33);
    const T nhi = (first == 32) ? hi : lo + width * (T)(first + 1) / T(33);
    lo = nlo;
    hi = nhi;
  }
  return T(0.5) * (lo + hi);
}

template <typename T>
__global__ void __launch_bounds__(32 * kRefineWarps, 4) tail_refine_kernel(
    const float2* __restrict__ coh, PointSet pts, int n, int ref, const unsigned char* __restrict__ ws,
    uint8_t* __restrict__ sing, float2* __restrict__ ph, float* __restrict__ quality, float* __restrict__ tcoh,
    double tol) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned char* mine = smem_raw + (size_t)wid * refine_warp_bytes(n);
  T* d = reinterpret_cast<T*>(mine);
  T* b = d + n;
  T* b2 = b + n;
  T* y = b2 + n;
  T* w1 = y + n;
  T* w2 = w1 + n;
  double* dd = reinterpret_cast<double*>(mine + align16(6 * (size_t)n * sizeof(float)));
  double* bd = dd + n;
  double* yd = bd + n;
  double* s1 = yd + n;
  double* s2 = s1 + n;
  double* s3 = s2 + n;
  float2* z32 = reinterpret_cast<float2*>(s1);  // FP32 work vector; s1 is scratch only inside the solve
  double2* dph = reinterpret_cast<double2*>(reinterpret_cast<unsigned char*>(dd) + align16(6 * (size_t)n * sizeof(double)));
  double2* v = dph + n;
  double2* t1 = v + n;
  const int64_t npairs = (int64_t)n * (n - 1) / 2;
  const float fnan = __int_as_float(0x7fffffff);
  const int64_t npt = pts.size();
  for (int64_t pt = (int64_t)blockIdx.x * kRefineWarps + wid; pt < npt; pt += (int64_t)gridDim.x * kRefineWarps) {
    const int64_t gp = pts[pt];
    const PointPtr<T, double> w(const_cast<unsigned char*>(ws), pt, n);
    const float2* c = coh + gp * npairs;
    // real tridiagonal R: b = |e|, phases delta_{k+1} = delta_k e_k/|e_k| (warp prefix product, FP64)
    double2 carry = make_double2(1, 0);
    for (int k0 = 0; k0 < n; k0 += 32) {
      const int k = k0 + lane;
      if (k < n) { d[k] = w.d[k]; dd[k] = (double)w.d[k]; }
      double2 f = make_double2(1, 0);
      if (k + 1 < n) {
        const typename C2<T>::type ek = w.e[k];
        const double ex = ek.x, ey = ek.y, a = sqrt(ex * ex + ey * ey);
        b[k] = (T)a;
        b2[k] = (T)a * (T)a;
        bd[k] = a;
        if (a > 0.0) f = make_double2(ex / a, ey / a);
      }
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const double ox = __shfl_up_sync(0xffffffffu, f.x, o), oy = __shfl_up_sync(0xffffffffu, f.y, o);
        if (lane >= o) f = cmul(make_double2(ox, oy), f);
      }
      const double2 dl = cmul(carry, f);
      if (k0 == 0 && lane == 0) dph[0] = make_double2(1, 0);
      if (k + 1 < n) dph[k + 1] = dl;
      carry = make_double2(__shfl_sync(0xffffffffu, dl.x, 31), __shfl_sync(0xffffffffu, dl.y, 31));
    }
    __syncwarp();
    // lambda_1 and lambda_2 of R (FP32 Sturm counts)
    T lo = Lim<T>::huge(), hi = -Lim<T>::huge(), tnorm = 0;
    for (int i = lane; i < n; i += 32) {
      const T r = (i > 0 ? b[i - 1] : T(0)) + (i + 1 < n ? b[i] : T(0));
      lo = fmin(lo, d[i] - r);
      hi = fmax(hi, d[i] + r);
      tnorm = fmax(tnorm, fabs(d[i]) + r);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
      tnorm = fmax(tnorm, __shfl_xor_sync(0xffffffffu, tnorm, o));
    }
    const T eps = Lim<T>::eps();
    const T pivmin = fmax(Lim<T>::tiny(), eps * eps * tnorm * tnorm) + Lim<T>::tiny();
    const T pad = T(2) * eps * fmax(tnorm, Lim<T>::tiny()) + T(2) * pivmin;
    lo -= pad;
    hi += pad;
    const T lam1 = multisect(d, b2, n, lo, hi, 1, pivmin, 64);
    // eigenvector y of R by inverse iteration (FP32, lane 0)
    for (int i = lane; i < n; i += 32) y[i] = T(1) + T(0.25) * (T)((i * 37) % 11) / T(11);
    __syncwarp();
    if (lane == 0) {
      const T tiny = eps * fmax(tnorm, Lim<T>::tiny());
      for (int it = 0; it < 2; ++it) {
        tridiag_solve_rcp(d, b, n, lam1, tiny, y, w1, w2, b2);  // b2 is free after the bisections
        T sc = 0;
        for (int i = 0; i < n; ++i) sc = fmax(sc, fabs(y[i]));
        if (!(sc > T(0)) || !isfinite(sc)) break;
        const T r = T(1) / sc;
        for (int i = 0; i < n; ++i) y[i] *= r;
      }
    }
    __syncwarp();
    // y to unit length in FP64; v = Q D y
    double yn = 0;
    for (int i = lane; i < n; i += 32) { yd[i] = (double)y[i]; yn += yd[i] * yd[i]; }
    yn = 1.0 / sqrt(warp_sum(yn));
    for (int i = lane; i < n; i += 32) {
      yd[i] *= yn;
      z32[i] = make_float2((float)(dph[i].x * yd[i]), (float)(dph[i].y * yd[i]));
    }
    __syncwarp();
    apply_q<float>(w, n, z32, false);
    for (int i = lane; i < n; i += 32) v[i] = make_double2(z32[i].x, z32[i].y);
    __syncwarp();
    // one correction step, then the check
    double lam = 0, rn = 0;
    for (int pass = 0; pass < 2; ++pass) {
      herm_matvec(w.ainv, c, n, v, t1);
      double vmv = 0, vv = 0;
      for (int i = lane; i < n; i += 32) {
        vmv += v[i].x * t1[i].x + v[i].y * t1[i].y;
        vv += v[i].x * v[i].x + v[i].y * v[i].y;
      }
      vv = warp_sum(vv);
      lam = warp_sum(vmv) / vv;
      double r2 = 0;
      for (int i = lane; i < n; i += 32) {
        t1[i] = make_double2(t1[i].x - lam * v[i].x, t1[i].y - lam * v[i].y);
        r2 += t1[i].x * t1[i].x + t1[i].y * t1[i].y;
      }
      rn = sqrt(warp_sum(r2) / vv);
      __syncwarp();
      if (pass == 1) break;
      // dv = Q D P (R - lam I)^-1 P D^H Q^H r; the reflectors are applied in FP32 (the factors
      // hold M only to FP32 accuracy anyway), the projected solve runs in FP64
      for (int i = lane; i < n; i += 32) z32[i] = make_float2((float)t1[i].x, (float)t1[i].y);
      __syncwarp();
      apply_q<float>(w, n, z32, true);
      double2 pr = make_double2(0, 0);
      for (int i = lane; i < n; i += 32) {
        t1[i] = cmulc(make_double2(z32[i].x, z32[i].y), dph[i]);  // D^H: times conj(delta_i)
        pr.x += yd[i] * t1[i].x;
        pr.y += yd[i] * t1[i].y;
      }
      pr.x = warp_sum(pr.x);
      pr.y = warp_sum(pr.y);
      for (int i = lane; i < n; i += 32) { t1[i].x -= yd[i] * pr.x; t1[i].y -= yd[i] * pr.y; }
      __syncwarp();
      if (lane == 0) tridiag_solve_rcp(dd, bd, n, lam, DBL_EPSILON * (double)tnorm + DBL_MIN, t1, s1, s2, s3);
      __syncwarp();
      pr = make_double2(0, 0);
      for (int i = lane; i < n; i += 32) { pr.x += yd[i] * t1[i].x; pr.y += yd[i] * t1[i].y; }
      pr.x = warp_sum(pr.x);
      pr.y = warp_sum(pr.y);
      for (int i = lane; i < n; i += 32) {
        const double2 x = cmul(make_double2(t1[i].x - yd[i] * pr.x, t1[i].y - yd[i] * pr.y), dph[i]);
        z32[i] = make_float2((float)x.x, (float)x.y);
      }
      __syncwarp();
      apply_q<float>(w, n, z32, false);
      double vn = 0;
      for (int i = lane; i < n; i += 32) {
        v[i] = make_double2(v[i].x - (double)z32[i].x, v[i].y - (double)z32[i].y);
        vn += v[i].x * v[i].x + v[i].y * v[i].y;
      }
      vn = 1.0 / sqrt(warp_sum(vn));
      for (int i = lane; i < n; i += 32) v[i] = make_double2(v[i].x * vn, v[i].y * vn);
      __syncwarp();
    }
    // phase error bound of the refined vector (v has unit length)
    double vmin = 1e300;
    for (int i = lane; i < n; i += 32) vmin = fmin(vmin, sqrt(v[i].x * v[i].x + v[i].y * v[i].y));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) vmin = fmin(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
    // |r'| / (gap min|v_i|) <= tol with gap = lambda_2(R) - lam - margin holds exactly when
    // lambda_2(R) >= sig = lam + margin + |r'| / (tol min|v_i|): one Sturm count at sig
    // (rounded up to FP32) answers it, without locating lambda_2
    const double sig = lam + 4.0 * (double)eps * (double)n * (double)tnorm + rn / (tol * vmin);
    for (int i = lane; i + 1 < n; i += 32) b2[i] = b[i] * b[i];  // b2 was the solves' scratch
    __syncwarp();
    float sg = (float)sig;
    if ((double)sg < sig) sg = nextafterf(sg, 3.4e38f);
    const bool gap_ok = sig < 3.0e38 && sturm_count(d, b2, n, (T)sg, pivmin) <= 1;  // NaN: false
    const bool singular = (sing[pt] & kRouteSingular) != 0;
    const bool small_pivot = (sing[pt] & kRouteCond) != 0;  // the sweep's inverse is not trusted
    const bool ok = singular || (!small_pivot && gap_ok);
    // normalise to the reference image
    const double2 zr = v[ref];
    for (int i = lane; i < n; i += 32) {
      const double2 q = cmulc(v[i], zr);
      const double a = sqrt(q.x * q.x + q.y * q.y);
      float2 o = make_float2((float)(q.x / a), (float)(q.y / a));
      if (singular) o = make_float2(fnan, fnan);
      ph[gp * n + i] = o;
      t1[i] = make_double2(o.x, o.y);
    }
    __syncwarp();
    if (lane == 0) {
      quality[gp] = singular ? fnan : (float)lam;
      sing[pt] = singular ? kRouteSingular : (ok ? 0 : kRouteCond);
    }
    if (tcoh) {  // |sum_q coh_q/|coh_q| conj(ph_m) ph_j| / n_pairs
      double tx = 0, ty = 0;
      int mm = 0, jj = 1 + lane;
      while (jj >= n && mm < n - 1) { mm += 1; jj = jj - n + mm + 1; }
      for (int64_t q = lane; q < npairs; q += 32) {
        const int m0 = mm, j0 = jj;
        jj += 32;
        while (jj >= n && mm < n - 1) { mm += 1; jj = jj - n + mm + 1; }
        const float2 g = c[q];
        const double ga = sqrt((double)g.x * g.x + (double)g.y * g.y);
        const double2 q2 = cmul(make_double2(g.x / ga, g.y / ga), cmulc(t1[j0], t1[m0]));
        tx += q2.x;
        ty += q2.y;
      }
      tx = warp_sum(tx);
      ty = warp_sum(ty);
      if (lane == 0) tcoh[gp] = (float)(sqrt(tx * tx + ty * ty) / (double)npairs);
    }
    __syncwarp();
  }
}

// ----------------------------------------------------------------- host side
template <class K>
int occupancy(K kernel, int threads, size_t smem) {
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, smem) != cudaSuccess) return 0;
  return occ;
}

// Most points of a sub-batch: its per-point workspace within 4 GiB (about 34,600 points at
// N = 100), so that each launch has enough points to keep every SM busy to its end.
template <typename T>
int64_t sub_batch(int n) {
  const PointWs<T> w(n);  // FP64 sub-batches also fit the refined layout (it is smaller)
  const int64_t def = (int64_t)std::max<size_t>(1024, std::min<size_t>(1 << 17, (size_t)(1ull << 32) / (w.bytes + 1)));
  const int64_t cap = g_sub_batch_cap.load();
  return cap > 0 ? std::min(cap, def) : def;
}

// Workspace of one sub-batch of `sub` points: per-point state of the widest arithmetic
// used and the route flags of the FP32 and FP64 passes; then, for all `n_list` points of the
// call, the list of points to redo in FP64 and its count. The redo runs once after every
// sub-batch, so the few routed points of a call share launches instead of running a
// nearly empty pass per sub-batch.
struct SubWs {
  unsigned char* pts;
  uint8_t* sing;
  uint8_t* sing2;
  int32_t* list;
  int32_t* count;
  static size_t bytes(int64_t sub, size_t point_bytes, int64_t n_list) {
    return align16((size_t)sub * point_bytes) + 2 * align16((size_t)sub) + align16(4 * (size_t)n_list) + 16;
  }
  SubWs(unsigned char* ws, int64_t sub, size_t point_bytes, int64_t n_list) {
    unsigned char* b = ws;
    pts = b;
    b += align16((size_t)sub * point_bytes);
    sing = b;
    b += align16((size_t)sub);
    sing2 = b;
    b += align16((size_t)sub);
    list = reinterpret_cast<int32_t*>(b);
    b += align16(4 * (size_t)n_list);
    count = reinterpret_cast<int32_t*>(b);
  }
};

// Appends the points of a sub-batch (global indices b0 + i) that are to be redone in FP64 to
// the list. `refined`: points singular in the (already FP64) inverse are not redone. With a
// device-held point count (dcount, the sub-batch starting at point doff of it) only the
// points below it are read.
__global__ void route_kernel(const uint8_t* __restrict__ sing, int64_t nb, int64_t b0, int32_t* __restrict__ list,
                             int32_t* __restrict__ count, uint8_t* __restrict__ route, bool refined,
                             const int64_t* __restrict__ dcount, int64_t doff) {
  if (dcount) {
    const int64_t c = *dcount - doff;
    nb = c < 0 ? 0 : (c < nb ? c : nb);
  }
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += (int64_t)gridDim.x * blockDim.x) {
    const uint8_t f = sing[i];
    if (route) route[i] = f;
    if (f && !(refined && f == kRouteSingular)) list[atomicAdd(count, 1)] = (int32_t)(b0 + i);  // order is free
  }
}

// Column groups of the Gauss-Jordan grid. 32 groups (512 threads, half the registers per
// thread) measured no faster than 16 in FP32 or FP64: one point per SM either way, and its
// serial pivot steps set the pace. With look-ahead pivoting the 512-thread tile stayed in
// local memory (128 registers per thread), twice as slow.
template <typename T>
constexpr int gj_cx() { return 16; }

template <typename T, int NB, typename TW>
int launch_inverse(const float2* coh, PointSet pts, int64_t grid_cap, int n, unsigned char* ws, uint8_t* sing,
                   float cond_max, cudaStream_t s) {
  constexpr int CX = gj_cx<T>();
  const int occ = std::max(1, occupancy(inverse_kernel<T, NB, CX, TW>, 16 * CX, 0));
  const int64_t grid = std::min<int64_t>(grid_cap, (int64_t)sm_count() * occ);
  KernelTimer kt(pts.list ? "emi inverse rerun" : sizeof(T) == 8 ? "emi inverse fp64" : "emi inverse fp32", s);
  inverse_kernel<T, NB, CX, TW><<<(unsigned)grid, 16 * CX, 0, s>>>(coh, pts, n, ws, sing, cond_max);
  return check_launch("emi inverse");
}

// inv(|Gamma|) in arithmetic TA into a workspace laid out for a reduction in T.
template <typename TA, typename T>
int run_inverse(const float2* c, PointSet pts, int n, unsigned char* ws, uint8_t* sing, float cond_max,
                cudaStream_t s) {
  const int64_t cap = pts.n_pc;  // grid bound: the most points this pass can see
  switch ((n + 15) / 16) {
    case 1: case 2: return launch_inverse<TA, 2, T>(c, pts, cap, n, ws, sing, cond_max, s);
    case 3: return launch_inverse<TA, 3, T>(c, pts, cap, n, ws, sing, cond_max, s);
    case 4: return launch_inverse<TA, 4, T>(c, pts, cap, n, ws, sing, cond_max, s);
    case 5: return launch_inverse<TA, 5, T>(c, pts, cap, n, ws, sing, cond_max, s);
    case 6: return launch_inverse<TA, 6, T>(c, pts, cap, n, ws, sing, cond_max, s);
    case 7: return launch_inverse<TA, 7, T>(c, pts, cap, n, ws, sing, cond_max, s);
    default: return launch_inverse<TA, 8, T>(c, pts, cap, n, ws, sing, cond_max, s);
  }
}

template <typename T, typename TA>
int run_reduce(const float2* c, PointSet pts, int n, unsigned char* ws, cudaStream_t s) {
  const size_t rsmem = tri_bytes<T>(n);
  if (int rc_ = allow_smem(reinterpret_cast<const void*>(reduce_kernel<T, TA>), (size_t)(rsmem))) return rc_;
  const int rocc = occupancy(reduce_kernel<T, TA>, kThreads, rsmem);
  if (rocc < 1) return fail(MR_ERR_UNSUPPORTED, "emi: %zu bytes of shared memory per CTA do not fit", rsmem);
  KernelTimer kt(pts.list ? "emi reduce rerun" : sizeof(T) == 8 ? "emi reduce fp64" : "emi reduce fp32", s);
  reduce_kernel<T, TA><<<(unsigned)std::min<int64_t>(pts.n_pc, (int64_t)sm_count() * rocc), kThreads, rsmem, s>>>(
      c, pts, n, ws);
  return check_launch("emi reduce");
}

// One pass of the three kernels over a sub-batch (pts.list == nullptr: all pts.n_pc points;
// else the listed ones, whose count is read on the device), inverse and reduction both in
// T. cond_max > 0 flags the points whose condition estimate exceeds it.
template <typename T>
int run_pass(const float2* c, PointSet pts, int n, int ref, float2* ph, float* quality, float* tcoh,
             unsigned char* ws, uint8_t* sing, float cond_max, cudaStream_t s) {
  if (int rc = run_inverse<T, T>(c, pts, n, ws, sing, cond_max, s)) return rc;
  if (int rc = run_reduce<T, T>(c, pts, n, ws, s)) return rc;
  const size_t tsmem = kTailWarps * tail_warp_bytes<T>(n);
  if (int rc_ = allow_smem(reinterpret_cast<const void*>(tail_kernel<T, T>), (size_t)(tsmem))) return rc_;
  const int tocc = std::max(1, occupancy(tail_kernel<T, T>, 32 * kTailWarps, tsmem));
  const int64_t tgrid = std::min<int64_t>((pts.n_pc + kTailWarps - 1) / kTailWarps, (int64_t)sm_count() * tocc);
  KernelTimer kt(pts.list ? "emi tail rerun" : sizeof(T) == 8 ? "emi tail fp64" : "emi tail fp32", s);
  tail_kernel<T, T><<<(unsigned)tgrid, 32 * kTailWarps, tsmem, s>>>(c, pts, n, ref, ws, sing, ph, quality, tcoh);
  return check_launch("emi tail");
}

template <int NB>
int launch_sweep(const float2* c, PointSet pts, int n, unsigned char* ws, uint8_t* sing, cudaStream_t s) {
  const int occ = std::max(1, occupancy(sweep_kernel<NB, float>, 256, 0));
  const int64_t grid = std::min<int64_t>(pts.n_pc, (int64_t)sm_count() * occ);
  KernelTimer kt(pts.list ? "emi sweep rerun" : "emi sweep fp64", s);
  sweep_kernel<NB, float><<<(unsigned)grid, 256, 0, s>>>(c, pts, n, ws, sing);
  return check_launch("emi sweep");
}

int run_sweep(const float2* c, PointSet pts, int n, unsigned char* ws, uint8_t* sing, cudaStream_t s) {
  switch ((n + 15) / 16) {
    case 1: case 2: return launch_sweep<2>(c, pts, n, ws, sing, s);
    case 3: return launch_sweep<3>(c, pts, n, ws, sing, s);
    case 4: return launch_sweep<4>(c, pts, n, ws, sing, s);
    case 5: return launch_sweep<5>(c, pts, n, ws, sing, s);
    case 6: return launch_sweep<6>(c, pts, n, ws, sing, s);
    case 7: return launch_sweep<7>(c, pts, n, ws, sing, s);
    default: return launch_sweep<8>(c, pts, n, ws, sing, s);
  }
}

// The refined pass: FP64 inverse (symmetric sweep), FP32 reduction, FP64-refined tail;
// sing[] ends with the points whose sweep met a small pivot or whose refined error bound
// exceeds `tol` flagged kRouteCond.
int run_refine_pass(const float2* c, PointSet pts, int n, int ref, float2* ph, float* quality, float* tcoh,
                    unsigned char* ws, uint8_t* sing, double tol, cudaStream_t s) {
  if (int rc = run_sweep(c, pts, n, ws, sing, s)) return rc;
  if (int rc = run_reduce<float, double>(c, pts, n, ws, s)) return rc;
  const size_t tsmem = kRefineWarps * refine_warp_bytes(n);
  if (int rc_ = allow_smem(reinterpret_cast<const void*>(tail_refine_kernel<float>), tsmem)) return rc_;
  const int tocc = std::max(1, occupancy(tail_refine_kernel<float>, 32 * kRefineWarps, tsmem));
  const int64_t tgrid = std::min<int64_t>((pts.n_pc + kRefineWarps - 1) / kRefineWarps, (int64_t)sm_count() * tocc);
  KernelTimer kt("emi refine tail", s);
  tail_refine_kernel<float><<<(unsigned)tgrid, 32 * kRefineWarps, tsmem, s>>>(c, pts, n, ref, ws, sing, ph,
                                                                                quality, tcoh, tol);
  return check_launch("emi refine tail");
}

size_t point_bytes_max(int n) {
  return std::max({PointWs<float>(n).bytes, PointWs<double>(n).bytes, PointWs<float, double>(n).bytes});
}

}  // namespace

int fast_supported(int n) { return n >= 2 && n <= kMaxFastN; }

size_t fast_workspace_bytes(int64_t n_pc, int n) {
  const int64_t s32 = std::min<int64_t>(n_pc, sub_batch<float>(n));
  const int64_t s64 = std::min<int64_t>(n_pc, sub_batch<double>(n));
  return std::max(SubWs::bytes(s32, PointWs<float>(n).bytes, n_pc), SubWs::bytes(s64, point_bytes_max(n), n_pc));
}

int fast_run(const float2* coh, int64_t n_pc, int n, int ref, int precision, float cond_max, float2* ph,
             float* quality, float* tcoh, uint8_t* route, void* workspace, cudaStream_t s,
             const int64_t* dcount, int64_t doff) {
  const bool f64 = precision == MR_PREC_FP64;
  const bool mixed = precision == MR_PREC_MIXED;
  const bool refine = precision == MR_PREC_REFINE;
  if (dcount && mixed) return fail(MR_ERR_UNSUPPORTED, "emi: device-counted points run in FP32, FP64 or refined");
  auto* ws = static_cast<unsigned char*>(workspace);
  // a mixed or refined sub-batch must hold its points in FP64 when all of them are routed
  const bool wide = f64 || mixed || refine;
  // sub-batches of equal size (none left nearly empty at the end)
  const int64_t cap = wide ? sub_batch<double>(n) : sub_batch<float>(n);
  const int64_t nsub = (n_pc + cap - 1) / cap;
  const int64_t sub = nsub > 0 ? (n_pc + nsub - 1) / nsub : 0;
  const SubWs w(ws, sub, wide ? point_bytes_max(n) : PointWs<float>(n).bytes, n_pc);
  const int64_t npairs = (int64_t)n * (n - 1) / 2;
  const bool routed = mixed || refine;
  if (routed) MR_CUDA_TRY(cudaMemsetAsync(w.count, 0, sizeof(int32_t), s));
  for (int64_t b0 = 0; b0 < n_pc; b0 += sub) {
    const int64_t nb = std::min<int64_t>(sub, n_pc - b0);
    const float2* c = coh + b0 * npairs;
    float2* p = ph + b0 * n;
    float* q = quality + b0;
    float* t = tcoh ? tcoh + b0 : nullptr;
    const PointSet all{nullptr, nullptr, nb, dcount, doff + b0};
    int rc;
    if (f64) {
      rc = run_pass<double>(c, all, n, ref, p, q, t, w.pts, w.sing, 0.f, s);
      if (!rc && route) MR_CUDA_TRY(cudaMemsetAsync(route + b0, 1, (size_t)nb, s));
    } else {
      rc = refine ? run_refine_pass(c, all, n, ref, p, q, t, w.pts, w.sing, (double)cond_max, s)
                  : run_pass<float>(c, all, n, ref, p, q, t, w.pts, w.sing, mixed ? cond_max : 0.f, s);
      if (!rc && routed) {
        const int grid = (int)std::min<int64_t>((nb + 255) / 256, (int64_t)sm_count() * 8);
        route_kernel<<<grid, 256, 0, s>>>(w.sing, nb, b0, w.list, w.count, route ? route + b0 : nullptr, refine,
                                          dcount, doff + b0);
        rc = check_launch("emi route");
      } else if (!rc && route) {
        MR_CUDA_TRY(cudaMemsetAsync(route + b0, 0, (size_t)nb, s));
      }
    }
    if (rc) return rc;
  }
  // the routed points of every sub-batch, in FP64, in windows of `sub` list entries (the
  // count is known only on the device: windows past it exit at once)
  if (routed) {
    for (int64_t l0 = 0; l0 < n_pc; l0 += sub) {
      const int rc = run_pass<double>(coh, PointSet{w.list, w.count, sub, nullptr, l0}, n, ref, ph, quality, tcoh,
                                      w.pts, w.sing2, 0.f, s);
      if (rc) return rc;
    }
  }
  return MR_OK;
}

}  // namespace emi
}  // namespace mr
