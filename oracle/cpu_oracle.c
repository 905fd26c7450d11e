/*
 * CPU oracle of the distributed-scatterer chain — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference algorithms, used by the tests, the package's
 * smoke check and the benchmark's CPU-baseline leg as the checker. It is never called by
 * the product path. Each function cites the reference file:line it follows
 * (kanglcn/moraine, paths inside that project).
 *
 * Build: see oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off -shared).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* moraine/shp.py:20-32: p = sum_{i=1..100} (-1)^(i-1) 2 exp(-2 i^2 x^2), stopping when the
 * partial sum repeats. Same operation order as the reference, in double. */
double oracle_ks_p(double x) {
  double x2 = -2 * x * x;
  double p = 0.0, p2 = 0.0;
  int sign = 1;
  for (int i = 1; i <= 100; ++i) {
    p += (double)(sign * 2) * exp(x2 * (double)i * (double)i);
    if (p == p2) return p;
    sign = -sign;
    p2 = p;
  }
  return p;
}

/* moraine/shp.py:36-44: merge of two ascending samples; ties advance both indices;
 * returns max |j2 - j1| (the statistic times n). */
static int ks_merge_count(const float* ref, const float* sec, int n) {
  int j1 = 0, j2 = 0, dmax = 0;
  while (j1 < n && j2 < n) {
    float f1 = ref[j1], f2 = sec[j2];
    if (f1 <= f2) j1 += 1;
    if (f1 >= f2) j2 += 1;
    int d = abs(j2 - j1);
    if (d > dmax) dmax = d;
  }
  return dmax;
}

/* ascending, NaN last (numpy.sort order) */
static int cmp_nan_last(const void* a, const void* b) {
  float x = *(const float*)a, y = *(const float*)b;
  int nx = isnan(x), ny = isnan(y);
  if (nx || ny) return nx - ny;
  return (x > y) - (x < y);
}

/* moraine/shp.py:117-125 (per-pixel sort) + :80-113 (window loop, NaN rules) +
 * :74-76 (x = (en + 0.12 + 0.11/en) * D). dist may be NULL. */
void oracle_ks_test(const float* rmli, int nlines, int width, int n, int azh, int rh, float* p,
                    float* dist, int nthreads) {
  const int64_t npix = (int64_t)nlines * width;
  const int az_win = 2 * azh + 1, r_win = 2 * rh + 1, win = az_win * r_win;
  float* sorted = (float*)malloc(sizeof(float) * npix * n);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
  for (int64_t i = 0; i < npix; ++i) {
    memcpy(sorted + i * n, rmli + i * n, sizeof(float) * n);
    qsort(sorted + i * n, n, sizeof(float), cmp_nan_last);
  }
  const double en = sqrt((double)n / 2);
  const double scale = en + 0.12 + 0.11 / en;
  const float fnan = nanf("");
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16)
#endif
  for (int64_t pix = 0; pix < npix; ++pix) {
    const int i = (int)(pix / width), j = (int)(pix % width);
    const float* ref = sorted + pix * n;
    const int ref_nan = isnan(ref[n - 1]);
    for (int l = -azh; l <= azh; ++l)
      for (int m = -rh; m <= rh; ++m) {
        const int64_t o = pix * win + (l + azh) * r_win + (m + rh);
        const int si = i + l, sj = j + m;
        if (ref_nan || si < 0 || si >= nlines || sj < 0 || sj >= width) {
          p[o] = fnan;
          if (dist) dist[o] = fnan;
          continue;
        }
        const float* sec = sorted + ((int64_t)si * width + sj) * n;
        if (isnan(sec[n - 1])) {
          p[o] = fnan;
          if (dist) dist[o] = fnan;
          continue;
        }
        const int k = ks_merge_count(ref, sec, n);
        const double d = fabs((double)k / (double)n);
        if (dist) dist[o] = (float)d;
        p[o] = (float)oracle_ks_p(scale * d);
      }
  }
  free(sorted);
}

/* ks_test followed by select_shp (moraine/shp.py:269-323) without the p array: p depends
 * only on the integer statistic k, so the decision (double)(float)p(k) < p_max is taken
 * from a table of p over k = 0..n built with the same expression as oracle_ks_test
 * (moraine/shp.py:74-76, :20-32). is_shp: (nlines, width, az_win, r_win) bytes; shp_num:
 * (nlines, width) counts. For whole scenes, where the float p array would not fit. */
void oracle_ks_select(const float* rmli, int nlines, int width, int n, int azh, int rh, double p_max,
                      uint8_t* is_shp, int32_t* shp_num, int nthreads) {
  const int64_t npix = (int64_t)nlines * width;
  const int az_win = 2 * azh + 1, r_win = 2 * rh + 1, win = az_win * r_win;
  const double en = sqrt((double)n / 2);
  const double scale = en + 0.12 + 0.11 / en;
  uint8_t* accept = (uint8_t*)malloc((size_t)n + 1);
  for (int k = 0; k <= n; ++k) {
    const double d = fabs((double)k / (double)n);
    accept[k] = (double)(float)oracle_ks_p(scale * d) < p_max;
  }
  float* sorted = (float*)malloc(sizeof(float) * npix * n);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
  for (int64_t i = 0; i < npix; ++i) {
    memcpy(sorted + i * n, rmli + i * n, sizeof(float) * n);
    qsort(sorted + i * n, n, sizeof(float), cmp_nan_last);
  }
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64)
#endif
  for (int64_t pix = 0; pix < npix; ++pix) {
    const int i = (int)(pix / width), j = (int)(pix % width);
    const float* ref = sorted + pix * n;
    const int ref_nan = isnan(ref[n - 1]);
    int32_t count = 0;
    for (int l = -azh; l <= azh; ++l)
      for (int m = -rh; m <= rh; ++m) {
        const int64_t o = pix * win + (l + azh) * r_win + (m + rh);
        const int si = i + l, sj = j + m;
        uint8_t a = 0;
        if (!ref_nan && si >= 0 && si < nlines && sj >= 0 && sj < width) {
          const float* sec = sorted + ((int64_t)si * width + sj) * n;
          if (!isnan(sec[n - 1])) a = accept[ks_merge_count(ref, sec, n)];
        }
        is_shp[o] = a;
        count += a;
      }
    shp_num[pix] = count;
  }
  free(sorted);
  free(accept);
}

/* moraine/co.py:209-226 (CPU path, float64 accumulation) and :164-187 (window order).
 * mask: (n_pc, az_win, r_win) bytes; pairs: (npairs, 2) int32; coh: complex128 out. */
void oracle_co_pc(const float* rslc /* complex64 interleaved */, int nlines, int width, int n,
                  const int32_t* idx, int64_t n_pc, const uint8_t* mask, int az_win, int r_win,
                  const int32_t* pairs, int npairs, double* coh /* complex128 interleaved */,
                  int nthreads) {
  const int azh = az_win / 2, rh = r_win / 2, win = az_win * r_win;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 8)
#endif
  for (int64_t i = 0; i < n_pc; ++i) {
    for (int q = 0; q < npairs; ++q) {
      const int mm = pairs[2 * q], jj = pairs[2 * q + 1];
      double nr = 0, ni = 0, am = 0, aj = 0;
      for (int k = 0; k < az_win; ++k)
        for (int l = 0; l < r_win; ++l) {
          const int a = idx[2 * i] - azh + k, r = idx[2 * i + 1] - rh + l;
          if (a >= 0 && a < nlines && r >= 0 && r < width && mask[i * win + k * r_win + l]) {
            const float* zm = rslc + 2 * (((int64_t)a * width + r) * n + mm);
            const float* zj = rslc + 2 * (((int64_t)a * width + r) * n + jj);
            const double xr = zm[0], xi = zm[1], yr = zj[0], yi = zj[1];
            am += xr * xr + xi * xi;
            aj += yr * yr + yi * yi;
            nr += xr * yr + xi * yi;
            ni += xi * yr - xr * yi;
          }
        }
      const double den = sqrt(am * aj);
      coh[2 * (i * npairs + q)] = nr / den;
      coh[2 * (i * npairs + q) + 1] = ni / den;
    }
  }
}

/* moraine/co.py:83-110: raster covariance (sum / n_shp) and coherence, every (m, j). */
void oracle_co_raster(const float* rslc, int nlines, int width, int n, const uint8_t* is_shp, int az_win,
                      int r_win, double* cov, double* coh, int nthreads) {
  const int azh = az_win / 2, rh = r_win / 2, win = az_win * r_win;
  const int64_t npix = (int64_t)nlines * width;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 8)
#endif
  for (int64_t pix = 0; pix < npix; ++pix) {
    const int ra = (int)(pix / width), rr = (int)(pix % width);
    for (int mm = 0; mm < n; ++mm)
      for (int jj = 0; jj < n; ++jj) {
        double nr = 0, ni = 0, am = 0, aj = 0;
        int cnt = 0;
        for (int k = 0; k < az_win; ++k)
          for (int l = 0; l < r_win; ++l) {
            const int a = ra - azh + k, r = rr - rh + l;
            if (is_shp[pix * win + k * r_win + l] && a >= 0 && a < nlines && r >= 0 && r < width) {
              const float* zm = rslc + 2 * (((int64_t)a * width + r) * n + mm);
              const float* zj = rslc + 2 * (((int64_t)a * width + r) * n + jj);
              const double xr = zm[0], xi = zm[1], yr = zj[0], yi = zj[1];
              am += xr * xr + xi * xi;
              aj += yr * yr + yi * yi;
              nr += xr * yr + xi * yi;
              ni += xi * yr - xr * yi;
              cnt += 1;
            }
          }
        const int64_t o = 2 * ((pix * n + mm) * n + jj);
        const double den = sqrt(am * aj);
        coh[o] = nr / den;
        coh[o + 1] = ni / den;
        cov[o] = nr / cnt;
        cov[o + 1] = ni / cnt;
      }
  }
}

/* moraine/pl.py:90-99 (ds_temp_coh, pqm = 0) and moraine/pqm.py:56-70 (temp_coh, pqm = 1):
 * double-precision sums over the pairs. */
void oracle_temp_coh(const float* intf, const float* ph, int64_t npts, int n, const int32_t* pairs, int npairs,
                     int pqm, double* out, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
  for (int64_t i = 0; i < npts; ++i) {
    double sr = 0, si = 0;
    for (int q = 0; q < npairs; ++q) {
      const int mm = pairs[2 * q], jj = pairs[2 * q + 1];
      const float* g = intf + 2 * (i * npairs + q);
      const float* pm = ph + 2 * (i * n + mm);
      const float* pj = ph + 2 * (i * n + jj);
      double gr = g[0], gi = g[1];
      double ga = sqrt(gr * gr + gi * gi);
      double mr = pm[0], mi = pm[1], jr = pj[0], ji = pj[1];
      if (pqm) {
        double ma = sqrt(mr * mr + mi * mi), ja = sqrt(jr * jr + ji * ji);
        mr /= ma; mi /= ma; jr /= ja; ji /= ja;
      }
      gr /= ga; gi /= ga;
      /* conj(ph_m) * ph_j */
      const double tr = mr * jr + mi * ji, ti = mr * ji - mi * jr;
      sr += gr * tr - gi * ti;
      si += gr * ti + gi * tr;
    }
    out[i] = sqrt(sr * sr + si * si) / npairs;
  }
}
