// Per-pixel symmetric 3x3 (or 1x1) pixel-matrix algebra on the device.
//
// Follows matrix.f90 of the reference: test_decoupling 15-51, invert_eig
// 53-126, invert_eig_s 132-179, invert_LU 287-327, and the pixmode rules of
// invert_pixelmatrix_cross / invert_pixelmatrix_map (map_routines.f90:83-321).
// LAPACK's DSYEV is replaced by cyclic Jacobi rotations, DPOTRF/DPOTRI by a
// Cholesky factor and the product of the inverse factors.
#pragma once

#include "params.h"

namespace madam {

#define MADAM_HD __host__ __device__ __forceinline__

// a is 3x3 column-major, upper triangle read.  w ascending, v columns.
MADAM_HD int jacobi3(int n, const double *a, double *w, double *v) {
  double A[9];
  for (int j = 0; j < n; ++j)
    for (int i = 0; i <= j; ++i) {
      A[i + 3 * j] = a[i + 3 * j];
      A[j + 3 * i] = a[i + 3 * j];
    }
  for (int i = 0; i < 9; ++i) v[i] = 0;
  for (int i = 0; i < n; ++i) v[i + 3 * i] = 1;
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = 0, diag = 0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        const double x = A[i + 3 * j] * A[i + 3 * j];
        if (i != j) off += x;
        else diag += x;
      }
    if (off == 0 || off <= 1e-34 * diag) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = A[p + 3 * q];
        if (apq == 0) continue;
        const double app = A[p + 3 * p], aqq = A[q + 3 * q];
        const double theta = (aqq - app) / (2 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
        if (isinf(theta)) t = 0.5 / theta;
        const double c = 1 / sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < n; ++k) {
          const double akp = A[k + 3 * p], akq = A[k + 3 * q];
          A[k + 3 * p] = c * akp - s * akq;
          A[k + 3 * q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = A[p + 3 * k], aqk = A[q + 3 * k];
          A[p + 3 * k] = c * apk - s * aqk;
          A[q + 3 * k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = v[k + 3 * p], vkq = v[k + 3 * q];
          v[k + 3 * p] = c * vkp - s * vkq;
          v[k + 3 * q] = s * vkp + c * vkq;
        }
      }
  }
  for (int i = 0; i < n; ++i) w[i] = A[i + 3 * i];
  for (int i = 0; i < n; ++i) {
    int m = i;
    for (int j = i + 1; j < n; ++j)
      if (w[j] < w[m]) m = j;
    if (m != i) {
      const double t = w[i];
      w[i] = w[m];
      w[m] = t;
      for (int k = 0; k < n; ++k) {
        const double tv = v[k + 3 * i];
        v[k + 3 * i] = v[k + 3 * m];
        v[k + 3 * m] = tv;
      }
    }
  }
  for (int i = 0; i < n; ++i)
    if (isnan(w[i])) return 1;
  return 0;
}

// Sub-block [s..3) x [s..3) of the 3x3 column-major matrix c.
MADAM_HD void invert_eig_sub(double *c, int s, bool incomplete, double &cdet, double &rcond,
                             bool &sing) {
  const int n = 3 - s;
  int good[3], nf = 0;
  if (incomplete) {
    for (int i = 0; i < n; ++i)
      if (fabs(c[(s + i) + 3 * (s + i)]) > fsp(1e-30f)) good[nf++] = s + i;
    if (nf == 0) good[nf++] = s;
  } else {
    for (int i = 0; i < n; ++i) good[nf++] = s + i;
  }
  double a[9] = {0}, w[3] = {0}, v[9];
  for (int j = 0; j < nf; ++j)
    for (int i = 0; i < nf; ++i) a[i + 3 * j] = c[good[i] + 3 * good[j]];
  const int info = jacobi3(nf, a, w, v);
  cdet = 1;
  double mn = w[0], mx = w[0];
  for (int i = 0; i < nf; ++i) {
    cdet *= w[i];
    mn = fmin(mn, w[i]);
    mx = fmax(mx, w[i]);
  }
  rcond = mn / mx;
  if (info != 0 || mx < fsp(1e-30f) || rcond < fsp(1e-12f)) {
    sing = true;
    for (int j = s; j < 3; ++j)
      for (int i = s; i < 3; ++i) c[i + 3 * j] = 0;
    cdet = 0;
    rcond = 0;
    return;
  }
  sing = false;
  for (int j = 0; j < nf; ++j)
    for (int i = 0; i < nf; ++i) {
      double acc = 0;
      for (int k = 0; k < nf; ++k) acc += (v[i + 3 * k] / w[k]) * v[j + 3 * k];
      c[good[i] + 3 * good[j]] = acc;
    }
}

MADAM_HD void invert_eig_s_sub(double *c, int s, double plim, double &cdet, double &rcond,
                               int &noeig) {
  const int n = 3 - s;
  double a[9] = {0}, w[3] = {0}, v[9];
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) a[i + 3 * j] = c[(s + i) + 3 * (s + j)];
  const int info = jacobi3(n, a, w, v);
  cdet = 1;
  double mn = w[0], mx = w[0];
  for (int i = 0; i < n; ++i) {
    cdet *= w[i];
    mn = fmin(mn, w[i]);
    mx = fmax(mx, w[i]);
  }
  rcond = mn / mx;
  if (info != 0 || mx < fsp(1e-30f)) {
    for (int j = s; j < 3; ++j)
      for (int i = s; i < 3; ++i) c[i + 3 * j] = 0;
    cdet = 0;
    rcond = 0;
    noeig = 0;
    return;
  }
  const double lim = fabs(plim * mx);
  noeig = 0;
  for (int i = 0; i < n; ++i) {
    if (w[i] < lim) w[i] = 0;
    else {
      w[i] = 1 / w[i];
      ++noeig;
    }
  }
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      double acc = 0;
      for (int k = 0; k < n; ++k) acc += (v[i + 3 * k] * w[k]) * v[j + 3 * k];
      c[(s + i) + 3 * (s + j)] = acc;
    }
}

MADAM_HD void invert_lu_sub(double *c, int s, double &cdet, bool &sing) {
  const int n = 3 - s;
  double u[9] = {0};
  for (int j = 0; j < n; ++j)
    for (int i = 0; i <= j; ++i) u[i + 3 * j] = c[(s + i) + 3 * (s + j)];
  for (int j = 0; j < n; ++j) {
    double acc = u[j + 3 * j];
    for (int k = 0; k < j; ++k) acc -= u[k + 3 * j] * u[k + 3 * j];
    if (!(acc > 0)) {
      sing = true;
      return;
    }
    const double ujj = sqrt(acc);
    u[j + 3 * j] = ujj;
    for (int i = j + 1; i < n; ++i) {
      double t = u[j + 3 * i];
      for (int k = 0; k < j; ++k) t -= u[k + 3 * j] * u[k + 3 * i];
      u[j + 3 * i] = t / ujj;
    }
  }
  cdet = 1;
  for (int i = 0; i < n; ++i) cdet *= u[i + 3 * i];
  double ui[9] = {0};
  for (int j = 0; j < n; ++j) {
    ui[j + 3 * j] = 1 / u[j + 3 * j];
    for (int i = j - 1; i >= 0; --i) {
      double acc = 0;
      for (int k = i + 1; k <= j; ++k) acc += u[i + 3 * k] * ui[k + 3 * j];
      ui[i + 3 * j] = -acc / u[i + 3 * i];
    }
  }
  for (int j = 0; j < n; ++j)
    for (int i = 0; i <= j; ++i) {
      double acc = 0;
      for (int k = j; k < n; ++k) acc += ui[i + 3 * k] * ui[j + 3 * k];
      c[(s + i) + 3 * (s + j)] = acc;
      c[(s + j) + 3 * (s + i)] = acc;
    }
  sing = false;
}

MADAM_HD int decoupling3(double *c, bool allow) {
  if (!allow) return 0;
  int istart = 1;
  for (int i = 0; i < 3; ++i) {
    const double cii = c[i + 3 * i];
    if (cii > fsp(1e-30f))
      for (int j = 1; j < 3; ++j)
        if (fabs(c[0 + 3 * j]) / cii > fsp(1e-10f)) istart = 0;
  }
  bool any = false;
  for (int i = 1; i < 3; ++i)
    if (fabs(c[i]) > fsp(1e-10f)) any = true;
  istart = any ? 0 : 1;
  if (istart == 1 && c[0] > fsp(1e-30f)) {
    c[0] = 1 / c[0];
    for (int i = 1; i < 3; ++i) {
      c[i] = 0;
      c[3 * i] = 0;
    }
  }
  return istart;
}

// Load the 6 stored values (upper triangle) into a column-major 3x3 with an
// empty lower triangle, as the reference's accumulated pixel matrices are.
MADAM_HD void load_upper(const double *s6, double *c) {
  c[0] = s6[0]; c[3] = s6[1]; c[6] = s6[2];
  c[4] = s6[3]; c[7] = s6[4]; c[8] = s6[5];
  c[1] = c[2] = c[5] = 0;
}

// Store the entries ccmultiply reads (diagonal and lower triangle).
MADAM_HD void store_lower(const double *c, double *s6) {
  s6[0] = c[0]; s6[1] = c[1]; s6[2] = c[2];
  s6[3] = c[4]; s6[4] = c[5]; s6[5] = c[8];
}

// invert_pixelmatrix_cross, one pixel (map_routines.f90:120-177)
MADAM_HD void invert_cross_pixel(double *s6, int pixmode, double pixlim, bool allow_dec,
                                 bool incomplete) {
  bool allz = true;
  for (int e = 0; e < 6; ++e)
    if (s6[e] != 0) allz = false;
  if (allz) return;
  double c[9];
  load_upper(s6, c);
  const int s = decoupling3(c, allow_dec);
  double cdet = 0, rc = 0, trace, tracen;
  bool sing = false;
  int noeig;
  bool zero = false;
  switch (pixmode) {
    case 0:
      invert_lu_sub(c, s, cdet, sing);
      zero = (cdet < pixlim || sing);
      break;
    case 1:
      trace = 0;
      for (int i = s; i < 3; ++i) trace += c[i + 3 * i];
      tracen = (fabs(trace) < fsp(1e-30f)) ? 0 : pow(3.0 / trace, 3);
      invert_lu_sub(c, s, cdet, sing);
      zero = (cdet * tracen < pixlim || sing);
      break;
    case 2:
      invert_eig_sub(c, s, incomplete, cdet, rc, sing);
      zero = (rc < pixlim || sing);
      break;
    case 3:
      if (c[0] > fsp(1e-30f)) {
        if (s == 0) c[0] = 1.0 / c[0];
        for (int j = 1; j < 3; ++j)
          for (int i = 0; i < 3; ++i) c[i + 3 * j] = 0;
        c[1] = c[2] = 0;
      } else {
        zero = true;
      }
      break;
    default:
      invert_eig_s_sub(c, s, pixlim, cdet, rc, noeig);
      break;
  }
  if (zero)
    for (int e = 0; e < 9; ++e) c[e] = 0;
  store_lower(c, s6);
}

// invert_pixelmatrix_map, one pixel (map_routines.f90:255-302); returns mask
MADAM_HD int invert_map_pixel(double *s6, int pixmode, double pixlim, bool allow_dec,
                              bool incomplete, float &crit) {
  bool allz = true;
  for (int e = 0; e < 6; ++e)
    if (s6[e] != 0) allz = false;
  if (allz) return 0;
  double c[9];
  load_upper(s6, c);
  const int s = decoupling3(c, allow_dec);
  double cdet = 0, rc = 0, pcrit = 0, trace, tracen;
  bool sing = false;
  if (pixmode == 0) {
    invert_lu_sub(c, s, cdet, sing);
    pcrit = cdet;
  } else if (pixmode == 1) {
    trace = 0;
    for (int i = s; i < 3; ++i) trace += c[i + 3 * i];
    tracen = (fabs(trace) < fsp(1e-30f)) ? 0 : pow(3.0 / trace, 3);
    invert_lu_sub(c, s, cdet, sing);
    pcrit = cdet * tracen;
  } else {
    invert_eig_sub(c, s, incomplete, cdet, rc, sing);
    pcrit = rc;
  }
  crit = (float)pcrit;
  if (pcrit < pixlim || sing) {
    for (int e = 0; e < 6; ++e) s6[e] = 0;
    return 0;
  }
  store_lower(c, s6);
  return 1;
}

}  // namespace madam
