/*
 * lu_small.c -- TEST INFRASTRUCTURE (oracle). Not part of the product.
 * See lu_small.h. Arithmetic follows LAPACK dgetf2 (pivot = first index of the
 * largest |a(i,j)|, column scaled by the reciprocal of the pivot when
 * |pivot| >= DBL_MIN, rank-1 update of the trailing block) and dgetrs (row
 * interchanges, unit-lower forward solve, upper back solve with division).
 */
#include <math.h>
#include <float.h>
#include "lu_small.h"

int orc_dgesv (int n, double *a, int *ipiv, double *b)
{
  int info = 0;

  for (int j = 0; j < n; j ++)
  {
    int p = j;
    double amax = fabs (a[j + j*n]);
    for (int i = j + 1; i < n; i ++)
    {
      double v = fabs (a[i + j*n]);
      if (v > amax) { amax = v; p = i; }
    }
    ipiv[j] = p + 1;

    if (a[p + j*n] != 0.0)
    {
      if (p != j)
      {
        for (int c = 0; c < n; c ++)
        {
          double t = a[j + c*n];
          a[j + c*n] = a[p + c*n];
          a[p + c*n] = t;
        }
      }
      double piv = a[j + j*n];
      if (fabs (piv) >= DBL_MIN)
      {
        double r = 1.0 / piv;
        for (int i = j + 1; i < n; i ++) a[i + j*n] *= r;
      }
      else
      {
        for (int i = j + 1; i < n; i ++) a[i + j*n] /= piv;
      }
    }
    else if (info == 0) info = j + 1;

    for (int c = j + 1; c < n; c ++)
    {
      double u = a[j + c*n];
      if (u != 0.0)
      {
        double t = -u;
        for (int i = j + 1; i < n; i ++) a[i + c*n] += a[i + j*n] * t;
      }
    }
  }

  if (info) return info;

  for (int i = 0; i < n; i ++)
  {
    int p = ipiv[i] - 1;
    if (p != i) { double t = b[i]; b[i] = b[p]; b[p] = t; }
  }
  for (int k = 0; k < n; k ++)
  {
    if (b[k] != 0.0)
      for (int i = k + 1; i < n; i ++) b[i] -= b[k] * a[i + k*n];
  }
  for (int k = n - 1; k >= 0; k --)
  {
    if (b[k] != 0.0)
    {
      b[k] /= a[k + k*n];
      for (int i = 0; i < k; i ++) b[i] -= b[k] * a[i + k*n];
    }
  }

  return 0;
}

int orc_dposv (int n, double *a, double *b)
{
  for (int j = 0; j < n; j ++)
  {
    double s = a[j + j*n];
    for (int k = 0; k < j; k ++) s -= a[k + j*n] * a[k + j*n];
    if (s <= 0.0 || isnan (s)) return j + 1;
    s = sqrt (s);
    a[j + j*n] = s;
    for (int c = j + 1; c < n; c ++)
    {
      double t = a[j + c*n];
      for (int k = 0; k < j; k ++) t -= a[k + j*n] * a[k + c*n];
      a[j + c*n] = t / s;
    }
  }
  for (int i = 0; i < n; i ++) /* U^T y = b */
  {
    double t = b[i];
    for (int k = 0; k < i; k ++) t -= a[k + i*n] * b[k];
    b[i] = t / a[i + i*n];
  }
  for (int i = n - 1; i >= 0; i --) /* U x = y */
  {
    double t = b[i];
    for (int k = i + 1; k < n; k ++) t -= a[i + k*n] * b[k];
    b[i] = t / a[i + i*n];
  }
  return 0;
}
