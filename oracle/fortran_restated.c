/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * C restatements of the three Fortran routines of the TIOGA reference, which
 * cannot be compiled here (no Fortran compiler).  They are linked into the
 * compiled reference (oracle/_ref) and into the C restatement of the hot path
 * (oracle/tioga_oracle.c).  Each follows its Fortran source statement by
 * statement, with Fortran's by-reference, 1-based, column-major calling
 * convention and double-precision literals (the reference builds Fortran
 * with -fdefault-real-8), so the floating-point operations happen in the same
 * order and with the same rounding.
 *
 *   median_       src/median.F90:59-210     partial quickselect; the ADT shape
 *                                            depends on its exact swap order
 *   kaiser_wrap_  src/kaiser.f:20-180       Kaiser (JK) eigen-decomposition of
 *                                            the 3x3 covariance (OBB axes)
 *   cellvolume_   src/cellVolume.f90:20-109 signed polyhedron volume by the
 *                                            divergence theorem
 */
#include <math.h>

/* ---------------------------------------------------------------------- */
/* src/median.F90:59-210                                                   */
/* ---------------------------------------------------------------------- */
void median_(int *ix, double *x, int *np, double *xmed_out) {
#define X_(i) x[(i)-1]
#define IX_(i) ix[(i)-1]
  const int n = *np;
  const int nby2 = n / 2;
  const int nby2p1 = nby2 + 1;
  int odd = 1;
  double temp, xhi, xlo, xmax, xmin, xmed;
  int hi, lo, mid, i, j, k, itemp;

  if (n == 2 * nby2) odd = 0;
  lo = 1;
  hi = n;
  if (n < 3) { /* :88-104 */
    if (n < 1) {
      *xmed_out = 0.0;
      return;
    }
    xmed = X_(1);
    if (n == 1) {
      *xmed_out = xmed;
      return;
    }
    xmed = 0.5 * (xmed + X_(2));
    if (X_(2) < X_(1)) {
      temp = X_(1); X_(1) = X_(2); X_(2) = temp;
      itemp = IX_(1); IX_(1) = IX_(2); IX_(2) = itemp;
    }
    *xmed_out = xmed;
    return;
  }

L10: /* median of first, middle and last values (:108-120) */
  mid = (lo + hi) / 2;
  xmed = X_(mid);
  xlo = X_(lo);
  xhi = X_(hi);
  if (xhi < xlo) {
    temp = xhi; xhi = xlo; xlo = temp;
  }
  if (xmed > xhi) {
    xmed = xhi;
  } else if (xmed < xlo) {
    xmed = xlo;
  }

  /* Hoare partition around xmed (:125-147) */
  i = lo;
  j = hi;
L50:
  for (;;) {
    if (X_(i) >= xmed) break;
    i = i + 1;
  }
  for (;;) {
    if (X_(j) <= xmed) break;
    j = j - 1;
  }
  if (i < j) {
    temp = X_(i); X_(i) = X_(j); X_(j) = temp;
    itemp = IX_(i); IX_(i) = IX_(j); IX_(j) = itemp;
    i = i + 1;
    j = j - 1;
    if (i <= j) goto L50;
  }

  /* decide which half holds the median (:149-164) */
  if (!odd) {
    if (j == nby2 && i == nby2p1) goto L130;
    if (j < nby2) lo = i;
    if (i > nby2p1) hi = j;
    if (i != j) goto L100;
    if (i == nby2) lo = nby2;
    if (j == nby2p1) hi = nby2p1;
  } else {
    if (j < nby2p1) lo = i;
    if (i > nby2p1) hi = j;
    if (i != j) goto L100;
    if (i == nby2p1) {
      *xmed_out = xmed;
      return;
    }
  }
L100:
  if (lo < hi - 1) goto L10;

  if (!odd) { /* :168-178 */
    if (X_(nby2p1) < X_(nby2)) {
      temp = X_(nby2p1); X_(nby2p1) = X_(nby2); X_(nby2) = temp;
      itemp = IX_(nby2p1); IX_(nby2p1) = IX_(nby2); IX_(nby2) = itemp;
    }
    xmed = 0.5 * (X_(nby2) + X_(nby2p1));
    *xmed_out = xmed;
    return;
  }
  temp = X_(lo); /* :179-188 */
  itemp = IX_(lo);
  if (temp > X_(hi)) {
    X_(lo) = X_(hi);
    X_(hi) = temp;
    IX_(lo) = IX_(hi);
    IX_(hi) = itemp;
  }
  xmed = X_(nby2p1);
  *xmed_out = xmed;
  return;

L130: /* N even, median between the halves (:195-207) */
  xmax = X_(1);
  for (k = lo; k <= j; k++) xmax = (xmax > X_(k)) ? xmax : X_(k);
  xmin = X_(n);
  for (k = i; k <= hi; k++) xmin = (xmin < X_(k)) ? xmin : X_(k);
  xmed = 0.5 * (xmin + xmax);
  *xmed_out = xmed;
#undef X_
#undef IX_
}

/* ---------------------------------------------------------------------- */
/* src/kaiser.f:29-180 (the wrapper at :20-27 forwards its arguments)      */
/* ---------------------------------------------------------------------- */
static void kaiser(double *a, int nrows, int n, double *eigenv, double *trace,
                   double *sume, int *ier) {
#define A_(i, j) a[((j)-1) * nrows + ((i)-1)]
  const double small = 1.0e-12, zero = 0.0, half = 0.5, one = 1.0;
  int i, iter, j, k, ncount, nn;
  double absp, absq, cs, ctn, eps, halfp, p, q, sn, ss, tn, temp, xj, xk;

  *ier = 1;
  if (n < 1 || n > nrows) return;
  *ier = 0;
  iter = 0;
  *trace = zero;
  ss = zero;
  for (j = 1; j <= n; j++) {
    *trace = *trace + A_(j, j);
    for (i = 1; i <= n; i++) ss = ss + A_(i, j) * A_(i, j);
  }
  *sume = zero;
  eps = small * ss / n;
  nn = n * (n - 1) / 2;
  ncount = nn;

L20:
  for (j = 1; j <= n - 1; j++) {
    for (k = j + 1; k <= n; k++) {
      halfp = zero;
      q = zero;
      for (i = 1; i <= n; i++) {
        xj = A_(i, j);
        xk = A_(i, k);
        halfp = halfp + xj * xk;
        q = q + (xj + xk) * (xj - xk);
      }
      p = halfp + halfp;
      absp = fabs(p);
      if (absp < eps && q >= zero) {
        ncount = ncount - 1;
        if (ncount <= 0) goto L160;
        continue;
      }
      absq = fabs(q);
      if (absp <= absq) {
        tn = absp / absq;
        cs = one / sqrt(one + tn * tn);
        sn = tn * cs;
      } else {
        ctn = absq / absp;
        sn = one / sqrt(one + ctn * ctn);
        cs = ctn * sn;
      }
      cs = sqrt((one + cs) * half);
      sn = sn / (cs + cs);
      if (q < zero) {
        temp = cs; cs = sn; sn = temp;
      }
      if (p < zero) sn = -sn;
      for (i = 1; i <= n; i++) {
        temp = A_(i, j);
        A_(i, j) = temp * cs + A_(i, k) * sn;
        A_(i, k) = -temp * sn + A_(i, k) * cs;
      }
    }
  }
  ncount = nn;
  iter = iter + 1;
  if (iter < 10) goto L20;
  *ier = 2;

L160:
  for (j = 1; j <= n; j++) {
    temp = 0.0;
    for (i = 1; i <= n; i++) temp = temp + A_(i, j) * A_(i, j);
    eigenv[j - 1] = sqrt(temp);
    *sume = *sume + eigenv[j - 1];
  }
  for (j = 1; j <= n; j++) {
    if (eigenv[j - 1] > zero) temp = one / eigenv[j - 1];
    else temp = zero;
    for (i = 1; i <= n; i++) A_(i, j) = A_(i, j) * temp;
  }
#undef A_
}

void kaiser_wrap_(double *a, int *nrows, int *n, double *eigenv, double *trace,
                  double *sume, int *ier) {
  kaiser(a, *nrows, *n, eigenv, trace, sume, ier);
}

/* ---------------------------------------------------------------------- */
/* src/cellVolume.f90:20-109                                               */
/* ---------------------------------------------------------------------- */
static double scalar_product(const double *a, const double *b, const double *c) {
  /* box product, evaluated left to right as written at :101-103 */
  return a[0] * b[1] * c[2] - a[0] * b[2] * c[1] + a[1] * b[2] * c[0] -
         a[1] * b[0] * c[2] + a[2] * b[0] * c[1] - a[2] * b[1] * c[0];
}

/* xc(3,nvert) column-major == xc[v][k]; fconn(4,nfaces) == fconn_row[4*f+j] */
void cellvolume_(double *vol, double xc[][3], int numverts[][6], int fconn[][24],
                 int *nfaces, int *nvert) {
  (void)nvert;
  const int *nverts = numverts[0];
  const int *fc = fconn[0];
  double v = 0.0;
  for (int f = 0; f < *nfaces; f++) {
    const double *p1 = xc[fc[4 * f + 0] - 1];
    const double *p2 = xc[fc[4 * f + 1] - 1];
    const double *p3 = xc[fc[4 * f + 2] - 1];
    if (nverts[f] == 3) {
      v = v - 0.5 * scalar_product(p1, p2, p3);
    } else {
      const double *p4 = xc[fc[4 * f + 3] - 1];
      v = v - 0.25 * scalar_product(p1, p2, p3);
      v = v - 0.25 * scalar_product(p1, p3, p4);
      v = v - 0.25 * scalar_product(p1, p2, p4);
      v = v - 0.25 * scalar_product(p2, p3, p4);
    }
  }
  *vol = v / 3.0;
}
