/* TEST INFRASTRUCTURE (not part of the product): the high-order callbacks a
 * solver hands to tioga_set_highorder_callback_ (src/tiogaInterface.C:273-285,
 * signatures src/MeshBlock.h:79-83), written here for Lagrange hexahedra of
 * degree p with equispaced nodes, to drive the oracle and the compiled
 * reference through the high-order path (tioga.C:162-178, highOrder.C).
 *
 * Element layout (the solver's): every cell owns (p+1)^3 degrees of freedom
 * stored element-major, node (i, j, k) of cell c at position
 * ((c * (p+1) + k) * (p+1) + j) * (p+1) + i, reference coordinates
 * (r, s, t) in [0, 1]^3 with node (i, j, k) at (i/p, j/p, k/p).  A solution
 * array holds nvar values per degree of freedom in that order (ROW).
 *
 * The callbacks receive no block id (the reference calls the same functions
 * for every block).  The oracle names the block before each call through
 * ho_set_block; a run of the compiled reference, which cannot, uses
 * ho_set_roles: receptor-side calls (points, modal conversion) then go to one
 * block and donor-side calls (inclusion test, fractions) to another.
 *
 * The element arithmetic (basis, Newton inversion, weights) is written out
 * in a fixed order that the library's device code repeats operation by
 * operation, so the FP64 results are the same bits. */
#include <math.h>
#include <string.h>

#define HO_MAXB 16
#define HO_MAXN 11 /* (p+1) per axis at most: NFRAC = 1331 = 11^3 */

static struct {
  int p, n1, npts, ncells;
  const double *xdof;
} HB[HO_MAXB];
static int g_block = 0, g_rec = -1, g_don = -1, g_nvar = 1;

void ho_register(int b, int p, int ncells, const double *xdof) {
  if (b < 0 || b >= HO_MAXB || p < 1 || p + 1 > HO_MAXN) return;
  HB[b].p = p;
  HB[b].n1 = p + 1;
  HB[b].npts = (p + 1) * (p + 1) * (p + 1);
  HB[b].ncells = ncells;
  HB[b].xdof = xdof;
}
void ho_set_block(int b) { g_block = b; }
void ho_set_roles(int rec_block, int don_block) {
  g_rec = rec_block;
  g_don = don_block;
}
void ho_set_nvar(int nvar) { g_nvar = nvar; }

static int rec_block(void) { return g_rec >= 0 ? g_rec : g_block; }
static int don_block(void) { return g_don >= 0 ? g_don : g_block; }

/* 1-D Lagrange basis on the nodes i/p and its derivative */
static void basis1(int p, double r, double *l, double *dl) {
  for (int i = 0; i <= p; i++) {
    const double xi = (double)i / p;
    double v = 1.0, d = 0.0;
    for (int m = 0; m <= p; m++) {
      if (m == i) continue;
      const double xm = (double)m / p;
      const double den = xi - xm;
      d = d * ((r - xm) / den) + v / den;
      v = v * ((r - xm) / den);
    }
    l[i] = v;
    dl[i] = d;
  }
}

/* map and Jacobian of the element at (r, s, t) */
static void ho_map(int p, const double *X, const double u[3], double x[3], double J[3][3]) {
  const int n1 = p + 1;
  double lr[HO_MAXN], ls[HO_MAXN], lt[HO_MAXN], dr[HO_MAXN], ds[HO_MAXN], dt[HO_MAXN];
  basis1(p, u[0], lr, dr);
  basis1(p, u[1], ls, ds);
  basis1(p, u[2], lt, dt);
  for (int a = 0; a < 3; a++) {
    x[a] = 0.0;
    J[a][0] = J[a][1] = J[a][2] = 0.0;
  }
  for (int k = 0; k < n1; k++)
    for (int j = 0; j < n1; j++)
      for (int i = 0; i < n1; i++) {
        const double *P = X + 3 * ((k * n1 + j) * n1 + i);
        const double w = (lr[i] * ls[j]) * lt[k];
        const double wr = (dr[i] * ls[j]) * lt[k];
        const double ws = (lr[i] * ds[j]) * lt[k];
        const double wt = (lr[i] * ls[j]) * dt[k];
        for (int a = 0; a < 3; a++) {
          x[a] = x[a] + w * P[a];
          J[a][0] = J[a][0] + wr * P[a];
          J[a][1] = J[a][1] + ws * P[a];
          J[a][2] = J[a][2] + wt * P[a];
        }
      }
}

/* Newton inversion from the element centre; returns 1 when the update fell
 * below 1e-14 within 50 steps */
static int ho_invert(int p, const double *X, const double *xp, double u[3]) {
  u[0] = u[1] = u[2] = 0.5;
  for (int it = 0; it < 50; it++) {
    double x[3], J[3][3];
    ho_map(p, X, u, x, J);
    const double f0 = xp[0] - x[0], f1 = xp[1] - x[1], f2 = xp[2] - x[2];
    const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
    if (!(fabs(det) > 1e-300)) return 0;
    /* Cramer's rule: du = J^-1 f */
    const double d0 = (f0 * c00 + f1 * (J[0][2] * J[2][1] - J[0][1] * J[2][2]) +
                       f2 * (J[0][1] * J[1][2] - J[0][2] * J[1][1])) / det;
    const double d1 = (f0 * c01 + f1 * (J[0][0] * J[2][2] - J[0][2] * J[2][0]) +
                       f2 * (J[0][2] * J[1][0] - J[0][0] * J[1][2])) / det;
    const double d2 = (f0 * c02 + f1 * (J[0][1] * J[2][0] - J[0][0] * J[2][1]) +
                       f2 * (J[0][0] * J[1][1] - J[0][1] * J[1][0])) / det;
    u[0] = u[0] + d0;
    u[1] = u[1] + d1;
    u[2] = u[2] + d2;
    if (fabs(d0) + fabs(d1) + fabs(d2) < 1e-14) return 1;
  }
  return 0;
}

#define HO_TOL 1e-10

/* f1: get_nodes_per_cell(icell, npts) */
void ho_nodes_per_cell(int *icell, int *npts) {
  (void)icell;
  *npts = HB[rec_block()].npts;
}

/* f2: get_receptor_nodes(icell, npts, xyz): the cell's own nodes */
void ho_receptor_nodes(int *icell, int *npts, double *xyz) {
  const int b = rec_block();
  memcpy(xyz, HB[b].xdof + 3 * (size_t)(*icell - 1) * HB[b].npts, sizeof(double) * 3 * (size_t)(*npts));
}

/* f3: donor_inclusion_test(icell, x, pass, rst) */
void ho_inclusion(int *icell, double *xp, int *pass, double *rst) {
  const int b = don_block();
  double u[3];
  const int ok = ho_invert(HB[b].p, HB[b].xdof + 3 * (size_t)(*icell - 1) * HB[b].npts, xp, u);
  *pass = ok && u[0] >= -HO_TOL && u[0] <= 1.0 + HO_TOL && u[1] >= -HO_TOL && u[1] <= 1.0 + HO_TOL &&
          u[2] >= -HO_TOL && u[2] <= 1.0 + HO_TOL;
  rst[0] = u[0];
  rst[1] = u[1];
  rst[2] = u[2];
}

/* f4: donor_frac(icell, x, nweights, inode, frac, rst, ndim): the weights
 * at the point's reference coordinates, inverted again from the point (the
 * reference leaves rst unset for a coincident point that was not searched
 * itself); inode[0] is the 1-based offset of the cell's first value */
void ho_frac(int *icell, double *xp, int *nw, int *inode, double *frac, double *rst, int *ndim) {
  const int b = don_block();
  const int p = HB[b].p, n1 = p + 1;
  double u[3], lr[HO_MAXN], ls[HO_MAXN], lt[HO_MAXN], d[HO_MAXN];
  (void)rst;
  ho_invert(p, HB[b].xdof + 3 * (size_t)(*icell - 1) * HB[b].npts, xp, u);
  basis1(p, u[0], lr, d);
  basis1(p, u[1], ls, d);
  basis1(p, u[2], lt, d);
  *nw = HB[b].npts < *ndim ? HB[b].npts : *ndim;
  int m = 0;
  for (int k = 0; k < n1; k++)
    for (int j = 0; j < n1; j++)
      for (int i = 0; i < n1; i++, m++)
        if (m < *nw) frac[m] = (lr[i] * ls[j]) * lt[k];
  inode[0] = (*icell - 1) * HB[b].npts * g_nvar + 1;
}

/* f5: convert_to_modal(icell, npts, qin, npout, index_out, qout): nodal
 * elements, the values stay as they are */
void ho_to_modal(int *icell, int *npts, double *qin, int *npout, int *index_out, double *qout) {
  const int b = rec_block();
  *npout = *npts;
  *index_out = (*icell - 1) * HB[b].npts * g_nvar + 1;
  memcpy(qout, qin, sizeof(double) * (size_t)(*npts) * g_nvar);
}
