/*
 * ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into the product library.
 *
 * A single-rank C restatement of the TIOGA overset-connectivity hot path:
 *   tioga_registergrid_data[_mb]_ -> tioga_preprocess_grids_ ->
 *   tioga_performconnectivity_ -> tioga_registersolution_ ->
 *   tioga_dataupdate[_mb]_   (+ donor-info queries and setters)
 * exporting the same C ABI as src/tiogaInterface.C:36-328.  The MPI exchange
 * steps of the reference are replaced by direct hand-offs between blocks in
 * the order in which a one-rank run delivers its self-messages, so every
 * order-dependent rule (ADT pre-order, donor-list ties, cancellation order)
 * is reproduced.  Each function cites the reference lines it restates.
 *
 * Floating point: all arithmetic is IEEE double, evaluated in the order the
 * reference writes it; the Makefile disables FMA contraction.
 */
#include <math.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define BIGVALUE 1.0e+15
#define BIGINT 2147483647
#define TOLV 1.0e-10
#define HOLEMAPSIZE 192
#define MAXBLOCKS 100

static double dmin(double a, double b) { return (a < b) ? a : b; }
static double dmax(double a, double b) { return (a > b) ? a : b; }

/* Fortran restatements (fortran_restated.c) */
void median_(int *ix, double *x, int *n, double *xmed);
void kaiser_wrap_(double *a, int *nrows, int *n, double *eigenv, double *trace,
                  double *sume, int *ier);
void cellvolume_(double *vol, double xc[][3], int numverts[][6], int fconn[][24],
                 int *nfaces, int *nvert);

typedef struct {
  double xc[3], dxc[3], vec[3][3];
} obb_t;

typedef struct {
  int exist;
  int nx[3];
  int *sam;
  double ext[6];
} holemap_t;

typedef struct { /* one donor candidate (src/codetypes.h:105-112) */
  int sender, mtag, remote;
  double dres, rres;
} cand_t;

typedef struct { /* src/codetypes.h:122-130 */
  int cancel, nw;
  int rinfo[3];
  int inode[9];
  double w[9];
} interp_t;

typedef struct {
  /* registered (caller-owned) */
  int tag, nnodes, ncells, nwbc, nobc, ntypes;
  double *x;
  int *iblank, *wbc, *obc;
  int nv[8], nc[8];
  int *vconn[8];
  int nfringe; /* copied at preprocess like tioga::profile (tioga.C:95-110) */
  double *user_nres, *user_cres;
  int *iblank_cell;
  int own_iblank_cell;
  /* preprocess */
  double *cellRes, *nodeRes;
  obb_t obb;
  int mapdims[3];
  double mapdx[3];
  int *icft, *invmap;
  /* search */
  int nsearch;
  double *xsearch, *res_search;
  int *isearch, *tagsearch, *donorId, *xtag;
  /* ADT over the culled cells */
  int nelem;
  int *elementList;
  double *elementBbox;
  int *adtInt;
  double *adtReal;
  double adtExt[6];
  /* donor lists per node (arrays of candidates) */
  int *dl_cnt, *dl_off;
  cand_t *dl;
  /* interpolation list */
  int ninterp;
  interp_t *interp;
  int *interp2donor;
  int ncancel;
  int *cancel_nodes;
  int cancel_cap;
  /* high-order path (highOrder.C): receptor cells, their points, point donors */
  int nrc, ntp;
  int *ctag, *ppc;
  double *rxyz, *rst;
  int ninterp2;
  int *i2_inode0, *i2_nw, *i2_rinfo; /* rinfo: point id, receptor block */
  double *i2_w;                      /* NFRAC per record */
  /* uniform-hex fast path (MeshBlock.h:96-117: check_uniform_hex_flag,
     uniform_hex, obh, dx, xlow, idims, uindx) */
  int check_uniform_flag, uniform_hex;
  /* node global ids (registerGridData's node_gid, MeshBlock.C:61) and, with
     the node-GID variant, the query points' ids (gid_search) */
  const uint64_t *node_gid;
  uint64_t *gid_search;
  obb_t obh;
  double hdx[3], xlow[3];
  int idims[3];
  int *uindx;
} block_t;

static struct {
  int alive;
  int nblocks;
  block_t *b[MAXBLOCKS];
  int isym, nfringe, mexclude;
  int nmesh;
  holemap_t *hm;
  int npairs; /* intersecting (receptor block, donor block) pairs */
  int *pair_ib, *pair_ob;
  obb_t *pair_obb;
  int nsend; /* 1 when any pair exists (self-message map), else 0 */
  double **qblock;
  /* high-order callbacks (src/MeshBlock.h:79-83) */
  int ihigh, ihighGlobal, ihigh_search;
  void (*get_nodes_per_cell)(int *, int *);
  void (*get_receptor_nodes)(int *, int *, double *);
  void (*donor_inclusion_test)(int *, double *, int *, double *);
  void (*donor_frac)(int *, double *, int *, int *, double *, double *, int *);
  void (*convert_to_modal)(int *, int *, double *, int *, int *, double *);
  void (*block_hook)(int); /* oracle only: names the block before callbacks */
  double *search_rst;      /* rst of the query being searched */
  int nodegid;             /* the TIOGA_HAS_NODEGID build's behaviour, switched at run time */
} G;

#define NFRAC 1331
static void data_update_points(int nvar, int itype);
static void ho_hook(int ib) {
  if (G.block_hook) G.block_hook(ib);
}

static int find_tag(int tag) {
  for (int i = 0; i < G.nblocks; i++)
    if (G.b[i]->tag == tag) return i;
  return -1;
}

/* locate the type and local index of a global cell id */
static void cell_type(const block_t *b, int icell, int *n_out, int *i_out) {
  int isum = 0, n;
  for (n = 0; n < b->ntypes; n++) {
    isum += b->nc[n];
    if (icell < isum) {
      *i_out = icell - (isum - b->nc[n]);
      break;
    }
  }
  *n_out = n;
}

/* ======================================================================= */
/* numerics: src/utils.c:25-165 (findOBB)                                  */
/* ======================================================================= */
static void find_obb(const double *x, int n, obb_t *o) {
  double *xc = o->xc, *dxc = o->dxc;
  double aa[9], eig[3], trace, sume, xd[3], xmin[3], xmax[3];
  int ier, nr = 3, ncol = 3;
  xc[0] = xc[1] = xc[2] = 0;
  for (int i = 0; i < n; i++) {
    xc[0] += x[3 * i];
    xc[1] += x[3 * i + 1];
    xc[2] += x[3 * i + 2];
  }
  xc[0] /= n;
  xc[1] /= n;
  xc[2] /= n;
  if (n < 4) {
    memset(o->vec, 0, sizeof(o->vec));
    o->vec[0][0] = o->vec[1][1] = o->vec[2][2] = 1;
    if (n == 1) {
      dxc[0] = dxc[1] = dxc[2] = 1e-3;
    } else if (n == 2) {
      for (int j = 0; j < 3; j++) dxc[j] = dmax(1e-3, fabs(x[3 + j] - x[j])) * 0.5;
    } else {
      for (int i = 0; i < n; i++)
        for (int j = 0; j < 3; j++) dxc[j] = dmax(1e-3, fabs(x[3 * i + j] - x[0]));
    }
    return;
  }
  for (int i = 0; i < 9; i++) aa[i] = 0;
  for (int i = 0; i < n; i++) {
    const double *p = x + 3 * i;
    aa[0] += ((p[0] - xc[0]) * (p[0] - xc[0]));
    aa[4] += ((p[1] - xc[1]) * (p[1] - xc[1]));
    aa[8] += ((p[2] - xc[2]) * (p[2] - xc[2]));
    aa[3] += ((p[0] - xc[0]) * (p[1] - xc[1]));
    aa[6] += ((p[0] - xc[0]) * (p[2] - xc[2]));
    aa[7] += ((p[1] - xc[1]) * (p[2] - xc[2]));
  }
  aa[1] = aa[3];
  aa[2] = aa[6];
  aa[5] = aa[7];
  kaiser_wrap_(aa, &nr, &ncol, eig, &trace, &sume, &ier);
  for (int i = 0, m = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) o->vec[i][j] = aa[m++];
  for (int j = 0; j < 3; j++) {
    xmax[j] = -BIGVALUE;
    xmin[j] = BIGVALUE;
  }
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < 3; j++) xd[j] = 0;
    for (int j = 0; j < 3; j++)
      for (int k = 0; k < 3; k++) xd[j] += (x[3 * i + k] - xc[k]) * o->vec[j][k];
    for (int j = 0; j < 3; j++) {
      xmax[j] = dmax(xmax[j], xd[j]);
      xmin[j] = dmin(xmin[j], xd[j]);
    }
  }
  for (int j = 0; j < 3; j++) {
    dxc[j] = (xmax[j] - xmin[j]) * 0.5 * 1.01;
    xd[j] = (xmax[j] + xmin[j]) * 0.5;
  }
  for (int j = 0; j < 3; j++)
    for (int k = 0; k < 3; k++) xc[j] += (xd[k] * o->vec[k][j]);
}

/* src/utils.c:386-400 (getobbcoords) */
static void obb_corners(const double xc[3], const double dxc[3], const double vec[3][3],
                        double xv[8][3]) {
  for (int i = 0; i < 8; i++) {
    for (int k = 0; k < 3; k++) xv[i][k] = xc[k];
    for (int k = 0; k < 3; k++) {
      int ik = (2 * ((i & (1 << k)) >> k) - 1);
      for (int j = 0; j < 3; j++) xv[i][j] += ik * dxc[k] * vec[k][j];
    }
  }
}

/* src/utils.c:402-411 (transform2OBB) */
static void to_obb(const double xv[3], const double xc[3], const double vec[3][3], double xd[3]) {
  for (int j = 0; j < 3; j++) {
    xd[j] = 0;
    for (int k = 0; k < 3; k++) xd[j] += (xv[k] - xc[k]) * vec[j][k];
  }
}

/* src/utils.c:297-384 (obbIntersectCheck): 15-axis separating-axis test */
static int obb_intersect(const double vA[3][3], const double xA[3], const double dxA[3],
                         const double vB[3][3], const double xB[3], const double dxB[3]) {
  const double eps = 1e-12;
  double D[3], c[3][3], r, r0, r1, d1, d2;
  for (int i = 0; i < 3; i++) D[i] = xB[i] - xA[i];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      c[i][j] = 0;
      for (int k = 0; k < 3; k++) c[i][j] = c[i][j] + vA[i][k] * vB[j][k];
    }
  for (int i = 0; i < 3; i++) {
    r0 = dxA[i];
    r1 = 0;
    r = 0;
    for (int j = 0; j < 3; j++) {
      r1 += dxB[j] * fabs(c[i][j]);
      r += fabs(vA[i][j]) * D[j];
    }
    if (r > (r0 + r1 + eps)) return 0;
  }
  for (int i = 0; i < 3; i++) {
    r1 = dxB[i];
    r0 = 0;
    r = 0;
    for (int j = 0; j < 3; j++) {
      r0 += dxA[j] * fabs(c[j][i]);
      r += fabs(vB[i][j]) * D[j];
    }
    if (r > (r0 + r1 + eps)) return 0;
  }
  for (int i = 0; i < 3; i++) {
    int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
    for (int j = 0; j < 3; j++) {
      int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
      r0 = dxA[i1] * fabs(c[i2][j]) + dxA[i2] * fabs(c[i1][j]);
      r1 = dxB[j1] * fabs(c[i][j2]) + dxB[j2] * fabs(c[i][j1]);
      d2 = 0;
      d1 = 0;
      for (int k = 0; k < 3; k++) {
        d2 += vA[i2][k] * D[k];
        d1 += vA[i1][k] * D[k];
      }
      r = fabs(c[i1][j] * d2 - c[i2][j] * d1);
      if (r > (r0 + r1 + eps)) return 0;
    }
  }
  return 1;
}

/* ======================================================================= */
/* numerics: src/math.c                                                    */
/* ======================================================================= */
/* src/math.c:25-81 (solvec): Gaussian elimination, pivot only if |a_ii|<1e-8 */
static int solve3(double a[3][3], double b[3]) {
  const int n = 3;
  const double eps = 1e-8;
  for (int i = 0; i < n; i++) {
    if (fabs(a[i][i]) < eps) {
      int flag = 1;
      for (int k = i + 1; k < n && flag; k++) {
        if (a[k][i] != 0) {
          flag = 0;
          for (int l = 0; l < n; l++) {
            double t = a[k][l];
            a[k][l] = a[i][l];
            a[i][l] = t;
          }
          double t = b[k];
          b[k] = b[i];
          b[i] = t;
        }
      }
      if (flag) return 0;
    }
    for (int k = i + 1; k < n; k++) {
      double fact = -a[k][i] / a[i][i];
      for (int j = 0; j < n; j++) a[k][j] += fact * a[i][j];
      b[k] += fact * b[i];
    }
  }
  for (int i = n - 1; i >= 0; i--) {
    double sum = 0;
    for (int j = i + 1; j < n; j++) sum += a[i][j] * b[j];
    b[i] = (b[i] - sum) / a[i][i];
  }
  return 1;
}

/* src/math.c:83-146 (newtonSolve): trilinear form, start (0.5,0.5,0.5),
 * <= 500 iterations, stop at ||res||_2 <= 1e-14; failure -> u=2 (reject) */
static void newton(double f[8][3], double *uo, double *vo, double *wo) {
  double u = 0.5, v = 0.5, w = 0.5, rhs[3], lhs[3][3];
  int iter, ok = 1;
  const int itmax = 500;
  for (iter = 0; iter < itmax; iter++) {
    double uv = u * v, vw = v * w, wu = w * u, uvw = u * v * w;
    for (int j = 0; j < 3; j++)
      rhs[j] = f[0][j] + f[1][j] * u + f[2][j] * v + f[3][j] * w + f[4][j] * uv + f[5][j] * vw +
               f[6][j] * wu + f[7][j] * uvw;
    double norm = rhs[0] * rhs[0] + rhs[1] * rhs[1] + rhs[2] * rhs[2];
    if (sqrt(norm) <= 1e-14) break;
    for (int j = 0; j < 3; j++) {
      lhs[j][0] = f[1][j] + f[4][j] * v + f[6][j] * w + f[7][j] * vw;
      lhs[j][1] = f[2][j] + f[5][j] * w + f[4][j] * u + f[7][j] * wu;
      lhs[j][2] = f[3][j] + f[6][j] * u + f[5][j] * v + f[7][j] * uv;
    }
    ok = solve3(lhs, rhs);
    if (!ok) break;
    u -= (rhs[0] * 1.0);
    v -= (rhs[1] * 1.0);
    w -= (rhs[2] * 1.0);
  }
  if (iter == itmax) {
    u = 2.0;
    v = w = 0.;
  }
  if (!ok) {
    u = 2.0;
    v = w = 0.;
  }
  *uo = u;
  *vo = v;
  *wo = w;
}

/* src/math.c:149-294 (computeNodalWeights) */
static void nodal_weights(double xv[8][3], const double *xp, double frac[8], int nvert) {
  double f[8][3], u, v, w;
  switch (nvert) {
    case 4: {
      double a[3][3], b[3];
      for (int k = 0; k < 3; k++) {
        for (int j = 0; j < 3; j++) a[j][k] = xv[k][j] - xv[3][j];
        b[k] = xp[k] - xv[3][k];
      }
      if (solve3(a, b)) {
        for (int k = 0; k < 3; k++) frac[k] = b[k];
        frac[3] = 1. - frac[0] - frac[1] - frac[2];
      } else {
        frac[0] = 1.0;
        frac[1] = frac[2] = frac[3] = 0;
      }
      break;
    }
    case 5:
      for (int j = 0; j < 3; j++) {
        f[0][j] = xv[0][j] - xp[j];
        f[1][j] = xv[1][j] - xv[0][j];
        f[2][j] = xv[3][j] - xv[0][j];
        f[3][j] = xv[4][j] - xv[0][j];
        f[4][j] = xv[0][j] - xv[1][j] + xv[2][j] - xv[3][j];
        f[5][j] = xv[0][j] - xv[3][j];
        f[6][j] = xv[0][j] - xv[1][j];
        f[7][j] = -xv[0][j] + xv[1][j] - xv[2][j] + xv[3][j];
      }
      newton(f, &u, &v, &w);
      frac[0] = (1.0 - u) * (1.0 - v) * (1.0 - w);
      frac[1] = u * (1.0 - v) * (1.0 - w);
      frac[2] = u * v * (1.0 - w);
      frac[3] = (1.0 - u) * v * (1.0 - w);
      frac[4] = w;
      break;
    case 6:
      for (int j = 0; j < 3; j++) {
        f[0][j] = xv[0][j] - xp[j];
        f[1][j] = xv[1][j] - xv[0][j];
        f[2][j] = xv[2][j] - xv[0][j];
        f[3][j] = xv[3][j] - xv[0][j];
        f[4][j] = 0;
        f[5][j] = xv[0][j] - xv[2][j] - xv[3][j] + xv[5][j];
        f[6][j] = xv[0][j] - xv[1][j] - xv[3][j] + xv[4][j];
        f[7][j] = 0.;
      }
      newton(f, &u, &v, &w);
      {
        double omuv = 1.0 - u - v, omw = 1.0 - w;
        frac[0] = omuv * omw;
        frac[1] = u * omw;
        frac[2] = v * omw;
        frac[3] = omuv * w;
        frac[4] = u * w;
        frac[5] = v * w;
      }
      break;
    case 8:
      for (int j = 0; j < 3; j++) {
        f[0][j] = xv[0][j] - xp[j];
        f[1][j] = xv[1][j] - xv[0][j];
        f[2][j] = xv[3][j] - xv[0][j];
        f[3][j] = xv[4][j] - xv[0][j];
        f[4][j] = xv[0][j] - xv[1][j] + xv[2][j] - xv[3][j];
        f[5][j] = xv[0][j] - xv[3][j] + xv[7][j] - xv[4][j];
        f[6][j] = xv[0][j] - xv[1][j] + xv[5][j] - xv[4][j];
        f[7][j] = -xv[0][j] + xv[1][j] - xv[2][j] + xv[3][j] + xv[4][j] - xv[5][j] + xv[6][j] - xv[7][j];
      }
      newton(f, &u, &v, &w);
      {
        double omu = 1.0 - u, omv = 1.0 - v, omw = 1.0 - w;
        frac[0] = omu * omv * omw;
        frac[1] = u * omv * omw;
        frac[2] = u * v * omw;
        frac[3] = omu * v * omw;
        frac[4] = omu * omv * w;
        frac[5] = u * omv * w;
        frac[6] = u * v * w;
        frac[7] = omu * v * w;
      }
      break;
    default:
      fprintf(stderr, "#tioga_oracle: no weights for cells with %d vertices\n", nvert);
      break;
  }
}

/* src/math.c:298-330 (computeCellVolume): face tables per cell type */
static double cell_volume(double xv[8][3], int nvert) {
  static int numverts[4][6] = {{3, 3, 3, 3, 0, 0}, {4, 3, 3, 3, 3, 0}, {3, 4, 4, 4, 3, 0}, {4, 4, 4, 4, 4, 4}};
  static int faces[4][24] = {
      {1, 2, 3, 0, 1, 4, 2, 0, 2, 4, 3, 0, 1, 3, 4, 0, 0, 0, 0, 0, 0, 0, 0, 0},
      {1, 2, 3, 4, 1, 5, 2, 0, 2, 5, 3, 0, 4, 3, 5, 0, 1, 4, 5, 0, 0, 0, 0, 0},
      {1, 2, 3, 0, 1, 4, 5, 2, 2, 5, 6, 3, 1, 3, 6, 4, 4, 6, 5, 0, 0, 0, 0, 0},
      {1, 2, 3, 4, 1, 5, 6, 2, 2, 6, 7, 3, 3, 7, 8, 4, 1, 4, 8, 5, 5, 8, 7, 6}};
  int itype = 3, nf = 6, nv = nvert;
  double vol;
  switch (nvert) {
    case 4: itype = 0; nf = 4; break;
    case 5: itype = 1; nf = 5; break;
    case 6: itype = 2; nf = 5; break;
    case 8: itype = 3; nf = 6; break;
  }
  cellvolume_(&vol, xv, &numverts[itype], &faces[itype], &nf, &nv);
  return vol;
}

static void gather_cell(const block_t *b, int n, int i, double xv[8][3], int inode[8]) {
  int nvert = b->nv[n];
  for (int m = 0; m < nvert; m++) {
    inode[m] = b->vconn[n][nvert * i + m] - 1;
    for (int j = 0; j < 3; j++) xv[m][j] = b->x[3 * inode[m] + j];
  }
}

/* ======================================================================= */
/* preprocess: src/MeshBlock.C:74-339                                      */
/* ======================================================================= */
static void tag_boundary(block_t *b) {
  int nn = b->nnodes;
  free(b->cellRes);
  free(b->nodeRes);
  b->cellRes = (double *)malloc(sizeof(double) * (b->ncells ? b->ncells : 1));
  b->nodeRes = (double *)malloc(sizeof(double) * (nn ? nn : 1));
  int *cnt = (int *)calloc(nn ? nn : 1, sizeof(int));
  int *ex0 = (int *)calloc(nn ? nn : 1, sizeof(int));
  int *ex1 = (int *)calloc(nn ? nn : 1, sizeof(int));
  double xv[8][3];
  int inode[8];
  const double scale = 1.0; /* resolutionScale (p4est mode is out of scope) */
  if (b->user_nres == NULL && b->user_cres == NULL) {
    for (int i = 0; i < nn; i++) b->nodeRes[i] = 0.0;
    int k = 0;
    for (int n = 0; n < b->ntypes; n++)
      for (int i = 0; i < b->nc[n]; i++) {
        gather_cell(b, n, i, xv, inode);
        double vol = cell_volume(xv, b->nv[n]);
        b->cellRes[k++] = (vol * scale);
        for (int m = 0; m < b->nv[n]; m++) {
          cnt[inode[m]]++;
          b->nodeRes[inode[m]] += (vol * scale);
        }
      }
  } else {
    for (int k = 0; k < b->ncells; k++) b->cellRes[k] = b->user_cres[k];
    for (int k = 0; k < nn; k++) b->nodeRes[k] = b->user_nres[k];
  }
  /* 10x10x10 node bins in the block's OBB frame, used to order query points
   * (MeshBlock.C:171-224); within a bin the nodes are in descending order */
  for (int j = 0; j < 3; j++) {
    b->mapdims[j] = 10;
    b->mapdx[j] = 2 * b->obb.dxc[j] / b->mapdims[j];
  }
  int nbin = b->mapdims[0] * b->mapdims[1] * b->mapdims[2];
  free(b->icft);
  free(b->invmap);
  b->icft = (int *)malloc(sizeof(int) * (nbin + 1));
  b->invmap = (int *)malloc(sizeof(int) * (nn ? nn : 1));
  int *head = (int *)malloc(sizeof(int) * (nbin + 1));
  int *nxt = (int *)malloc(sizeof(int) * (nn ? nn : 1));
  for (int i = 0; i < nbin + 1; i++) head[i] = -1;
  for (int i = 0; i < nn; i++) {
    double xd[3];
    int idx[3];
    if (cnt[i] != 0) b->nodeRes[i] /= cnt[i];
    for (int j = 0; j < 3; j++) {
      xd[j] = b->obb.dxc[j];
      for (int k = 0; k < 3; k++) xd[j] += (b->x[3 * i + k] - b->obb.xc[k]) * b->obb.vec[j][k];
      idx[j] = xd[j] / b->mapdx[j];
    }
    int indx = idx[2] * b->mapdims[1] * b->mapdims[0] + idx[1] * b->mapdims[0] + idx[0];
    nxt[i] = head[indx + 1];
    head[indx + 1] = i;
  }
  b->icft[0] = 0;
  for (int i = 0, kc = 0; i < nbin; i++) {
    int m = 0;
    for (int ip = head[i + 1]; ip != -1; ip = nxt[ip]) {
      b->invmap[kc++] = ip;
      m++;
    }
    b->icft[i + 1] = b->icft[i] + m;
  }
  free(head);
  free(nxt);
  /* mandatory receptors: every node of a cell touching an overset-boundary
   * node gets nodeRes = BIG (MeshBlock.C:230-284) */
  int *obcf = (int *)calloc(nn ? nn : 1, sizeof(int));
  for (int i = 0; i < b->nobc; i++) obcf[b->obc[i] - 1] = 1;
  for (int n = 0; n < b->ntypes; n++)
    for (int i = 0; i < b->nc[n]; i++) {
      int itag = 0, nvert = b->nv[n];
      for (int m = 0; m < nvert; m++)
        if (obcf[b->vconn[n][nvert * i + m] - 1]) itag = 1;
      if (itag)
        for (int m = 0; m < nvert; m++) {
          int v = b->vconn[n][nvert * i + m] - 1;
          b->nodeRes[v] = BIGVALUE;
          ex0[v] = ex1[v] = 1;
        }
    }
  free(obcf);
  /* mexclude rounds: cells touching tagged nodes are no donors
   * (MeshBlock.C:307-335) */
  for (int iex = 0; iex < G.mexclude; iex++) {
    int k = 0;
    for (int n = 0; n < b->ntypes; n++) {
      int nvert = b->nv[n];
      for (int i = 0; i < b->nc[n]; i++) {
        for (int m = 0; m < nvert; m++)
          if (ex0[b->vconn[n][nvert * i + m] - 1] == 1) {
            b->cellRes[k] = BIGVALUE;
            break;
          }
        if (b->cellRes[k] == BIGVALUE)
          for (int m = 0; m < nvert; m++) {
            int v = b->vconn[n][nvert * i + m] - 1;
            if (ex0[v] != 1) ex1[v] = 1;
          }
        k++;
      }
    }
    for (int i = 0; i < nn; i++) ex0[i] = ex1[i];
  }
  free(cnt);
  free(ex0);
  free(ex1);
}

/* ======================================================================= */
/* hole maps: src/holeMap.C:40-188, MeshBlock.C:637-772, utils.c:170-295    */
/* ======================================================================= */
static void free_holemaps(void) {
  if (G.hm) {
    for (int i = 0; i < G.nmesh; i++) free(G.hm[i].sam);
    free(G.hm);
  }
  G.hm = NULL;
  G.nmesh = 0;
}

static void fill_holemap(int *h, const int ix[3], int isym) {
  int ns2 = ix[0] * ix[1];
  for (int kk = 0; kk < ix[2]; kk += (ix[2] - 1))
    for (int jj = 0; jj < ix[1]; jj++)
      for (int ii = 0; ii < ix[0]; ii++) h[kk * ns2 + jj * ix[0] + ii] = 1;
  for (int kk = 0; kk < ix[2]; kk++)
    for (int jj = 0; jj < ix[1]; jj += (ix[1] - 1))
      for (int ii = 0; ii < ix[0]; ii++) h[kk * ns2 + jj * ix[0] + ii] = 1;
  for (int kk = 0; kk < ix[2]; kk++)
    for (int jj = 0; jj < ix[1]; jj++)
      for (int ii = 0; ii < ix[0]; ii += (ix[0] - 1)) h[kk * ns2 + jj * ix[0] + ii] = 1;
  int npaint = ns2 * ix[2];
  while (npaint > 0) {
    npaint = 0;
    for (int k = 1; k < ix[2] - 1; k++)
      for (int j = 1; j < ix[1] - 1; j++)
        for (int i = 1; i < ix[0] - 1; i++) {
          int m = k * ns2 + j * ix[0] + i;
          if (h[m] != 0) continue;
          int mk[6], nneig;
          if (isym == 1) { /* y and z neighbours */
            mk[0] = m - ns2; mk[1] = m + ns2; mk[2] = m - ix[0]; mk[3] = m + ix[0];
            nneig = 4;
          } else if (isym == 2) { /* x and z neighbours */
            mk[0] = m - ns2; mk[1] = m + ns2; mk[2] = m - 1; mk[3] = m + 1;
            nneig = 4;
          } else if (isym == 3) { /* x and y neighbours */
            mk[0] = m - ix[0]; mk[1] = m + ix[0]; mk[2] = m - 1; mk[3] = m + 1;
            nneig = 4;
          } else {
            mk[0] = m - ns2; mk[1] = m + ns2; mk[2] = m - ix[0]; mk[3] = m + ix[0];
            mk[4] = m - 1; mk[5] = m + 1;
            nneig = 6;
          }
          int paint = 0;
          for (int q = 0; q < nneig && !paint; q++) paint = (h[mk[q]] == 1);
          if (paint) {
            h[m] = 1;
            npaint++;
          }
        }
  }
  for (int i = 0; i < ix[2] * ix[1] * ix[0]; i++) h[i] = (h[i] == 0 || h[i] == 2);
}

static void get_holemaps(void) {
  int maxtag = -BIGINT;
  for (int i = 0; i < G.nblocks; i++)
    if (G.b[i]->tag > maxtag) maxtag = G.b[i]->tag;
  free_holemaps();
  G.nmesh = maxtag;
  G.hm = (holemap_t *)calloc(maxtag, sizeof(holemap_t));
  double *bb = (double *)malloc(sizeof(double) * 6 * maxtag);
  for (int i = 0; i < maxtag; i++) {
    bb[6 * i + 0] = bb[6 * i + 1] = bb[6 * i + 2] = BIGVALUE;
    bb[6 * i + 3] = bb[6 * i + 4] = bb[6 * i + 5] = -BIGVALUE;
  }
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *b = G.b[ib];
    int t = b->tag - 1;
    G.hm[t].exist = (b->nwbc > 0);
    if (b->nwbc <= 0) { /* getWallBounds returns zeros (MeshBlock.C:643-646) */
      for (int j = 0; j < 6; j++) bb[6 * t + j] = 0;
      continue;
    }
    double w[6] = {BIGVALUE, BIGVALUE, BIGVALUE, -BIGVALUE, -BIGVALUE, -BIGVALUE};
    for (int i = 0; i < b->nwbc; i++) {
      const double *p = b->x + 3 * (b->wbc[i] - 1);
      for (int j = 0; j < 3; j++) {
        w[j] = dmin(w[j], p[j]);
        w[j + 3] = dmax(w[j + 3], p[j]);
      }
    }
    for (int j = 0; j < 6; j++) bb[6 * t + j] = w[j];
  }
  for (int i = 0; i < maxtag; i++) {
    holemap_t *h = &G.hm[i];
    if (!h->exist) continue;
    double ds[3];
    for (int j = 0; j < 3; j++) {
      h->ext[j] = bb[6 * i + j];
      h->ext[j + 3] = bb[6 * i + j + 3];
      ds[j] = h->ext[j + 3] - h->ext[j];
    }
    double dsmax = dmax(dmax(ds[0], ds[1]), ds[2]);
    double dsbox = dsmax / HOLEMAPSIZE;
    for (int j = 0; j < 3; j++) {
      h->ext[j] -= (2 * dsbox);
      h->ext[j + 3] += (2 * dsbox);
      h->nx[j] = floor(dmax((h->ext[j + 3] - h->ext[j]) / dsbox, 1));
    }
    h->sam = (int *)calloc((size_t)h->nx[0] * h->nx[1] * h->nx[2], sizeof(int));
  }
  free(bb);
  /* mark wall-touching cells' index boxes with 2 (MeshBlock.C:666-772) */
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *b = G.b[ib];
    holemap_t *h = &G.hm[b->tag - 1];
    if (!h->exist) continue;
    int *wn = (int *)calloc(b->nnodes ? b->nnodes : 1, sizeof(int));
    for (int i = 0; i < b->nwbc; i++) wn[b->wbc[i] - 1] = 1;
    double ds[3];
    for (int k = 0; k < 3; k++) ds[k] = (h->ext[k + 3] - h->ext[k]) / h->nx[k];
    for (int n = 0; n < b->ntypes; n++) {
      int nvert = b->nv[n];
      for (int i = 0; i < b->nc[n]; i++) {
        int wall = 0;
        for (int j = 0; j < nvert; j++)
          if (wn[b->vconn[n][nvert * i + j] - 1] == 1) {
            wall = 1;
            break;
          }
        if (!wall) continue;
        int imin[3] = {BIGINT, BIGINT, BIGINT}, imax[3] = {-BIGINT, -BIGINT, -BIGINT};
        for (int j = 0; j < nvert; j++) {
          const double *p = b->x + 3 * (b->vconn[n][nvert * i + j] - 1);
          for (int k = 0; k < 3; k++) {
            int iv = floor((p[k] - h->ext[k]) / ds[k]);
            if (iv < imin[k]) imin[k] = iv;
            if (iv > imax[k]) imax[k] = iv;
          }
        }
        for (int j = 0; j < 3; j++) {
          if (imin[j] < 0) imin[j] = 0;
          if (imax[j] > h->nx[j] - 1) imax[j] = h->nx[j] - 1;
        }
        for (int kk = imin[2]; kk < imax[2] + 1; kk++)
          for (int jj = imin[1]; jj < imax[1] + 1; jj++)
            for (int ii = imin[0]; ii < imax[0] + 1; ii++)
              h->sam[kk * h->nx[1] * h->nx[0] + jj * h->nx[0] + ii] = 2;
      }
    }
    free(wn);
  }
  for (int i = 0; i < maxtag; i++)
    if (G.hm[i].exist) fill_holemap(G.hm[i].sam, G.hm[i].nx, G.isym);
}

/* src/utils.c:170-185: truncation toward zero, outside the map -> 0 */
static int check_holemap(const double *x, const holemap_t *h) {
  double dx[3];
  int ix[3];
  for (int i = 0; i < 3; i++) dx[i] = (h->ext[i + 3] - h->ext[i]) / h->nx[i];
  for (int i = 0; i < 3; i++) {
    ix[i] = (x[i] - h->ext[i]) / dx[i];
    if (ix[i] < 0 || ix[i] > h->nx[i] - 1) return 0;
  }
  return h->sam[ix[2] * h->nx[1] * h->nx[0] + ix[1] * h->nx[0] + ix[0]];
}

/* ======================================================================= */
/* boxes: src/exchangeBoxes.C:34-272 + MeshBlock.C:774-838                  */
/* ======================================================================= */
/* Region of block b's cells whose boxes overlap OBB obc, in b's OBB frame,
 * widened by 2% (getReducedOBB). */
static void reduced_obb(const block_t *b, const obb_t *obc, obb_t *out) {
  double rd[6] = {BIGVALUE, BIGVALUE, BIGVALUE, -BIGVALUE, -BIGVALUE, -BIGVALUE};
  for (int n = 0; n < b->ntypes; n++) {
    int nvert = b->nv[n];
    for (int i = 0; i < b->nc[n]; i++) {
      double bbox[6] = {BIGVALUE, BIGVALUE, BIGVALUE, -BIGVALUE, -BIGVALUE, -BIGVALUE}, xd[3];
      for (int m = 0; m < nvert; m++) {
        const double *p = b->x + 3 * (b->vconn[n][nvert * i + m] - 1);
        for (int j = 0; j < 3; j++) xd[j] = 0;
        for (int j = 0; j < 3; j++)
          for (int k = 0; k < 3; k++) xd[j] += (p[k] - obc->xc[k]) * obc->vec[j][k];
        for (int j = 0; j < 3; j++) bbox[j] = dmin(bbox[j], xd[j]);
        for (int j = 0; j < 3; j++) bbox[j + 3] = dmax(bbox[j + 3], xd[j]);
      }
      int skip = 0;
      for (int j = 0; j < 3; j++) skip = (skip || (bbox[j] > obc->dxc[j]));
      if (skip) continue;
      for (int j = 0; j < 3; j++) skip = (skip || (bbox[j + 3] < -obc->dxc[j]));
      if (skip) continue;
      for (int m = 0; m < nvert; m++) {
        const double *p = b->x + 3 * (b->vconn[n][nvert * i + m] - 1);
        for (int j = 0; j < 3; j++) xd[j] = 0;
        for (int j = 0; j < 3; j++)
          for (int k = 0; k < 3; k++) xd[j] += (p[k] - b->obb.xc[k]) * b->obb.vec[j][k];
        for (int j = 0; j < 3; j++) rd[j] = dmin(rd[j], xd[j]);
        for (int j = 0; j < 3; j++) rd[j + 3] = dmax(rd[j + 3], xd[j]);
      }
    }
  }
  for (int j = 0; j < 3; j++) {
    out->xc[j] = b->obb.xc[j];
    for (int k = 0; k < 3; k++) out->xc[j] += ((rd[k] + rd[k + 3]) * 0.5) * b->obb.vec[k][j];
    out->dxc[j] = (rd[j + 3] - rd[j]) * 0.51;
  }
}

/* Pairs (receptor block ib, donor block ob) whose OBBs intersect, listed with
 * ob outer and ib inner like the reference loop (exchangeBoxes.C:133-160).
 * pair_obb[p] is donor ob's region that overlaps ib, with ob's axes. */
static void exchange_boxes(void) {
  free(G.pair_ib);
  free(G.pair_ob);
  free(G.pair_obb);
  int cap = G.nblocks * G.nblocks + 1;
  G.pair_ib = (int *)malloc(sizeof(int) * cap);
  G.pair_ob = (int *)malloc(sizeof(int) * cap);
  G.pair_obb = (obb_t *)malloc(sizeof(obb_t) * cap);
  G.npairs = 0;
  for (int ob = 0; ob < G.nblocks; ob++)
    for (int ib = 0; ib < G.nblocks; ib++) {
      block_t *a = G.b[ib], *o = G.b[ob];
      if (abs(o->tag) == a->tag) continue;
      if (obb_intersect(a->obb.vec, a->obb.xc, a->obb.dxc, o->obb.vec, o->obb.xc, o->obb.dxc) ||
          obb_intersect(o->obb.vec, o->obb.xc, o->obb.dxc, a->obb.vec, a->obb.xc, a->obb.dxc)) {
        G.pair_ib[G.npairs] = ib;
        G.pair_ob[G.npairs] = ob;
        G.npairs++;
      }
    }
  G.nsend = (G.npairs > 0);
  for (int p = 0; p < G.npairs; p++) {
    block_t *rec = G.b[G.pair_ib[p]], *don = G.b[G.pair_ob[p]];
    obb_t r;
    reduced_obb(don, &rec->obb, &r);
    memcpy(r.vec, don->obb.vec, sizeof(r.vec));
    G.pair_obb[p] = r;
  }
}

/* ======================================================================= */
/* query points: src/exchangeSearchData.C:27-263 + MeshBlock.C:953-1117      */
/* ======================================================================= */
/* nodes of block b inside box obc, visited bin by bin (getQueryPoints2) */
static int query_points(const block_t *b, const obb_t *obc, int *out) {
  double xv[8][3], xd[3], xc[3], xmin[3], xmax[3], mdx[3];
  int imin[3], imax[3], nq = 0;
  const obb_t *o = &b->obb;
  obb_corners(obc->xc, obc->dxc, obc->vec, xv);
  for (int j = 0; j < 3; j++) {
    xmin[j] = BIGVALUE;
    xmax[j] = -BIGVALUE;
  }
  for (int n = 0; n < 8; n++) {
    to_obb(xv[n], o->xc, o->vec, xd);
    for (int j = 0; j < 3; j++) {
      xmin[j] = dmin(xmin[j], xd[j] + o->dxc[j]);
      xmax[j] = dmax(xmax[j], xd[j] + o->dxc[j]);
    }
  }
  for (int j = 0; j < 3; j++) {
    double delta = 0.01 * (xmax[j] - xmin[j]);
    xmin[j] -= delta;
    xmax[j] += delta;
    imin[j] = (xmin[j] / b->mapdx[j]) > (0) ? (xmin[j] / b->mapdx[j]) : (0);
    imax[j] = (xmax[j] / b->mapdx[j]) < (b->mapdims[j] - 1) ? (xmax[j] / b->mapdx[j]) : (b->mapdims[j] - 1);
    mdx[j] = 0.5 * b->mapdx[j];
  }
  obb_corners(obc->xc, mdx, o->vec, xv);
  for (int j = 0; j < 3; j++) {
    xmin[j] = BIGVALUE;
    xmax[j] = -BIGVALUE;
  }
  for (int m = 0; m < 8; m++) {
    to_obb(xv[m], obc->xc, obc->vec, xd);
    for (int j = 0; j < 3; j++) {
      xmin[j] = dmin(xmin[j], xd[j]);
      xmax[j] = dmax(xmax[j], xd[j]);
    }
  }
  for (int l = imin[2]; l <= imax[2]; l++)
    for (int k = imin[1]; k <= imax[1]; k++)
      for (int j = imin[0]; j <= imax[0]; j++) {
        xd[0] = -o->dxc[0] + j * b->mapdx[0] + b->mapdx[0] * 0.5;
        xd[1] = -o->dxc[1] + k * b->mapdx[1] + b->mapdx[1] * 0.5;
        xd[2] = -o->dxc[2] + l * b->mapdx[2] + b->mapdx[2] * 0.5;
        for (int n = 0; n < 3; n++) {
          xc[n] = o->xc[n];
          for (int ij = 0; ij < 3; ij++) xc[n] += (xd[ij] * o->vec[ij][n]);
        }
        to_obb(xc, obc->xc, obc->vec, xd);
        int off = 0;
        for (int ij = 0; ij < 3 && !off; ij++) off = (off || (xmin[ij] + xd[ij] > obc->dxc[ij]));
        if (off) continue;
        off = 0;
        for (int ij = 0; ij < 3 && !off; ij++) off = (off || (xmax[ij] + xd[ij] < -obc->dxc[ij]));
        if (off) continue;
        int indx = l * b->mapdims[1] * b->mapdims[0] + k * b->mapdims[0] + j;
        for (int m = b->icft[indx]; m < b->icft[indx + 1]; m++) {
          int node = b->invmap[m];
          to_obb(b->x + 3 * node, obc->xc, obc->vec, xd);
          if (fabs(xd[0]) <= obc->dxc[0] && fabs(xd[1]) <= obc->dxc[1] && fabs(xd[2]) <= obc->dxc[2])
            out[nq++] = node;
        }
      }
  return nq;
}

static void exchange_search_data(void) {
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *b = G.b[ib];
    b->nsearch = 0;
    free(b->xsearch); b->xsearch = NULL;
    free(b->isearch); b->isearch = NULL;
    free(b->tagsearch); b->tagsearch = NULL;
    free(b->donorId); b->donorId = NULL;
    free(b->res_search); b->res_search = NULL;
    free(b->gid_search); b->gid_search = NULL;
  }
  int **lists = (int **)malloc(sizeof(int *) * (G.npairs + 1));
  int *counts = (int *)malloc(sizeof(int) * (G.npairs + 1));
  for (int p = 0; p < G.npairs; p++) {
    block_t *rec = G.b[G.pair_ib[p]];
    lists[p] = (int *)malloc(sizeof(int) * (rec->nnodes ? rec->nnodes : 1));
    counts[p] = query_points(rec, &G.pair_obb[p], lists[p]);
    G.b[G.pair_ob[p]]->nsearch += counts[p];
  }
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *b = G.b[ib];
    if (b->nsearch < 1) continue;
    b->xsearch = (double *)malloc(sizeof(double) * 3 * b->nsearch);
    b->res_search = (double *)malloc(sizeof(double) * b->nsearch);
    b->isearch = (int *)malloc(sizeof(int) * 3 * b->nsearch);
    b->tagsearch = (int *)malloc(sizeof(int) * b->nsearch);
    b->donorId = (int *)malloc(sizeof(int) * b->nsearch);
    if (G.nodegid) b->gid_search = (uint64_t *)malloc(sizeof(uint64_t) * b->nsearch);
  }
  int *fill = (int *)calloc(G.nblocks, sizeof(int));
  for (int p = 0; p < G.npairs; p++) {
    block_t *rec = G.b[G.pair_ib[p]], *don = G.b[G.pair_ob[p]];
    int ob = G.pair_ob[p];
    for (int j = 0; j < counts[p]; j++) {
      int node = lists[p][j], q = fill[ob]++;
      don->isearch[3 * q] = 0;
      don->isearch[3 * q + 1] = node;
      don->isearch[3 * q + 2] = G.pair_ib[p];
      don->tagsearch[q] = rec->tag;
      for (int k = 0; k < 3; k++) don->xsearch[3 * q + k] = rec->x[3 * node + k];
      don->res_search[q] = rec->nodeRes[node];
      if (G.nodegid) don->gid_search[q] = rec->node_gid ? rec->node_gid[node] : 0; /* exchangeSearchData.C:226-231 */
    }
    free(lists[p]);
  }
  free(fill);
  free(lists);
  free(counts);
}

/* ======================================================================= */
/* ADT: src/ADT.C:34-135, buildADTrecursion.c:24-116, searchADTrecursion.C  */
/* ======================================================================= */
static void adt_recurse(block_t *b, double *work, int *avail, int *count, int side, int parent,
                        int level, int nav) {
  const int ndim = 6, nd = 3;
  if (nav > 1) {
    int dimcut = level % ndim;
    for (int i = 0; i < nav; i++) work[i] = b->elementBbox[ndim * avail[i] + dimcut];
    double mid;
    median_(avail, work, &nav, &mid);
    int nleft = (nav + 1) / 2;
    (*count)++;
    int node = *count;
    b->adtInt[4 * node] = avail[nleft - 1];
    b->adtInt[4 * node + 1] = -1;
    b->adtInt[4 * node + 2] = -1;
    b->adtInt[4 * node + 3] = -1;
    for (int i = 0; i < nd; i++) {
      b->adtReal[ndim * node + i] = BIGVALUE;
      b->adtReal[ndim * node + i + nd] = -BIGVALUE;
    }
    for (int i = 0; i < nav; i++)
      for (int j = 0; j < nd; j++) {
        int ii = ndim * node + j, jj = ndim * avail[i] + j;
        b->adtReal[ii] = dmin(b->adtReal[ii], b->elementBbox[jj]);
        b->adtReal[ii + nd] = dmax(b->adtReal[ii + nd], b->elementBbox[jj + nd]);
      }
    if (side > 0) b->adtInt[4 * parent + side] = avail[nleft - 1];
    if (nleft > 1) adt_recurse(b, work, avail, count, 1, node, level + 1, nleft - 1);
    adt_recurse(b, work, avail + nleft, count, 2, node, level + 1, nav - nleft);
  } else if (nav == 1) {
    (*count)++;
    int node = *count;
    b->adtInt[4 * node] = avail[0];
    b->adtInt[4 * node + 1] = -1;
    b->adtInt[4 * node + 2] = -1;
    b->adtInt[4 * node + 3] = -1;
    for (int j = 0; j < ndim; j++) b->adtReal[ndim * node + j] = b->elementBbox[ndim * avail[0] + j];
    if (side > 0) b->adtInt[4 * parent + side] = avail[0];
  }
}

static void adt_build(block_t *b) {
  int ne = b->nelem;
  free(b->adtInt);
  free(b->adtReal);
  b->adtInt = (int *)malloc(sizeof(int) * 4 * (ne ? ne : 1));
  b->adtReal = (double *)malloc(sizeof(double) * 6 * (ne ? ne : 1));
  for (int i = 0; i < 3; i++) {
    b->adtExt[2 * i] = BIGVALUE;
    b->adtExt[2 * i + 1] = -BIGVALUE;
  }
  for (int j = 0; j < ne; j++) {
    for (int i = 0; i < 3; i++) b->adtExt[2 * i] = dmin(b->adtExt[2 * i], b->elementBbox[6 * j + i]);
    for (int i = 0; i < 3; i++)
      b->adtExt[2 * i + 1] = dmax(b->adtExt[2 * i + 1], b->elementBbox[6 * j + i + 3]);
  }
  for (int i = 0; i < 3; i++) {
    double delta = 0.01 * (b->adtExt[2 * i + 1] - b->adtExt[2 * i]);
    b->adtExt[2 * i] -= delta;
    b->adtExt[2 * i + 1] += delta;
  }
  int *avail = (int *)malloc(sizeof(int) * (ne ? ne : 1));
  double *work = (double *)malloc(sizeof(double) * (ne ? ne : 1));
  for (int i = 0; i < ne; i++) avail[i] = i;
  int count = -1;
  adt_recurse(b, work, avail, &count, 0, 0, 0, ne);
  for (int i = 0; i < ne; i++) b->adtInt[4 * b->adtInt[4 * i] + 3] = i;
  free(avail);
  free(work);
}

/* src/checkContainment.C:27-84: cellIndex[0] = cell or -1, cellIndex[1] = 1
 * for an accept on a face (|frac|<TOL) of a no-donor (BIG) cell */
static void check_containment(block_t *b, int *cellIndex, int elem, const double *xs) {
  int icell = b->elementList[elem], n, i;
  if (G.ihigh_search) { /* checkContainment.C:86-94 */
    int icell1 = icell + 1, pass = 0;
    cellIndex[0] = -1;
    cellIndex[1] = 0;
    G.donor_inclusion_test(&icell1, (double *)xs, &pass, G.search_rst);
    if (pass) cellIndex[0] = icell;
    return;
  }
  double xv[8][3], frac[8];
  int inode[8];
  cell_type(b, icell, &n, &i);
  int nvert = b->nv[n];
  gather_cell(b, n, i, xv, inode);
  nodal_weights(xv, xs, frac, nvert);
  cellIndex[0] = icell;
  cellIndex[1] = 0;
  for (int m = 0; m < nvert; m++) {
    if ((frac[m] + TOLV) * (frac[m] - 1.0 - TOLV) > 0) {
      cellIndex[0] = -1;
      return;
    }
    if (fabs(frac[m]) < TOLV && b->cellRes[icell] == BIGVALUE) cellIndex[1] = 1;
  }
}

static int in_box(const double *xs, const double *e) {
  int flag = 1;
  for (int i = 0; i < 3; i++) flag = (flag && (xs[i] >= e[i] - TOLV));
  for (int i = 3; i < 6; i++) flag = (flag && (xs[i - 3] <= e[i] + TOLV));
  return flag;
}

static void adt_visit(block_t *b, int *cellIndex, int node, const double *xs) {
  if (in_box(xs, b->elementBbox + 6 * b->adtInt[4 * node])) {
    check_containment(b, cellIndex, b->adtInt[4 * node], xs);
    if (cellIndex[0] > -1 && cellIndex[1] == 0) return;
  }
  for (int d = 1; d < 3; d++) {
    int child = b->adtInt[4 * node + d];
    if (child > -1) {
      child = b->adtInt[4 * child + 3];
      if (in_box(xs, b->adtReal + 6 * child)) {
        adt_visit(b, cellIndex, child, xs);
        if (cellIndex[0] > -1 && cellIndex[1] == 0) return;
      }
    }
  }
}

static void adt_search(block_t *b, int *cellIndex, const double *xs) {
  cellIndex[0] = -1;
  cellIndex[1] = 0;
  int flag = 1;
  for (int i = 0; i < 3; i++) flag = (flag && (xs[i] >= b->adtExt[2 * i] - TOLV));
  for (int i = 0; i < 3; i++) flag = (flag && (xs[i] <= b->adtExt[2 * i + 1] + TOLV));
  if (flag && b->nelem > 0) adt_visit(b, cellIndex, 0, xs);
}

/* ======================================================================= */
/* duplicate query points: src/utils.c:622-737 (uniqNodesTree)              */
/* ======================================================================= */
static void uniq_tree(const double *coord, int *itag, double *rtag, const int *mtag, int *avail,
                      int nav) {
  int check = 1;
  if (nav > 20) {
    double xmin[3] = {BIGVALUE, BIGVALUE, BIGVALUE}, xmax[3] = {-BIGVALUE, -BIGVALUE, -BIGVALUE};
    double xmid[3], dx[3], xp[3];
    int npts[8], iv[3], cft[9];
    check = 0;
    for (int i = 0; i < nav; i++)
      for (int j = 0; j < 3; j++) {
        xmin[j] = dmin(xmin[j], coord[3 * avail[i] + j]);
        xmax[j] = dmax(xmax[j], coord[3 * avail[i] + j]);
      }
    for (int j = 0; j < 3; j++) {
      xmid[j] = (xmax[j] + xmin[j]) * 0.5;
      dx[j] = (xmax[j] - xmin[j]) * 0.5 + TOLV;
    }
    for (int j = 0; j < 8; j++) npts[j] = 0;
    for (int i = 0; i < nav; i++) {
      for (int j = 0; j < 3; j++) {
        xp[j] = coord[3 * avail[i] + j] - xmid[j];
        iv[j] = floor(xp[j] / dx[j]) + 1;
      }
      npts[4 * iv[0] + 2 * iv[1] + iv[2]]++;
    }
    for (int j = 0; j < 8; j++)
      if (npts[j] == nav) check = 1;
    if (!check) {
      cft[0] = 0;
      for (int j = 0; j < 8; j++) cft[j + 1] = cft[j] + npts[j];
      int *tmp = (int *)malloc(sizeof(int) * nav);
      for (int i = 0; i < nav; i++) {
        for (int j = 0; j < 3; j++) {
          xp[j] = coord[3 * avail[i] + j] - xmid[j];
          iv[j] = floor(xp[j] / dx[j]) + 1;
        }
        int box = 4 * iv[0] + 2 * iv[1] + iv[2];
        npts[box] = npts[box] - 1;
        tmp[npts[box] + cft[box]] = avail[i];
      }
      memcpy(avail, tmp, sizeof(int) * nav);
      free(tmp);
      for (int j = 0; j < 8; j++)
        if (cft[j + 1] > cft[j]) uniq_tree(coord, itag, rtag, mtag, avail + cft[j], cft[j + 1] - cft[j]);
    }
  }
  if (check) {
    for (int i = 0; i < nav; i++) {
      int p1 = avail[i];
      for (int j = i + 1; j < nav; j++) {
        int p2 = avail[j];
        if (fabs(coord[3 * p1] - coord[3 * p2]) + fabs(coord[3 * p1 + 1] - coord[3 * p2 + 1]) +
                    fabs(coord[3 * p1 + 2] - coord[3 * p2 + 2]) < TOLV &&
            mtag[p1] == mtag[p2]) {
          if (p1 > p2) {
            rtag[p2] = dmax(rtag[p1], rtag[p2]);
            itag[p1] = itag[p2];
          } else {
            rtag[p1] = dmax(rtag[p1], rtag[p2]);
            itag[p2] = itag[p1];
          }
        }
      }
    }
  }
}

/* ======================================================================= */
/* search: src/search.C:78-269                                             */
/* ======================================================================= */
/* uniquenode_map (search.C:48-74), the TIOGA_HAS_NODEGID build's merge of
   coincident query points: the first query with a node id is the
   representative of every later one with that id, its resolution the
   maximum over them, copied to all of them.  (The reference uses a hash map;
   a sort by id gives the same first occurrences.) */
static int cmp_gid_pos(const void *a, const void *b) {
  const uint64_t *x = (const uint64_t *)a, *y = (const uint64_t *)b;
  if (x[0] != y[0]) return x[0] < y[0] ? -1 : 1;
  return x[1] < y[1] ? -1 : (x[1] > y[1]);
}

static void uniquenode_map(const uint64_t *ids, double *res, int *itag, int n) {
  uint64_t *kv = (uint64_t *)malloc(sizeof(uint64_t) * 2 * (n ? n : 1));
  for (int i = 0; i < n; i++) {
    kv[2 * i] = ids[i];
    kv[2 * i + 1] = (uint64_t)i;
  }
  qsort(kv, n, 2 * sizeof(uint64_t), cmp_gid_pos);
  for (int s = 0; s < n;) {
    int e = s + 1;
    while (e < n && kv[2 * e] == kv[2 * s]) e++;
    const int first = (int)kv[2 * s + 1];
    itag[first] = first;
    for (int k = s + 1; k < e; k++) { /* in index order, as the sequential loop visits them */
      const int i = (int)kv[2 * k + 1];
      itag[i] = first;
      res[first] = (res[first] > res[i]) ? res[first] : res[i];
    }
    s = e;
  }
  for (int i = 0; i < n; i++) res[i] = res[itag[i]];
  free(kv);
}

static void merge_coincident(block_t *b) {
  free(b->xtag);
  b->xtag = (int *)malloc(sizeof(int) * b->nsearch);
  if (G.nodegid) {
    uniquenode_map(b->gid_search, b->res_search, b->xtag, b->nsearch);
    return;
  }
  int *avail = (int *)malloc(sizeof(int) * b->nsearch);
  for (int i = 0; i < b->nsearch; i++) avail[i] = b->xtag[i] = i;
  uniq_tree(b->xsearch, b->xtag, b->res_search, b->tagsearch, avail, b->nsearch);
  free(avail);
}

void tioga_oracle_set_node_gid(int btag, const uint64_t *gid) {
  int ib = find_tag(btag);
  if (ib >= 0) G.b[ib]->node_gid = gid;
}

void tioga_oracle_set_nodegid_merge(int on) { G.nodegid = on; }

/* ----------------------------------------------------------------------- */
/* uniform-hex fast path: MeshBlock::check_for_uniform_hex (MeshBlock.C:1249-  */
/* 1372), create_hex_cell_map (:1374-1409), search_uniform_hex (search.C:     */
/* 271-341)                                                                 */
/* ----------------------------------------------------------------------- */
static double tdot(const double a[3], const double b[3], const double c[3]) { /* math.c:331-337 */
  double dp = 0.0;
  for (int k = 0; k < 3; k++) dp += ((a[k] - c[k]) * (b[k] - c[k]));
  return dp;
}

static void check_for_uniform_hex(block_t *b) {
  double xv[8][3];
  int hex_present = 0;
  if (b->ntypes > 1) return;
  for (int n = 0; n < b->ntypes; n++) {
    int nvert = b->nv[n];
    if (nvert != 8) continue;
    hex_present = 1;
    for (int i = 0; i < b->nc[n]; i++) {
      int vold = -1;
      for (int m = 0; m < nvert; m++) {
        if (b->vconn[n][nvert * i + m] == vold) return; /* degenerate hex */
        vold = b->vconn[n][nvert * i + m];
        int i3 = 3 * (vold - 1);
        for (int k = 0; k < 3; k++) xv[m][k] = b->x[i3 + k];
      }
      /* rectangular faces at vertex 0 and the corner at vertex 6 */
      if (fabs(tdot(xv[1], xv[3], xv[0])) > TOLV) return;
      if (fabs(tdot(xv[1], xv[3], xv[2])) > TOLV) return;
      if (fabs(tdot(xv[3], xv[4], xv[0])) > TOLV) return;
      if (fabs(tdot(xv[3], xv[4], xv[7])) > TOLV) return;
      if (fabs(tdot(xv[4], xv[1], xv[0])) > TOLV) return;
      if (fabs(tdot(xv[4], xv[1], xv[5])) > TOLV) return;
      if (fabs(tdot(xv[5], xv[7], xv[6])) > TOLV) return;
      /* the same squared edge lengths as the first hex */
      if (i == 0) {
        b->hdx[0] = tdot(xv[1], xv[1], xv[0]);
        b->hdx[1] = tdot(xv[3], xv[3], xv[0]);
        b->hdx[2] = tdot(xv[4], xv[4], xv[0]);
      } else {
        if (fabs(b->hdx[0] - tdot(xv[1], xv[1], xv[0])) > TOLV) return;
        if (fabs(b->hdx[1] - tdot(xv[3], xv[3], xv[0])) > TOLV) return;
        if (fabs(b->hdx[2] - tdot(xv[4], xv[4], xv[0])) > TOLV) return;
      }
    }
  }
  if (!hex_present) return;
  for (int j = 0; j < 3; j++) b->hdx[j] = sqrt(b->hdx[j]);
  b->uniform_hex = 1;
  obb_t *o = &b->obh;
  for (int j = 0; j < 3; j++)
    for (int k = 0; k < 3; k++) o->vec[j][k] = 0;
  /* axes from the last hex's edges, lengths from the first hex's */
  for (int k = 0; k < 3; k++) o->vec[0][k] = (xv[1][k] - xv[0][k]) / b->hdx[0];
  for (int k = 0; k < 3; k++) o->vec[1][k] = (xv[3][k] - xv[0][k]) / b->hdx[1];
  for (int k = 0; k < 3; k++) o->vec[2][k] = (xv[4][k] - xv[0][k]) / b->hdx[2];
  double xd[3], xmax[3] = {-BIGVALUE, -BIGVALUE, -BIGVALUE}, xmin[3] = {BIGVALUE, BIGVALUE, BIGVALUE};
  for (int i = 0; i < b->nnodes; i++) {
    for (int j = 0; j < 3; j++) xd[j] = 0;
    for (int j = 0; j < 3; j++)
      for (int k = 0; k < 3; k++) xd[j] += b->x[3 * i + k] * o->vec[j][k];
    for (int j = 0; j < 3; j++) {
      xmax[j] = dmax(xmax[j], xd[j]);
      xmin[j] = dmin(xmin[j], xd[j]);
    }
  }
  for (int j = 0; j < 3; j++) {
    xmax[j] += TOLV;
    xmin[j] -= TOLV;
    o->dxc[j] = (xmax[j] - xmin[j]) * 0.5;
    xd[j] = (xmax[j] + xmin[j]) * 0.5;
  }
  for (int j = 0; j < 3; j++) {
    o->xc[j] = 0.0;
    for (int k = 0; k < 3; k++) o->xc[j] += (xd[k] * o->vec[k][j]);
  }
}

/* The reference writes uindx without a bounds check; a centroid outside the
   map (which a uniform block cannot have) is skipped here. */
static void create_hex_cell_map(block_t *b) {
  const obb_t *o = &b->obh;
  for (int j = 0; j < 3; j++) {
    b->xlow[j] = o->xc[j];
    for (int k = 0; k < 3; k++) b->xlow[j] -= (o->dxc[k] * o->vec[k][j]);
    b->idims[j] = (int)round(2 * o->dxc[j] / b->hdx[j]);
    b->hdx[j] = (2 * o->dxc[j]) / b->idims[j];
  }
  const long long nmap = (long long)b->idims[0] * b->idims[1] * b->idims[2];
  free(b->uindx);
  b->uindx = (int *)malloc(sizeof(int) * (nmap > 0 ? nmap : 1));
  for (long long i = 0; i < nmap; i++) b->uindx[i] = -1;
  for (int i = 0; i < b->nc[0]; i++) {
    double xc[3], xd[3];
    int idx[3];
    for (int j = 0; j < 3; j++) {
      int lnode = b->vconn[0][8 * i] - 1, tnode = b->vconn[0][8 * i + 6] - 1;
      xc[j] = 0.5 * (b->x[3 * lnode + j] + b->x[3 * tnode + j]);
    }
    int ok = 1;
    for (int j = 0; j < 3; j++) {
      xd[j] = 0;
      for (int k = 0; k < 3; k++) xd[j] += (xc[k] - b->xlow[k]) * o->vec[j][k];
      idx[j] = (int)(xd[j] / b->hdx[j]);
      ok = ok && idx[j] >= 0 && idx[j] < b->idims[j];
    }
    if (ok) b->uindx[(long long)idx[2] * b->idims[1] * b->idims[0] + idx[1] * b->idims[0] + idx[0]] = i;
  }
}

/* search.C:271-341.  The reference's loop over the eight corners of a cube
   of side 4 TOL runs while "dId[0] == -1 || dID[1]", where dId is a freshly
   malloc'd, never written array (search.C:291, 311); its first word is not -1
   in practice, so the loop runs while the current pick is missing (-1) or a
   cell of BIG resolution, as restated here. */
static void search_uniform_hex(block_t *b) {
  merge_coincident(b);
  double xvec[8][3];
  for (int jj = 0; jj < 8; jj++)
    for (int k = 0; k < 3; k++) xvec[jj][k] = (2 * ((jj & (1 << k)) >> k) - 1) * 2 * TOLV;
  const obb_t *o = &b->obh;
  const int *d = b->idims;
  for (int i = 0; i < b->nsearch; i++) {
    if (b->xtag[i] != i) {
      b->donorId[i] = b->donorId[b->xtag[i]];
      continue;
    }
    double xd[3];
    int idx[3];
    for (int j = 0; j < 3; j++) {
      xd[j] = 0;
      for (int k = 0; k < 3; k++) xd[j] += (b->xsearch[3 * i + k] - b->xlow[k]) * o->vec[j][k];
      idx[j] = (int)(xd[j] / b->hdx[j]);
    }
    if (xd[0] > -TOLV && xd[0] < d[0] * b->hdx[0] + TOLV && xd[1] > -TOLV && xd[1] < d[1] * b->hdx[1] + TOLV &&
        xd[2] > -TOLV && xd[2] < d[2] * b->hdx[2] + TOLV) {
      for (int k = 0; k < 3; k++)
        if (idx[k] == d[k]) idx[k]--;
      int id0 = b->uindx[(long long)idx[2] * d[1] * d[0] + idx[1] * d[0] + idx[0]];
      int big = (id0 > -1) ? (b->cellRes[id0] == BIGVALUE) : 1;
      for (int jj = 0; jj < 8 && big; jj++) {
        for (int k = 0; k < 3; k++) {
          idx[k] = (int)((xd[k] + xvec[jj][k]) / b->hdx[k]);
          if (idx[k] == d[k]) idx[k]--;
        }
        int dtest = b->uindx[(long long)idx[2] * d[1] * d[0] + idx[1] * d[0] + idx[0]];
        big = (dtest > -1) ? (b->cellRes[dtest] == BIGVALUE) : 1;
        id0 = (id0 == -1) ? dtest : (!big ? dtest : id0);
      }
      b->donorId[i] = id0;
    } else {
      b->donorId[i] = -1;
    }
  }
}

int tioga_oracle_uniform_hex(int btag) {
  int ib = find_tag(btag);
  return ib >= 0 ? G.b[ib]->uniform_hex : -1;
}

void tioga_oracle_set_uniform_hex_flag(int btag, int flag) {
  int ib = find_tag(btag);
  if (ib >= 0) G.b[ib]->check_uniform_flag = flag;
}

static void search_block(block_t *b) {
  if (b->nsearch == 0) return;
  if (b->uniform_hex) {
    search_uniform_hex(b);
    return;
  }
  obb_t q;
  find_obb(b->xsearch, b->nsearch, &q);
  /* cells whose box overlaps the query OBB, pushed LIFO (:123-167) */
  int *icell = (int *)malloc(sizeof(int) * (b->ncells ? b->ncells : 1));
  int top = -1, cnt = 0, p = 0;
  for (int n = 0; n < b->ntypes; n++) {
    int nvert = b->nv[n];
    for (int i = 0; i < b->nc[n]; i++, p++) {
      double xmin[3] = {BIGVALUE, BIGVALUE, BIGVALUE}, xmax[3] = {-BIGVALUE, -BIGVALUE, -BIGVALUE};
      double xd[3], dxc[3];
      for (int m = 0; m < nvert; m++) {
        const double *pt = b->x + 3 * (b->vconn[n][nvert * i + m] - 1);
        for (int j = 0; j < 3; j++) {
          xd[j] = 0;
          for (int k = 0; k < 3; k++) xd[j] += (pt[k] - q.xc[k]) * q.vec[j][k];
          xmin[j] = dmin(xmin[j], xd[j]);
          xmax[j] = dmax(xmax[j], xd[j]);
        }
      }
      for (int j = 0; j < 3; j++) {
        xd[j] = (xmax[j] + xmin[j]) * 0.5;
        dxc[j] = (xmax[j] - xmin[j]) * 0.5;
      }
      if (fabs(xd[0]) <= (dxc[0] + q.dxc[0]) && fabs(xd[1]) <= (dxc[1] + q.dxc[1]) &&
          fabs(xd[2]) <= (dxc[2] + q.dxc[2])) {
        icell[p] = top;
        top = p;
        cnt++;
      }
    }
  }
  free(b->elementBbox);
  free(b->elementList);
  b->nelem = cnt;
  b->elementBbox = (double *)malloc(sizeof(double) * 6 * (cnt ? cnt : 1));
  b->elementList = (int *)malloc(sizeof(int) * (cnt ? cnt : 1));
  for (int k = top, e = 0; k != -1; k = icell[k], e++) {
    int n, i;
    cell_type(b, k, &n, &i);
    int nvert = b->nv[n];
    double xmin[3] = {BIGVALUE, BIGVALUE, BIGVALUE}, xmax[3] = {-BIGVALUE, -BIGVALUE, -BIGVALUE};
    for (int m = 0; m < nvert; m++) {
      const double *pt = b->x + 3 * (b->vconn[n][nvert * i + m] - 1);
      for (int j = 0; j < 3; j++) {
        xmin[j] = dmin(xmin[j], pt[j]);
        xmax[j] = dmax(xmax[j], pt[j]);
      }
    }
    for (int j = 0; j < 3; j++) {
      b->elementBbox[6 * e + j] = xmin[j];
      b->elementBbox[6 * e + j + 3] = xmax[j];
    }
    b->elementList[e] = k;
  }
  free(icell);
  adt_build(b);
  merge_coincident(b);
  for (int i = 0; i < b->nsearch; i++) {
    if (b->xtag[i] == i) {
      int ci[2];
      G.search_rst = b->rst ? b->rst + 3 * i : NULL;
      adt_search(b, ci, b->xsearch + 3 * i);
      b->donorId[i] = ci[0];
    } else {
      b->donorId[i] = b->donorId[b->xtag[i]];
    }
  }
}

/* ======================================================================= */
/* donors: src/exchangeDonors.C:25-301, bookKeeping.C:74-648, linklist.c    */
/* ======================================================================= */
/* linklist.c:62-104: insert before the first entry with |dres| > new dres */
static void list_insert(cand_t *list, int *len, cand_t c) {
  int pos = *len;
  for (int k = 0; k < *len; k++)
    if (fabs(list[k].dres) > c.dres) {
      pos = k;
      break;
    }
  for (int k = *len; k > pos; k--) list[k] = list[k - 1];
  list[pos] = c;
  (*len)++;
}

static void cancel_push(block_t *b, int v) {
  if (b->ncancel == b->cancel_cap) {
    b->cancel_cap = b->cancel_cap ? 2 * b->cancel_cap : 64;
    b->cancel_nodes = (int *)realloc(b->cancel_nodes, sizeof(int) * b->cancel_cap);
  }
  b->cancel_nodes[b->ncancel++] = v;
}

/* bookKeeping.C:385-535 (findInterpData) on donor block b for query q */
static void find_interp(block_t *b, int q, double rres2) {
  double rres = fabs(rres2), xv[8][3], xp[3], frac[8];
  int inode[8], n, i, accept = 1, mtagrecv = b->tagsearch[q];
  for (int k = 0; k < 3; k++) xp[k] = b->xsearch[3 * q + k];
  cell_type(b, b->donorId[q], &n, &i);
  int nvert = b->nv[n];
  gather_cell(b, n, i, xv, inode);
  for (int m = 0; m < nvert; m++) {
    int v = inode[m];
    if (b->iblank[v] <= 0 && rres2 > 0.0) {
      if (b->nodeRes[v] == BIGVALUE) accept = 0;
      if (abs(b->iblank[v]) == mtagrecv) accept = 0;
    }
  }
  if (rres == BIGVALUE) { /* resolutionScale == 1 here */
    for (int m = 0; m < nvert; m++) {
      int v = inode[m];
      if (b->iblank[v] <= 0 && b->nodeRes[v] != BIGVALUE) {
        if (b->iblank[v] < 0) b->iblank[v] = 1;
        cancel_push(b, v);
      }
    }
  }
  nodal_weights(xv, xp, frac, nvert);
  interp_t *it = &b->interp[b->ninterp];
  b->interp2donor[q] = b->ninterp;
  it->cancel = 0;
  it->nw = nvert;
  it->rinfo[0] = b->isearch[3 * q];
  it->rinfo[1] = b->isearch[3 * q + 1];
  it->rinfo[2] = b->isearch[3 * q + 2];
  for (int m = 0; m < nvert; m++) {
    it->inode[m] = inode[m];
    it->w[m] = frac[m];
    if (frac[m] < -0.2 || frac[m] > 1.2)
      fprintf(stderr, "#tioga_oracle: weight %g outside [-0.2,1.2] (the reference aborts)\n", frac[m]);
  }
  it->inode[nvert] = b->donorId[q];
  it->w[nvert] = 0.0;
  if (accept == 0 && rres != BIGVALUE) it->cancel = 1;
  b->ninterp++;
}

static void exchange_donors(void) {
  if (!G.nsend) return;
  /* comm1: found donors, in donor-block order then query order */
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *r = G.b[ib];
    free(r->dl_cnt);
    free(r->dl_off);
    free(r->dl);
    r->dl_cnt = (int *)calloc(r->nnodes + 1, sizeof(int));
    r->dl_off = (int *)calloc(r->nnodes + 1, sizeof(int));
    r->dl = NULL;
  }
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *d = G.b[ib];
    for (int q = 0; q < d->nsearch; q++)
      if (d->donorId[q] > -1) G.b[d->isearch[3 * q + 2]]->dl_cnt[d->isearch[3 * q + 1]]++;
  }
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *r = G.b[ib];
    int tot = 0;
    for (int i = 0; i < r->nnodes; i++) {
      r->dl_off[i] = tot;
      tot += r->dl_cnt[i];
      r->dl_cnt[i] = 0;
    }
    r->dl = (cand_t *)malloc(sizeof(cand_t) * (tot ? tot : 1));
  }
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *d = G.b[ib];
    for (int q = 0; q < d->nsearch; q++) {
      if (d->donorId[q] < 0) continue;
      block_t *r = G.b[d->isearch[3 * q + 2]];
      int node = d->isearch[3 * q + 1];
      cand_t c = {0, d->tag, q, d->cellRes[d->donorId[q]], d->res_search[d->xtag[q]]};
      list_insert(r->dl + r->dl_off[node], &r->dl_cnt[node], c);
    }
  }
  /* processDonors per receptor block (bookKeeping.C:143-355) */
  int *nrec = (int *)calloc(G.nblocks, sizeof(int));
  int **rec_node = (int **)calloc(G.nblocks, sizeof(int *));
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *r = G.b[ib];
    int nn = r->nnodes;
    int *seen = (int *)malloc(sizeof(int) * (G.nmesh ? G.nmesh : 1));
    for (int i = 0; i < nn; i++) {
      r->iblank[i] = 1;
      const double *xi = r->x + 3 * i;
      if (r->dl_cnt[i] == 0) {
        for (int j = 0; j < G.nmesh; j++)
          if (j != r->tag - 1 && G.hm[j].exist && check_holemap(xi, &G.hm[j])) {
            r->iblank[i] = 0;
            break;
          }
      } else {
        for (int j = 0; j < G.nmesh; j++) seen[j] = 0;
        for (int c = 0; c < r->dl_cnt[i]; c++) {
          const cand_t *cd = &r->dl[r->dl_off[i] + c];
          seen[cd->mtag - 1] = 1;
          r->nodeRes[i] = dmax(r->nodeRes[i], cd->rres);
        }
        for (int j = 0; j < G.nmesh; j++)
          if (j != r->tag - 1 && G.hm[j].exist && !seen[j] && check_holemap(xi, &G.hm[j])) {
            r->iblank[i] = 0;
            break;
          }
      }
    }
    free(seen);
    for (int i = 0; i < r->nwbc; i++)
      if (r->iblank[r->wbc[i] - 1] == 0)
        fprintf(stderr, "#tioga_oracle: wall node %d of mesh %d is tagged as a hole\n", r->wbc[i] - 1, r->tag);
    /* nfringe layers around holes become mandatory receptors */
    int *m0 = (int *)malloc(sizeof(int) * (nn ? nn : 1));
    int *m1 = (int *)malloc(sizeof(int) * (nn ? nn : 1));
    for (int i = 0; i < nn; i++) m0[i] = m1[i] = (r->iblank[i] == 0);
    for (int it = 0; it < r->nfringe; it++) {
      for (int n = 0; n < r->ntypes; n++) {
        int nvert = r->nv[n];
        for (int i = 0; i < r->nc[n]; i++) {
          const int *cv = r->vconn[n] + nvert * i;
          for (int m = 0; m < nvert; m++)
            if (m0[cv[m] - 1] == 1)
              for (int mm = 0; mm < nvert; mm++)
                if (m != mm && m0[cv[mm] - 1] != 1) m1[cv[mm] - 1] = 1;
        }
      }
      for (int i = 0; i < nn; i++) m0[i] = m1[i];
    }
    for (int i = 0; i < nn; i++)
      if (m1[i] && r->iblank[i]) r->nodeRes[i] = BIGVALUE;
    free(m0);
    free(m1);
    /* fringes: the first candidate finer than the node (sorted list) */
    rec_node[ib] = (int *)malloc(sizeof(int) * (nn ? nn : 1));
    for (int i = 0; i < nn; i++) {
      if (r->dl_cnt[i] == 0 || r->iblank[i] == 0) continue;
      for (int c = 0; c < r->dl_cnt[i]; c++) {
        const cand_t *cd = &r->dl[r->dl_off[i] + c];
        if (cd->dres < r->nodeRes[i]) {
          r->iblank[i] = -cd->mtag;
          rec_node[ib][nrec[ib]++] = i;
          break;
        }
      }
    }
  }
  /* comm2: chosen donors, receptor block order then node order */
  int *ninterp = (int *)calloc(G.nblocks, sizeof(int));
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *r = G.b[ib];
    for (int k = 0; k < nrec[ib]; k++) {
      int i = rec_node[ib][k];
      for (int c = 0; c < r->dl_cnt[i]; c++) {
        const cand_t *cd = &r->dl[r->dl_off[i] + c];
        if (cd->dres < r->nodeRes[i]) {
          ninterp[find_tag(cd->mtag)]++;
          break;
        }
      }
    }
  }
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *d = G.b[ib];
    free(d->interp);
    free(d->interp2donor);
    d->interp = (interp_t *)malloc(sizeof(interp_t) * (ninterp[ib] ? ninterp[ib] : 1));
    d->ninterp = 0;
    d->ncancel = 0;
    d->interp2donor = (int *)malloc(sizeof(int) * (d->nsearch ? d->nsearch : 1));
    for (int q = 0; q < d->nsearch; q++) d->interp2donor[q] = -1;
  }
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *r = G.b[ib];
    for (int k = 0; k < nrec[ib]; k++) {
      int i = rec_node[ib][k];
      for (int c = 0; c < r->dl_cnt[i]; c++) {
        const cand_t *cd = &r->dl[r->dl_off[i] + c];
        if (cd->dres < r->nodeRes[i]) {
          find_interp(G.b[find_tag(cd->mtag)], cd->remote, r->nodeRes[i]);
          break;
        }
      }
    }
  }
  /* comm3: cancellations through each cancelled node's head donor */
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *d = G.b[ib];
    for (int c = 0; c < d->ncancel; c++) {
      int v = d->cancel_nodes[c];
      if (d->dl_cnt[v] == 0) continue;
      const cand_t *h = &d->dl[d->dl_off[v]];
      block_t *dd = G.b[find_tag(h->mtag)];
      int ip = dd->interp2donor[h->remote];
      if (ip > -1) dd->interp[ip].cancel = 1;
    }
  }
  /* resetCoincident (bookKeeping.C:572-597) */
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *d = G.b[ib];
    int *reset = (int *)malloc(sizeof(int) * (d->nsearch ? d->nsearch : 1));
    for (int q = 0; q < d->nsearch; q++) reset[q] = 1;
    for (int q = 0; q < d->nsearch; q++) {
      int ip = d->interp2donor[q];
      if (ip > -1 && d->interp[ip].cancel < reset[d->xtag[q]]) reset[d->xtag[q]] = d->interp[ip].cancel;
    }
    for (int q = 0; q < d->nsearch; q++) {
      int ip = d->interp2donor[q];
      if (ip > -1 && d->interp[ip].cancel == 1) d->interp[ip].cancel = reset[d->xtag[q]];
    }
    free(reset);
  }
  /* comm4: surviving interpolations set receptor iblank = -1 */
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *r = G.b[ib];
    for (int i = 0; i < r->nnodes; i++)
      if (r->iblank[i] < 0) r->iblank[i] = 1;
  }
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *d = G.b[ib];
    for (int k = 0; k < d->ninterp; k++)
      if (!d->interp[k].cancel) G.b[d->interp[k].rinfo[2]]->iblank[d->interp[k].rinfo[1]] = -1;
  }
  for (int ib = 0; ib < G.nblocks; ib++) free(rec_node[ib]);
  free(rec_node);
  free(nrec);
  free(ninterp);
}

/* src/highOrder.C:88-150 */
static void cell_iblanks(block_t *b) {
  if (b->iblank_cell == NULL) {
    b->iblank_cell = (int *)malloc(sizeof(int) * (b->ncells ? b->ncells : 1));
    b->own_iblank_cell = 1;
  }
  int icell = 0;
  for (int n = 0; n < b->ntypes; n++) {
    int nvert = b->nv[n];
    for (int i = 0; i < b->nc[n]; i++, icell++) {
      int flag = 1, ncount = 0;
      b->iblank_cell[icell] = 1;
      for (int m = 0; m < nvert && flag; m++) {
        int v = b->vconn[n][nvert * i + m] - 1;
        if (b->iblank[v] == 0) {
          b->iblank_cell[icell] = 0;
          flag = 0;
        }
        ncount = ncount + (b->iblank[v] == -1);
      }
      if (flag && ncount == nvert) b->iblank_cell[icell] = -1;
    }
  }
}

/* ======================================================================= */
/* the C API (src/tiogaInterface.C:36-328, tioga.C:64-570)                  */
/* ======================================================================= */
static void free_block(block_t *b) {
  free(b->cellRes); free(b->nodeRes); free(b->icft); free(b->invmap);
  free(b->xsearch); free(b->res_search); free(b->isearch); free(b->tagsearch);
  free(b->donorId); free(b->xtag); free(b->elementList); free(b->elementBbox);
  free(b->adtInt); free(b->adtReal); free(b->dl_cnt); free(b->dl_off); free(b->dl);
  free(b->interp); free(b->interp2donor); free(b->cancel_nodes);
  free(b->ctag); free(b->ppc); free(b->rxyz); free(b->rst);
  free(b->i2_inode0); free(b->i2_nw); free(b->i2_rinfo); free(b->i2_w);
  free(b->uindx); free(b->gid_search);
  if (b->own_iblank_cell) free(b->iblank_cell);
  free(b);
}

void tioga_init_(intptr_t comm) {
  (void)comm;
  memset(&G, 0, sizeof(G));
  G.alive = 1;
  G.isym = 3;
  G.nfringe = 1;
  G.mexclude = 3;
}

void tioga_init_f90_(int *fcomm) {
  (void)fcomm;
  tioga_init_(0);
}

static void register_va(int btag, int nnodes, double *xyz, int *ibl, int nwbc, int nobc, int *wbc,
                        int *obc, int ntypes, va_list ap) {
  int ib = find_tag(btag);
  block_t *b;
  if (ib < 0) {
    if (G.nblocks >= MAXBLOCKS) {
      fprintf(stderr, "#tioga_oracle: too many blocks\n");
      return;
    }
    b = (block_t *)calloc(1, sizeof(block_t));
    G.b[G.nblocks++] = b;
  } else {
    b = G.b[ib];
  }
  b->tag = btag;
  b->nnodes = nnodes;
  b->x = xyz;
  b->iblank = ibl;
  b->nwbc = nwbc;
  b->nobc = nobc;
  b->wbc = wbc;
  b->obc = obc;
  b->ntypes = ntypes;
  b->ncells = 0;
  for (int i = 0; i < ntypes; i++) {
    b->nv[i] = *va_arg(ap, int *);
    b->nc[i] = *va_arg(ap, int *);
    b->vconn[i] = va_arg(ap, int *);
    b->ncells += b->nc[i];
  }
}

void tioga_registergrid_data_(int *btag, int *nnodes, double *xyz, int *ibl, int *nwbc, int *nobc,
                              int *wbcnode, int *obcnode, int *ntypes, ...) {
  va_list ap;
  va_start(ap, ntypes);
  register_va(*btag, *nnodes, xyz, ibl, *nwbc, *nobc, wbcnode, obcnode, *ntypes, ap);
  va_end(ap);
}

void tioga_registergrid_data_mb_(int *bid, int *btag, int *nnodes, double *xyz, int *ibl, int *nwbc,
                                 int *nobc, int *wbcnode, int *obcnode, int *ntypes, ...) {
  (void)bid;
  va_list ap;
  va_start(ap, ntypes);
  register_va(*btag, *nnodes, xyz, ibl, *nwbc, *nobc, wbcnode, obcnode, *ntypes, ap);
  va_end(ap);
}

void tioga_preprocess_grids_(void) {
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *b = G.b[ib];
    b->nfringe = G.nfringe;
    for (int i = 0; i < b->nnodes; i++) b->iblank[i] = 1;
    if (b->check_uniform_flag) { /* MeshBlock.C:84-87 */
      check_for_uniform_hex(b);
      if (b->uniform_hex) create_hex_cell_map(b);
    }
    find_obb(b->x, b->nnodes, &b->obb);
    tag_boundary(b);
  }
}

void tioga_performconnectivity_(void) {
  get_holemaps();
  exchange_boxes();
  exchange_search_data();
  for (int ib = 0; ib < G.nblocks; ib++) {
    G.b[ib]->ninterp = 0;
    search_block(G.b[ib]);
  }
  exchange_donors();
  G.ihighGlobal = G.ihigh; /* tioga.C:138 */
  for (int ib = 0; ib < G.nblocks; ib++) cell_iblanks(G.b[ib]);
  free(G.qblock);
  G.qblock = (double **)calloc(G.nblocks ? G.nblocks : 1, sizeof(double *));
}

void tioga_registersolution_(int *btag, double *q) {
  int ib = find_tag(*btag);
  if (ib < 0 || G.qblock == NULL) {
    fprintf(stderr, "#tioga_oracle: registersolution before connectivity or unknown tag\n");
    return;
  }
  G.qblock[ib] = q;
}

/* tioga.C:336-524 + dataUpdate.C:27-119 */
static void data_update(int nvar, int itype) {
  for (int ib = 0; ib < G.nblocks; ib++)
    if (G.qblock == NULL || G.qblock[ib] == NULL) {
      printf("Solution data not set, cannot update \n");
      return;
    }
  if (!G.nsend) return;
  size_t tot = 0;
  for (int ib = 0; ib < G.nblocks; ib++) tot += (size_t)G.b[ib]->ninterp;
  double *vals = (double *)malloc(sizeof(double) * (tot * nvar + 1));
  size_t r = 0;
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *d = G.b[ib];
    const double *q = G.qblock[ib];
    for (int k = 0; k < d->ninterp; k++) {
      const interp_t *it = &d->interp[k];
      if (it->cancel) continue;
      double *qq = vals + r * nvar;
      for (int v = 0; v < nvar; v++) qq[v] = 0;
      for (int m = 0; m < it->nw; m++) {
        int node = it->inode[m];
        double w = it->w[m];
        for (int v = 0; v < nvar; v++)
          qq[v] += (itype == 0 ? q[node * nvar + v] : q[v * d->nnodes + node]) * w;
      }
      r++;
    }
  }
  r = 0;
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *d = G.b[ib];
    for (int k = 0; k < d->ninterp; k++) {
      const interp_t *it = &d->interp[k];
      if (it->cancel) continue;
      int rb = it->rinfo[2], node = it->rinfo[1];
      block_t *rcv = G.b[rb];
      double *q = G.qblock[rb];
      for (int v = 0; v < nvar; v++) {
        if (itype == 0) q[node * nvar + v] = vals[r * nvar + v];
        else q[rcv->nnodes * v + node] = vals[r * nvar + v];
      }
      r++;
    }
  }
  free(vals);
}

void tioga_dataupdate_mb_(int *nvar, char *itype) {
  int t;
  if (strstr(itype, "row")) t = 0;
  else if (strstr(itype, "column")) t = 1;
  else {
    printf("#tiogaInterface.C:dataupdate_:unknown data orientation\n");
    return;
  }
  if (G.ihighGlobal) data_update_points(*nvar, t); /* tiogaInterface.C:194-214 */
  else data_update(*nvar, t);
}

/* The reference looks up mesh tag 0 here, which never exists (undefined
 * behaviour); this restatement binds q to the only block. */
void tioga_dataupdate_(double *q, int *nvar, char *itype) {
  if (G.qblock && G.nblocks > 0) G.qblock[0] = q;
  tioga_dataupdate_mb_(nvar, itype);
}

void tioga_getdonorcount_(int *btag, int *dcount, int *fcount) {
  *dcount = *fcount = 0;
  if (!G.nsend) return;
  int ib = find_tag(*btag);
  if (ib < 0) return;
  block_t *d = G.b[ib];
  for (int k = 0; k < d->ninterp; k++)
    if (!d->interp[k].cancel) {
      (*dcount)++;
      (*fcount) += d->interp[k].nw + 1;
    }
}

void tioga_getdonorinfo_(int *btag, int *receptors, int *indices, double *frac, int *dcount) {
  (void)dcount;
  if (!G.nsend) return;
  int ib = find_tag(*btag);
  if (ib < 0) return;
  block_t *d = G.b[ib];
  int j = 0, k = 0;
  for (int i = 0; i < d->ninterp; i++) {
    const interp_t *it = &d->interp[i];
    if (it->cancel) continue;
    for (int m = 0; m < it->nw + 1; m++) {
      indices[j] = it->inode[m];
      frac[j] = it->w[m];
      j++;
    }
    receptors[k++] = 0; /* the receptor's rank (sndMap of the only slot) */
    receptors[k++] = it->rinfo[1];
    receptors[k++] = it->rinfo[2];
    receptors[k++] = it->nw;
  }
}

void tioga_setsymmetry_(int *isym) { G.isym = *isym; }
void tioga_setnfringe_(int *nfringe) { G.nfringe = *nfringe; }
void tioga_setmexclude_(int *mexclude) { G.mexclude = *mexclude; }

void tioga_setresolutions_(double *nres, double *cres) {
  if (G.nblocks < 1) return;
  G.b[0]->user_nres = nres;
  G.b[0]->user_cres = cres;
}

void tioga_setresolutions_multi_(int *btag, double *nres, double *cres) {
  int ib = find_tag(*btag);
  if (ib < 0) return;
  G.b[ib]->user_nres = nres;
  G.b[ib]->user_cres = cres;
}

void tioga_setcelliblank_(int *iblank_cell) {
  if (G.nblocks < 1) return;
  block_t *b = G.b[0];
  if (b->own_iblank_cell) free(b->iblank_cell);
  b->own_iblank_cell = 0;
  b->iblank_cell = iblank_cell;
}

void tioga_delete_(void) {
  for (int i = 0; i < G.nblocks; i++) free_block(G.b[i]);
  free_holemaps();
  free(G.pair_ib);
  free(G.pair_ob);
  free(G.pair_obb);
  free(G.qblock);
  memset(&G, 0, sizeof(G));
}

/* tioga::reduce_fringes (src/tioga.C:737-885) with MeshBlock::reduce_fringes
 * (src/bookKeeping.C:650-760): keep only the receptors within nfringe+1
 * layers of the field, cancel the others through their head donor
 * (getCancellationData, cancelDonor: bookKeeping.C:542-570), resetCoincident,
 * then clearIblanks (receptors -> 1, nodes outside the reduced set -> 0,
 * bookKeeping.C:615-625) and setIblanks for the surviving interpolations. */
void tioga_reduce_fringes_(void) {
  int **red = (int **)calloc(G.nblocks ? G.nblocks : 1, sizeof(int *));
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *r = G.b[ib];
    int nn = r->nnodes;
    red[ib] = (int *)malloc(sizeof(int) * (nn ? nn : 1));
    int *tmp = (int *)malloc(sizeof(int) * (nn ? nn : 1));
    for (int i = 0; i < nn; i++) red[ib][i] = r->iblank[i] > 0 ? r->iblank[i] : 0;
    for (int i = 0; i < nn; i++) tmp[i] = red[ib][i];
    for (int iter = 0; iter < r->nfringe + 1; iter++) {
      for (int n = 0; n < r->ntypes; n++) {
        int nvert = r->nv[n];
        for (int i = 0; i < r->nc[n]; i++) {
          const int *cv = r->vconn[n] + nvert * i;
          int ncount = 0;
          for (int m = 0; m < nvert; m++) {
            int v = cv[m] - 1;
            ncount = ncount + (red[ib][v] == 1 || red[ib][v] < 0);
          }
          if (ncount > 0 && ncount < nvert)
            for (int m = 0; m < nvert; m++) {
              int v = cv[m] - 1;
              if (tmp[v] == 0 && r->iblank[v] < 0) tmp[v] = r->iblank[v];
            }
        }
      }
      for (int i = 0; i < nn; i++) red[ib][i] = tmp[i];
    }
    free(tmp);
  }
  /* cancellations through each cancelled node's head donor, node order */
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *r = G.b[ib];
    for (int v = 0; v < r->nnodes; v++) {
      if (!(r->iblank[v] < 0 && red[ib][v] == 0)) continue;
      if (r->dl_cnt == NULL || r->dl_cnt[v] == 0) continue;
      const cand_t *h = &r->dl[r->dl_off[v]];
      block_t *dd = G.b[find_tag(h->mtag)];
      int ip = dd->interp2donor[h->remote];
      if (ip > -1) dd->interp[ip].cancel = 1;
    }
  }
  /* resetCoincident (bookKeeping.C:572-597) */
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *d = G.b[ib];
    if (d->interp2donor == NULL) continue;
    int *reset = (int *)malloc(sizeof(int) * (d->nsearch ? d->nsearch : 1));
    for (int q = 0; q < d->nsearch; q++) reset[q] = 1;
    for (int q = 0; q < d->nsearch; q++) {
      int ip = d->interp2donor[q];
      if (ip > -1 && d->interp[ip].cancel < reset[d->xtag[q]]) reset[d->xtag[q]] = d->interp[ip].cancel;
    }
    for (int q = 0; q < d->nsearch; q++) {
      int ip = d->interp2donor[q];
      if (ip > -1 && d->interp[ip].cancel == 1) d->interp[ip].cancel = reset[d->xtag[q]];
    }
    free(reset);
  }
  /* clearIblanks, then setIblanks for the surviving interpolations */
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *r = G.b[ib];
    for (int i = 0; i < r->nnodes; i++)
      if (r->iblank[i] < 0) r->iblank[i] = 1;
    for (int i = 0; i < r->nnodes; i++)
      if (red[ib][i] == 0) r->iblank[i] = 0;
    free(red[ib]);
  }
  free(red);
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *d = G.b[ib];
    for (int k = 0; k < d->ninterp; k++)
      if (!d->interp[k].cancel) G.b[d->interp[k].rinfo[2]]->iblank[d->interp[k].rinfo[1]] = -1;
  }
}

/* ======================================================================= */
/* high-order path: tioga.C:162-178, highOrder.C:152-566, exchangeSearchData  */
/* ======================================================================= */
void tioga_set_highorder_callback_(void (*f1)(int *, int *), void (*f2)(int *, int *, double *),
                                   void (*f3)(int *, double *, int *, double *),
                                   void (*f4)(int *, double *, int *, int *, double *, double *, int *),
                                   void (*f5)(int *, int *, double *, int *, int *, double *)) {
  G.get_nodes_per_cell = f1;
  G.get_receptor_nodes = f2;
  G.donor_inclusion_test = f3;
  G.donor_frac = f4;
  G.convert_to_modal = f5;
  G.ihigh = 1; /* tioga.h:211-223 */
}

/* oracle only: fn(block index) is called before the callbacks of a block */
void tioga_oracle_set_block_hook(void (*fn)(int)) { G.block_hook = fn; }

/* highOrder.C:208-247: receptor cells (iblank_cell == -1) and their points */
static void get_internal_nodes(int ib) {
  block_t *b = G.b[ib];
  free(b->ctag);
  b->ctag = (int *)malloc(sizeof(int) * (b->ncells ? b->ncells : 1));
  b->nrc = 0;
  for (int i = 0; i < b->ncells; i++)
    if (b->iblank_cell[i] == -1) b->ctag[b->nrc++] = i + 1;
  free(b->ppc);
  b->ppc = (int *)malloc(sizeof(int) * (b->nrc ? b->nrc : 1));
  b->ntp = 0;
  ho_hook(ib);
  for (int i = 0; i < b->nrc; i++) {
    G.get_nodes_per_cell(&b->ctag[i], &b->ppc[i]);
    b->ntp += b->ppc[i];
  }
  free(b->rxyz);
  b->rxyz = (double *)malloc(sizeof(double) * 3 * (b->ntp ? b->ntp : 1));
  for (int i = 0, m = 0; i < b->nrc; i++) {
    G.get_receptor_nodes(&b->ctag[i], &b->ppc[i], b->rxyz + m);
    m += 3 * b->ppc[i];
  }
}

/* exchangeSearchData(at_points = 1) + getExtraQueryPoints (highOrder.C:272-319):
 * every receptor point inside the pair's box, in point order, res = BIG */
static void exchange_search_points(void) {
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *b = G.b[ib];
    b->nsearch = 0;
    free(b->xsearch); b->xsearch = NULL;
    free(b->isearch); b->isearch = NULL;
    free(b->tagsearch); b->tagsearch = NULL;
    free(b->donorId); b->donorId = NULL;
    free(b->res_search); b->res_search = NULL;
    free(b->rst); b->rst = NULL;
  }
  int **lists = (int **)malloc(sizeof(int *) * (G.npairs + 1));
  int *counts = (int *)calloc(G.npairs + 1, sizeof(int));
  for (int p = 0; p < G.npairs; p++) {
    block_t *rec = G.b[G.pair_ib[p]];
    const obb_t *o = &G.pair_obb[p];
    lists[p] = (int *)malloc(sizeof(int) * (rec->ntp ? rec->ntp : 1));
    for (int i = 0; i < rec->ntp; i++) {
      double xd[3];
      for (int j = 0; j < 3; j++) xd[j] = 0;
      for (int j = 0; j < 3; j++)
        for (int k = 0; k < 3; k++) xd[j] += (rec->rxyz[3 * i + k] - o->xc[k]) * o->vec[j][k];
      if (fabs(xd[0]) <= o->dxc[0] && fabs(xd[1]) <= o->dxc[1] && fabs(xd[2]) <= o->dxc[2])
        lists[p][counts[p]++] = i;
    }
    G.b[G.pair_ob[p]]->nsearch += counts[p];
  }
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *b = G.b[ib];
    if (b->nsearch < 1) continue;
    b->xsearch = (double *)malloc(sizeof(double) * 3 * b->nsearch);
    b->res_search = (double *)malloc(sizeof(double) * b->nsearch);
    b->isearch = (int *)malloc(sizeof(int) * 3 * b->nsearch);
    b->tagsearch = (int *)malloc(sizeof(int) * b->nsearch);
    b->donorId = (int *)malloc(sizeof(int) * b->nsearch);
    b->rst = (double *)calloc(3 * (size_t)b->nsearch, sizeof(double));
  }
  int *fill = (int *)calloc(G.nblocks, sizeof(int));
  for (int p = 0; p < G.npairs; p++) {
    block_t *rec = G.b[G.pair_ib[p]], *don = G.b[G.pair_ob[p]];
    int ob = G.pair_ob[p];
    for (int j = 0; j < counts[p]; j++) {
      int pt = lists[p][j], q = fill[ob]++;
      don->isearch[3 * q] = 0;
      don->isearch[3 * q + 1] = pt;
      don->isearch[3 * q + 2] = G.pair_ib[p];
      don->tagsearch[q] = rec->tag;
      for (int k = 0; k < 3; k++) don->xsearch[3 * q + k] = rec->rxyz[3 * pt + k];
      don->res_search[q] = BIGVALUE;
    }
    free(lists[p]);
  }
  free(fill);
  free(lists);
  free(counts);
}

/* highOrder.C:321-419 (ihigh branch): point donors that are field cells */
static void process_point_donors(int ib) {
  block_t *b = G.b[ib];
  free(b->i2_inode0); free(b->i2_nw); free(b->i2_rinfo); free(b->i2_w);
  b->ninterp2 = 0;
  for (int i = 0; i < b->nsearch; i++)
    if (b->donorId[i] > -1 && b->iblank_cell[b->donorId[i]] == 1) b->ninterp2++;
  const int n = b->ninterp2 ? b->ninterp2 : 1;
  b->i2_inode0 = (int *)malloc(sizeof(int) * n);
  b->i2_nw = (int *)malloc(sizeof(int) * n);
  b->i2_rinfo = (int *)malloc(sizeof(int) * 2 * n);
  b->i2_w = (double *)malloc(sizeof(double) * NFRAC * (size_t)n);
  ho_hook(ib);
  for (int i = 0, m = 0; i < b->nsearch; i++) {
    if (b->donorId[i] > -1 && b->iblank_cell[b->donorId[i]] == 1) {
      int icell = b->donorId[i] + 1, ndim = NFRAC;
      b->i2_nw[m] = 0;
      G.donor_frac(&icell, b->xsearch + 3 * i, &b->i2_nw[m], &b->i2_inode0[m], b->i2_w + (size_t)NFRAC * m,
                   b->rst + 3 * i, &ndim);
      b->i2_rinfo[2 * m] = b->isearch[3 * i + 1];
      b->i2_rinfo[2 * m + 1] = b->isearch[3 * i + 2];
      m++;
    }
  }
}

void tioga_performconnectivity_highorder_(void) {
  if (!G.ihigh) {
    fprintf(stderr, "#tioga_oracle: performconnectivity_highorder without callbacks is not restated\n");
    return;
  }
  for (int ib = 0; ib < G.nblocks; ib++) get_internal_nodes(ib);
  exchange_search_points();
  G.ihigh_search = 1;
  for (int ib = 0; ib < G.nblocks; ib++) {
    ho_hook(ib);
    search_block(G.b[ib]);
    process_point_donors(ib);
  }
  G.ihigh_search = 0;
}

/* tioga.C:336-524 with at_points = 1, ROW (getInterpolatedSolutionAtPoints
 * ihigh branch, highOrder.C:421-477; receptor side, clearOrphans 152-205,
 * updatePointData 479-566).  A point reached by several donors keeps the
 * last one in packet order (donor blocks in order, then list order). */
static void data_update_points(int nvar, int itype) {
  for (int ib = 0; ib < G.nblocks; ib++)
    if (G.qblock == NULL || G.qblock[ib] == NULL) {
      printf("Solution data not set, cannot update \n");
      return;
    }
  if (!G.nsend) return;
  if (itype != 0) {
    fprintf(stderr, "#tioga_oracle: high-order data update is ROW only (highOrder.C:474)\n");
    return;
  }
  double **qtmp = (double **)malloc(sizeof(double *) * G.nblocks);
  int **itmp = (int **)malloc(sizeof(int *) * G.nblocks);
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *b = G.b[ib];
    qtmp[ib] = (double *)calloc((size_t)(b->ntp ? b->ntp : 1) * nvar, sizeof(double));
    itmp[ib] = (int *)calloc(b->ntp ? b->ntp : 1, sizeof(int));
  }
  double *qq = (double *)malloc(sizeof(double) * nvar);
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *d = G.b[ib];
    const double *q = G.qblock[ib];
    for (int i = 0; i < d->ninterp2; i++) {
      for (int k = 0; k < nvar; k++) qq[k] = 0;
      const int inode = d->i2_inode0[i] - 1;
      for (int m = 0; m < d->i2_nw[i]; m++) {
        const double w = d->i2_w[(size_t)NFRAC * i + m];
        for (int k = 0; k < nvar; k++) qq[k] += q[inode + m * nvar + k] * w;
      }
      const int pt = d->i2_rinfo[2 * i], rb = d->i2_rinfo[2 * i + 1];
      for (int k = 0; k < nvar; k++) qtmp[rb][(size_t)pt * nvar + k] = qq[k];
      itmp[rb][pt] = 1;
    }
  }
  free(qq);
  for (int ib = 0; ib < G.nblocks; ib++) {
    block_t *b = G.b[ib];
    /* clearOrphans: the last orphan point of a cell decides */
    for (int i = 0, m = 0; i < b->nrc; i++) {
      int reject = 0;
      for (int j = 0; j < b->ppc[i]; j++, m++) {
        if (itmp[ib][m] == 0) {
          reject = 2;
          for (int k = 0; k < G.nmesh; k++)
            if (k != b->tag - 1 && G.hm[k].exist && check_holemap(b->rxyz + 3 * m, &G.hm[k])) {
              reject = 1;
              break;
            }
        }
      }
      if (reject == 1) b->iblank_cell[b->ctag[i] - 1] = 0;
      else if (reject == 2) b->iblank_cell[b->ctag[i] - 1] = 1;
    }
    /* updatePointData */
    double *qout = (double *)malloc(sizeof(double) * (size_t)nvar * NFRAC);
    ho_hook(ib);
    for (int i = 0, m = 0; i < b->nrc; i++) {
      if (b->iblank_cell[b->ctag[i] - 1] == -1) {
        int npts = NFRAC, index_out = 0;
        G.convert_to_modal(&b->ctag[i], &b->ppc[i], qtmp[ib] + m, &npts, &index_out, qout);
        index_out -= 1;
        for (int j = 0, k = 0; j < npts; j++)
          for (int n = 0; n < nvar; n++, k++) G.qblock[ib][index_out + j * nvar + n] = qout[k];
      }
      m += b->ppc[i] * nvar;
    }
    free(qout);
    free(qtmp[ib]);
    free(itmp[ib]);
  }
  free(qtmp);
  free(itmp);
}

/* oracle only: point donors of block btag's list, in list order: for each
 * record (receptor block, point id, donor cell 0-based, weights count) */
int tioga_oracle_pointdonors(int btag, int *out, double *w) {
  int ib = find_tag(btag);
  if (ib < 0) return 0;
  block_t *b = G.b[ib];
  if (out)
    for (int i = 0; i < b->ninterp2; i++) {
      out[4 * i] = b->i2_rinfo[2 * i + 1];
      out[4 * i + 1] = b->i2_rinfo[2 * i];
      out[4 * i + 2] = b->i2_inode0[i];
      out[4 * i + 3] = b->i2_nw[i];
      if (w) memcpy(w + (size_t)NFRAC * i, b->i2_w + (size_t)NFRAC * i, sizeof(double) * b->i2_nw[i]);
    }
  return b->ninterp2;
}

/* ---- oracle-only diagnostics for the tests ---------------------------- */
/* Cell iblank of block btag (computed for every block, not only the one a
 * solver registered through tioga_setcelliblank_). */
void tioga_oracle_getcelliblank(int btag, int *out) {
  int ib = find_tag(btag);
  if (ib < 0) return;
  block_t *b = G.b[ib];
  if (b->iblank_cell) memcpy(out, b->iblank_cell, sizeof(int) * b->ncells);
}

/* Number of query points and found donors of block btag. */
void tioga_oracle_searchstats(int btag, int *nsearch, int *ndonor) {
  int ib = find_tag(btag);
  *nsearch = *ndonor = 0;
  if (ib < 0) return;
  block_t *b = G.b[ib];
  *nsearch = b->nsearch;
  for (int q = 0; q < b->nsearch; q++) *ndonor += (b->donorId[q] > -1);
}
