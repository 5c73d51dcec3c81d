/*
 * fesom_oracle.c -- CPU oracle (test infrastructure) for the FESOM2 tracer
 * advection step.  Every routine restates the reference loop it names, with
 * the same loop bounds, the same evaluation order of floating-point
 * expressions and no fused multiply-add (built with -ffp-contract=off), so
 * that a CUDA kernel that follows the same order can be compared bit for bit.
 *
 * Reference: suvarchal/fesom2_tracer_dwarf.  File:line citations below are
 * relative to that project's root.
 *
 * Indices: A2(a,i,j,ld) is the Fortran element a(i,j) of an array whose
 * leading dimension is ld; all mesh index arrays are 1-based as in Fortran.
 *
 * Parity anchors: the UPW1/UPW1/NONE path on the 20x20x10 periodic mesh is
 * pinned against the reference's printed golden numbers (README.md:51-52);
 * MUSCL/MFCT/PPM/QR4C/CDIFF/FCT are not pinned by any reference test and are
 * checked through invariants (conservation, FCT bounds, constant
 * preservation) in tests/.
 */
#include "fesom_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define A2(a, i, j, ld) (a)[(size_t)((j)-1) * (size_t)(ld) + (size_t)((i)-1)]
#define A3(a, i, j, k, ld1, ld2) \
  (a)[((size_t)((k)-1) * (size_t)(ld2) + (size_t)((j)-1)) * (size_t)(ld1) + (size_t)((i)-1)]

/* lib/oce_modules.F90:19,24 */
static const double PI_F = 3.14159265358979;
static const double R_EARTH = 6367500.0;
/* lib/gen_modules_config.F90:83 (degrees; never fires on the analytic mesh) */
static const double CYCLIC_LENGTH = 360.0;

/* Fortran MAX/MIN as used throughout: the first argument wins ties. */
static inline double fmax2(double a, double b) { return (b > a) ? b : a; }
static inline double fmin2(double a, double b) { return (b < a) ? b : a; }
static inline double fmax3(double a, double b, double c) { return fmax2(fmax2(a, b), c); }
static inline double fmin3(double a, double b, double c) { return fmin2(fmin2(a, b), c); }
static inline int imax2(int a, int b) { return a > b ? a : b; }
static inline int imin2(int a, int b) { return a < b ? a : b; }

struct om_mesh {
  int nx, ny, nl, periodic, full_rings;
  double Lx, Ly, max_depth;
  double cyclic;            /* cyclic_length in the units of coord         */
  int nod2D, nod2D_total, elem2D, edge2D, max_nie;
  double *coord;            /* (2, nod2D_total), radians                   */
  int *elem2D_nodes;        /* (3, elem2D), after the periodic remap       */
  int *edges;               /* (2, edge2D), after the periodic remap       */
  int *edge_tri;            /* (2, edge2D)                                 */
  int *nlevels, *ulevels;   /* (elem2D)                                    */
  int *nlevels_nod2D, *ulevels_nod2D;          /* (nod2D_total)            */
  int *nlevels_nod2D_min, *ulevels_nod2D_max;  /* (nod2D)                  */
  int *nod_in_elem2D_num;   /* (nod2D_total)                               */
  int *nod_in_elem2D;       /* (max_nie, nod2D_total)                      */
  double *elem_area;        /* (elem2D) m^2                                */
  double *area, *areasvol;  /* (nl, nod2D_total) m^2                       */
  double *edge_dxdy;        /* (2, edge2D) radians                         */
  double *edge_cross_dxdy;  /* (4, edge2D) m                               */
  double *gradient_sca;     /* (6, elem2D)                                 */
  double *elem_cos;         /* (elem2D)                                    */
  double *zbar, *Z;         /* (nl), (nl-1)                                */
  double *hnode, *hnode_new;/* (nl-1, nod2D)                               */
  double *helem;            /* (nl-1, elem2D)                              */
  double *zbar_3d_n;        /* (nl, nod2D)                                 */
  double *Z_3d_n;           /* (nl-1, nod2D)                               */
  int *edge_up_dn_tri;      /* (2, edge2D)                                 */
  int *nboundary_lay;       /* (nod2D)                                     */
  struct om_work_s *work;   /* step workspace, allocated on first use      */
};

/* ------------------------------------------------------------------------ */
/* threads                                                                   */
/* ------------------------------------------------------------------------ */
void om_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
int om_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* Owned node range of the calling thread.  Edge scatters are parallelised by
 * letting every thread walk all edges in order and apply only the updates of
 * the nodes it owns, so every node receives its contributions in edge order
 * (the serial order of the reference's scatter loops). */
static void own_range(int nod2D, int *lo, int *hi) {
#ifdef _OPENMP
  int t = omp_get_thread_num(), nt = omp_get_num_threads();
#else
  int t = 0, nt = 1;
#endif
  *lo = (int)((long long)nod2D * t / nt) + 1;
  *hi = (int)((long long)nod2D * (t + 1) / nt);
}

/* ------------------------------------------------------------------------ */
/* analytic mesh: lib/analytic_mesh.F90:114-829                             */
/* ------------------------------------------------------------------------ */
static void trim_cyclic(double *b) { /* lib/gen_modules_rotate_grid.F90:216-223 */
  if (*b > CYCLIC_LENGTH / 2.0) *b = *b - CYCLIC_LENGTH;
  if (*b < -CYCLIC_LENGTH / 2.0) *b = *b + CYCLIC_LENGTH;
}

/* trim_cyclic with the mesh's cyclic length */
static void trim_cyc(double *b, double L) {
  if (*b > L / 2.0) *b = *b - L;
  if (*b < -L / 2.0) *b = *b + L;
}

/* lib/oce_mesh.F90:2001-2019 */
static void edge_center(const om_mesh *m, int n1, int n2, double *x, double *y) {
  const double L = m->cyclic;
  double a1 = A2(m->coord, 1, n1, 2), a2 = A2(m->coord, 2, n1, 2);
  double b1 = A2(m->coord, 1, n2, 2), b2 = A2(m->coord, 2, n2, 2);
  if (a1 - b1 > L / 2.0) a1 = a1 - L;
  if (a1 - b1 < -L / 2.0) b1 = b1 - L;
  *x = 0.5 * (a1 + b1);
  *y = 0.5 * (a2 + b2);
}

/* lib/oce_mesh.F90:2021-2041 */
static void elem_center(const om_mesh *m, const int *elnodes, double *x, double *y) {
  double ax[3];
  for (int k = 0; k < 3; k++) ax[k] = A2(m->coord, 1, elnodes[k], 2);
  double amin = fmin3(ax[0], ax[1], ax[2]);
  for (int k = 0; k < 3; k++) {
    if (ax[k] - amin >= m->cyclic / 2.0) ax[k] = ax[k] - m->cyclic;
    if (ax[k] - amin < -m->cyclic / 2.0) ax[k] = ax[k] + m->cyclic;
  }
  *x = ((ax[0] + ax[1]) + ax[2]) / 3.0;
  *y = ((A2(m->coord, 2, elnodes[0], 2) + A2(m->coord, 2, elnodes[1], 2)) +
        A2(m->coord, 2, elnodes[2], 2)) / 3.0;
}

/* Minimum-image wrap of a coordinate difference on the periodic analytic mesh
 * (period P in radians).  Replaces the reference's cyclic_length trim, which
 * never fires on a Cartesian mesh measured in radians
 * (lib/oce_muscl_adv.F90:248-249,266-269). */
static void trim_period(double *v, double P) {
  if (*v > 0.5 * P) *v = *v - P;
  if (*v < -0.5 * P) *v = *v + P;
}

/* lib/oce_muscl_adv.F90:166-357 (up/down-wind triangle search), with the
 * minimum-image wrap on periodic meshes; e_nodes/coord_elem are the remapped
 * element nodes and their coordinates. */
static void find_up_downwind_triangles(om_mesh *m) {
  const int periodic = m->periodic;
  const double Px = m->Lx / R_EARTH, Py = m->Ly / R_EARTH;
  for (int n = 1; n <= m->edge2D; n++) {
    int ed1 = A2(m->edges, 1, n, 2), ed2 = A2(m->edges, 2, n, 2);
    for (int side = 0; side < 2; side++) {
      int ednode = side == 0 ? ed1 : ed2;
      double x[2];
      x[0] = A2(m->coord, 1, ed2, 2) - A2(m->coord, 1, ed1, 2);
      x[1] = A2(m->coord, 2, ed2, 2) - A2(m->coord, 2, ed1, 2);
      trim_cyc(&x[0], m->cyclic);
      if (periodic) { trim_period(&x[0], Px); trim_period(&x[1], Py); }
      if (side == 0) { x[0] = -x[0]; x[1] = -x[1]; }
      for (int k = 1; k <= m->nod_in_elem2D_num[ednode - 1]; k++) {
        int elem = A2(m->nod_in_elem2D, k, ednode, m->max_nie);
        const int *en = &A2(m->elem2D_nodes, 1, elem, 3);
        int i0, i1, i2;
        if (en[0] == ednode) { i0 = 0; i1 = 1; i2 = 2; }
        else if (en[1] == ednode) { i0 = 1; i1 = 0; i2 = 2; }
        else { i0 = 2; i1 = 0; i2 = 1; }
        double b[2], c[2];
        b[0] = A2(m->coord, 1, en[i1], 2) - A2(m->coord, 1, en[i0], 2);
        b[1] = A2(m->coord, 2, en[i1], 2) - A2(m->coord, 2, en[i0], 2);
        c[0] = A2(m->coord, 1, en[i2], 2) - A2(m->coord, 1, en[i0], 2);
        c[1] = A2(m->coord, 2, en[i2], 2) - A2(m->coord, 2, en[i0], 2);
        trim_cyc(&b[0], m->cyclic);
        trim_cyc(&c[0], m->cyclic);
        if (periodic) {
          trim_period(&b[0], Px); trim_period(&b[1], Py);
          trim_period(&c[0], Px); trim_period(&c[1], Py);
        }
        double cr = c[0] * c[0] + c[1] * c[1];
        double bx = (b[0] * c[0] + b[1] * c[1]) / cr;
        double by = (-b[0] * c[1] + b[1] * c[0]) / cr;
        double xx = (x[0] * c[0] + x[1] * c[1]) / cr;
        double xy = (-x[0] * c[1] + x[1] * c[0]) / cr;
        double ab = atan2(by, bx);
        double ax = atan2(xy, xx);
        /* "cycle" continues the search: the last match wins. */
        if ((ab > 0.0) && (ax > 0.0) && (ax < ab)) { A2(m->edge_up_dn_tri, side + 1, n, 2) = elem; continue; }
        if ((ab < 0.0) && (ax < 0.0) && (ax > ab)) { A2(m->edge_up_dn_tri, side + 1, n, 2) = elem; continue; }
        if ((ab == ax) || (ax == 0.0)) { A2(m->edge_up_dn_tri, side + 1, n, 2) = elem; continue; }
      }
    }
  }
}

/* lib/oce_muscl_adv.F90:96-161 */
static void init_nboundary_lay(om_mesh *m) {
  for (int n = 1; n <= m->nod2D; n++) m->nboundary_lay[n - 1] = m->nl - 1;
  for (int n = 1; n <= m->edge2D; n++) {
    int n1 = A2(m->edges, 1, n, 2), n2 = A2(m->edges, 2, n, 2);
    int t1 = A2(m->edge_tri, 1, n, 2), t2 = A2(m->edge_tri, 2, n, 2);
    if (t1 <= 0 || t2 <= 0) {
      m->nboundary_lay[n1 - 1] = 0;
      m->nboundary_lay[n2 - 1] = 0;
    } else {
      int mn = imin2(m->nlevels[t1 - 1], m->nlevels[t2 - 1]) - 1;
      m->nboundary_lay[n1 - 1] = imin2(m->nboundary_lay[n1 - 1], mn);
      m->nboundary_lay[n2 - 1] = imin2(m->nboundary_lay[n2 - 1], mn);
    }
  }
}

static void build_nod_in_elem(om_mesh *m, int nnodes) {
  free(m->nod_in_elem2D_num);
  free(m->nod_in_elem2D);
  m->nod_in_elem2D_num = (int *)calloc((size_t)nnodes, sizeof(int));
  for (int e = 1; e <= m->elem2D; e++)
    for (int j = 1; j <= 3; j++) m->nod_in_elem2D_num[A2(m->elem2D_nodes, j, e, 3) - 1]++;
  int mx = 0;
  for (int n = 0; n < nnodes; n++) mx = imax2(mx, m->nod_in_elem2D_num[n]);
  m->max_nie = mx;
  m->nod_in_elem2D = (int *)calloc((size_t)mx * nnodes, sizeof(int));
  memset(m->nod_in_elem2D_num, 0, sizeof(int) * (size_t)nnodes);
  for (int e = 1; e <= m->elem2D; e++)
    for (int j = 1; j <= 3; j++) {
      int node = A2(m->elem2D_nodes, j, e, 3);
      m->nod_in_elem2D_num[node - 1]++;
      A2(m->nod_in_elem2D, m->nod_in_elem2D_num[node - 1], node, mx) = e;
    }
}

om_mesh *om_mesh_analytic(int nx, int ny, int nl, double Lx, double Ly,
                          double max_depth, int periodic, int options,
                          const int *node_K) {
  if (nx < 2 || ny < 2 || nl < 3) return NULL;
  om_mesh *m = (om_mesh *)calloc(1, sizeof(om_mesh));
  m->cyclic = CYCLIC_LENGTH;
  m->nx = nx; m->ny = ny; m->nl = nl; m->periodic = periodic ? 1 : 0;
  m->full_rings = (options & OM_FULL_RINGS) ? 1 : 0;
  const int left = (options & OM_LEFT_ORIENTED) ? 1 : 0;
  m->Lx = Lx; m->Ly = Ly; m->max_depth = max_depth;

  /* 1b. sizes (lib/analytic_mesh.F90:175-190) */
  int nod_local, eDim, n_total_edges;
  if (periodic) {
    nod_local = (nx - 1) * (ny - 1);
    eDim = (nx - 1) + (ny - 1) + 1;
    n_total_edges = 3 * (nx - 1) * (ny - 1);
  } else {
    nod_local = nx * ny;
    eDim = 0;
    n_total_edges = (nx - 1) * ny + nx * (ny - 1) + (nx - 1) * (ny - 1);
  }
  const int nod_total = nod_local + eDim;
  m->nod2D = nod_local;
  m->nod2D_total = nod_total;
  m->elem2D = 2 * (nx - 1) * (ny - 1);
  m->edge2D = n_total_edges;

#define PNODE(i, j)                                                          \
  (((i) <= nx - 1 && (j) <= ny - 1) ? ((j)-1) * (nx - 1) + (i)               \
   : ((i) == nx && (j) <= ny - 1)   ? nod_local + (j)                        \
   : ((i) <= nx - 1 && (j) == ny)   ? nod_local + (ny - 1) + (i)             \
                                    : nod_total)

  /* 1c. coordinates (lib/analytic_mesh.F90:268-305) */
  const double dx = Lx / (double)(nx - 1), dy = Ly / (double)(ny - 1);
  m->coord = (double *)calloc((size_t)2 * nod_total, sizeof(double));
  if (periodic) {
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        int n = (j - 1) * (nx - 1) + i;
        A2(m->coord, 1, n, 2) = (double)(i - 1) * dx / R_EARTH;
        A2(m->coord, 2, n, 2) = (double)(j - 1) * dy / R_EARTH;
      }
    for (int j = 1; j <= ny - 1; j++) {
      int n = nod_local + j;
      A2(m->coord, 1, n, 2) = Lx / R_EARTH;
      A2(m->coord, 2, n, 2) = (double)(j - 1) * dy / R_EARTH;
    }
    for (int i = 1; i <= nx - 1; i++) {
      int n = nod_local + (ny - 1) + i;
      A2(m->coord, 1, n, 2) = (double)(i - 1) * dx / R_EARTH;
      A2(m->coord, 2, n, 2) = Ly / R_EARTH;
    }
    A2(m->coord, 1, nod_total, 2) = Lx / R_EARTH;
    A2(m->coord, 2, nod_total, 2) = Ly / R_EARTH;
  } else {
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        int n = (j - 1) * nx + i;
        A2(m->coord, 1, n, 2) = (double)(i - 1) * dx / R_EARTH;
        A2(m->coord, 2, n, 2) = (double)(j - 1) * dy / R_EARTH;
      }
  }

  /* 1d. elements, clockwise (lib/analytic_mesh.F90:310-354) */
  m->elem2D_nodes = (int *)calloc((size_t)3 * m->elem2D, sizeof(int));
  {
    int e = 0;
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        int n1, n2, n3, n4;
        if (periodic) {
          n1 = PNODE(i, j); n2 = PNODE(i + 1, j); n3 = PNODE(i + 1, j + 1); n4 = PNODE(i, j + 1);
        } else {
          n1 = (j - 1) * nx + i; n2 = (j - 1) * nx + i + 1; n3 = j * nx + i + 1; n4 = j * nx + i;
        }
        e++;
        A2(m->elem2D_nodes, 1, e, 3) = n1; A2(m->elem2D_nodes, 2, e, 3) = n3; A2(m->elem2D_nodes, 3, e, 3) = n2;
        e++;
        A2(m->elem2D_nodes, 1, e, 3) = n1; A2(m->elem2D_nodes, 2, e, 3) = n4; A2(m->elem2D_nodes, 3, e, 3) = n3;
      }
  }

  /* 1e. vertical levels (lib/analytic_mesh.F90:359-369) */
  m->zbar = (double *)calloc((size_t)nl, sizeof(double));
  m->Z = (double *)calloc((size_t)nl, sizeof(double));
  for (int k = 1; k <= nl; k++) m->zbar[k - 1] = -((double)(k - 1) * max_depth / (double)(nl - 1));
  for (int k = 1; k <= nl - 1; k++) m->Z[k - 1] = 0.5 * (m->zbar[k - 1] + m->zbar[k]);

  /* 1f. edges and edge_tri (lib/analytic_mesh.F90:383-596) */
  m->edges = (int *)calloc((size_t)2 * n_total_edges, sizeof(int));
  m->edge_tri = (int *)calloc((size_t)2 * n_total_edges, sizeof(int));
  {
    int *en = (int *)calloc((size_t)2 * n_total_edges, sizeof(int));
    int *ee = (int *)calloc((size_t)2 * n_total_edges, sizeof(int));
    int c = 0;
    if (periodic) {
      for (int j = 1; j <= ny - 1; j++)
        for (int i = 1; i <= nx - 1; i++) {
          c++;
          A2(en, 1 + left, c, 2) = PNODE(i, j); A2(en, 2 - left, c, 2) = PNODE(i + 1, j);
          int e_lower = 2 * ((j - 1) * (nx - 1) + (i - 1)) + 1;
          int e_upper = (j >= 2) ? 2 * ((j - 2) * (nx - 1) + (i - 1)) + 2
                                 : 2 * ((ny - 2) * (nx - 1) + (i - 1)) + 2;
          A2(ee, 1, c, 2) = e_upper; A2(ee, 2, c, 2) = e_lower;
        }
      for (int j = 1; j <= ny - 1; j++)
        for (int i = 1; i <= nx - 1; i++) {
          c++;
          A2(en, 1 + left, c, 2) = PNODE(i, j); A2(en, 2 - left, c, 2) = PNODE(i, j + 1);
          int e_upper = 2 * ((j - 1) * (nx - 1) + (i - 1)) + 2;
          int e_lower = (i >= 2) ? 2 * ((j - 1) * (nx - 1) + (i - 2)) + 1
                                 : 2 * ((j - 1) * (nx - 1) + (nx - 2)) + 1;
          A2(ee, 1, c, 2) = e_upper; A2(ee, 2, c, 2) = e_lower;
        }
      for (int j = 1; j <= ny - 1; j++)
        for (int i = 1; i <= nx - 1; i++) {
          c++;
          A2(en, 1, c, 2) = PNODE(i, j); A2(en, 2, c, 2) = PNODE(i + 1, j + 1);
          A2(ee, 1, c, 2) = 2 * ((j - 1) * (nx - 1) + (i - 1)) + 2;
          A2(ee, 2, c, 2) = 2 * ((j - 1) * (nx - 1) + (i - 1)) + 1;
        }
      memcpy(m->edges, en, sizeof(int) * 2 * (size_t)n_total_edges);
      memcpy(m->edge_tri, ee, sizeof(int) * 2 * (size_t)n_total_edges);
    } else {
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx - 1; i++) {
          c++;
          A2(en, 1 + left, c, 2) = (j - 1) * nx + i; A2(en, 2 - left, c, 2) = (j - 1) * nx + i + 1;
          int e_lower = (j <= ny - 1) ? 2 * ((j - 1) * (nx - 1) + (i - 1)) + 1 : 0;
          int e_upper = (j >= 2) ? 2 * ((j - 2) * (nx - 1) + (i - 1)) + 2 : 0;
          A2(ee, 1, c, 2) = e_upper; A2(ee, 2, c, 2) = e_lower;
        }
      for (int j = 1; j <= ny - 1; j++)
        for (int i = 1; i <= nx; i++) {
          c++;
          A2(en, 1 + left, c, 2) = (j - 1) * nx + i; A2(en, 2 - left, c, 2) = j * nx + i;
          int e_upper = (i <= nx - 1) ? 2 * ((j - 1) * (nx - 1) + (i - 1)) + 2 : 0;
          int e_lower = (i >= 2) ? 2 * ((j - 1) * (nx - 1) + (i - 2)) + 1 : 0;
          A2(ee, 1, c, 2) = e_upper; A2(ee, 2, c, 2) = e_lower;
        }
      for (int j = 1; j <= ny - 1; j++)
        for (int i = 1; i <= nx - 1; i++) {
          c++;
          A2(en, 1, c, 2) = (j - 1) * nx + i; A2(en, 2, c, 2) = j * nx + i + 1;
          A2(ee, 1, c, 2) = 2 * ((j - 1) * (nx - 1) + (i - 1)) + 2;
          A2(ee, 2, c, 2) = 2 * ((j - 1) * (nx - 1) + (i - 1)) + 1;
        }
      /* zero into position 2 (lib/analytic_mesh.F90:534-539) */
      for (int n = 1; n <= n_total_edges; n++)
        if (A2(ee, 1, n, 2) == 0 && A2(ee, 2, n, 2) > 0) {
          A2(ee, 1, n, 2) = A2(ee, 2, n, 2);
          A2(ee, 2, n, 2) = 0;
        }
      /* internal edges first, boundary edges after (lib/analytic_mesh.F90:542-588) */
      int eidx = 0;
      for (int pass = 0; pass < 2; pass++)
        for (int n = 1; n <= n_total_edges; n++) {
          int bnd = !(A2(ee, 1, n, 2) > 0 && A2(ee, 2, n, 2) > 0);
          if (bnd != pass) continue;
          eidx++;
          A2(m->edges, 1, eidx, 2) = A2(en, 1, n, 2); A2(m->edges, 2, eidx, 2) = A2(en, 2, n, 2);
          A2(m->edge_tri, 1, eidx, 2) = A2(ee, 1, n, 2); A2(m->edge_tri, 2, eidx, 2) = A2(ee, 2, n, 2);
        }
    }
    free(en);
    free(ee);
  }

  /* halo -> real map (lib/analytic_mesh.F90:744-754) */
  int *h2r = (int *)calloc((size_t)(eDim > 0 ? eDim : 1), sizeof(int));
  if (periodic) {
    for (int h = 1; h <= ny - 1; h++) h2r[h - 1] = (h - 1) * (nx - 1) + 1;
    for (int h = 1; h <= nx - 1; h++) h2r[(ny - 1) + h - 1] = h;
    h2r[eDim - 1] = 1;
  }
#define REAL_OF(n) ((n) > nod_local ? h2r[(n)-nod_local - 1] : (n))

  /* 1g. levels (lib/analytic_mesh.F90:601-608); with node_K the element
   * level is the minimum over its nodes and the node level the maximum over
   * the elements around it (the FESOM convention). */
  m->nlevels = (int *)calloc((size_t)m->elem2D, sizeof(int));
  m->ulevels = (int *)calloc((size_t)m->elem2D, sizeof(int));
  m->nlevels_nod2D = (int *)calloc((size_t)nod_total, sizeof(int));
  m->ulevels_nod2D = (int *)calloc((size_t)nod_total, sizeof(int));
  for (int e = 0; e < m->elem2D; e++) { m->nlevels[e] = nl; m->ulevels[e] = 1; }
  for (int n = 0; n < nod_total; n++) { m->nlevels_nod2D[n] = nl; m->ulevels_nod2D[n] = 1; }
  if (node_K) {
    for (int e = 1; e <= m->elem2D; e++) {
      int k = nl;
      for (int j = 1; j <= 3; j++) k = imin2(k, node_K[REAL_OF(A2(m->elem2D_nodes, j, e, 3)) - 1]);
      m->nlevels[e - 1] = k;
    }
    for (int n = 0; n < nod_total; n++) m->nlevels_nod2D[n] = 0;
    for (int e = 1; e <= m->elem2D; e++)
      for (int j = 1; j <= 3; j++) {
        int r = REAL_OF(A2(m->elem2D_nodes, j, e, 3));
        m->nlevels_nod2D[r - 1] = imax2(m->nlevels_nod2D[r - 1], m->nlevels[e - 1]);
      }
    for (int n = nod_local + 1; n <= nod_total; n++) m->nlevels_nod2D[n - 1] = m->nlevels_nod2D[REAL_OF(n) - 1];
  }

  /* test_tri (lib/oce_mesh.F90:1565-1615): make every triangle clockwise */
  for (int e = 1; e <= m->elem2D; e++) {
    int *el = &A2(m->elem2D_nodes, 1, e, 3);
    double a1 = A2(m->coord, 1, el[0], 2), a2 = A2(m->coord, 2, el[0], 2);
    double b1 = A2(m->coord, 1, el[1], 2) - a1, b2 = A2(m->coord, 2, el[1], 2) - a2;
    double c1 = A2(m->coord, 1, el[2], 2) - a1, c2 = A2(m->coord, 2, el[2], 2) - a2;
    trim_cyclic(&b1);
    trim_cyclic(&c1);
    double r = b1 * c2 - b2 * c1;
    if (r > 0.0) { int t = el[1]; el[1] = el[2]; el[2] = t; }
  }

  /* nod_in_elem2D before the remap (lib/analytic_mesh.F90:675-694) */
  build_nod_in_elem(m, nod_total);

  /* find_levels_min_e2n (lib/oce_mesh.F90:1522-1560) is evaluated below,
   * after the ring mode is fixed. */

  /* mesh_areas (lib/oce_mesh.F90:2043-2309), cartesian, no cavity */
  m->elem_area = (double *)calloc((size_t)m->elem2D, sizeof(double));
  for (int n = 1; n <= m->elem2D; n++) {
    const int *el = &A2(m->elem2D_nodes, 1, n, 3);
    double ay = 1.0; /* cartesian */
    double a1 = A2(m->coord, 1, el[1], 2) - A2(m->coord, 1, el[0], 2);
    double a2 = A2(m->coord, 2, el[1], 2) - A2(m->coord, 2, el[0], 2);
    double b1 = A2(m->coord, 1, el[2], 2) - A2(m->coord, 1, el[0], 2);
    double b2 = A2(m->coord, 2, el[2], 2) - A2(m->coord, 2, el[0], 2);
    trim_cyclic(&a1);
    trim_cyclic(&b1);
    a1 = a1 * ay;
    b1 = b1 * ay;
    m->elem_area[n - 1] = 0.5 * fabs(a1 * b2 - b1 * a2);
  }
  m->area = (double *)calloc((size_t)nl * nod_total, sizeof(double));
  m->areasvol = (double *)calloc((size_t)nl * nod_total, sizeof(double));
  for (int n = 1; n <= nod_total; n++)
    for (int j = 1; j <= m->nod_in_elem2D_num[n - 1]; j++) {
      int elem = A2(m->nod_in_elem2D, j, n, m->max_nie);
      for (int nz = m->ulevels[elem - 1]; nz <= m->nlevels[elem - 1] - 1; nz++)
        A2(m->area, nz, n, nl) = A2(m->area, nz, n, nl) + m->elem_area[elem - 1] / 3.0;
    }
  for (int n = 1; n <= nod_total; n++)
    for (int nz = m->ulevels_nod2D[n - 1]; nz <= m->nlevels_nod2D[n - 1] - 1; nz++)
      A2(m->areasvol, nz, n, nl) = A2(m->area, nz, n, nl);
  for (int e = 0; e < m->elem2D; e++) m->elem_area[e] = m->elem_area[e] * R_EARTH * R_EARTH;
  for (size_t i = 0; i < (size_t)nl * nod_total; i++) {
    m->area[i] = m->area[i] * R_EARTH * R_EARTH;
    m->areasvol[i] = m->areasvol[i] * R_EARTH * R_EARTH;
  }

  /* mesh_auxiliary_arrays (lib/oce_mesh.F90:2313-2680), hot-path subset */
  m->elem_cos = (double *)calloc((size_t)m->elem2D, sizeof(double));
  double *center_x = (double *)calloc((size_t)m->elem2D, sizeof(double));
  double *center_y = (double *)calloc((size_t)m->elem2D, sizeof(double));
  for (int n = 1; n <= m->elem2D; n++) {
    double ax, ay;
    elem_center(m, &A2(m->elem2D_nodes, 1, n, 3), &ax, &ay);
    center_x[n - 1] = ax;
    center_y[n - 1] = ay;
    m->elem_cos[n - 1] = 1.0; /* cartesian (lib/oce_mesh.F90:2418-2421) */
  }
  m->edge_dxdy = (double *)calloc((size_t)2 * m->edge2D, sizeof(double));
  m->edge_cross_dxdy = (double *)calloc((size_t)4 * m->edge2D, sizeof(double));
  for (int n = 1; n <= m->edge2D; n++) {
    int ed1 = A2(m->edges, 1, n, 2), ed2 = A2(m->edges, 2, n, 2);
    double a1 = A2(m->coord, 1, ed2, 2) - A2(m->coord, 1, ed1, 2);
    double a2 = A2(m->coord, 2, ed2, 2) - A2(m->coord, 2, ed1, 2);
    trim_cyclic(&a1);
    A2(m->edge_dxdy, 1, n, 2) = a1;
    A2(m->edge_dxdy, 2, n, 2) = a2;
  }
  for (int n = 1; n <= m->edge2D; n++) {
    int ed1 = A2(m->edges, 1, n, 2), ed2 = A2(m->edges, 2, n, 2);
    int el1 = A2(m->edge_tri, 1, n, 2), el2 = A2(m->edge_tri, 2, n, 2);
    double a1, a2;
    edge_center(m, ed1, ed2, &a1, &a2);
    double b1 = center_x[el1 - 1] - a1, b2 = center_y[el1 - 1] - a2;
    trim_cyclic(&b1);
    b1 = b1 * m->elem_cos[el1 - 1];
    b1 = b1 * R_EARTH;
    b2 = b2 * R_EARTH;
    A2(m->edge_cross_dxdy, 1, n, 4) = b1;
    A2(m->edge_cross_dxdy, 2, n, 4) = b2;
    if (el2 > 0) {
      b1 = center_x[el2 - 1] - a1;
      b2 = center_y[el2 - 1] - a2;
      trim_cyclic(&b1);
      b1 = b1 * m->elem_cos[el2 - 1];
      b1 = b1 * R_EARTH;
      b2 = b2 * R_EARTH;
      A2(m->edge_cross_dxdy, 3, n, 4) = b1;
      A2(m->edge_cross_dxdy, 4, n, 4) = b2;
    } else {
      A2(m->edge_cross_dxdy, 3, n, 4) = 0.0;
      A2(m->edge_cross_dxdy, 4, n, 4) = 0.0;
    }
  }
  m->gradient_sca = (double *)calloc((size_t)6 * m->elem2D, sizeof(double));
  for (int elem = 1; elem <= m->elem2D; elem++) {
    const int *el = &A2(m->elem2D_nodes, 1, elem, 3);
    double dX31 = A2(m->coord, 1, el[2], 2) - A2(m->coord, 1, el[0], 2);
    trim_cyclic(&dX31);
    dX31 = m->elem_cos[elem - 1] * dX31;
    double dX21 = A2(m->coord, 1, el[1], 2) - A2(m->coord, 1, el[0], 2);
    trim_cyclic(&dX21);
    dX21 = m->elem_cos[elem - 1] * dX21;
    double dY31 = A2(m->coord, 2, el[2], 2) - A2(m->coord, 2, el[0], 2);
    double dY21 = A2(m->coord, 2, el[1], 2) - A2(m->coord, 2, el[0], 2);
    double dfactor = -(0.5 * R_EARTH / m->elem_area[elem - 1]);
    A2(m->gradient_sca, 1, elem, 6) = (-dY31 + dY21) * dfactor;
    A2(m->gradient_sca, 2, elem, 6) = dY31 * dfactor;
    A2(m->gradient_sca, 3, elem, 6) = -(dY21 * dfactor);
    A2(m->gradient_sca, 4, elem, 6) = (dX31 - dX21) * dfactor;
    A2(m->gradient_sca, 5, elem, 6) = -(dX31 * dfactor);
    A2(m->gradient_sca, 6, elem, 6) = dX21 * dfactor;
  }
  free(center_x);
  free(center_y);

  /* 1j. periodic post-remap (lib/analytic_mesh.F90:736-827) */
  if (periodic) {
    const double half_Lx = 0.5 * Lx, half_Ly = 0.5 * Ly;
    for (int n = 1; n <= m->edge2D; n++)
      for (int k = 1; k <= 3; k += 2) {
        double val = A2(m->edge_cross_dxdy, k, n, 4);
        if (fabs(val) > half_Lx) A2(m->edge_cross_dxdy, k, n, 4) = val - copysign(Lx, val);
        val = A2(m->edge_cross_dxdy, k + 1, n, 4);
        if (fabs(val) > half_Ly) A2(m->edge_cross_dxdy, k + 1, n, 4) = val - copysign(Ly, val);
      }
    for (int h = 1; h <= eDim; h++) {
      int r = h2r[h - 1];
      for (int nz = 1; nz <= nl - 1; nz++) {
        A2(m->area, nz, r, nl) = A2(m->area, nz, r, nl) + A2(m->area, nz, nod_local + h, nl);
        A2(m->areasvol, nz, r, nl) = A2(m->areasvol, nz, r, nl) + A2(m->areasvol, nz, nod_local + h, nl);
      }
    }
    for (int n = 1; n <= m->elem2D; n++)
      for (int k = 1; k <= 3; k++) {
        int h = A2(m->elem2D_nodes, k, n, 3);
        if (h > nod_local) A2(m->elem2D_nodes, k, n, 3) = h2r[h - nod_local - 1];
      }
    for (int n = 1; n <= m->edge2D; n++)
      for (int k = 1; k <= 2; k++) {
        int h = A2(m->edges, k, n, 2);
        if (h > nod_local) A2(m->edges, k, n, 2) = h2r[h - nod_local - 1];
      }
    if (m->full_rings) build_nod_in_elem(m, nod_local);
  }
  free(h2r);
#undef PNODE
#undef REAL_OF

  /* find_levels_min_e2n (lib/oce_mesh.F90:1522-1560) over the ring lists */
  m->nlevels_nod2D_min = (int *)calloc((size_t)m->nod2D, sizeof(int));
  m->ulevels_nod2D_max = (int *)calloc((size_t)m->nod2D, sizeof(int));
  for (int node = 1; node <= m->nod2D; node++) {
    int k = m->nod_in_elem2D_num[node - 1];
    int mn = 1 << 30, mx = -(1 << 30);
    for (int j = 1; j <= k; j++) {
      int e = A2(m->nod_in_elem2D, j, node, m->max_nie);
      mn = imin2(mn, m->nlevels[e - 1]);
      mx = imax2(mx, m->ulevels[e - 1]);
    }
    m->nlevels_nod2D_min[node - 1] = mn;
    m->ulevels_nod2D_max[node - 1] = mx;
  }

  /* ALE arrays of the analytic driver (src/fesom_analytic.F90:206-244) */
  const int nz = nl - 1;
  m->hnode = (double *)calloc((size_t)nz * m->nod2D, sizeof(double));
  m->hnode_new = (double *)calloc((size_t)nz * m->nod2D, sizeof(double));
  m->helem = (double *)calloc((size_t)nz * m->elem2D, sizeof(double));
  m->zbar_3d_n = (double *)calloc((size_t)nl * m->nod2D, sizeof(double));
  m->Z_3d_n = (double *)calloc((size_t)nz * m->nod2D, sizeof(double));
  for (int n = 1; n <= m->nod2D; n++) {
    for (int k = 1; k <= nz; k++) {
      A2(m->hnode, k, n, nz) = m->zbar[k - 1] - m->zbar[k];
      A2(m->hnode_new, k, n, nz) = A2(m->hnode, k, n, nz);
      A2(m->Z_3d_n, k, n, nz) = m->Z[k - 1];
    }
    for (int k = 1; k <= nl; k++) A2(m->zbar_3d_n, k, n, nl) = m->zbar[k - 1];
  }
  for (int e = 1; e <= m->elem2D; e++)
    for (int k = 1; k <= nz; k++) A2(m->helem, k, e, nz) = m->zbar[k - 1] - m->zbar[k];

  /* MUSCL set-up (lib/oce_muscl_adv.F90:38-357) */
  m->edge_up_dn_tri = (int *)calloc((size_t)2 * m->edge2D, sizeof(int));
  m->nboundary_lay = (int *)calloc((size_t)m->nod2D, sizeof(int));
  find_up_downwind_triangles(m);
  init_nboundary_lay(m);
  return m;
}

/* ------------------------------------------------------------------------ */
/* mesh from the ASCII mesh files: mesh_setup (lib/oce_mesh.F90:49-94) on one */
/* process, followed by the ALE arrays of tracer_init_ale_arrays             */
/* (lib/tracer_c_interface.F90:875-929) and the MUSCL set-up                 */
/* ------------------------------------------------------------------------ */

/* r2g_matrix (lib/gen_modules_rotate_grid.F90:33-56); R[i][j] = r2g_matrix(i+1, j+1) */
static void rot_matrix(double al, double be, double ga, double R[3][3]) {
  R[0][0] = cos(ga) * cos(al) - sin(ga) * cos(be) * sin(al);
  R[0][1] = cos(ga) * sin(al) + sin(ga) * cos(be) * cos(al);
  R[0][2] = sin(ga) * sin(be);
  R[1][0] = -sin(ga) * cos(al) - cos(ga) * cos(be) * sin(al);
  R[1][1] = -sin(ga) * sin(al) + cos(ga) * cos(be) * cos(al);
  R[1][2] = cos(ga) * sin(be);
  R[2][0] = sin(be) * sin(al);
  R[2][1] = -sin(be) * cos(al);
  R[2][2] = cos(be);
}

/* lib/gen_modules_rotate_grid.F90:58-80 (rotated -> geographical) */
static void rot_r2g(double R[3][3], double rlon, double rlat, double *glon, double *glat) {
  double xr = cos(rlat) * cos(rlon), yr = cos(rlat) * sin(rlon), zr = sin(rlat);
  double xg = R[0][0] * xr + R[1][0] * yr + R[2][0] * zr;
  double yg = R[0][1] * xr + R[1][1] * yr + R[2][1] * zr;
  double zg = R[0][2] * xr + R[1][2] * yr + R[2][2] * zr;
  *glat = asin(zg);
  *glon = (yg == 0.0 && xg == 0.0) ? 0.0 : atan2(yg, xg);
}

/* lib/gen_modules_rotate_grid.F90:84-106 (geographical -> rotated) */
static void rot_g2r(double R[3][3], double glon, double glat, double *rlon, double *rlat) {
  double xg = cos(glat) * cos(glon), yg = cos(glat) * sin(glon), zg = sin(glat);
  double xr = R[0][0] * xg + R[0][1] * yg + R[0][2] * zg;
  double yr = R[1][0] * xg + R[1][1] * yg + R[1][2] * zg;
  double zr = R[2][0] * xg + R[2][1] * yg + R[2][2] * zg;
  *rlat = asin(zr);
  *rlon = (yr == 0.0 && xr == 0.0) ? 0.0 : atan2(yr, xr);
}

static FILE *open_mesh_file(const char *dir, const char *name, char *err, int errlen) {
  char path[4096];
  snprintf(path, sizeof path, "%s/%s", dir, name);
  FILE *f = fopen(path, "r");
  if (!f && err) snprintf(err, (size_t)errlen, "cannot open %s", path);
  return f;
}

static int read_ints(FILE *f, int *v, long n) {
  for (long i = 0; i < n; i++)
    if (fscanf(f, "%d", &v[i]) != 1) return -1;
  return 0;
}
static int read_dbls(FILE *f, double *v, long n) {
  for (long i = 0; i < n; i++)
    if (fscanf(f, "%lf", &v[i]) != 1) return -1;
  return 0;
}

#define MESH_FAIL(...)                                          \
  do {                                                          \
    if (err) snprintf(err, (size_t)errlen, __VA_ARGS__);        \
    if (f) fclose(f);                                           \
    om_mesh_free(m);                                            \
    return NULL;                                                \
  } while (0)

om_mesh *om_mesh_from_files(const char *dir, int rotate, double alpha, double beta, double gamma,
                            double angle_scale, double cyclic_length, char *err, int errlen) {
  om_mesh *m = (om_mesh *)calloc(1, sizeof(om_mesh));
  FILE *f = NULL;
  const double rad = PI_F / 180.0; /* lib/oce_modules.F90:20 */
  double R[3][3];
  rot_matrix(alpha * angle_scale, beta * angle_scale, gamma * angle_scale, R);
  m->cyclic = cyclic_length;
  m->full_rings = 1;

  /* nod2d.out and the rotation (lib/oce_mesh.F90:221-368) */
  if (!(f = open_mesh_file(dir, "nod2d.out", err, errlen))) MESH_FAIL("cannot open nod2d.out");
  int N = 0;
  if (fscanf(f, "%d", &N) != 1 || N < 3) MESH_FAIL("nod2d.out: bad node count");
  m->nod2D = m->nod2D_total = N;
  m->coord = (double *)calloc((size_t)2 * N, sizeof(double));
  double xp, yp;
  rot_r2g(R, 0.0 * rad, 90.0 * rad, &xp, &yp);
  xp = xp / rad;
  yp = yp / rad;
  const double dbox = 2.5;
  int isrot = 0, mustrot = 1;
  for (int n = 1; n <= N; n++) {
    int id, flag;
    double lon, lat;
    if (fscanf(f, "%d %lf %lf %d", &id, &lon, &lat, &flag) != 4) MESH_FAIL("nod2d.out: short record %d", n);
    double offset = 0.0;
    if (lon > 180.0) offset = -360.0;
    else if (lon < -180.0) offset = 360.0;
    int inbox = lon + offset >= xp - dbox && lon + offset <= xp + dbox && lat >= yp - dbox && lat <= yp + dbox;
    if (rotate && inbox) isrot = 1;
    if (!rotate && inbox) mustrot = 0;
    double x = lon * rad, y = lat * rad;
    if (rotate) {
      double rx = x, ry = y;
      rot_g2r(R, rx, ry, &x, &y);
    }
    A2(m->coord, 1, n, 2) = x;
    A2(m->coord, 2, n, 2) = y;
  }
  fclose(f);
  f = NULL;
  if (rotate && isrot) MESH_FAIL("the mesh seems to be rotated already (ocean nodes next to the rotated pole)");
  if (!rotate && mustrot) MESH_FAIL("the mesh seems to be unrotated (no ocean nodes next to the rotated pole)");

  /* elem2d.out (lib/oce_mesh.F90:370-437) and test_tri (:1565-1615) */
  if (!(f = open_mesh_file(dir, "elem2d.out", err, errlen))) MESH_FAIL("cannot open elem2d.out");
  int T = 0;
  if (fscanf(f, "%d", &T) != 1 || T < 1) MESH_FAIL("elem2d.out: bad element count");
  m->elem2D = T;
  m->elem2D_nodes = (int *)calloc((size_t)3 * T, sizeof(int));
  if (read_ints(f, m->elem2D_nodes, 3L * T)) MESH_FAIL("elem2d.out: short file");
  fclose(f);
  f = NULL;
  for (long i = 0; i < 3L * T; i++)
    if (m->elem2D_nodes[i] < 1 || m->elem2D_nodes[i] > N) MESH_FAIL("elem2d.out: node out of range");
  for (int e = 1; e <= T; e++) {
    int *el = &A2(m->elem2D_nodes, 1, e, 3);
    double a1 = A2(m->coord, 1, el[0], 2), a2 = A2(m->coord, 2, el[0], 2);
    double b1 = A2(m->coord, 1, el[1], 2) - a1, b2 = A2(m->coord, 2, el[1], 2) - a2;
    double c1 = A2(m->coord, 1, el[2], 2) - a1, c2 = A2(m->coord, 2, el[2], 2) - a2;
    trim_cyc(&b1, m->cyclic);
    trim_cyc(&c1, m->cyclic);
    double r = b1 * c2 - b2 * c1;
    if (r > 0.0) {
      int t = el[1];
      el[1] = el[2];
      el[2] = t;
    }
  }

  /* aux3d.out: levels and depths (lib/oce_mesh.F90:439-600) */
  if (!(f = open_mesh_file(dir, "aux3d.out", err, errlen))) MESH_FAIL("cannot open aux3d.out");
  int nl = 0;
  if (fscanf(f, "%d", &nl) != 1 || nl < 3) MESH_FAIL("aux3d.out: nl < 3");
  m->nl = nl;
  m->zbar = (double *)calloc((size_t)nl, sizeof(double));
  m->Z = (double *)calloc((size_t)nl - 1, sizeof(double));
  if (read_dbls(f, m->zbar, nl)) MESH_FAIL("aux3d.out: short level list");
  if (m->zbar[1] > 0.0)
    for (int k = 0; k < nl; k++) m->zbar[k] = -m->zbar[k];
  for (int k = 0; k < nl - 1; k++) m->Z[k] = 0.5 * (m->zbar[k] + m->zbar[k + 1]);
  double *depth = (double *)calloc((size_t)N, sizeof(double));
  int bad = read_dbls(f, depth, N);
  free(depth);
  if (bad) MESH_FAIL("aux3d.out: short depth list");
  fclose(f);
  f = NULL;
  m->max_depth = -m->zbar[nl - 1];

  /* edgenum.out, edges.out, edge_tri.out (lib/oce_mesh.F90:1617-1848) */
  if (!(f = open_mesh_file(dir, "edgenum.out", err, errlen))) MESH_FAIL("cannot open edgenum.out");
  int E = 0, E_in = 0;
  if (fscanf(f, "%d %d", &E, &E_in) != 2 || E < 1) MESH_FAIL("edgenum.out: bad edge count");
  fclose(f);
  f = NULL;
  m->edge2D = E;
  m->edges = (int *)calloc((size_t)2 * E, sizeof(int));
  m->edge_tri = (int *)calloc((size_t)2 * E, sizeof(int));
  if (!(f = open_mesh_file(dir, "edges.out", err, errlen))) MESH_FAIL("cannot open edges.out");
  if (read_ints(f, m->edges, 2L * E)) MESH_FAIL("edges.out: short file");
  fclose(f);
  f = NULL;
  if (!(f = open_mesh_file(dir, "edge_tri.out", err, errlen))) MESH_FAIL("cannot open edge_tri.out");
  if (read_ints(f, m->edge_tri, 2L * E)) MESH_FAIL("edge_tri.out: short file");
  fclose(f);
  f = NULL;
  for (long i = 0; i < 2L * E; i++) {
    if (m->edges[i] < 1 || m->edges[i] > N) MESH_FAIL("edges.out: node out of range");
    if (m->edge_tri[i] < 0) m->edge_tri[i] = 0;
    if (m->edge_tri[i] > T) MESH_FAIL("edge_tri.out: element out of range");
  }
  for (int e = 1; e <= E; e++)
    if (A2(m->edge_tri, 1, e, 2) < 1) MESH_FAIL("edge_tri.out: edge %d has no first element", e);

  /* find_neighbors (lib/oce_mesh.F90:1850-1999): nod_in_elem2D in ascending
   * element order, and every element needs at least two neighbours */
  build_nod_in_elem(m, N);
  {
    int *cnt = (int *)calloc((size_t)T, sizeof(int));
    int *nb = (int *)calloc((size_t)T, sizeof(int));
    for (int e = 1; e <= E; e++)
      for (int k = 1; k <= 2; k++) {
        int q = A2(m->edge_tri, k, e, 2);
        if (q > 0) {
          cnt[q - 1]++;
          int other = A2(m->edge_tri, 3 - k, e, 2);
          if (other > 0) nb[q - 1]++;
        }
      }
    int ok = 1;
    for (int t = 0; t < T; t++)
      if (cnt[t] != 3 || nb[t] < 2) ok = 0;
    free(cnt);
    free(nb);
    if (!ok) MESH_FAIL("an element has not three edges or fewer than two neighbours");
  }

  /* find_levels (lib/oce_mesh.F90:807-1001): elvls.out, nlvls.out */
  m->nlevels = (int *)calloc((size_t)T, sizeof(int));
  m->ulevels = (int *)calloc((size_t)T, sizeof(int));
  m->nlevels_nod2D = (int *)calloc((size_t)N, sizeof(int));
  m->ulevels_nod2D = (int *)calloc((size_t)N, sizeof(int));
  if (!(f = open_mesh_file(dir, "elvls.out", err, errlen))) MESH_FAIL("cannot open elvls.out");
  if (read_ints(f, m->nlevels, T)) MESH_FAIL("elvls.out: short file");
  fclose(f);
  f = NULL;
  if (!(f = open_mesh_file(dir, "nlvls.out", err, errlen))) MESH_FAIL("cannot open nlvls.out");
  if (read_ints(f, m->nlevels_nod2D, N)) MESH_FAIL("nlvls.out: short file");
  fclose(f);
  f = NULL;
  for (int t = 0; t < T; t++) {
    m->ulevels[t] = 1;
    if (m->nlevels[t] < 3 || m->nlevels[t] > nl) MESH_FAIL("elvls.out: level outside [3, nl]");
  }
  for (int n = 0; n < N; n++) {
    m->ulevels_nod2D[n] = 1;
    if (m->nlevels_nod2D[n] < 3 || m->nlevels_nod2D[n] > nl) MESH_FAIL("nlvls.out: level outside [3, nl]");
  }

  /* find_levels_min_e2n (lib/oce_mesh.F90:1522-1560) */
  m->nlevels_nod2D_min = (int *)calloc((size_t)N, sizeof(int));
  m->ulevels_nod2D_max = (int *)calloc((size_t)N, sizeof(int));
  for (int node = 1; node <= N; node++) {
    int mn = 1 << 30, mx = -(1 << 30);
    for (int j = 1; j <= m->nod_in_elem2D_num[node - 1]; j++) {
      int e = A2(m->nod_in_elem2D, j, node, m->max_nie);
      mn = imin2(mn, m->nlevels[e - 1]);
      mx = imax2(mx, m->ulevels[e - 1]);
    }
    m->nlevels_nod2D_min[node - 1] = mn;
    m->ulevels_nod2D_max[node - 1] = mx;
  }

  /* mesh_areas (lib/oce_mesh.F90:2043-2309), no cavities */
  m->elem_area = (double *)calloc((size_t)T, sizeof(double));
  m->area = (double *)calloc((size_t)nl * N, sizeof(double));
  m->areasvol = (double *)calloc((size_t)nl * N, sizeof(double));
  for (int e = 1; e <= T; e++) {
    const int *el = &A2(m->elem2D_nodes, 1, e, 3);
    double ay = (A2(m->coord, 2, el[0], 2) + A2(m->coord, 2, el[1], 2) + A2(m->coord, 2, el[2], 2)) / 3.0;
    ay = cos(ay);
    double a1 = A2(m->coord, 1, el[1], 2) - A2(m->coord, 1, el[0], 2);
    double a2 = A2(m->coord, 2, el[1], 2) - A2(m->coord, 2, el[0], 2);
    double b1 = A2(m->coord, 1, el[2], 2) - A2(m->coord, 1, el[0], 2);
    double b2 = A2(m->coord, 2, el[2], 2) - A2(m->coord, 2, el[0], 2);
    trim_cyc(&a1, m->cyclic);
    trim_cyc(&b1, m->cyclic);
    a1 = a1 * ay;
    b1 = b1 * ay;
    m->elem_area[e - 1] = 0.5 * fabs(a1 * b2 - b1 * a2);
  }
  for (int n = 1; n <= N; n++)
    for (int j = 1; j <= m->nod_in_elem2D_num[n - 1]; j++) {
      int elem = A2(m->nod_in_elem2D, j, n, m->max_nie);
      for (int nz = m->ulevels[elem - 1]; nz <= m->nlevels[elem - 1] - 1; nz++)
        A2(m->area, nz, n, nl) = A2(m->area, nz, n, nl) + m->elem_area[elem - 1] / 3.0;
    }
  for (int n = 1; n <= N; n++)
    for (int nz = m->ulevels_nod2D[n - 1]; nz <= m->nlevels_nod2D[n - 1] - 1; nz++)
      A2(m->areasvol, nz, n, nl) = A2(m->area, nz, n, nl);
  for (int e = 0; e < T; e++) m->elem_area[e] = m->elem_area[e] * R_EARTH * R_EARTH;
  for (long i = 0; i < (long)nl * N; i++) {
    m->area[i] = m->area[i] * R_EARTH * R_EARTH;
    m->areasvol[i] = m->areasvol[i] * R_EARTH * R_EARTH;
  }

  /* mesh_auxiliary_arrays (lib/oce_mesh.F90:2313-2534), the arrays the
   * advection reads */
  m->elem_cos = (double *)calloc((size_t)T, sizeof(double));
  double *cx = (double *)calloc((size_t)T, sizeof(double));
  double *cy = (double *)calloc((size_t)T, sizeof(double));
  for (int e = 1; e <= T; e++) {
    elem_center(m, &A2(m->elem2D_nodes, 1, e, 3), &cx[e - 1], &cy[e - 1]);
    m->elem_cos[e - 1] = cos(cy[e - 1]);
  }
  m->edge_dxdy = (double *)calloc((size_t)2 * E, sizeof(double));
  m->edge_cross_dxdy = (double *)calloc((size_t)4 * E, sizeof(double));
  for (int n = 1; n <= E; n++) {
    int ed1 = A2(m->edges, 1, n, 2), ed2 = A2(m->edges, 2, n, 2);
    double a1 = A2(m->coord, 1, ed2, 2) - A2(m->coord, 1, ed1, 2);
    double a2 = A2(m->coord, 2, ed2, 2) - A2(m->coord, 2, ed1, 2);
    trim_cyc(&a1, m->cyclic);
    A2(m->edge_dxdy, 1, n, 2) = a1;
    A2(m->edge_dxdy, 2, n, 2) = a2;
    double ex, ey;
    edge_center(m, ed1, ed2, &ex, &ey);
    for (int s = 1; s <= 2; s++) {
      int el = A2(m->edge_tri, s, n, 2);
      if (el <= 0) {
        A2(m->edge_cross_dxdy, 2 * s - 1, n, 4) = 0.0;
        A2(m->edge_cross_dxdy, 2 * s, n, 4) = 0.0;
        continue;
      }
      double b1 = cx[el - 1] - ex, b2 = cy[el - 1] - ey;
      trim_cyc(&b1, m->cyclic);
      b1 = b1 * m->elem_cos[el - 1];
      b1 = b1 * R_EARTH;
      b2 = b2 * R_EARTH;
      A2(m->edge_cross_dxdy, 2 * s - 1, n, 4) = b1;
      A2(m->edge_cross_dxdy, 2 * s, n, 4) = b2;
    }
  }
  free(cx);
  free(cy);
  m->gradient_sca = (double *)calloc((size_t)6 * T, sizeof(double));
  for (int e = 1; e <= T; e++) {
    const int *el = &A2(m->elem2D_nodes, 1, e, 3);
    double dX31 = A2(m->coord, 1, el[2], 2) - A2(m->coord, 1, el[0], 2);
    trim_cyc(&dX31, m->cyclic);
    dX31 = m->elem_cos[e - 1] * dX31;
    double dX21 = A2(m->coord, 1, el[1], 2) - A2(m->coord, 1, el[0], 2);
    trim_cyc(&dX21, m->cyclic);
    dX21 = m->elem_cos[e - 1] * dX21;
    double dY31 = A2(m->coord, 2, el[2], 2) - A2(m->coord, 2, el[0], 2);
    double dY21 = A2(m->coord, 2, el[1], 2) - A2(m->coord, 2, el[0], 2);
    double fac = -0.5 * R_EARTH / m->elem_area[e - 1];
    double *gs = &A2(m->gradient_sca, 1, e, 6);
    gs[0] = (-dY31 + dY21) * fac;
    gs[1] = dY31 * fac;
    gs[2] = -dY21 * fac;
    gs[3] = (dX31 - dX21) * fac;
    gs[4] = -dX31 * fac;
    gs[5] = dX21 * fac;
  }

  /* coordinate extents (the domain box of the seeded synthetic fields) */
  double x0 = A2(m->coord, 1, 1, 2), x1 = x0, y0 = A2(m->coord, 2, 1, 2), y1 = y0;
  for (int n = 2; n <= N; n++) {
    x0 = fmin2(x0, A2(m->coord, 1, n, 2)); x1 = fmax2(x1, A2(m->coord, 1, n, 2));
    y0 = fmin2(y0, A2(m->coord, 2, n, 2)); y1 = fmax2(y1, A2(m->coord, 2, n, 2));
  }
  m->Lx = (x1 - x0) * R_EARTH;
  m->Ly = (y1 - y0) * R_EARTH;

  /* ALE arrays (lib/tracer_c_interface.F90:875-929) */
  const int nz = nl - 1;
  m->hnode = (double *)calloc((size_t)nz * N, sizeof(double));
  m->hnode_new = (double *)calloc((size_t)nz * N, sizeof(double));
  m->helem = (double *)calloc((size_t)nz * T, sizeof(double));
  m->zbar_3d_n = (double *)calloc((size_t)nl * N, sizeof(double));
  m->Z_3d_n = (double *)calloc((size_t)nz * N, sizeof(double));
  for (int n = 1; n <= N; n++) {
    for (int k = 1; k <= nz; k++) {
      A2(m->hnode, k, n, nz) = m->zbar[k - 1] - m->zbar[k];
      A2(m->hnode_new, k, n, nz) = A2(m->hnode, k, n, nz);
      A2(m->Z_3d_n, k, n, nz) = m->Z[k - 1];
    }
    for (int k = 1; k <= nl; k++) A2(m->zbar_3d_n, k, n, nl) = m->zbar[k - 1];
  }
  for (int e = 1; e <= T; e++)
    for (int k = 1; k <= nz; k++) A2(m->helem, k, e, nz) = m->zbar[k - 1] - m->zbar[k];

  /* MUSCL set-up (lib/oce_muscl_adv.F90:38-357) */
  m->edge_up_dn_tri = (int *)calloc((size_t)2 * E, sizeof(int));
  m->nboundary_lay = (int *)calloc((size_t)N, sizeof(int));
  find_up_downwind_triangles(m);
  init_nboundary_lay(m);
  return m;
}
#undef MESH_FAIL

/* ------------------------------------------------------------------------ */
/* mesh from given arrays (every table as passed, the MUSCL ones included)   */
/* ------------------------------------------------------------------------ */
static void *dup_bytes(const void *src, size_t bytes) {
  void *p = malloc(bytes ? bytes : 1);
  if (bytes) memcpy(p, src, bytes);
  return p;
}

om_mesh *om_mesh_from_arrays(int nl, int nod2D, int elem2D, int edge2D, int periodic, double Lx, double Ly,
                             const double *coord, const int *elem2D_nodes, const int *edges, const int *edge_tri,
                             const int *nlevels, const int *nlevels_nod2D, const int *nlevels_nod2D_min,
                             const int *ring_num, const int *ring_elem, const double *elem_area, const double *area,
                             const double *areasvol, const double *edge_dxdy, const double *edge_cross_dxdy,
                             const double *gradient_sca, const double *elem_cos, const double *zbar,
                             const double *hnode, const double *hnode_new, const double *helem,
                             const int *edge_up_dn_tri, const int *nboundary_lay) {
  if (nl < 3 || nod2D < 1 || elem2D < 1 || edge2D < 1) return NULL;
  om_mesh *m = (om_mesh *)calloc(1, sizeof(om_mesh));
  const size_t N = (size_t)nod2D, T = (size_t)elem2D, E = (size_t)edge2D, L = (size_t)nl - 1;
  m->nl = nl;
  m->nod2D = m->nod2D_total = nod2D;
  m->elem2D = elem2D;
  m->edge2D = edge2D;
  m->periodic = periodic;
  m->full_rings = 1;
  m->Lx = Lx;
  m->Ly = Ly;
  m->cyclic = CYCLIC_LENGTH;
  m->coord = (double *)dup_bytes(coord, 2 * N * sizeof(double));
  m->elem2D_nodes = (int *)dup_bytes(elem2D_nodes, 3 * T * sizeof(int));
  m->edges = (int *)dup_bytes(edges, 2 * E * sizeof(int));
  m->edge_tri = (int *)dup_bytes(edge_tri, 2 * E * sizeof(int));
  m->nlevels = (int *)dup_bytes(nlevels, T * sizeof(int));
  m->nlevels_nod2D = (int *)dup_bytes(nlevels_nod2D, N * sizeof(int));
  m->nlevels_nod2D_min = (int *)dup_bytes(nlevels_nod2D_min, N * sizeof(int));
  m->ulevels = (int *)malloc(T * sizeof(int));
  for (size_t t = 0; t < T; t++) m->ulevels[t] = 1;
  m->ulevels_nod2D = (int *)malloc(N * sizeof(int));
  m->ulevels_nod2D_max = (int *)malloc(N * sizeof(int));
  for (size_t n = 0; n < N; n++) m->ulevels_nod2D[n] = m->ulevels_nod2D_max[n] = 1;
  int mx = 0;
  for (size_t n = 0; n < N; n++) mx = imax2(mx, ring_num[n]);
  m->max_nie = mx;
  m->nod_in_elem2D_num = (int *)dup_bytes(ring_num, N * sizeof(int));
  m->nod_in_elem2D = (int *)calloc((size_t)mx * N, sizeof(int));
  for (size_t n = 0, p = 0; n < N; n++)
    for (int j = 1; j <= ring_num[n]; j++) A2(m->nod_in_elem2D, j, (int)n + 1, mx) = ring_elem[p++];
  m->elem_area = (double *)dup_bytes(elem_area, T * sizeof(double));
  m->area = (double *)dup_bytes(area, (size_t)nl * N * sizeof(double));
  m->areasvol = (double *)dup_bytes(areasvol, (size_t)nl * N * sizeof(double));
  m->edge_dxdy = (double *)dup_bytes(edge_dxdy, 2 * E * sizeof(double));
  m->edge_cross_dxdy = (double *)dup_bytes(edge_cross_dxdy, 4 * E * sizeof(double));
  m->gradient_sca = (double *)dup_bytes(gradient_sca, 6 * T * sizeof(double));
  m->elem_cos = (double *)dup_bytes(elem_cos, T * sizeof(double));
  m->zbar = (double *)dup_bytes(zbar, (size_t)nl * sizeof(double));
  m->Z = (double *)malloc(L * sizeof(double));
  for (size_t k = 0; k < L; k++) m->Z[k] = 0.5 * (m->zbar[k] + m->zbar[k + 1]);
  m->max_depth = -m->zbar[nl - 1];
  m->hnode = (double *)dup_bytes(hnode, L * N * sizeof(double));
  m->hnode_new = (double *)dup_bytes(hnode_new, L * N * sizeof(double));
  m->helem = (double *)dup_bytes(helem, L * T * sizeof(double));
  m->zbar_3d_n = (double *)malloc((size_t)nl * N * sizeof(double));
  m->Z_3d_n = (double *)malloc(L * N * sizeof(double));
  for (size_t n = 0; n < N; n++) {
    for (size_t k = 0; k < (size_t)nl; k++) m->zbar_3d_n[n * nl + k] = m->zbar[k];
    for (size_t k = 0; k < L; k++) m->Z_3d_n[n * L + k] = m->Z[k];
  }
  m->edge_up_dn_tri = (int *)dup_bytes(edge_up_dn_tri, 2 * E * sizeof(int));
  m->nboundary_lay = (int *)dup_bytes(nboundary_lay, N * sizeof(int));
  return m;
}

static void work_free(struct om_work_s *w);
void om_mesh_free(om_mesh *m) {
  if (!m) return;
  if (m->work) { work_free(m->work); free(m->work); }
  void *p[] = {m->coord, m->elem2D_nodes, m->edges, m->edge_tri, m->nlevels, m->ulevels,
               m->nlevels_nod2D, m->ulevels_nod2D, m->nlevels_nod2D_min, m->ulevels_nod2D_max,
               m->nod_in_elem2D_num, m->nod_in_elem2D, m->elem_area, m->area, m->areasvol,
               m->edge_dxdy, m->edge_cross_dxdy, m->gradient_sca, m->elem_cos, m->zbar, m->Z,
               m->hnode, m->hnode_new, m->helem, m->zbar_3d_n, m->Z_3d_n, m->edge_up_dn_tri,
               m->nboundary_lay};
  for (size_t i = 0; i < sizeof(p) / sizeof(p[0]); i++) free(p[i]);
  free(m);
}

void om_mesh_dims(const om_mesh *m, int *d) {
  d[0] = m->nl; d[1] = m->nod2D; d[2] = m->elem2D; d[3] = m->edge2D; d[4] = m->max_nie;
  d[5] = m->periodic;
}

typedef struct { const char *name; int is_int; const void *ptr; long len; } om_field;

static int lookup(const om_mesh *m, const char *name, om_field *f) {
  const long N = m->nod2D, E = m->edge2D, T = m->elem2D, nl = m->nl;
  om_field tab[] = {
      {"coord", 0, m->coord, 2 * N},
      {"elem2D_nodes", 1, m->elem2D_nodes, 3 * T},
      {"edges", 1, m->edges, 2 * E},
      {"edge_tri", 1, m->edge_tri, 2 * E},
      {"nlevels", 1, m->nlevels, T},
      {"ulevels", 1, m->ulevels, T},
      {"nlevels_nod2D", 1, m->nlevels_nod2D, N},
      {"ulevels_nod2D", 1, m->ulevels_nod2D, N},
      {"nlevels_nod2D_min", 1, m->nlevels_nod2D_min, N},
      {"ulevels_nod2D_max", 1, m->ulevels_nod2D_max, N},
      {"nod_in_elem2D_num", 1, m->nod_in_elem2D_num, N},
      {"nod_in_elem2D", 1, m->nod_in_elem2D, (long)m->max_nie * N},
      {"elem_area", 0, m->elem_area, T},
      {"area", 0, m->area, nl * N},
      {"areasvol", 0, m->areasvol, nl * N},
      {"edge_dxdy", 0, m->edge_dxdy, 2 * E},
      {"edge_cross_dxdy", 0, m->edge_cross_dxdy, 4 * E},
      {"gradient_sca", 0, m->gradient_sca, 6 * T},
      {"elem_cos", 0, m->elem_cos, T},
      {"zbar", 0, m->zbar, nl},
      {"Z", 0, m->Z, nl - 1},
      {"hnode", 0, m->hnode, (nl - 1) * N},
      {"hnode_new", 0, m->hnode_new, (nl - 1) * N},
      {"helem", 0, m->helem, (nl - 1) * T},
      {"zbar_3d_n", 0, m->zbar_3d_n, nl * N},
      {"Z_3d_n", 0, m->Z_3d_n, (nl - 1) * N},
      {"edge_up_dn_tri", 1, m->edge_up_dn_tri, 2 * E},
      {"nboundary_lay", 1, m->nboundary_lay, N},
  };
  for (size_t i = 0; i < sizeof(tab) / sizeof(tab[0]); i++)
    if (strcmp(tab[i].name, name) == 0) { *f = tab[i]; return 0; }
  return -1;
}

long om_mesh_len(const om_mesh *m, const char *name) {
  om_field f;
  return lookup(m, name, &f) ? -1 : f.len;
}
int om_mesh_get_int(const om_mesh *m, const char *name, int *out) {
  om_field f;
  if (lookup(m, name, &f) || !f.is_int) return -1;
  memcpy(out, f.ptr, sizeof(int) * (size_t)f.len);
  return 0;
}
int om_mesh_get_dbl(const om_mesh *m, const char *name, double *out) {
  om_field f;
  if (lookup(m, name, &f) || f.is_int) return -1;
  memcpy(out, f.ptr, sizeof(double) * (size_t)f.len);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* initial fields: src/fesom_analytic.F90:251-256, 306-331                   */
/* ------------------------------------------------------------------------ */
void om_analytic_fields(const om_mesh *m, double *T, double *S, double *uv, double *w) {
  const int nz = m->nl - 1;
  const double Lx = m->Lx, Ly = m->Ly, xc = 0.5 * Lx, yc = 0.5 * Ly;
  for (int n = 1; n <= m->nod2D; n++) {
    double xn = A2(m->coord, 1, n, 2) * R_EARTH, yn = A2(m->coord, 2, n, 2) * R_EARTH;
    double r = sqrt((xn - xc) * (xn - xc) + (yn - yc) * (yn - yc));
    for (int k = 1; k <= nz; k++) {
      double zn = (double)(k - 1) / (double)(nz - 1);
      if (T) A2(T, k, n, nz) = 15.0 + 5.0 * sin(2.0 * PI_F * xn / Lx) * cos(2.0 * PI_F * yn / Ly) - 10.0 * zn;
      if (S) A2(S, k, n, nz) = 34.0 + 2.0 * exp(-(r * r) / ((0.1 * Lx) * (0.1 * Lx))) * (1.0 - zn);
    }
  }
  if (uv)
    for (size_t i = 0; i < (size_t)nz * m->elem2D; i++) { uv[2 * i] = 0.1; uv[2 * i + 1] = 0.0; }
  if (w) memset(w, 0, sizeof(double) * (size_t)m->nl * m->nod2D);
}

/* ------------------------------------------------------------------------ */
/* the hot path                                                              */
/* ------------------------------------------------------------------------ */
typedef struct om_work_s {
  double *fct_LO, *adv_flux_hor, *adv_flux_ver, *fct_ttf_max, *fct_ttf_min;
  double *fct_plus, *fct_minus, *edge_up_dn_grad, *tr_xy, *aux, *tvert_max, *tvert_min;
  double *dttf_h, *dttf_v;
} om_work;

static void work_alloc(const om_mesh *m, om_work *w) {
  const size_t L = (size_t)m->nl - 1, nl = (size_t)m->nl, N = (size_t)m->nod2D,
               E = (size_t)m->edge2D, T = (size_t)m->elem2D;
  w->fct_LO = calloc(L * N, 8); w->adv_flux_hor = calloc(L * E, 8);
  w->adv_flux_ver = calloc(nl * N, 8); w->fct_ttf_max = calloc(L * N, 8);
  w->fct_ttf_min = calloc(L * N, 8); w->fct_plus = calloc(L * N, 8);
  w->fct_minus = calloc(L * N, 8); w->edge_up_dn_grad = calloc(4 * L * E, 8);
  w->tr_xy = calloc(2 * L * T, 8); w->aux = calloc(2 * L * T, 8);
  w->tvert_max = calloc(L * N, 8); w->tvert_min = calloc(L * N, 8);
  w->dttf_h = calloc(L * N, 8); w->dttf_v = calloc(L * N, 8);
}
static om_work *mesh_work(const om_mesh *cm) {
  om_mesh *m = (om_mesh *)cm;
  if (!m->work) {
    m->work = (om_work *)calloc(1, sizeof(om_work));
    work_alloc(m, m->work);
  }
  return m->work;
}
static void work_free(om_work *w) {
  void *p[] = {w->fct_LO, w->adv_flux_hor, w->adv_flux_ver, w->fct_ttf_max, w->fct_ttf_min,
               w->fct_plus, w->fct_minus, w->edge_up_dn_grad, w->tr_xy, w->aux,
               w->tvert_max, w->tvert_min, w->dttf_h, w->dttf_v};
  for (size_t i = 0; i < sizeof(p) / sizeof(p[0]); i++) free(p[i]);
}

#define NIE(k, n) A2(m->nod_in_elem2D, k, n, m->max_nie)

/* element tracer gradient tr_xy (absent from the reference; upstream FESOM2's
 * tracer_gradient_elements): tr_xy(1,nz,e) = sum(gradient_sca(1:3,e)*T(nz,nodes)),
 * tr_xy(2,nz,e) = sum(gradient_sca(4:6,e)*T(nz,nodes)), gradient_sca from
 * lib/oce_mesh.F90:2512-2534, summed left to right. */
static void tracer_gradient_elements(const om_mesh *m, const double *ttf, double *tr_xy) {
  const int L = m->nl - 1;
#pragma omp parallel for schedule(static)
  for (int elem = 1; elem <= m->elem2D; elem++) {
    const int *en = &A2(m->elem2D_nodes, 1, elem, 3);
    const double *gs = &A2(m->gradient_sca, 1, elem, 6);
    for (int nz = m->ulevels[elem - 1]; nz <= m->nlevels[elem - 1] - 1; nz++) {
      double t1 = A2(ttf, nz, en[0], L), t2 = A2(ttf, nz, en[1], L), t3 = A2(ttf, nz, en[2], L);
      A3(tr_xy, 1, nz, elem, 2, L) = (gs[0] * t1 + gs[1] * t2) + gs[2] * t3;
      A3(tr_xy, 2, nz, elem, 2, L) = (gs[3] * t1 + gs[4] * t2) + gs[5] * t3;
    }
  }
}

/* area-weighted mean of tr_xy over the ring of node n at level nz
 * (lib/oce_muscl_adv.F90:394-409 and its three copies) */
static void ring_mean(const om_mesh *m, const double *tr_xy, int n, int nz, double *gx, double *gy) {
  const int L = m->nl - 1;
  double tvol = 0.0, tx = 0.0, ty = 0.0;
  for (int k = 1; k <= m->nod_in_elem2D_num[n - 1]; k++) {
    int elem = NIE(k, n);
    if (m->nlevels[elem - 1] - 1 < nz || nz < m->ulevels[elem - 1]) continue;
    tvol = tvol + m->elem_area[elem - 1];
    tx = tx + A3(tr_xy, 1, nz, elem, 2, L) * m->elem_area[elem - 1];
    ty = ty + A3(tr_xy, 2, nz, elem, 2, L) * m->elem_area[elem - 1];
  }
  *gx = tx / tvol;
  *gy = ty / tvol;
}

/* lib/oce_muscl_adv.F90:361-530 */
static void fill_up_dn_grad(const om_mesh *m, const double *tr_xy, double *g) {
  const int L = m->nl - 1;
#pragma omp parallel for schedule(static)
  for (int edge = 1; edge <= m->edge2D; edge++) {
    int n1 = A2(m->edges, 1, edge, 2), n2 = A2(m->edges, 2, edge, 2);
    int up = A2(m->edge_up_dn_tri, 1, edge, 2), dn = A2(m->edge_up_dn_tri, 2, edge, 2);
    double gx, gy;
    if (up != 0 && dn != 0) {
      int nzmin = imax2(m->ulevels_nod2D_max[n1 - 1], m->ulevels_nod2D_max[n2 - 1]);
      int nzmax = imin2(m->nlevels_nod2D_min[n1 - 1], m->nlevels_nod2D_min[n2 - 1]);
      for (int nz = m->ulevels_nod2D[n1 - 1]; nz <= nzmin - 1; nz++) {
        ring_mean(m, tr_xy, n1, nz, &gx, &gy);
        A3(g, 1, nz, edge, 4, L) = gx; A3(g, 3, nz, edge, 4, L) = gy;
      }
      for (int nz = m->ulevels_nod2D[n2 - 1]; nz <= nzmin - 1; nz++) {
        ring_mean(m, tr_xy, n2, nz, &gx, &gy);
        A3(g, 2, nz, edge, 4, L) = gx; A3(g, 4, nz, edge, 4, L) = gy;
      }
      for (int nz = nzmin; nz <= nzmax - 1; nz++) {
        A3(g, 1, nz, edge, 4, L) = A3(tr_xy, 1, nz, up, 2, L);
        A3(g, 2, nz, edge, 4, L) = A3(tr_xy, 1, nz, dn, 2, L);
        A3(g, 3, nz, edge, 4, L) = A3(tr_xy, 2, nz, up, 2, L);
        A3(g, 4, nz, edge, 4, L) = A3(tr_xy, 2, nz, dn, 2, L);
      }
      for (int nz = nzmax; nz <= m->nlevels_nod2D[n1 - 1] - 1; nz++) {
        ring_mean(m, tr_xy, n1, nz, &gx, &gy);
        A3(g, 1, nz, edge, 4, L) = gx; A3(g, 3, nz, edge, 4, L) = gy;
      }
      for (int nz = nzmax; nz <= m->nlevels_nod2D[n2 - 1] - 1; nz++) {
        ring_mean(m, tr_xy, n2, nz, &gx, &gy);
        A3(g, 2, nz, edge, 4, L) = gx; A3(g, 4, nz, edge, 4, L) = gy;
      }
    } else {
      for (int nz = m->ulevels_nod2D[n1 - 1]; nz <= m->nlevels_nod2D[n1 - 1] - 1; nz++) {
        ring_mean(m, tr_xy, n1, nz, &gx, &gy);
        A3(g, 1, nz, edge, 4, L) = gx; A3(g, 3, nz, edge, 4, L) = gy;
      }
      for (int nz = m->ulevels_nod2D[n2 - 1]; nz <= m->nlevels_nod2D[n2 - 1] - 1; nz++) {
        ring_mean(m, tr_xy, n2, nz, &gx, &gy);
        A3(g, 2, nz, edge, 4, L) = gx; A3(g, 4, nz, edge, 4, L) = gy;
      }
    }
  }
}

/* Level segments shared by every edge loop (lib/oce_adv_tra_hor.F90:123-164). */
typedef struct { int n1, n2, el1, el2, nl1, nu1, nl2, nu2, nl12, nu12; double dX1, dY1, dX2, dY2, a; } edge_geo;
static void edge_geometry(const om_mesh *m, int edge, edge_geo *g) {
  g->n1 = A2(m->edges, 1, edge, 2); g->n2 = A2(m->edges, 2, edge, 2);
  g->el1 = A2(m->edge_tri, 1, edge, 2); g->el2 = A2(m->edge_tri, 2, edge, 2);
  g->nl1 = m->nlevels[g->el1 - 1] - 1;
  g->nu1 = m->ulevels[g->el1 - 1];
  g->dX1 = A2(m->edge_cross_dxdy, 1, edge, 4);
  g->dY1 = A2(m->edge_cross_dxdy, 2, edge, 4);
  g->a = R_EARTH * m->elem_cos[g->el1 - 1];
  g->nl2 = 0; g->nu2 = 0; g->dX2 = 0.0; g->dY2 = 0.0;
  if (g->el2 > 0) {
    g->dX2 = A2(m->edge_cross_dxdy, 3, edge, 4);
    g->dY2 = A2(m->edge_cross_dxdy, 4, edge, 4);
    g->nl2 = m->nlevels[g->el2 - 1] - 1;
    g->nu2 = m->ulevels[g->el2 - 1];
    g->a = 0.5 * (g->a + R_EARTH * m->elem_cos[g->el2 - 1]);
  }
  g->nl12 = imin2(g->nl1, g->nl2);
  g->nu12 = imax2(g->nu1, g->nu2);
}

/* volume flux through the edge's dual segments at level nz; side 1, 2 or both
 * (lib/oce_adv_tra_hor.F90:174,194,215-216) */
static inline double vflux_at(const om_mesh *m, const edge_geo *g, const double *vel, int nz, int which) {
  const int L = m->nl - 1;
  double v1 = 0.0, v2 = 0.0;
  if (which & 1)
    v1 = (-A3(vel, 2, nz, g->el1, 2, L) * g->dX1 + A3(vel, 1, nz, g->el1, 2, L) * g->dY1) * A2(m->helem, nz, g->el1, L);
  if (which & 2)
    v2 = (A3(vel, 2, nz, g->el2, 2, L) * g->dX2 - A3(vel, 1, nz, g->el2, 2, L) * g->dY2) * A2(m->helem, nz, g->el2, L);
  if (which == 3) return v1 + v2;
  return (which & 1) ? v1 : v2;
}

/* adv_tra_hor_upw1 (lib/oce_adv_tra_hor.F90:64-261) */
static void adv_tra_hor_upw1(const om_mesh *m, const double *vel, const double *ttf, double *flux, int init_zero) {
  const int L = m->nl - 1;
  if (init_zero) memset(flux, 0, sizeof(double) * (size_t)L * m->edge2D);
#pragma omp parallel for schedule(static)
  for (int edge = 1; edge <= m->edge2D; edge++) {
    edge_geo g;
    edge_geometry(m, edge, &g);
    /* segments run A, B, C, D, E in this order, as in the reference */
    int lo[5] = {g.nu1, g.nu2 > 0 ? g.nu2 : 1, g.nu12, g.nl12 + 1, g.nl12 + 1};
    int hi[5] = {g.nu12 - 1, g.nu2 > 0 ? g.nu12 - 1 : 0, g.nl12, g.nl1, g.nl2};
    int wh[5] = {1, 2, 3, 1, 2};
    for (int s = 0; s < 5; s++)
      for (int nz = lo[s]; nz <= hi[s]; nz++) {
        double vflux = vflux_at(m, &g, vel, nz, wh[s]);
        A2(flux, nz, edge, L) = -0.5 * (A2(ttf, nz, g.n1, L) * (vflux + fabs(vflux)) +
                                        A2(ttf, nz, g.n2, L) * (vflux - fabs(vflux))) -
                                A2(flux, nz, edge, L);
      }
  }
}

/* adv_tra_hor_muscl / adv_tra_hor_mfct (lib/oce_adv_tra_hor.F90:265-550,
 * 554-846); use_clo = 1 for MUSCL (c_lo switch of :364-365), 0 for MFCT. */
static void adv_tra_hor_muscl(const om_mesh *m, const double *vel, const double *ttf, double num_ord,
                              double *flux, const double *g4, int use_clo, int init_zero) {
  const int L = m->nl - 1;
  if (init_zero) memset(flux, 0, sizeof(double) * (size_t)L * m->edge2D);
#pragma omp parallel for schedule(static)
  for (int edge = 1; edge <= m->edge2D; edge++) {
    edge_geo g;
    edge_geometry(m, edge, &g);
    const double ex = A2(m->edge_dxdy, 1, edge, 2), ey = A2(m->edge_dxdy, 2, edge, 2);
    int lo[5] = {g.nu1, g.nu2 > 0 ? g.nu2 : 1, g.nu12, g.nl12 + 1, g.nl12 + 1};
    int hi[5] = {g.nu12 - 1, g.nu2 > 0 ? g.nu12 - 1 : 0, g.nl12, g.nl1, g.nl2};
    int wh[5] = {1, 2, 3, 1, 2};
    for (int s = 0; s < 5; s++)
      for (int nz = lo[s]; nz <= hi[s]; nz++) {
        double t1 = A2(ttf, nz, g.n1, L), t2 = A2(ttf, nz, g.n2, L);
        double Tmean2, Tmean1;
        if (use_clo) {
          /* real(max(sign(1, nboundary_lay(n)-nz), 0)): 1 when nboundary_lay(n) >= nz */
          double c_lo1 = (m->nboundary_lay[g.n1 - 1] - nz >= 0) ? 1.0 : 0.0;
          double c_lo2 = (m->nboundary_lay[g.n2 - 1] - nz >= 0) ? 1.0 : 0.0;
          Tmean2 = t2 - (2.0 * (t2 - t1) + ex * g.a * A3(g4, 2, nz, edge, 4, L) +
                         ey * R_EARTH * A3(g4, 4, nz, edge, 4, L)) / 6.0 * c_lo2;
          Tmean1 = t1 + (2.0 * (t2 - t1) + ex * g.a * A3(g4, 1, nz, edge, 4, L) +
                         ey * R_EARTH * A3(g4, 3, nz, edge, 4, L)) / 6.0 * c_lo1;
        } else {
          Tmean2 = t2 - (2.0 * (t2 - t1) + ex * g.a * A3(g4, 2, nz, edge, 4, L) +
                         ey * R_EARTH * A3(g4, 4, nz, edge, 4, L)) / 6.0;
          Tmean1 = t1 + (2.0 * (t2 - t1) + ex * g.a * A3(g4, 1, nz, edge, 4, L) +
                         ey * R_EARTH * A3(g4, 3, nz, edge, 4, L)) / 6.0;
        }
        double vflux = vflux_at(m, &g, vel, nz, wh[s]);
        double cHO = (vflux + fabs(vflux)) * Tmean1 + (vflux - fabs(vflux)) * Tmean2;
        A2(flux, nz, edge, L) = -(0.5 * (1.0 - num_ord) * cHO) -
                                vflux * num_ord * 0.5 * (Tmean1 + Tmean2) - A2(flux, nz, edge, L);
      }
  }
}

/* adv_tra_ver_upw1 (lib/oce_adv_tra_ver.F90:248-335) */
static void adv_tra_ver_upw1(const om_mesh *m, const double *W, const double *ttf, double *flux, int init_zero) {
  const int L = m->nl - 1, nl = m->nl;
  if (init_zero) memset(flux, 0, sizeof(double) * (size_t)nl * m->nod2D);
#pragma omp parallel for schedule(static)
  for (int n = 1; n <= m->nod2D; n++) {
    int nzmax = m->nlevels_nod2D[n - 1], nzmin = m->ulevels_nod2D[n - 1];
    int nz = nzmin;
    A2(flux, nz, n, nl) = -(A2(W, nz, n, nl) * A2(ttf, nz, n, L) * A2(m->area, nz, n, nl)) - A2(flux, nz, n, nl);
    nz = nzmax;
    A2(flux, nz, n, nl) = 0.0 - A2(flux, nz, n, nl);
    for (nz = nzmin + 1; nz <= nzmax - 1; nz++) {
      double Wz = A2(W, nz, n, nl);
      A2(flux, nz, n, nl) = -(0.5 * (A2(ttf, nz, n, L) * (Wz + fabs(Wz)) + A2(ttf, nz - 1, n, L) * (Wz - fabs(Wz))) *
                              A2(m->area, nz, n, nl)) - A2(flux, nz, n, nl);
    }
  }
}

/* adv_tra_ver_qr4c (lib/oce_adv_tra_ver.F90:339-444); assignments in the
 * reference's order, including its overlaps on short columns. */
static void adv_tra_ver_qr4c(const om_mesh *m, const double *W, const double *ttf, double num_ord, double *flux, int init_zero) {
  const int L = m->nl - 1, nl = m->nl;
  if (init_zero) memset(flux, 0, sizeof(double) * (size_t)nl * m->nod2D);
#pragma omp parallel for schedule(static)
  for (int n = 1; n <= m->nod2D; n++) {
    int nzmax = m->nlevels_nod2D[n - 1], nzmin = m->ulevels_nod2D[n - 1];
#define T_(k) A2(ttf, k, n, L)
#define W_(k) A2(W, k, n, nl)
#define AR_(k) A2(m->area, k, n, nl)
#define F_(k) A2(flux, k, n, nl)
#define Z_(k) A2(m->Z_3d_n, k, n, L)
#define ZB_(k) A2(m->zbar_3d_n, k, n, nl)
    int nz = nzmin;
    F_(nz) = -(T_(nz) * W_(nz) * AR_(nz)) - F_(nz);
    nz = nzmin + 1;
    F_(nz) = -(0.5 * (T_(nz - 1) + T_(nz)) * W_(nz) * AR_(nz)) - F_(nz);
    nz = nzmax - 1;
    F_(nz) = -(0.5 * (T_(nz - 1) + T_(nz)) * W_(nz) * AR_(nz)) - F_(nz);
    nz = nzmax;
    F_(nz) = 0.0 - F_(nz);
    for (nz = nzmin + 2; nz <= nzmax - 2; nz++) {
      double qc = (T_(nz - 1) - T_(nz)) / (Z_(nz - 1) - Z_(nz));
      double qu = (T_(nz) - T_(nz + 1)) / (Z_(nz) - Z_(nz + 1));
      double qd = (T_(nz - 2) - T_(nz - 1)) / (Z_(nz - 2) - Z_(nz - 1));
      double Tmean1 = T_(nz) + (2.0 * qc + qu) * (ZB_(nz) - Z_(nz)) / 3.0;
      double Tmean2 = T_(nz - 1) + (2.0 * qc + qd) * (ZB_(nz) - Z_(nz - 1)) / 3.0;
      double Tmean = (W_(nz) + fabs(W_(nz))) * Tmean1 + (W_(nz) - fabs(W_(nz))) * Tmean2;
      F_(nz) = (-(0.5 * (1.0 - num_ord) * Tmean) - num_ord * (0.5 * (Tmean1 + Tmean2)) * W_(nz)) * AR_(nz) - F_(nz);
    }
#undef T_
#undef W_
#undef AR_
#undef F_
#undef Z_
#undef ZB_
  }
}

/* adv_tra_vert_ppm (lib/oce_adv_tra_ver.F90:448-644) */
static void adv_tra_vert_ppm(const om_mesh *m, double dt, const double *W, const double *ttf, double *flux, int init_zero) {
  const int L = m->nl - 1, nl = m->nl;
  if (init_zero) memset(flux, 0, sizeof(double) * (size_t)nl * m->nod2D);
#pragma omp parallel
  {
    double *tv = (double *)malloc(sizeof(double) * (size_t)nl);
    double *tvert = (double *)malloc(sizeof(double) * (size_t)nl);
#pragma omp for schedule(static)
    for (int n = 1; n <= m->nod2D; n++) {
#define T_(k) A2(ttf, k, n, L)
#define W_(k) A2(W, k, n, nl)
#define HN_(k) A2(m->hnode_new, k, n, L)
      int nzmax = m->nlevels_nod2D[n - 1], nzmin = m->ulevels_nod2D[n - 1];
      tv[nzmin - 1] = T_(nzmin);
      tv[nzmin] = 0.5 * (T_(nzmin) + T_(nzmin + 1));
      tv[nzmax - 2] = -T_(nzmax - 2) * fmin2(copysign(1.0, W_(nzmax - 1)), 0.0) +
                      T_(nzmax - 1) * fmax2(copysign(1.0, W_(nzmax - 1)), 0.0);
      tv[nzmax - 1] = T_(nzmax - 1);
      for (int nz = nzmin + 1; nz <= nzmax - 3; nz++) {
        double dzjm1 = HN_(nz - 1), dzj = HN_(nz), dzjp1 = HN_(nz + 1), dzjp2 = HN_(nz + 2);
        double deltaj = dzj / (dzjm1 + dzj + dzjp1) *
                        ((2.0 * dzjm1 + dzj) / (dzjp1 + dzj) * (T_(nz + 1) - T_(nz)) +
                         (dzj + 2.0 * dzjp1) / (dzjm1 + dzj) * (T_(nz) - T_(nz - 1)));
        double deltajp1 = dzjp1 / (dzj + dzjp1 + dzjp2) *
                          ((2.0 * dzj + dzjp1) / (dzjp2 + dzjp1) * (T_(nz + 2) - T_(nz + 1)) +
                           (dzjp1 + 2.0 * dzjp2) / (dzj + dzjp1) * (T_(nz + 1) - T_(nz)));
        if ((T_(nz + 1) - T_(nz)) * (T_(nz) - T_(nz - 1)) > 0.0)
          deltaj = fmin3(fabs(deltaj), 2.0 * fabs(T_(nz + 1) - T_(nz)), 2.0 * fabs(T_(nz) - T_(nz - 1))) *
                   copysign(1.0, deltaj);
        else
          deltaj = 0.0;
        if ((T_(nz + 2) - T_(nz + 1)) * (T_(nz + 1) - T_(nz)) > 0.0)
          deltajp1 = fmin3(fabs(deltajp1), 2.0 * fabs(T_(nz + 2) - T_(nz + 1)), 2.0 * fabs(T_(nz + 1) - T_(nz))) *
                     copysign(1.0, deltajp1);
        else
          deltajp1 = 0.0;
        tv[nz] = T_(nz) + dzj / (dzj + dzjp1) * (T_(nz + 1) - T_(nz)) +
                 1.0 / (dzjm1 + dzj + dzjp1 + dzjp2) *
                     ((2.0 * dzjp1 * dzj) / (dzj + dzjp1) *
                          ((dzjm1 + dzj) / (2.0 * dzj + dzjp1) - (dzjp2 + dzjp1) / (2.0 * dzjp1 + dzj)) *
                          (T_(nz + 1) - T_(nz)) -
                      dzj * (dzjm1 + dzj) / (2.0 * dzj + dzjp1) * deltajp1 +
                      dzjp1 * (dzjp1 + dzjp2) / (dzj + 2.0 * dzjp1) * deltaj);
      }
      for (int k = 0; k < nzmax; k++) tvert[k] = 0.0;
      for (int nz = nzmin; nz <= nzmax - 1; nz++) {
        if ((W_(nz) <= 0.0) && (W_(nz + 1) >= 0.0)) continue;
        double Tc = T_(nz);
        double aL = tv[nz - 1], aR = tv[nz];
        if ((aR - Tc) * (Tc - aL) <= 0.0) { aL = Tc; aR = Tc; }
        if ((aR - aL) * (Tc - 0.5 * (aL + aR)) > (aR - aL) * (aR - aL) / 6.0) aL = 3.0 * Tc - 2.0 * aR;
        if ((aR - aL) * (Tc - 0.5 * (aR + aL)) < -((aR - aL) * (aR - aL) / 6.0)) aR = 3.0 * Tc - 2.0 * aL;
        double dzj = A2(m->hnode, nz, n, L);
        double aj = 6.0 * (Tc - 0.5 * (aL + aR));
        if (W_(nz) > 0.0) {
          double x = fmin2(W_(nz) * dt / dzj, 1.0);
          double t = (-aL - 0.5 * x * (aR - aL + (1.0 - 2.0 / 3.0 * x) * aj));
          tvert[nz - 1] = t * A2(m->area, nz, n, nl) * W_(nz);
        }
        if (W_(nz + 1) < 0.0) {
          double x = fmin2(-(W_(nz + 1) * dt / dzj), 1.0);
          double t = (-aR + 0.5 * x * (aR - aL - (1.0 - 2.0 / 3.0 * x) * aj));
          tvert[nz] = t * A2(m->area, nz + 1, n, nl) * W_(nz + 1);
        }
      }
      tvert[nzmin - 1] = -(tv[nzmin - 1] * W_(nzmin) * A2(m->area, nzmin, n, nl));
      tvert[nzmax - 1] = 0.0;
      for (int k = nzmin; k <= nzmax; k++) A2(flux, k, n, nl) = tvert[k - 1] - A2(flux, k, n, nl);
#undef T_
#undef W_
#undef HN_
    }
    free(tv);
    free(tvert);
  }
}

/* adv_tra_ver_cdiff (lib/oce_adv_tra_ver.F90:648-712) */
static void adv_tra_ver_cdiff(const om_mesh *m, const double *W, const double *ttf, double *flux, int init_zero) {
  const int L = m->nl - 1, nl = m->nl;
  if (init_zero) memset(flux, 0, sizeof(double) * (size_t)nl * m->nod2D);
#pragma omp parallel for schedule(static)
  for (int n = 1; n <= m->nod2D; n++) {
    int nzmax = m->nlevels_nod2D[n - 1] - 1, nzmin = m->ulevels_nod2D[n - 1];
    double tvert[1024];
    tvert[nzmin - 1] = -(A2(W, nzmin, n, nl) * A2(ttf, nzmin, n, L) * A2(m->area, nzmin, n, nl));
    tvert[nzmax] = 0.0;
    for (int nz = nzmin + 1; nz <= nzmax; nz++) {
      double tv = 0.5 * (A2(ttf, nz - 1, n, L) + A2(ttf, nz, n, L));
      tvert[nz - 1] = -(tv * A2(W, nz, n, nl) * A2(m->area, nz, n, nl));
    }
    for (int k = nzmin; k <= nzmax; k++) A2(flux, k, n, nl) = tvert[k - 1] - A2(flux, k, n, nl);
  }
}

/* oce_tra_adv_fct (lib/oce_adv_tra_fct.F90:53-483) */
static void oce_tra_adv_fct(const om_mesh *m, double dt, const double *ttf, const double *LO, double *adf_h,
                            double *adf_v, om_work *w) {
  const int L = m->nl - 1, nl = m->nl;
  const double flux_eps = (double)1e-16f; /* real(MP) :: flux_eps=1e-16 (default-real literal) */
  const double bignumber = 1e3;
  double *fmax_ = w->fct_ttf_max, *fmin_ = w->fct_ttf_min, *fp = w->fct_plus, *fm = w->fct_minus;
  /* a1 */
#pragma omp parallel for schedule(static)
  for (int n = 1; n <= m->nod2D; n++)
    for (int nz = m->ulevels_nod2D[n - 1]; nz <= m->nlevels_nod2D[n - 1] - 1; nz++) {
      A2(fmax_, nz, n, L) = fmax2(A2(LO, nz, n, L), A2(ttf, nz, n, L));
      A2(fmin_, nz, n, L) = fmin2(A2(LO, nz, n, L), A2(ttf, nz, n, L));
    }
  /* a2 */
#pragma omp parallel for schedule(static)
  for (int elem = 1; elem <= m->elem2D; elem++) {
    const int *en = &A2(m->elem2D_nodes, 1, elem, 3);
    int nu1 = m->ulevels[elem - 1], nl1 = m->nlevels[elem - 1];
    for (int nz = nu1; nz <= nl1 - 1; nz++) {
      A3(w->aux, 1, nz, elem, 2, L) = fmax3(A2(fmax_, nz, en[0], L), A2(fmax_, nz, en[1], L), A2(fmax_, nz, en[2], L));
      A3(w->aux, 2, nz, elem, 2, L) = fmin3(A2(fmin_, nz, en[0], L), A2(fmin_, nz, en[1], L), A2(fmin_, nz, en[2], L));
    }
    if (nl1 <= nl - 1)
      for (int nz = nl1; nz <= nl - 1; nz++) {
        A3(w->aux, 1, nz, elem, 2, L) = -bignumber;
        A3(w->aux, 2, nz, elem, 2, L) = bignumber;
      }
  }
  /* a3 */
#pragma omp parallel for schedule(static)
  for (int n = 1; n <= m->nod2D; n++) {
    int nu1 = m->ulevels_nod2D[n - 1], nl1 = m->nlevels_nod2D[n - 1];
    for (int nz = nu1; nz <= nl1 - 1; nz++) {
      A2(w->tvert_max, nz, n, L) = A3(w->aux, 1, nz, NIE(1, n), 2, L);
      A2(w->tvert_min, nz, n, L) = A3(w->aux, 2, nz, NIE(1, n), 2, L);
      for (int elem = 2; elem <= m->nod_in_elem2D_num[n - 1]; elem++) {
        A2(w->tvert_max, nz, n, L) = fmax2(A2(w->tvert_max, nz, n, L), A3(w->aux, 1, nz, NIE(elem, n), 2, L));
        A2(w->tvert_min, nz, n, L) = fmin2(A2(w->tvert_min, nz, n, L), A3(w->aux, 2, nz, NIE(elem, n), 2, L));
      }
    }
  }
#pragma omp parallel for schedule(static)
  for (int n = 1; n <= m->nod2D; n++) {
    int nu1 = m->ulevels_nod2D[n - 1], nl1 = m->nlevels_nod2D[n - 1];
    A2(fmax_, nu1, n, L) = A2(w->tvert_max, nu1, n, L) - A2(LO, nu1, n, L);
    A2(fmin_, nu1, n, L) = A2(w->tvert_min, nu1, n, L) - A2(LO, nu1, n, L);
    for (int nz = nu1 + 1; nz <= nl1 - 2; nz++) {
      A2(fmax_, nz, n, L) = fmax3(A2(w->tvert_max, nz - 1, n, L), A2(w->tvert_max, nz, n, L), A2(w->tvert_max, nz + 1, n, L)) - A2(LO, nz, n, L);
      A2(fmin_, nz, n, L) = fmin3(A2(w->tvert_min, nz - 1, n, L), A2(w->tvert_min, nz, n, L), A2(w->tvert_min, nz + 1, n, L)) - A2(LO, nz, n, L);
    }
    int nz = nl1 - 1;
    A2(fmax_, nz, n, L) = A2(w->tvert_max, nz, n, L) - A2(LO, nz, n, L);
    A2(fmin_, nz, n, L) = A2(w->tvert_min, nz, n, L) - A2(LO, nz, n, L);
  }
  /* b1: zero, vertical, horizontal edge scatter in edge order */
#pragma omp parallel for schedule(static)
  for (int n = 1; n <= m->nod2D; n++)
    for (int nz = m->ulevels_nod2D[n - 1]; nz <= m->nlevels_nod2D[n - 1] - 1; nz++) {
      A2(fp, nz, n, L) = 0.0;
      A2(fm, nz, n, L) = 0.0;
    }
#pragma omp parallel for schedule(static)
  for (int n = 1; n <= m->nod2D; n++)
    for (int nz = m->ulevels_nod2D[n - 1]; nz <= m->nlevels_nod2D[n - 1] - 1; nz++) {
      A2(fp, nz, n, L) = A2(fp, nz, n, L) + (fmax2(0.0, A2(adf_v, nz, n, nl)) + fmax2(0.0, -A2(adf_v, nz + 1, n, nl)));
      A2(fm, nz, n, L) = A2(fm, nz, n, L) + (fmin2(0.0, A2(adf_v, nz, n, nl)) + fmin2(0.0, -A2(adf_v, nz + 1, n, nl)));
    }
#pragma omp parallel
  {
    int own_lo, own_hi;
    own_range(m->nod2D, &own_lo, &own_hi);
    for (int edge = 1; edge <= m->edge2D; edge++) {
      int n1 = A2(m->edges, 1, edge, 2), n2 = A2(m->edges, 2, edge, 2);
      int el1 = A2(m->edge_tri, 1, edge, 2), el2 = A2(m->edge_tri, 2, edge, 2);
      int nl1 = m->nlevels[el1 - 1] - 1, nu1 = m->ulevels[el1 - 1], nl2 = 0, nu2 = 0;
      if (el2 > 0) { nl2 = m->nlevels[el2 - 1] - 1; nu2 = m->ulevels[el2 - 1]; }
      int nl12 = imax2(nl1, nl2), nu12 = nu1;
      if (nu2 > 0) nu12 = imin2(nu1, nu2);
      if (n1 >= own_lo && n1 <= own_hi)
        for (int nz = nu12; nz <= nl12; nz++) {
          A2(fp, nz, n1, L) = A2(fp, nz, n1, L) + fmax2(0.0, A2(adf_h, nz, edge, L));
          A2(fm, nz, n1, L) = A2(fm, nz, n1, L) + fmin2(0.0, A2(adf_h, nz, edge, L));
        }
      if (n2 >= own_lo && n2 <= own_hi)
        for (int nz = nu12; nz <= nl12; nz++) {
          A2(fp, nz, n2, L) = A2(fp, nz, n2, L) + fmax2(0.0, -A2(adf_h, nz, edge, L));
          A2(fm, nz, n2, L) = A2(fm, nz, n2, L) + fmin2(0.0, -A2(adf_h, nz, edge, L));
        }
    }
  }
  /* b2 */
#pragma omp parallel for schedule(static)
  for (int n = 1; n <= m->nod2D; n++)
    for (int nz = m->ulevels_nod2D[n - 1]; nz <= m->nlevels_nod2D[n - 1] - 1; nz++) {
      double flux = A2(fp, nz, n, L) * dt / A2(m->areasvol, nz, n, nl) + flux_eps;
      A2(fp, nz, n, L) = fmin2(1.0, A2(fmax_, nz, n, L) / flux);
      flux = A2(fm, nz, n, L) * dt / A2(m->areasvol, nz, n, nl) - flux_eps;
      A2(fm, nz, n, L) = fmin2(1.0, A2(fmin_, nz, n, L) / flux);
    }
  /* b3 vertical */
#pragma omp parallel for schedule(static)
  for (int n = 1; n <= m->nod2D; n++) {
    int nu1 = m->ulevels_nod2D[n - 1], nl1 = m->nlevels_nod2D[n - 1];
    int nz = nu1;
    double ae = 1.0, flux = A2(adf_v, nz, n, nl);
    if (flux >= 0.0) ae = fmin2(ae, A2(fp, nz, n, L));
    else ae = fmin2(ae, A2(fm, nz, n, L));
    A2(adf_v, nz, n, nl) = ae * A2(adf_v, nz, n, nl);
    for (nz = nu1 + 1; nz <= nl1 - 1; nz++) {
      ae = 1.0;
      flux = A2(adf_v, nz, n, nl);
      if (flux >= 0.0) {
        ae = fmin2(ae, A2(fm, nz - 1, n, L));
        ae = fmin2(ae, A2(fp, nz, n, L));
      } else {
        ae = fmin2(ae, A2(fp, nz - 1, n, L));
        ae = fmin2(ae, A2(fm, nz, n, L));
      }
      A2(adf_v, nz, n, nl) = ae * A2(adf_v, nz, n, nl);
    }
  }
  /* b3 horizontal */
#pragma omp parallel for schedule(static)
  for (int edge = 1; edge <= m->edge2D; edge++) {
    int n1 = A2(m->edges, 1, edge, 2), n2 = A2(m->edges, 2, edge, 2);
    int el1 = A2(m->edge_tri, 1, edge, 2), el2 = A2(m->edge_tri, 2, edge, 2);
    int nu1 = m->ulevels[el1 - 1], nl1 = m->nlevels[el1 - 1] - 1, nl2 = 0, nu2 = 0;
    if (el2 > 0) { nu2 = m->ulevels[el2 - 1]; nl2 = m->nlevels[el2 - 1] - 1; }
    int nl12 = imax2(nl1, nl2), nu12 = nu1;
    if (nu2 > 0) nu12 = imin2(nu1, nu2);
    for (int nz = nu12; nz <= nl12; nz++) {
      double ae = 1.0, flux = A2(adf_h, nz, edge, L);
      if (flux >= 0.0) {
        ae = fmin2(ae, A2(fp, nz, n1, L));
        ae = fmin2(ae, A2(fm, nz, n2, L));
      } else {
        ae = fmin2(ae, A2(fm, nz, n1, L));
        ae = fmin2(ae, A2(fp, nz, n2, L));
      }
      A2(adf_h, nz, edge, L) = ae * A2(adf_h, nz, edge, L);
    }
  }
}

/* oce_tra_adv_flux2dtracer (lib/oce_adv_tra_driver.F90:298-450) */
static void flux2dtracer(const om_mesh *m, double dt, double *dttf_h, double *dttf_v, const double *flux_h,
                         const double *flux_v, int use_lo, const double *ttf, const double *LO) {
  const int L = m->nl - 1, nl = m->nl;
  if (use_lo) {
#pragma omp parallel for schedule(static)
    for (int n = 1; n <= m->nod2D; n++)
      for (int nz = m->ulevels_nod2D[n - 1]; nz <= m->nlevels_nod2D[n - 1] - 1; nz++)
        A2(dttf_v, nz, n, L) = A2(dttf_v, nz, n, L) - A2(ttf, nz, n, L) * A2(m->hnode, nz, n, L) +
                               A2(LO, nz, n, L) * A2(m->hnode_new, nz, n, L);
  }
#pragma omp parallel for schedule(static)
  for (int n = 1; n <= m->nod2D; n++)
    for (int nz = m->ulevels_nod2D[n - 1]; nz <= m->nlevels_nod2D[n - 1] - 1; nz++)
      A2(dttf_v, nz, n, L) = A2(dttf_v, nz, n, L) +
                             (A2(flux_v, nz, n, nl) - A2(flux_v, nz + 1, n, nl)) * dt / A2(m->areasvol, nz, n, nl);
#pragma omp parallel
  {
    int own_lo, own_hi;
    own_range(m->nod2D, &own_lo, &own_hi);
    for (int edge = 1; edge <= m->edge2D; edge++) {
      int n1 = A2(m->edges, 1, edge, 2), n2 = A2(m->edges, 2, edge, 2);
      int el1 = A2(m->edge_tri, 1, edge, 2), el2 = A2(m->edge_tri, 2, edge, 2);
      int nl1 = m->nlevels[el1 - 1] - 1, nu1 = m->ulevels[el1 - 1], nl2 = 0, nu2 = 0;
      if (el2 > 0) { nl2 = m->nlevels[el2 - 1] - 1; nu2 = m->ulevels[el2 - 1]; }
      int nl12 = imax2(nl1, nl2), nu12 = nu1;
      if (nu2 > 0) nu12 = imin2(nu1, nu2);
      if (n1 >= own_lo && n1 <= own_hi)
        for (int nz = nu12; nz <= nl12; nz++)
          A2(dttf_h, nz, n1, L) = A2(dttf_h, nz, n1, L) + A2(flux_h, nz, edge, L) * dt / A2(m->areasvol, nz, n1, nl);
      if (n2 >= own_lo && n2 <= own_hi)
        for (int nz = nu12; nz <= nl12; nz++)
          A2(dttf_h, nz, n2, L) = A2(dttf_h, nz, n2, L) - A2(flux_h, nz, edge, L) * dt / A2(m->areasvol, nz, n2, nl);
    }
  }
}

/* do_oce_adv_tra (lib/oce_adv_tra_driver.F90:23-294); W = WI = WE. */
static void do_oce_adv_tra(const om_mesh *m, int hor, int ver, int lim, double opth, double optv, double dt,
                           const double *vel, const double *W, const double *ttf, const double *ttfAB, om_work *w) {
  const int L = m->nl - 1, nl = m->nl;
  double *fct_LO = w->fct_LO, *adv_flux_hor = w->adv_flux_hor, *adv_flux_ver = w->adv_flux_ver;
  if (lim == OM_LIM_FCT) {
    adv_tra_hor_upw1(m, vel, ttf, adv_flux_hor, 1);
    memset(fct_LO, 0, sizeof(double) * (size_t)L * m->nod2D);
#pragma omp parallel
    {
      int own_lo, own_hi;
      own_range(m->nod2D, &own_lo, &own_hi);
      for (int e = 1; e <= m->edge2D; e++) {
        int n1 = A2(m->edges, 1, e, 2), n2 = A2(m->edges, 2, e, 2);
        int el1 = A2(m->edge_tri, 1, e, 2), el2 = A2(m->edge_tri, 2, e, 2);
        int nl1 = m->nlevels[el1 - 1] - 1, nu1 = m->ulevels[el1 - 1], nl2 = 0, nu2 = 0;
        if (el2 > 0) { nl2 = m->nlevels[el2 - 1] - 1; nu2 = m->ulevels[el2 - 1]; }
        int nl12 = imax2(nl1, nl2), nu12 = nu1;
        if (nu2 > 0) nu12 = imin2(nu1, nu2);
        if (n1 >= own_lo && n1 <= own_hi)
          for (int nz = nu12; nz <= nl12; nz++) A2(fct_LO, nz, n1, L) = A2(fct_LO, nz, n1, L) + A2(adv_flux_hor, nz, e, L);
        if (n2 >= own_lo && n2 <= own_hi)
          for (int nz = nu12; nz <= nl12; nz++) A2(fct_LO, nz, n2, L) = A2(fct_LO, nz, n2, L) - A2(adv_flux_hor, nz, e, L);
      }
    }
    adv_tra_ver_upw1(m, W, ttf, adv_flux_ver, 1);
#pragma omp parallel for schedule(static)
    for (int n = 1; n <= m->nod2D; n++)
      for (int nz = m->ulevels_nod2D[n - 1]; nz <= m->nlevels_nod2D[n - 1] - 1; nz++)
        A2(fct_LO, nz, n, L) = (A2(ttf, nz, n, L) * A2(m->hnode, nz, n, L) +
                                (A2(fct_LO, nz, n, L) + (A2(adv_flux_ver, nz, n, nl) - A2(adv_flux_ver, nz + 1, n, nl))) *
                                    dt / A2(m->areasvol, nz, n, nl)) /
                               A2(m->hnode_new, nz, n, L);
  }
  const int zero = (lim == OM_LIM_FCT) ? 0 : 1;
  switch (hor) {
    case OM_HOR_MUSCL: adv_tra_hor_muscl(m, vel, ttfAB, opth, adv_flux_hor, w->edge_up_dn_grad, 1, zero); break;
    case OM_HOR_MFCT: adv_tra_hor_muscl(m, vel, ttfAB, opth, adv_flux_hor, w->edge_up_dn_grad, 0, zero); break;
    default: adv_tra_hor_upw1(m, vel, ttfAB, adv_flux_hor, zero); break;
  }
  switch (ver) {
    case OM_VER_QR4C: adv_tra_ver_qr4c(m, W, ttfAB, optv, adv_flux_ver, zero); break;
    case OM_VER_CDIFF: adv_tra_ver_cdiff(m, W, ttfAB, adv_flux_ver, zero); break;
    case OM_VER_PPM: adv_tra_vert_ppm(m, dt, W, ttfAB, adv_flux_ver, zero); break;
    default: adv_tra_ver_upw1(m, W, ttfAB, adv_flux_ver, zero); break;
  }
  if (lim == OM_LIM_FCT) {
    oce_tra_adv_fct(m, dt, ttf, fct_LO, adv_flux_hor, adv_flux_ver, w);
    flux2dtracer(m, dt, w->dttf_h, w->dttf_v, adv_flux_hor, adv_flux_ver, 1, ttf, fct_LO);
  } else {
    flux2dtracer(m, dt, w->dttf_h, w->dttf_v, adv_flux_hor, adv_flux_ver, 0, NULL, NULL);
  }
}

static void step_one(const om_mesh *m, int hor, int ver, int lim, double ph, double pv, double dt, const double *uv,
                     const double *w, double *values, const double *valuesAB, om_work *wk) {
  const int L = m->nl - 1;
  /* src/fesom_analytic.F90:407-413 */
  memset(wk->dttf_h, 0, sizeof(double) * (size_t)L * m->nod2D);
  memset(wk->dttf_v, 0, sizeof(double) * (size_t)L * m->nod2D);
  if (hor == OM_HOR_MUSCL || hor == OM_HOR_MFCT) {
    tracer_gradient_elements(m, valuesAB, wk->tr_xy);
    fill_up_dn_grad(m, wk->tr_xy, wk->edge_up_dn_grad);
  }
  do_oce_adv_tra(m, hor, ver, lim, ph, pv, dt, uv, w, values, valuesAB, wk);
  /* src/fesom_analytic.F90:419-437: del_ttf = 0 + h + v; values += del/h_new */
#pragma omp parallel for schedule(static)
  for (int n = 1; n <= m->nod2D; n++)
    for (int kz = m->ulevels_nod2D[n - 1]; kz <= m->nlevels_nod2D[n - 1] - 1; kz++) {
      double del = 0.0 + A2(wk->dttf_h, kz, n, L) + A2(wk->dttf_v, kz, n, L);
      A2(values, kz, n, L) = A2(values, kz, n, L) + del / A2(m->hnode_new, kz, n, L);
    }
}

int om_tracer_step(const om_mesh *m, int hor, int ver, int lim, double ph, double pv, double dt, const double *uv,
                   const double *w, double *values, const double *valuesAB, double *del_h, double *del_v, double *lo) {
  if (!m) return -1;
  const size_t LN = (size_t)(m->nl - 1) * m->nod2D;
  om_work *wk = mesh_work(m);
  step_one(m, hor, ver, lim, ph, pv, dt, uv, w, values, valuesAB, wk);
  if (del_h) memcpy(del_h, wk->dttf_h, LN * 8);
  if (del_v) memcpy(del_v, wk->dttf_v, LN * 8);
  if (lo) memcpy(lo, wk->fct_LO, LN * 8);
  return 0;
}

int om_run(const om_mesh *m, int hor, int ver, int lim, double ph, double pv, double dt, const double *uv,
           const double *w, int ntracers, int nsteps, double *values, double *valuesAB, int refresh_ab) {
  if (!m) return -1;
  const size_t LN = (size_t)(m->nl - 1) * m->nod2D;
  om_work *wk = mesh_work(m);
  for (int s = 0; s < nsteps; s++)
    for (int t = 0; t < ntracers; t++) {
      if (refresh_ab) memcpy(valuesAB + t * LN, values + t * LN, LN * 8);
      step_one(m, hor, ver, lim, ph, pv, dt, uv, w, values + t * LN, valuesAB + t * LN, wk);
    }
  return 0;
}

void om_stats(const om_mesh *m, const double *values, double *out) {
  const size_t LN = (size_t)(m->nl - 1) * m->nod2D;
  double mn = values[0], mx = values[0], sm = 0.0, nan = 0.0;
  for (size_t i = 0; i < LN; i++) {
    double v = values[i];
    if (v < mn) mn = v;
    if (v > mx) mx = v;
    sm += v;
    if (v != v) nan += 1.0;
  }
  out[0] = mn; out[1] = mx; out[2] = sm; out[3] = nan;
}

/* ------------------------------------------------------------------------ */
/* Seeded synthetic inputs of the benchmark workloads, restated here so that  */
/* the CPU baseline builds its inputs without the product library.  They are  */
/* the same functions of the same seeds as the library's generators: a CPU    */
/* test checks the two bit for bit.                                           */
/* ------------------------------------------------------------------------ */

/* MT19937-64 (Matsumoto & Nishimura, "Mersenne Twister 64-bit", 2004): the
 * published recurrence, tempering and seeding, which are also those of the
 * C++ std::mt19937_64 engine. */
typedef struct { uint64_t s[312]; int i; } mt64;
static void mt64_seed(mt64 *g, uint64_t seed) {
  g->s[0] = seed;
  for (int i = 1; i < 312; i++) g->s[i] = 6364136223846793005ULL * (g->s[i - 1] ^ (g->s[i - 1] >> 62)) + (uint64_t)i;
  g->i = 312;
}
static uint64_t mt64_next(mt64 *g) {
  if (g->i >= 312) {
    const uint64_t UM = 0xFFFFFFFF80000000ULL, LM = 0x7FFFFFFFULL, A = 0xB5026F5AA96619E9ULL;
    for (int k = 0; k < 312; k++) {
      const uint64_t x = (g->s[k] & UM) | (g->s[(k + 1) % 312] & LM);
      g->s[k] = g->s[(k + 156) % 312] ^ (x >> 1) ^ ((x & 1ULL) ? A : 0ULL);
    }
    g->i = 0;
  }
  uint64_t x = g->s[g->i++];
  x ^= (x >> 29) & 0x5555555555555555ULL;
  x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
  x ^= (x << 37) & 0xFFF7EEE000000000ULL;
  x ^= x >> 43;
  return x;
}
static double mt64_uni(mt64 *g) { return (double)(mt64_next(g) >> 11) * 0x1.0p-53; } /* [0, 1) */
static double mt64_normal(mt64 *g) { /* Box-Muller, first variate */
  double u1 = mt64_uni(g), u2 = mt64_uni(g);
  if (u1 < 1e-300) u1 = 1e-300;
  return sqrt(-2.0 * log(u1)) * cos(2.0 * PI_F * u2);
}

/* six Fourier modes with integer wave numbers, periodic on [0,Lx) x [0,Ly) */
typedef struct { int kx[6], ky[6]; double amp[6], ph[6]; } om_modes;
static void modes_draw(om_modes *md, mt64 *g) {
  for (int q = 0; q < 6; q++) {
    md->kx[q] = 1 + (int)(mt64_next(g) % 4);
    md->ky[q] = 1 + (int)(mt64_next(g) % 4);
    md->amp[q] = 0.5 + mt64_uni(g);
    md->ph[q] = 2.0 * PI_F * mt64_uni(g);
  }
}
static double modes_eval(const om_modes *md, double x, double y, double Lx, double Ly) {
  double s = 0.0;
  for (int q = 0; q < 6; q++) s += md->amp[q] * sin(2.0 * PI_F * (md->kx[q] * x / Lx + md->ky[q] * y / Ly) + md->ph[q]);
  return s;
}

void om_synth_bathymetry_smooth(int nx, int ny, int periodic, int nl, double corr_cells, unsigned long long seed, int *K) {
  mt64 g;
  mt64_seed(&g, seed);
  enum { NM = 48 };
  double kx[NM], ky[NM], ph[NM];
  const double cmax = (double)(nx > ny ? nx : ny);
  const double cc = corr_cells > 1.0 ? corr_cells : 1.0;
  const double kmax = fmax(1.0, cmax / cc);
  for (int q = 0; q < NM; q++) {
    double a, b;
    do {
      a = floor((2.0 * mt64_uni(&g) - 1.0) * (kmax + 1.0));
      b = floor((2.0 * mt64_uni(&g) - 1.0) * (kmax + 1.0));
    } while (a == 0.0 && b == 0.0);
    kx[q] = a; ky[q] = b;
    ph[q] = 2.0 * PI_F * mt64_uni(&g);
  }
  const int ni = periodic ? nx - 1 : nx, nj = periodic ? ny - 1 : ny;
  const double norm = sqrt(2.0 / NM);
  for (int j = 0; j < nj; j++)
    for (int i = 0; i < ni; i++) {
      const double x = (double)i / (double)(nx - 1), y = (double)j / (double)(ny - 1);
      double gg = 0.0;
      for (int q = 0; q < NM; q++) gg += cos(2.0 * PI_F * (kx[q] * x + ky[q] * y) + ph[q]);
      gg *= norm;
      const double u = 0.5 * erfc(-gg / sqrt(2.0));
      int k = 3 + (int)(u * (double)(nl - 2));
      K[(size_t)j * ni + i] = imin2(nl, imax2(3, k));
    }
}

void om_synth_velocity(const om_mesh *m, unsigned long long seed, double umax, double mode1_frac, double mode2_frac,
                       double baro_frac, double *uv, double *W) {
  const int N = m->nod2D, T = m->elem2D, E = m->edge2D, nl = m->nl, L = nl - 1;
  mt64 g;
  mt64_seed(&g, seed);
  double *xm = malloc(sizeof(double) * N), *ym = malloc(sizeof(double) * N);
  for (int n = 0; n < N; n++) {
    xm[n] = A2(m->coord, 1, n + 1, 2) * R_EARTH;
    ym[n] = A2(m->coord, 2, n + 1, 2) * R_EARTH;
  }
  om_modes p1, p2, chi, p0;
  modes_draw(&p1, &g);
  modes_draw(&p2, &g);
  modes_draw(&chi, &g);
  if (baro_frac != 0.0) modes_draw(&p0, &g);
  double *f1 = malloc(sizeof(double) * N), *f2 = malloc(sizeof(double) * N), *f3 = malloc(sizeof(double) * N);
  for (int n = 0; n < N; n++) {
    f1[n] = modes_eval(&p1, xm[n], ym[n], m->Lx, m->Ly);
    f2[n] = modes_eval(&p2, xm[n], ym[n], m->Lx, m->Ly);
    f3[n] = modes_eval(&chi, xm[n], ym[n], m->Lx, m->Ly);
  }
  const size_t nuv = (size_t)2 * L * T;
  memset(uv, 0, nuv * sizeof(double));
  /* barotropic part curl(psi0), psi0 zero at nodes of an element dry at the
   * level and on walls */
  if (baro_frac != 0.0) {
    int *shallowest = malloc(sizeof(int) * N);
    char *wall = calloc(N, 1);
    double *f0 = malloc(sizeof(double) * N);
    for (int n = 0; n < N; n++) shallowest[n] = nl;
    for (int e = 0; e < T; e++)
      for (int q = 0; q < 3; q++) {
        const int nd = m->elem2D_nodes[3 * e + q] - 1;
        shallowest[nd] = imin2(shallowest[nd], m->nlevels[e]);
      }
    for (int e = 0; e < E; e++)
      if (m->edge_tri[2 * e + 1] <= 0) { wall[m->edges[2 * e] - 1] = 1; wall[m->edges[2 * e + 1] - 1] = 1; }
    for (int n = 0; n < N; n++) f0[n] = wall[n] ? 0.0 : baro_frac * modes_eval(&p0, xm[n], ym[n], m->Lx, m->Ly);
    for (int e = 0; e < T; e++) {
      const int *en = &m->elem2D_nodes[3 * e];
      const double *gs = &m->gradient_sca[6 * e];
      for (int k = 0; k < m->nlevels[e] - 1; k++) {
        double psi[3];
        for (int q = 0; q < 3; q++) psi[q] = (k + 1) > shallowest[en[q] - 1] - 1 ? 0.0 : f0[en[q] - 1];
        uv[2 * ((size_t)e * L + k)] += -(gs[3] * psi[0] + gs[4] * psi[1] + gs[5] * psi[2]);
        uv[2 * ((size_t)e * L + k) + 1] += gs[0] * psi[0] + gs[1] * psi[1] + gs[2] * psi[2];
      }
    }
    free(shallowest); free(wall); free(f0);
  }
  double *c1 = malloc(sizeof(double) * (L > 0 ? L : 1)), *c2 = malloc(sizeof(double) * (L > 0 ? L : 1));
  for (int e = 0; e < T; e++) {
    const int a0 = m->elem2D_nodes[3 * e] - 1, a1 = m->elem2D_nodes[3 * e + 1] - 1, a2 = m->elem2D_nodes[3 * e + 2] - 1;
    const double *gs = &m->gradient_sca[6 * e];
#define GX(f) (gs[0] * (f)[a0] + gs[1] * (f)[a1] + gs[2] * (f)[a2])
#define GY(f) (gs[3] * (f)[a0] + gs[4] * (f)[a1] + gs[5] * (f)[a2])
    const double u1 = -GY(f1), v1 = GX(f1);
    const double u2 = -GY(f2) + GX(f3), v2 = GX(f2) + GY(f3);
#undef GX
#undef GY
    const int M = m->nlevels[e] - 1;
    const double *h = &m->helem[(size_t)e * L];
    double s1 = 0.0, s2 = 0.0, hs = 0.0;
    for (int k = 0; k < M; k++) {
      c1[k] = cos(PI_F * ((double)k + 0.5) / (double)M);
      c2[k] = cos(2.0 * PI_F * ((double)k + 0.5) / (double)M);
      s1 += c1[k] * h[k];
      s2 += c2[k] * h[k];
      hs += h[k];
    }
    s1 /= hs;
    s2 /= hs;
    for (int k = 0; k < M; k++) {
      const double b1 = mode1_frac * (c1[k] - s1), b2 = mode2_frac * (c2[k] - s2);
      uv[2 * ((size_t)e * L + k)] += b1 * u1 + b2 * u2;
      uv[2 * ((size_t)e * L + k) + 1] += b1 * v1 + b2 * v2;
    }
  }
  double vmax = 0.0;
  for (size_t i = 0; i < nuv / 2; i++) vmax = fmax(vmax, hypot(uv[2 * i], uv[2 * i + 1]));
  const double scale = umax < 0.0 ? -umax : (vmax > 0.0 ? umax / vmax : 0.0);
  for (size_t i = 0; i < nuv; i++) uv[i] *= scale;
  /* horizontal divergence of the edge volume fluxes, then W from the bottom up */
  double *D = calloc((size_t)L * N, sizeof(double));
  for (int e = 0; e < E; e++) {
    const int n1 = m->edges[2 * e] - 1, n2 = m->edges[2 * e + 1] - 1;
    const int t1 = m->edge_tri[2 * e] - 1, t2 = m->edge_tri[2 * e + 1] - 1;
    const int nl1 = m->nlevels[t1] - 1, nl2 = t2 >= 0 ? m->nlevels[t2] - 1 : 0;
    const double *c = &m->edge_cross_dxdy[4 * e];
    for (int k = 0; k < imax2(nl1, nl2); k++) {
      double v = 0.0;
      if (k < nl1) v += (-uv[2 * ((size_t)t1 * L + k) + 1] * c[0] + uv[2 * ((size_t)t1 * L + k)] * c[1]) * m->helem[(size_t)t1 * L + k];
      if (k < nl2) v += (uv[2 * ((size_t)t2 * L + k) + 1] * c[2] - uv[2 * ((size_t)t2 * L + k)] * c[3]) * m->helem[(size_t)t2 * L + k];
      D[(size_t)n1 * L + k] += v;
      D[(size_t)n2 * L + k] -= v;
    }
  }
  memset(W, 0, (size_t)nl * N * sizeof(double));
  for (int n = 0; n < N; n++) {
    const int nlev = m->nlevels_nod2D[n];
    for (int i = nlev - 1; i >= 2; i--) {
      const double Ai = m->area[(size_t)n * nl + i - 1], Ai1 = m->area[(size_t)n * nl + i];
      const double flux_below = W[(size_t)n * nl + i] * Ai1;
      W[(size_t)n * nl + i - 1] = Ai > 0.0 ? (flux_below - D[(size_t)n * L + i - 1]) / Ai : 0.0;
    }
    W[(size_t)n * nl + 0] = 0.0;
  }
  free(D); free(c1); free(c2); free(f1); free(f2); free(f3); free(xm); free(ym);
}

void om_synth_tracer(const om_mesh *m, unsigned long long seed, int kind, double *T) {
  const int N = m->nod2D, L = m->nl - 1;
  mt64 g;
  mt64_seed(&g, seed);
  memset(T, 0, (size_t)L * N * sizeof(double));
  if (kind == 0) {
    double bx[8], by[8], bs[8], ba[8];
    for (int b = 0; b < 8; b++) {
      bx[b] = mt64_uni(&g) * m->Lx; by[b] = mt64_uni(&g) * m->Ly;
      bs[b] = (0.03 + 0.07 * mt64_uni(&g)) * m->Lx; ba[b] = 5.0 + 10.0 * mt64_uni(&g);
    }
    for (int n = 0; n < N; n++) {
      const double x = A2(m->coord, 1, n + 1, 2) * R_EARTH, y = A2(m->coord, 2, n + 1, 2) * R_EARTH;
      double blob = 0.0;
      for (int b = 0; b < 8; b++) {
        double dx = fabs(x - bx[b]), dy = fabs(y - by[b]);
        if (m->periodic) { dx = fmin(dx, m->Lx - dx); dy = fmin(dy, m->Ly - dy); }
        blob += ba[b] * exp(-(dx * dx + dy * dy) / (bs[b] * bs[b]));
      }
      for (int k = 0; k < m->nlevels_nod2D[n] - 1; k++) T[(size_t)n * L + k] = 20.0 * mt64_uni(&g) + blob;
    }
  } else {
    for (int n = 0; n < N; n++)
      for (int k = 0; k < m->nlevels_nod2D[n] - 1; k++) T[(size_t)n * L + k] = 35.0 + 0.5 * mt64_normal(&g);
  }
}
