/*
 * fesom_oracle.h -- CPU oracle for the FESOM2 tracer advection step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library restates, loop by loop, the
 * reference's FP64 algorithm for do_oce_adv_tra (suvarchal/fesom2_tracer_dwarf,
 * lib/oce_adv_tra_driver.F90:23-450 and the routines it calls) together with the
 * analytic mesh generator it runs on (lib/analytic_mesh.F90:114-829,
 * lib/oce_mesh.F90:1522-1560,2001-2534).  It is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * it.  The product never links it.
 *
 * Conventions: every array is stored in Fortran column-major order with
 * 1-based indices in the index arrays (0 = "no element"), exactly like the
 * reference's derived types (lib/MOD_MESH.F90:24-166, lib/MOD_TRACER.F90:10-62).
 */
#ifndef FESOM_ORACLE_H
#define FESOM_ORACLE_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct om_mesh om_mesh;

/* Scheme codes (lib/oce_adv_tra_driver.F90:244-283). */
enum { OM_HOR_UPW1 = 0, OM_HOR_MUSCL = 1, OM_HOR_MFCT = 2 };
enum { OM_VER_UPW1 = 0, OM_VER_PPM = 1, OM_VER_QR4C = 2, OM_VER_CDIFF = 3 };
enum { OM_LIM_NONE = 0, OM_LIM_FCT = 1 };

/* Build the analytic mesh of lib/analytic_mesh.F90:114 (periodic or closed).
 * options bit 0 (OM_FULL_RINGS): 0 keeps the reference's periodic
 * nod_in_elem2D lists, which are built before the halo remap and are therefore
 * incomplete on the wrap rows (lib/analytic_mesh.F90:674-694); 1 rebuilds them
 * after the remap.  options bit 1 (OM_LEFT_ORIENTED): reverse the node order
 * of the horizontal and vertical edges so that edge_tri(1) lies to the left of
 * edges(1)->edges(2) on every edge, as it does on the diagonals of the
 * reference mesh (lib/analytic_mesh.F90:386-441 puts it on the right of the
 * horizontal and vertical edges).
 * node_K (length nod2D, nullable) gives a per-node bottom level index in
 * [3, nl]; NULL reproduces the reference's flat bottom (nlevels = nl). */
enum { OM_FULL_RINGS = 1, OM_LEFT_ORIENTED = 2 };
om_mesh *om_mesh_analytic(int nx, int ny, int nl, double Lx, double Ly,
                          double max_depth, int periodic, int options,
                          const int *node_K);
/* Build a mesh from the reference's ASCII mesh files in dir (nod2d.out,
 * elem2d.out, aux3d.out, edgenum.out, edges.out, edge_tri.out, elvls.out,
 * nlvls.out) as mesh_setup does on one process (lib/oce_mesh.F90:49-94):
 * node coordinates in degrees -> radians, rotated by the Euler angles
 * (alpha, beta, gamma) x angle_scale when rotate != 0, elements oriented by
 * test_tri, levels from elvls/nlvls, spherical areas and auxiliary arrays with
 * the given cyclic_length (in radians of longitude), then the ALE thicknesses
 * of tracer_init_ale_arrays and the MUSCL tables.  The reference's defaults
 * are rotate = 1, (50, 15, -90), angle_scale = 1 (its
 * set_mesh_transform_matrix passes the values to cos/sin as they are) and
 * cyclic_length = 360.  NULL on failure, with a message in err. */
om_mesh *om_mesh_from_files(const char *dir, int rotate, double alpha, double beta, double gamma,
                            double angle_scale, double cyclic_length, char *err, int errlen);
/* A mesh from arrays in the layouts above (index arrays 1-based, 0 = none;
 * the node rings as counts and their concatenated element lists), with the
 * MUSCL tables (edge_up_dn_tri, nboundary_lay) taken as given, and
 * thicknesses as given (zbar_3d_n, Z_3d_n from zbar).  Checks mesh parts of
 * a domain decomposition against the whole mesh. */
om_mesh *om_mesh_from_arrays(int nl, int nod2D, int elem2D, int edge2D, int periodic, double Lx, double Ly,
                             const double *coord, const int *elem2D_nodes, const int *edges, const int *edge_tri,
                             const int *nlevels, const int *nlevels_nod2D, const int *nlevels_nod2D_min,
                             const int *ring_num, const int *ring_elem, const double *elem_area, const double *area,
                             const double *areasvol, const double *edge_dxdy, const double *edge_cross_dxdy,
                             const double *gradient_sca, const double *elem_cos, const double *zbar,
                             const double *hnode, const double *hnode_new, const double *helem,
                             const int *edge_up_dn_tri, const int *nboundary_lay);
void om_mesh_free(om_mesh *m);

/* dims[0..5] = nl, nod2D, elem2D, edge2D, max_nod_in_elem, periodic */
void om_mesh_dims(const om_mesh *m, int *dims);
/* Length and contents of a named mesh array (see om_mesh fields). */
long om_mesh_len(const om_mesh *m, const char *name);
int om_mesh_get_int(const om_mesh *m, const char *name, int *out);
int om_mesh_get_dbl(const om_mesh *m, const char *name, double *out);

/* Initial fields of the analytic driver (src/fesom_analytic.F90:251-256,
 * 306-331): T, S of shape (nl-1, nod2D); uv (2, nl-1, elem2D); w (nl, nod2D). */
void om_analytic_fields(const om_mesh *m, double *T, double *S, double *uv,
                        double *w);

/* One do_oce_adv_tra call for one tracer (lib/oce_adv_tra_driver.F90:23),
 * preceded by the element gradient tr_xy and fill_up_dn_grad when the
 * horizontal scheme is MUSCL or MFCT, followed by the host update of
 * src/fesom_analytic.F90:407-437:  values += (del_h + del_v) / hnode_new.
 * w is used as w, w_i and w_e (use_wsplit = .false.).  Optional outputs
 * (nullable): del_h, del_v (nl-1, nod2D), lo (nl-1, nod2D). */
int om_tracer_step(const om_mesh *m, int hor, int ver, int lim, double ph,
                   double pv, double dt, const double *uv, const double *w,
                   double *values, const double *valuesAB, double *del_h,
                   double *del_v, double *lo);

/* Advance ntracers tracers nsteps steps.  values / valuesAB hold ntracers
 * consecutive (nl-1, nod2D) arrays.  refresh_ab = 1 sets valuesAB := values
 * before every step; 0 keeps valuesAB frozen like the analytic driver. */
int om_run(const om_mesh *m, int hor, int ver, int lim, double ph, double pv,
           double dt, const double *uv, const double *w, int ntracers,
           int nsteps, double *values, double *valuesAB, int refresh_ab);

/* min, max, sum(dble()) and NaN count over values(:, 1:nod2D)
 * (src/fesom_analytic.F90:441-446). */
void om_stats(const om_mesh *m, const double *values, double *out4);

/* Seeded synthetic inputs of the benchmark workloads (the same functions of
 * the same seeds as the library's generators, restated so that the CPU
 * baseline does not load the product): a smooth bottom-level field K (per
 * analytic grid node, uniform marginal on [3, nl]); a layered flow uv
 * (2, nl-1, elem2D) and w (nl, nod2D) that is discretely divergence-free;
 * tracer fields (nl-1, nod2D): kind 0 temperature-like U[0,20] + blobs,
 * kind 1 salinity-like 35 + N(0, 0.5). */
void om_synth_bathymetry_smooth(int nx, int ny, int periodic, int nl, double corr_cells,
                                unsigned long long seed, int *K);
void om_synth_velocity(const om_mesh *m, unsigned long long seed, double umax, double mode1_frac,
                       double mode2_frac, double baro_frac, double *uv, double *w);
void om_synth_tracer(const om_mesh *m, unsigned long long seed, int kind, double *T);

/* Threads used by the OpenMP build (no-op in the serial build). */
void om_set_threads(int n);
int om_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
