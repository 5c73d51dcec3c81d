/*
 * fesom_tracer.h -- C ABI of libfesom_tracer.so, the B200 (sm_100a) tracer
 * advection library.
 *
 * The first group of entry points keeps the names, argument meaning, value /
 * pointer passing and return convention (0 = success, -1 = not initialised,
 * bad id or unsupported input, message on stderr prefixed "### error:") of the
 * reference's Fortran bind(C) interface, lib/tracer_c_interface.F90 in
 * suvarchal/fesom2_tracer_dwarf; each declaration cites the function it
 * replaces.  Arrays are Fortran column-major doubles, copied in and out, never
 * aliased.  One global instance, not thread-safe, as in the reference.
 *
 * Behaviour that differs from the reference on purpose (reference bugs):
 *  - tracer_advect_step advances every allocated tracer (the reference
 *    advanced tracer 1 only, lib/tracer_c_interface.F90:188-190,210) and
 *    zeroes the tendency each step (the reference accumulated del_ttf,
 *    :177-203);
 *  - w is used as w, w_i and w_e (use_wsplit = .false.); the reference's
 *    array path left w_e zero and sized by edges (:711-712);
 *  - tracer_set_velocity reads uv as (nl-1, n, 2) with n the number of
 *    ELEMENTS, the mesh entity velocity lives on; the reference allocated it
 *    by edges and the kernels then read it as (2, nl-1, elem) (:694-725).
 * Restart files (tracer_init, tracer_finalize, tracer_run_workflow,
 * tracer_load_mesh_partition) use the reference's derived-type binary
 * format (lib/io_restart_derivedtype.F90:33-199) for one process:
 * <dir>/np1/t_mesh.0, t_partit.0, t_tracer.0, t_dynamics.0 and
 * <dir>/meta.time.  Meshes also come from tracer_init_analytic,
 * tracer_set_mesh_arrays or the ASCII mesh files
 * (tracer_load_mesh_from_files, one process, no partition files).
 */
#ifndef FESOM_TRACER_H
#define FESOM_TRACER_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- reference interface (lib/tracer_c_interface.F90) ------------------ */

/* :46 tracer_init_mpi -- no MPI in a one-GPU build; always 0. */
int tracer_init_mpi(int mpi_comm);
/* :89 tracer_finalize_mpi -- always 0. */
int tracer_finalize_mpi(void);
/* :113 tracer_init -- mesh, tracers (values, valuesAB, schemes) and flow
 * (uv, w) from the restart in restart_dir/np1; valuesAB is kept as read
 * (not refreshed per step), as in the reference's drivers.  -1 with a
 * message naming the file and field when a record does not parse, the
 * partition is not one process's, or ulevels /= 1. */
int tracer_init(const char *restart_dir);
/* :163 tracer_advect_step -- one step of every tracer. */
int tracer_advect_step(double dt);
/* :228 tracer_get_stats -- min, max, sum of tracer 1 over (nl-1, nod2D). */
int tracer_get_stats(double *tmin, double *tmax, double *tsum);
/* :255 tracer_get_size -- nz = nl-1, nn = nod2D. */
int tracer_get_size(int *nz, int *nn);
/* :280 tracer_get_values -- tracer 1 into values(nz, nn). */
int tracer_get_values(double *values, int nz, int nn);
/* :308 tracer_finalize -- writes the restart of the current state into
 * output_dir/np1 and output_dir/meta.time; the state is then no longer
 * initialised (as in the reference). */
int tracer_finalize(const char *output_dir);
/* :356 tracer_run_workflow -- tracer_init, nsteps steps each followed by
 * tracer_get_stats (printed), tracer_finalize into the same directory. */
int tracer_run_workflow(const char *restart_dir, int nsteps, double dt);
/* :391 tracer_cleanup -- releases every host and device resource. */
int tracer_cleanup(void);
/* :415 tracer_set_mesh_dims */
int tracer_set_mesh_dims(int nl, int nod2D, int edge2D, int elem2D);
/* :441 tracer_set_levels -- nlevels_nod2D and ulevels_nod2D (ulevels must be 1). */
int tracer_set_levels(const int *nlevels, const int *ulevels, int nod2D);
/* :477 tracer_set_thickness -- hnode_new(nl-1, nod2D). */
int tracer_set_thickness(const double *hnode, int nl, int nod2D);
/* :510 tracer_set_partition -- one GPU: eDim_nod2D must be 0. */
int tracer_set_partition(int myDim_nod2D, int eDim_nod2D);
/* :539 tracer_allocate_tracers -- defaults UPW1/UPW1/NONE, ph = pv = 1. */
int tracer_allocate_tracers(int num_tracers, int nl, int nod2D, int AB_order);
/* :613 tracer_set_values -- values, valuesAB (and valuesold) of one tracer. */
int tracer_set_values(int tracer_id, const double *values, int nl, int nod2D);
/* :652 tracer_set_velocity_zero */
int tracer_set_velocity_zero(int nl, int nod2D, int edge2D);
/* :694 tracer_set_velocity -- uv(nl-1, elem2D, 2), w(nl, nod2D). */
int tracer_set_velocity(const double *uv, const double *w, int nl, int nod2D, int nelem);
/* :749 tracer_init_complete */
int tracer_init_complete(void);
/* :769 tracer_load_mesh_partition -- mesh and flow from a restart directory
 * (its tracer record, when present, supplies only the MUSCL tables). */
int tracer_load_mesh_partition(const char *restart_dir);
/* :830 tracer_load_mesh_from_files -- reads the mesh directory's nod2d.out,
 * elem2d.out, aux3d.out, edgenum.out, edges.out, edge_tri.out, elvls.out and
 * nlvls.out as mesh_setup does (lib/oce_mesh.F90:49-94), on one process
 * (the reference reads them through its dist_<npes> partition lists), with
 * the reference's conventions: rotation by the Euler angles (50, 15, -90)
 * given to cos/sin as they are (lib/gen_modules_rotate_grid.F90:42-44) and
 * cyclic_length = 360 against coordinates in radians, which leaves elements
 * that straddle the longitude seam with their unwrapped (oversized) geometry
 * exactly as the reference computes it.  Layer thicknesses are those of
 * tracer_init_ale_arrays.  -1 with a message on a missing or malformed file. */
int tracer_load_mesh_from_files(const char *mesh_path);
/* :875 tracer_init_ale_arrays -- hnode = hnode_new = zbar(k)-zbar(k+1). */
int tracer_init_ale_arrays(void);
/* :931 tracer_init_for_advection -- allocates the device state. */
int tracer_init_for_advection(void);

/* ---- additive extensions ------------------------------------------------ */

/* tracer_load_mesh_from_files with explicit conventions: rotate (0/1), Euler
 * angles alpha, beta, gamma multiplied by angle_scale before cos/sin, and the
 * cyclic length in radians of longitude.  (1, 50, 15, -90, 1, 360) is the
 * reference's behaviour; (1, 50, 15, -90, pi/180, 2 pi) gives FESOM2's
 * (angles in degrees, longitude wrapped at the seam). */
int tracer_load_mesh_from_files_opts(const char *mesh_path, int rotate, double alpha, double beta, double gamma,
                                     double angle_scale, double cyclic_length);

/* Analytic mesh of lib/analytic_mesh.F90:114 (generate_analytic_mesh) with
 * the ALE arrays of src/fesom_analytic.F90:206-244.  node_K (nullable,
 * length nod2D) is a per-node bottom level index in [3, nl].  options bit 0:
 * 1 rebuilds the periodic nod_in_elem2D lists after the halo remap, 0 keeps
 * the reference's incomplete ones.  options bit 1: reverse the horizontal and
 * vertical edges so that edge_tri(1) lies left of edges(1)->edges(2) on every
 * edge (the reference mesh has it on the right of those edges and on the left
 * of the diagonals, so its fluxes across them point against the flow). */
int tracer_init_analytic(int nx, int ny, int nl, double Lx, double Ly, double max_depth,
                         int periodic, int options, const int *node_K);
/* Number of nodes of the analytic mesh (nx, ny, periodic). */
int tracer_analytic_nodes(int nx, int ny, int periodic);
/* Generic mesh from arrays (1-based Fortran indices, 0 = no element):
 * elem2D_nodes(3, elem2D), edges(2, edge2D), edge_tri(2, edge2D),
 * nlevels(elem2D), nlevels_nod2D(nod2D), nod_in_elem2D given by
 * ring_num(nod2D) and ring(max_ring, nod2D), elem_area(elem2D),
 * area(nl, nod2D), areasvol(nl, nod2D), edge_dxdy(2, edge2D),
 * edge_cross_dxdy(4, edge2D), gradient_sca(6, elem2D), elem_cos(elem2D),
 * zbar(nl), hnode(nl-1, nod2D), hnode_new(nl-1, nod2D), helem(nl-1, elem2D),
 * coord_nod2D(2, nod2D) (radians).  Up/down-wind triangles, nboundary_lay and
 * the edge tables are derived.  Lx, Ly > 0 mark a doubly periodic domain. */
int tracer_set_mesh_arrays(int nl, int nod2D, int elem2D, int edge2D, int max_ring,
                           const int *elem2D_nodes, const int *edges, const int *edge_tri,
                           const int *nlevels, const int *nlevels_nod2D, const int *ring_num,
                           const int *ring, const double *elem_area, const double *area,
                           const double *areasvol, const double *edge_dxdy,
                           const double *edge_cross_dxdy, const double *gradient_sca,
                           const double *elem_cos, const double *zbar, const double *hnode,
                           const double *hnode_new, const double *helem,
                           const double *coord_nod2D, double Lx, double Ly);
/* Per-tracer schemes, as the strings of lib/MOD_TRACER.F90:18-20:
 * hor "UPW1"|"MUSCL"|"MFCT", ver "UPW1"|"PPM"|"QR4C"|"CDIFF", lim "NONE"|"FCT". */
int tracer_set_scheme(int tracer_id, const char *hor, const char *ver, const char *lim,
                      double ph, double pv);
/* Element velocity in the kernels' own layout uv(2, nl-1, elem2D), w(nl, nod2D). */
int tracer_set_velocity_elem(const double *uv, const double *w, int nl, int nod2D, int elem2D);
/* valuesAB of one tracer (the field the high-order fluxes are built from). */
int tracer_set_values_ab(int tracer_id, const double *values, int nl, int nod2D);
/* 1: valuesAB := values before every step; 0 (default, as the reference
 * drivers): valuesAB stays as set. */
int tracer_set_ab_refresh(int on);
/* Arithmetic mode of the device state: 0 FP64 (default, bit-identical to the
 * reference algorithm), 1 FP32, 2 BF16 tracer storage with FP32 arithmetic, 3
 * FP16 tracer storage with FP32 arithmetic, 4 FP64 with the kernels built
 * with FMA contraction (each a*b+c the compiler fuses rounds once: results
 * within about 1e-13 relative of mode 0, fewer FP64 instructions); in modes
 * 1-3 the FCT ratio denominators are formed in FP64.  Changing it rebuilds
 * the device state and keeps the tracer values. */
int tracer_set_precision(int mode);
/* Rounding of new tracer values into 16-bit storage (modes 2, 3):
 * 0 = to nearest (default), 1 = stochastic (round up with probability equal
 * to the distance from the lower neighbour over the spacing; a reproducible
 * counter-based stream per tracer, step and cell).  16-bit storage holds
 * T - off on wet cells, off = the FP32-rounded wet-cell mean of the tracer's
 * latest full upload (tracer_set_values); tracer_storage_offset returns it
 * (0 in modes 0, 1). */
int tracer_set_rounding(int mode);
/* Step kernels (no counterpart in the reference): 1 (default) = the
 * five-kernel path (gradients, edges, LO solution, FCT ratios, update) with
 * the intermediates in device memory; 0 = one fused kernel per tracer, a
 * thread block per mesh patch that keeps the patch and three halo rings on
 * chip and writes only the new values, wherever the scheme allows it (FP64
 * or FP32 modes, PPM or UPW1 vertical, no learned flux) -- it moves about a
 * third of the DRAM bytes but runs slower on B200 (one 12-warp block per SM,
 * five block barriers per level).  Both paths give bit-identical FP64
 * results.  tracer_step_info reports out4[0] = the path,
 * out4[1] = 1 when tracer 1 runs the fused kernel, out4[2] = patches of the
 * fused kernel's plan, out4[3] = the plan's LO-solution nodes per mesh node
 * (its halo redundancy). */
int tracer_set_step_path(int path);
int tracer_step_info(double *out4);
/* Owned nodes per patch of the fused kernel's plan (0 = the default, 225);
 * every size gives the same results, small ones recompute more halo. */
int tracer_set_patch_size(int owned);
/* Most wet cells per thread block of the five-kernel path's schedules (0 =
 * the default, 512; 32..576); every size gives the same results. */
int tracer_set_cells_per_block(int cells);
/* Failure detection (no counterpart in the reference): the update kernels
 * count, on the device, every new tracer value that is not finite.
 * tracer_step_status returns that count since its last call (and resets
 * it); with tracer_set_nan_check(1), tracer_advect_step / _steps return -1
 * with a message when the steps of the call produced any. */
int tracer_set_nan_check(int on);
/* One step with host I/O (no counterpart in the reference): values_in[t]
 * (nullable) becomes tracer t+1's values (and valuesAB), every tracer is
 * advanced once, values_out[t] (nullable) receives its new values; arrays
 * (nl-1, nod2D).  When every array is page-locked (tracer_host_register)
 * and the storage is FP64 or FP32, the uploads, the per-tracer steps and the
 * downloads are pipelined on three streams (tracer t+1 uploads and tracer
 * t-1 downloads while tracer t steps); otherwise the same operations run one
 * after the other.  ntracers must equal the allocated tracers.  FP64 results
 * are those of tracer_set_values + tracer_advect_step + tracer_get_values bit
 * for bit; in FP32 the pipelined form steps each tracer alone where
 * tracer_advect_step batches up to four, and the FP32 kernels of different
 * batch sizes may contract different multiply-adds (an ulp or so). */
int tracer_advect_step_io(double dt, const double *const *values_in, double *const *values_out, int ntracers);
int tracer_step_status(long long *nonfinite);
/* Builds the fused kernel's patch plan for the loaded mesh on the host (no
 * device needed) with patches of about max_owned owned nodes, checks it
 * against the mesh (every node owned once, three halo rings, incidence lists
 * in ascending edge id, up/down triangles, rings) and returns out8 =
 * {patches, smallest owned count, largest N2 and N3 region, largest edge and
 * element counts, LO-solution nodes per mesh node, edges per mesh edge};
 * -1 with a message when a check fails. */
int tracer_tile_plan_check(int max_owned, double *out8);
/* Page-lock a host range (cudaHostRegister) so that tracer_set_values*,
 * tracer_get_values* and tracer_advect_* transfers from / to arrays inside it
 * take one DMA each way instead of going through the library's pinned
 * staging ring.  Register once, before the time loop; unregister before
 * freeing the memory.  No counterpart in the reference (whose host arrays are
 * Fortran-owned and never cross a PCIe bus). */
int tracer_host_register(void *ptr, long long bytes);
int tracer_host_unregister(void *ptr);
int tracer_storage_offset(int tracer_id, double *off);
/* Compensated FP64 sums over the wet cells of one tracer, on the device:
 * out2[0] = Sum T, out2[1] = Sum T*areasvol*hnode_new (conserved content). */
int tracer_volume_sum(int tracer_id, double *out2);
/* nsteps steps of every tracer. */
int tracer_advect_steps(int nsteps, double dt);
/* Values / stats of tracer tracer_id (1-based). stats4 = min, max, sum, nan. */
int tracer_get_values_id(int tracer_id, double *values, int nz, int nn);
int tracer_get_stats_id(int tracer_id, double *stats4);
/* Fields of the analytic driver for the current analytic mesh:
 * T, S (nl-1, nod2D), uv (2, nl-1, elem2D), w (nl, nod2D); any may be NULL. */
int tracer_analytic_fields(double *T, double *S, double *uv, double *w);
/* Seeded synthetic inputs: bathymetry K(nnodes) in [3, nl]; a layered flow
 * for the current mesh (two zero-column-mean vertical modes weighted by
 * mode1_frac and mode2_frac, plus baro_frac times a depth-independent
 * non-divergent part, which needs a left-oriented mesh; w from the discrete
 * continuity; |u| scaled to umax, or multiplied by -umax when umax < 0); a
 * tracer field (kind 0 temperature-like, 1 salinity-like, 2 smooth blobs and
 * fronts that do not depend on the resolution). */
int tracer_synth_bathymetry(int nnodes, int nl, uint64_t seed, int *K);
int tracer_synth_velocity(uint64_t seed, double umax, double mode1_frac, double mode2_frac, double baro_frac,
                          double *uv, double *w);
/* Smooth seeded bathymetry of the analytic grid (tracer_analytic_nodes
 * entries): a random field of correlation length ~corr_cells cells with a
 * uniform marginal on [3, nl]. */
int tracer_synth_bathymetry_smooth(int nx, int ny, int periodic, int nl, double corr_cells, uint64_t seed, int *K);
int tracer_synth_tracer(uint64_t seed, int kind, double *values);
/* Mesh sizes: nl, nod2D, elem2D, edge2D, wet cells (low 31 bits), level stride. */
int tracer_mesh_dims(int *dims6);
/* Copy a named mesh array out in the reference's layout (1-based indices):
 * int: "elem2D_nodes", "edges", "edge_tri", "nlevels", "nlevels_nod2D",
 * "nlevels_nod2D_min", "edge_up_dn_tri", "nboundary_lay", "ring_num";
 * double: "coord", "elem_area", "area", "areasvol", "edge_dxdy",
 * "edge_cross_dxdy", "gradient_sca", "hnode", "hnode_new", "helem", "zbar". */
long tracer_mesh_len(const char *name);
int tracer_mesh_get_int(const char *name, int *out);
int tracer_mesh_get_dbl(const char *name, double *out);
/* Device time of nsteps steps of every tracer, CUDA events on the engine's
 * stream (inputs already resident). */
int tracer_time_steps(int nsteps, double dt, float *ms);
/* Per-kernel device time over nsteps steps (an event pair around every
 * launch): ms[kind] summed per kernel kind, names[kind] its name (up to
 * nkinds entries); *launches = kernel launches issued. */
int tracer_profile_steps(int nsteps, double dt, double *ms, const char **names, int nkinds, int *launches);
/* CUDA device the engine runs on (before the first step; default 0). */
int tracer_set_device(int device);
/* Number of kernel launches one tracer_advect_step issues. */
int tracer_launches_per_step(void);
/* Device memory held by the engine, in bytes. */
long long tracer_device_bytes(void);
/* Checks on the GPU that the reciprocal-based division of the FP64 kernels
 * returns the same bits as IEEE a / b for n random operand pairs;
 * *mismatches = number of differing results, example4 = (a, b, got,
 * expected) of the first one. */
int tracer_selftest_division(long long n, uint64_t seed, long long *mismatches, double *example4);
/* Checks on the GPU the stochastic rounding of 16-bit stores (fmt 0 BF16,
 * 1 FP16) on n random inputs with `draws` roundings each: *outside = results
 * that are not one of the input's two storage neighbours; *z = standardized
 * total of (rounded-up count - expected count), ~N(0, 1) when unbiased. */
int tracer_selftest_sround(int fmt, long long n, int draws, uint32_t seed, long long *outside, double *z);
/* No counterpart in the reference.  One step of tracer tracer_id (its scheme,
 * the loaded mesh and flow) on caller-owned DEVICE buffers, allocating no
 * device memory: for callers whose runtime has reserved the GPU's memory for
 * its own pool, or whose time loop must not allocate.  T_dev, TAB_dev (in) and
 * T_out_dev (out, not aliasing either) hold nod2D columns of level stride S
 * (tracer_mesh_dims()[5]) of doubles.  Work space comes from a 64 MiB
 * static device array (tracer_noalloc_scratch_bytes()) shared by every call:
 * meshes needing more are rejected with -1; calls that overlap on the GPU
 * race.  The device state must exist (tracer_init_for_advection, which also
 * commits the static array on the engine's device and looks up its address,
 * so it should come before the host reserves its memory pool and before any
 * stream capture).  The step runs on the engine's device whatever the
 * calling thread's current device, and first waits for all work already
 * queued on that device (so inputs written asynchronously by the caller are
 * complete).  Returns after the step has finished. */
int tracer_advect_device_noalloc(int tracer_id, const double *T_dev, const double *TAB_dev,
                                 double *T_out_dev, double dt);
/* Size in bytes of the static work array of tracer_advect_device_noalloc. */
long long tracer_noalloc_scratch_bytes(void);
/* ---- multi-member batch: no counterpart in the reference -----------------
 * Many tracers of many ensemble members, each on its own analytic mesh (any
 * sizes, periodic or closed), advanced together in FP32.  Three step paths
 * (tracer_batch_set_path): path 1 (default) runs one persistent launch per
 * phase (gradients, edge fluxes, vertical fluxes and LO solution, FCT ratios,
 * limiting and update) and wave of tracer batches over every member's work;
 * path 0 runs the whole step as one persistent cooperative launch with
 * grid-wide barriers between the phases (bounded waits: a timed-out barrier
 * makes the step return -1); path 2 runs the members' own launches.
 * tracer_batch_steps with use_graph = 1 replays the launches from a CUDA
 * graph.  The three paths give the same bits.  Members are
 * numbered from 0, tracers from 1.  Supported schemes: MUSCL+PPM or
 * UPW1+UPW1, with or without FCT, one scheme for all tracers. */
int tracer_batch_create(void);
int tracer_batch_destroy(void);
/* Adds a member on the analytic mesh of tracer_init_analytic's arguments with
 * ntracers (a multiple of 4) tracers; returns its index or -1. */
int tracer_batch_add_member(int nx, int ny, int nl, double Lx, double Ly, double max_depth, int periodic,
                            int options, const int *node_K, int ntracers);
/* dims4 = nl, nod2D, elem2D, edge2D of a member. */
int tracer_batch_member_dims(int member, int *dims4);
/* uv (2, nl-1, elem2D), w (nl, nod2D); values (nl-1, nod2D), FP64 host arrays. */
int tracer_batch_set_velocity(int member, const double *uv, const double *w);
int tracer_batch_set_values(int member, int tracer_id, const double *values);
int tracer_batch_get_values(int member, int tracer_id, double *values);
/* One scheme for every tracer, dt[num_members], refresh_ab = 1: valuesAB :=
 * values each step.  Builds the work arrays and task table for the current
 * tile. */
int tracer_batch_configure(const char *hor, const char *ver, const char *lim, double ph, double pv, const double *dt,
                           int refresh_ab);
/* Tile: most wet cells per block (32..576), threads per block (64..256),
 * persistent blocks per SM (capped by occupancy), 4-tracer batches in flight
 * per member. */
int tracer_batch_set_tile(int cells_per_block, int threads, int blocks_per_sm, int wave);
int tracer_batch_get_tile(int *tile4);
/* Times every candidate (path and tile) on steps_per_candidate steps (the
 * tracer state is restored afterwards) and keeps the fastest; log receives
 * one line per candidate (truncated to log_capacity). */
int tracer_batch_autotune(int steps_per_candidate, char *log, int log_capacity);
/* Step path: 0 one cooperative launch per step, 1 one persistent launch per
 * phase and wave, 2 the members' own per-batch launches on their streams
 * (tracer_batch_steps_separate).  get returns the path or -1. */
int tracer_batch_set_path(int path);
int tracer_batch_get_path(void);
/* Learned antidiffusive flux (no counterpart in the reference) on every
 * member's MUSCL tracers: params as for tracer_learn_set (NULL keeps each
 * member's), on = 0/1.  While on, the batch steps on path 2 (the members'
 * own launches, which evaluate the MLP between their edge and column
 * kernels), tracer_batch_set_path(0 or 1) and tracer_batch_add_member
 * return -1, and the autotuner times path 2's tiles only. */
int tracer_batch_learn_set(const float *params, int on);
int tracer_batch_steps(int nsteps, int use_graph);
/* Device time (CUDA events) of nsteps steps of the selected path,
 * milliseconds; path 2 behaves as tracer_batch_time_separate (one more,
 * untimed step first, host time between device synchronisations). */
int tracer_batch_time_steps(int nsteps, int use_graph, double *ms);
/* The same steps as per-member launches of the four-to-five step kernels per
 * 4-tracer batch (the path tracer_advect_step takes) on the members' own
 * streams; use_graph = 1 replays them from a CUDA graph of two steps forked
 * from and joined into the batch's stream.  The timed variant runs one
 * untimed step first (nsteps + 1 in all) and returns the wall time of nsteps
 * between device synchronisations. */
int tracer_batch_steps_separate(int nsteps, int use_graph);
int tracer_batch_time_separate(int nsteps, int use_graph, double *ms);
/* info4 = members, wet cells x tracers, work-array bytes, graph captured. */
int tracer_batch_info(long long *info4);
/* Runs a grid barrier that waits for one block more than the grid holds:
 * returns 1 when the wait ran out after `limit` polls and was reported (the
 * expected outcome), 0 if it passed, -1 on a CUDA error. */
int tracer_selftest_barrier_timeout(long long limit);

/* Tensor-core self-test (tcgen05.mma, no counterpart in the reference):
 * D[128 x N] = A[128 x K] * B[N x K]^T with A, B given as BF16 bit patterns
 * (row-major) and D FP32 row-major; N, K multiples of 16 up to 256.  Returns
 * 0, -1 on a CUDA error or bad arguments, -2 if the MMA did not complete. */
int tracer_selftest_umma(int N, int K, const uint16_t *A, const uint16_t *B, float *D);

/* ---- learned antidiffusive flux: no counterpart in the reference ----------
 * Per-edge-level MLP 16 -> 64 -> 64 -> 1 with GELU, BF16 weights and
 * activations on the tensor cores (tcgen05), FP32 accumulation.  Parameters
 * are FP32, packed: W1[64][16], b1[64], W2[64][64], b2[64], w3[64], b3
 * (tracer_mlp_num_params() floats).  Features X are BF16 bit patterns [S][16]. */
int tracer_mlp_num_params(void);
/* y[S] = MLP(X) (host arrays; device buffers are allocated per call). */
int tracer_mlp_forward(const uint16_t *X, long long S, const float *params, float *y);
/* grads = d/dparams sum_s dy[s] * y(X[s]) (host arrays). */
int tracer_mlp_grads(const uint16_t *X, const float *dy, long long S, const float *params, float *grads);
/* The learned flux inside the engine (precision mode 1, FP32; MUSCL
 * tracers): set the parameters (NULL keeps them; an engine never given any
 * has the zero network, whose correction is 0) and switch it on or off.  On,
 * every MUSCL edge flux becomes HO - LO + scale * MLP(features) before the
 * vertical fluxes and the unchanged FCT limiter.  A precision change drops it. */
int tracer_learn_set(const float *params, int on);
int tracer_learn_get(float *params);
/* Gradient of the loss of the last updating tracer_learn_step, taken before
 * that step's parameter update. */
int tracer_learn_grad(float *grad);
/* One training step on tracer 1 (see Engine::learn_step): values := T_in,
 * one MUSCL+PPM step with the learned correction (fct = 0: no limiter;
 * 1: FCT, the gradient taken through the limiter's ratios R+/-; 2: FCT, the
 * limiter's factors held fixed in the gradient), *loss = volume-weighted mean
 * squared difference to T_target; update = 1 applies one Adam step of rate
 * lr.  T_in, T_target (nl-1, nod2D). */
int tracer_learn_step(const double *T_in, const double *T_target, double dt, double lr, int update, int fct,
                      double *loss);

/* ---- raw binary output for the reference's plotting scripts ---------------
 * The files of lib/mesh_output.F90:19-161 (read by visualization/plot_mesh.py
 * and plot_scalars.py).  tracer_write_mesh replaces write_mesh_for_python
 * (:19): mesh_info.txt, coord_nod2D.bin (metres), elem2D_nodes.bin (0-based),
 * zbar.bin, depth.bin (bottom of each node's column).  The scalar calls
 * replace open_scalar_output (:97), write_scalar_step (:136) and
 * close_scalar_output (:154): one FP64 (nl-1, nod2D) frame of every
 * allocated tracer per write (temperature.bin, salinity.bin, tracer3.bin, ...;
 * wp = 8, 4 or 2 after the precision mode). */
int tracer_write_mesh(const char *output_dir);
int tracer_scalar_output_open(const char *output_dir, int nsteps);
int tracer_scalar_output_write(void);
int tracer_scalar_output_close(void);

/* Last error message of this thread ("" if none). */
const char *tracer_last_error(void);

/* ---- domain decomposition ------------------------------------------------
 * Parts of the loaded mesh, each owning a set of nodes (node_part, nod2D
 * entries in [0, nparts)) and holding `rings` (>= 3) rings of halo nodes;
 * every part runs the ordinary step on its local mesh and only the halo
 * values are exchanged after a step (the reference exchanges the LO
 * solution, the FCT ratios and the new values: lib/oce_adv_tra_driver.F90:234,
 * lib/oce_adv_tra_fct.F90:383, partitioned by lib/gen_modules_partitioning.F90).
 * Owned values are bit-identical to a step of the whole mesh.  FP64 and FP32
 * modes. */
/* node -> part map (0-based) of a partition directory dist_<n> of the loaded
 * mesh: rpart.out and the owned nodes of every my_list<part>.out
 * (lib/oce_mesh.F90:150-200) */
int tracer_partition_read_dist(const char *dist_dir, int *node_part, int *nparts);
/* 1-based global ids of the nodes `from` owns in the halo of `to`, ascending;
 * returns their count (or -1) */
int tracer_partition_halo(const int *node_part, int nparts, int from, int to, int rings, int *out, int capacity);
/* owned nodes, local nodes, local elements, local edges of one part (host only) */
int tracer_partition_part_dims(const int *node_part, int nparts, int part, int rings, int *dims4);
/* host only: make part `part`'s local mesh the current mesh (for inspection
 * and host-side checks), dims4 as tracer_partition_part_dims; its 1-based
 * global node and element ids (local order) by tracer_partition_part_ids */
int tracer_partition_install_part(const int *node_part, int nparts, int part, int rings, int *dims4);
int tracer_partition_part_ids(int *nodes, int *elems);
/* engines for local_parts[0..nlocal) of the decomposition, on this process's GPU */
int tracer_dd_setup(const int *node_part, int nparts, const int *local_parts, int nlocal, int rings);
int tracer_dd_destroy(void);
/* part id, owned nodes, local nodes, local elements, local edges of local part i */
int tracer_dd_part_info(int i, int *info5);
int tracer_dd_allocate_tracers(int ntr);
int tracer_dd_set_scheme(int tracer_id, const char *hor, const char *ver, const char *lim, double ph, double pv);
/* whole-mesh arrays: uv(2, nl-1, elem2D), w(nl, nod2D), values(nl-1, nod2D) */
int tracer_dd_set_velocity(const double *uv, const double *w);
int tracer_dd_set_values(int tracer_id, const double *values);
/* writes the rows of the nodes the local parts own */
int tracer_dd_get_values(int tracer_id, double *values);
/* nsteps steps of every tracer on every local part; exchange != 0 exchanges
 * the halos between the local parts after each step */
int tracer_dd_steps(int nsteps, double dt, int refresh_ab, int exchange);
/* halo transfer of local part i with part `peer`: node count (send != 0: to
 * the peer), and packing / unpacking of one tracer as (nl-1) x n FP64 values
 * in device memory, in ascending global node order */
int tracer_dd_transfer_nodes(int i, int peer, int send);
int tracer_dd_pack(int i, int tracer_id, int peer, double *dev_out);
int tracer_dd_unpack(int i, int tracer_id, int peer, const double *dev_in);

#ifdef __cplusplus
}
#endif
#endif
