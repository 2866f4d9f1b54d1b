/*
 * asohf_gpu.h -- C ABI of libasohf_gpu.so, the B200 (sm_100a) implementation
 * of the ASOHF particle hot path.
 *
 * Each entry point replaces one subroutine of the reference Fortran driver
 * (dvallesp/ASOHF) and keeps its argument meaning; the Fortran side binds
 * them with ISO_C_BINDING (fortran/asohf_gpu_mod.f90).  All calls:
 *   - return 0 on success or an ASOHF_ERR_* status (asohf_types.h), the
 *     reference's `STOP 1` exits; asohf_strerror() gives the message;
 *   - run on the context's CUDA stream and return once their results are in
 *     the output arrays (host outputs) or enqueued (device outputs);
 *   - never fall back to the CPU: without a usable device they return
 *     ASOHF_ERR_NO_DEVICE.
 * `on_device` = 0: array arguments are host pointers (the library stages
 * them); 1: they are device pointers of the context's device.
 * A context is not re-entrant: one host thread drives it at a time.
 */
#ifndef ASOHF_GPU_H
#define ASOHF_GPU_H

#include <stdint.h>
#include "asohf_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct asohf_ctx asohf_ctx;

/* Status text (for the Fortran shim's `WRITE(*,*)` before `STOP 1`). */
const char *asohf_strerror(int code);
/* Detail of the last CUDA failure seen by the library in this process. */
const char *asohf_last_error_detail(void);

/* Context: device, stream, device particle store and scratch arena. */
int asohf_create(int device, asohf_ctx **out);
int asohf_destroy(asohf_ctx *ctx);
/* The stream the context's kernels run on.  The size tiers of the per-halo
   kernels run on side streams created at this stream's priority; the
   deferred patch deposit (asohf_set_density_overlap) runs at the least
   priority, so a caller that runs the hot path on a high-priority stream
   lets the deposit fill the gaps the halo finder leaves. */
int asohf_set_stream(asohf_ctx *ctx, void *cuda_stream);
int asohf_synchronize(asohf_ctx *ctx);
/* Number of kernels this context has launched (diagnostics). */
int64_t asohf_launch_count(asohf_ctx *ctx);
/* Diagnostics, no counterpart in the reference: with profiling on, the main
 * kernels are bracketed by CUDA events on the context stream; stats entry i
 * gives a kernel's name, summed device time (ms) and launch count since
 * profiling was (re)enabled. */
int asohf_set_profiling(asohf_ctx *ctx, int on);
int asohf_kernel_stats(asohf_ctx *ctx, int i, const char **name, double *total_ms,
                       int64_t *launches);
/* Diagnostics, no counterpart in the reference: 8 work counters (entry 0:
 * element-passes of the halo kernel, 1: of the subhalo kernel), optionally
 * reset after reading. */
int asohf_work_counters(asohf_ctx *ctx, int64_t *out8, int reset);
/* Host I/O, no counterpart in the reference: enqueues on `cuda_stream`
 * (the context stream when NULL) a copy of `bytes` bytes from device memory
 * of this context's GPU to page-locked host memory, made by SM stores
 * rather than a copy engine so that it overlaps the context's own host
 * copies.  Both pointers and bytes must be multiples of 16 and host_dst must
 * hold `bytes` bytes; the copy is complete when the stream reaches it. */
int asohf_copy_to_host_sm(asohf_ctx *ctx, void *host_dst, const void *dev_src, int64_t bytes,
                          void *cuda_stream);
/* Host I/O, no counterpart in the reference: copies `bytes` bytes from
 * device memory of this context's GPU to page-locked host memory on a copy
 * engine, after the work the context has issued so far (a deferred patch
 * deposit included), and returns at once.  A helper thread issues the copy
 * in chunks, one at a time: the copy engine serves copies in the order they
 * were queued, so the short copies the context makes meanwhile wait for one
 * chunk at most.  asohf_copy_wait makes cuda_stream (the host, when NULL)
 * wait for every such copy issued so far. */
int asohf_copy_to_host_async(asohf_ctx *ctx, void *host_dst, const void *dev_src, int64_t bytes);
int asohf_copy_wait(asohf_ctx *ctx, void *cuda_stream);
/* Tuning, no counterpart in the reference: with on = 1, asohf_density
 * called with device outputs returns before its AMR-patch deposit is done:
 * that work runs on a stream of the context's own (at the least priority),
 * from buffers no other call reuses, beside whatever the caller issues next
 * (the x-slab sort and the halo finder do not read U11), and
 * asohf_renorm_density's patch scaling follows it there.  U11 is complete
 * once asohf_density_wait has made a stream wait for it, or after
 * asohf_synchronize.  U1 is complete on return as before. */
int asohf_set_density_overlap(asohf_ctx *ctx, int on);
/* Makes cuda_stream wait (device side) for a deferred patch deposit. */
int asohf_density_wait(asohf_ctx *ctx, void *cuda_stream);
/* Seed of COMPUTE_EPOT's sampling estimator (haloes_particles.f:1568-1626),
 * used for bound lists of MAX_PART_DSUM entries or more when energies are
 * on.  The reference draws its particle pairs from RANDOM_NUMBER after an
 * unseeded RANDOM_SEED(), so its estimate changes from run to run; here the
 * draws come from a counter-based generator keyed by (seed, catalogue row,
 * draw), so a run is reproducible and equals the oracle's bit for bit.
 * Default 1. */
int asohf_set_epot_seed(asohf_ctx *ctx, uint32_t seed);
/* Tuning, no counterpart in the reference: haloes with at least
 * min_members members are refined by a thread-block cluster, the others by
 * one CTA each (results are the same either way).  0 restores the default
 * (32768); 1 sends every halo to the cluster path. */
int asohf_set_cluster_threshold(asohf_ctx *ctx, int64_t min_members);
/* Tuning, no counterpart in the reference: the halo kernel gives a
 * cluster-tier halo 16 CTAs above 8 x members_per_cta members, 8 above
 * 4 x, else 4 (results are the same for every width).  0 restores the
 * default (32768). */
int asohf_set_cluster_share(asohf_ctx *ctx, int64_t members_per_cta);
/* Tuning, no counterpart in the reference: haloes below the cluster
 * threshold are refined by one CTA of 256 threads from tier2_members
 * members, of 128 threads from tier1_members, else of 32 threads; a halo
 * whose growth sphere outgrows its CTA moves to a larger one.  0 restores
 * a default (256, 2048). */
int asohf_set_group_tiers(asohf_ctx *ctx, int64_t tier1_members, int64_t tier2_members);

/* MODULE PARTICLES (particles.f:1-14) / READ_AND_ALLOC_PARTICLES
 * (alloc.f:196-528): copies the particle arrays into the device store,
 * which stays resident across calls.  Download copies the store back (in
 * its current order: the sorts below permute it in place, as the Fortran
 * permutes RXPA.., ORIPA). */
int asohf_upload_particles(asohf_ctx *ctx, const asohf_particles *src, int on_device);
int asohf_download_particles(asohf_ctx *ctx, asohf_particles *dst, int on_device);
/* Tuning, no counterpart in the reference: starts copying the host arrays
 * of a coming asohf_upload_particles (page-locked, for the copy to overlap)
 * on a copy stream of the context's own into a staging store, while the
 * context stream runs what was issued before.  The next upload of exactly
 * these arrays (same pointers and count, on_device = 0) takes the staged
 * store: the context stream waits for the copy instead of copying again.
 * The arrays must not change until that upload. */
int asohf_prefetch_particles(asohf_ctx *ctx, const asohf_particles *src);

/* SORT_DM_PARTICLES_LOCALDENSITY (reader.f:140-336): NGP density on the
 * NX^3 grid, species INT(LOG(rho)/LOG(8)) in [0, N_ESP-1], stable sort of
 * the store by species.  npart_esp: host array of N_ESP counts (out). */
int asohf_sort_dm_particles_localdensity(asohf_ctx *ctx, int nx, float dx, float rodo,
                                         float re0, int32_t *npart_esp);

/* DENSITY (grids.f:710-994) with COMPUTE_KERNELS (grids.f:997-1067): kernel
 * deposit of the store (species-sorted, counts npart_esp) onto the periodic
 * base grid u1 (NX^3, column-major) and the patches u11 (32^3 per patch,
 * sum(mesh->npatch) patches). */
int asohf_density(asohf_ctx *ctx, int nx, float lado0, float dx, float rote, float rete,
                  const int32_t *npart_esp, const asohf_mesh *mesh, int interp_degree,
                  float *u1, float *u11, int on_device);

/* RENORM_DENSITY (grids.f:2668-2722): u1, u11 /= fdm in place. */
int asohf_renorm_density(asohf_ctx *ctx, int nx, const asohf_mesh *mesh, float fdm,
                         float *u1, float *u11, int on_device);

/* INTERPOLATE_DENSITY_TSC (grids.f:1070-1398): true TSC deposit of the store
 * onto u1 and u11.  radx: host array RADX(0:NX+1) from MALLA. */
int asohf_interpolate_density_tsc(asohf_ctx *ctx, int nx, float lado0, float dx,
                                  const float *radx, float rote, float rete,
                                  const asohf_mesh *mesh, float *u1, float *u11, int on_device);

/* MOMENTO + POFFT3D (poisson.f:98-249): periodic potential of `batch`
 * fields rho (NX^3 each) into pot.  Green's function -(DX/2)^2/sum sin^2,
 * zero mode from the 1e30 denominator.  Each field is solved on its own
 * (no rounding of one reaches another); results equal an FFT solve within
 * float32 rounding. */
int asohf_poisson_fft(asohf_ctx *ctx, int nx, float dx, int batch, const float *rho,
                      float *pot, int on_device);

/* Deposit + Poisson for `batch` particle sets of n_per particles each
 * (device arrays of batch*n_per): base-grid TSC of INTERPOLATE_DENSITY_TSC
 * (grids.f:1163-1239, periodic) scaled by 1/(DX^3 ROTE RETE^3), then the
 * FFT solve; rho and pot receive batch*NX^3 values.  No counterpart routine
 * in the reference: it chains the two routines POISSON calls
 * (poisson.f:41-51) for the differentiable layer. */
int asohf_tsc_poisson_forward(asohf_ctx *ctx, int nx, float lado0, float dx, const float *radx,
                              float rote, float rete, int batch, int64_t n_per,
                              const float *x, const float *y, const float *z, const float *m,
                              float *rho, float *pot);
/* Adjoint of asohf_tsc_poisson_forward: given w = dL/dpot (batch*NX^3),
 * writes dL/dx, dL/dy, dL/dz (batch*n_per) and, if grad_m is not NULL,
 * dL/dm.  The Green's multiply is self-adjoint; the deposit's adjoint is a
 * TSC gather of the gradient of G*w. */
int asohf_tsc_poisson_adjoint(asohf_ctx *ctx, int nx, float lado0, float dx, const float *radx,
                              float rote, float rete, int batch, int64_t n_per,
                              const float *x, const float *y, const float *z, const float *m,
                              const float *w, float *grad_x, float *grad_y, float *grad_z,
                              float *grad_m);

/* SORT_DM_PARTICLES_X (grids.f:2726-2838): ARGSORT of x with its tie rule
 * (num.f:150-203), store permuted, slab table NDMPART_X(0:NX) written to
 * the host array ndmpart_x (nx+1 entries).  Also builds the (y,z) column
 * index the per-halo queries use. */
int asohf_sort_dm_particles_x(asohf_ctx *ctx, int nx, float lado0, int32_t *ndmpart_x);

/* PRUNE_POOR_HALOES (haloes_particles.f:185-256) over haloes low1..low2
 * (Fortran 1-based, inclusive). */
int asohf_prune_poor_haloes(asohf_ctx *ctx, const asohf_consts *k, asohf_catalogue *cat,
                            int low1, int low2, float facrad, int do_need_to_count,
                            int on_device);

/* CREATE_MESH particle counts of the base grid (grids.f:107-143), on the
 * uploaded store in species order: cr0[(kz*nx + jy)*nx + ix] (IX fastest,
 * nx^3 int32) = particles of species 0 plus refine_thr per particle of a
 * heavier species in each cell, IX = INT((x - XL)/DX)+1 clamped to 1..nx
 * with XL = -nx*dx/2, then zero within bor cells of the faces.  The species
 * of store index i is the range of npart_esp (N_ESP counts) holding it, 0
 * past the last.  The greedy patch placement that reads CR0 stays with the
 * caller. */
int asohf_mesh_base_counts(asohf_ctx *ctx, int nx, float dx, int refine_thr, int bor, const int32_t *npart_esp,
                           int32_t *cr0, int on_device);
/* CREATE_MESH particle counts on the npatch patches of level irpa
 * (grids.f:341-380): per patch NAMRX^3 int32 (IX fastest), IX =
 * FLOOR((x - XL)/DXPA)+1 kept when 1 <= IX <= PATCHNX, XL = PATCHRX - DXPA,
 * DXPA = dx/2^irpa; 1 per particle of species <= irpa, refine_thr otherwise;
 * zero within boramr cells of the patch faces and outside the patch.
 * patchnx..patchrz: host arrays of the level's patches (the slice
 * LOW1..LOW2 of the reference's patch table); nx, lado0 size the particle
 * bins. */
int asohf_mesh_patch_counts(asohf_ctx *ctx, int nx, float lado0, float dx, int irpa, int refine_thr, int boramr,
                            const int32_t *npart_esp, int npatch, const int32_t *patchnx, const int32_t *patchny,
                            const int32_t *patchnz, const float *patchrx, const float *patchry,
                            const float *patchrz, int32_t *cr01, int on_device);

/* VEINSGRID_REDUCED (grids.f:1771-2073), called by CREATE_MESH after the
 * patch counts of level ir: on the npatch patches of the level (host arrays,
 * the slice LOW1..LOW2), patch I in order marks every cell of each
 * neighbour J (intersecting cell boxes on the level's grid, origin RADX(1) -
 * DX/2 + DXPA/2 with radx1 = RADX(1)) that faces an unmarked cell of I,
 * when the overlap covers more than 0.1 of J, and zeroes CR01 and CONTA11
 * there (NAMRX^3 int32 per patch, IX fastest; conta11 may be NULL).  The
 * sequential order is reproduced exactly.  ASOHF_ERR_CAPACITY when a patch
 * has more than max_neighbours neighbours (NPALEV2; the reference stops).
 * Cells outside the NAMRX^3 arrays are skipped. */
int asohf_veinsgrid_reduced(asohf_ctx *ctx, int ir, float dx, float radx1, int npatch, const int32_t *patchnx,
                            const int32_t *patchny, const int32_t *patchnz, const float *patchrx,
                            const float *patchry, const float *patchrz, int max_neighbours, int32_t *cr01,
                            int32_t *conta11, int on_device);

/* CHECK_RUBISH (haloes_particles.f:259-318), called after each level's
 * refinement (asohf.f:672-673): a halo of the window low1..low2 (1-based,
 * inclusive) is removed (REALCLUS=0) when a live halo of a lower level lies
 * within 1.01 times the smaller radius, with mass ratio above 0.2 and
 * relative speed difference below 3.  Requires levels that never decrease
 * with the catalogue index (the driver's order; ASOHF_ERR_INVALID
 * otherwise).  A zero speed leaves the Fortran's speed ratio at the
 * previous pair's value; when that alone would decide a removal the call
 * returns ASOHF_ERR_UNSUPPORTED.  *removed (may be NULL) receives KONTA. */
int asohf_check_rubish(asohf_ctx *ctx, asohf_catalogue *cat, int nclus, int low1, int low2, int on_device,
                       int32_t *removed);
/* ACCIDENTAL_SUBSTRUCTURE (haloes_particles.f:321-364), asohf.f:674-675: a
 * confirmed halo (REALCLUS=-1) wholly inside a confirmed halo of a lower
 * level (DIS + R <= R of the other) is removed.  Same level-order
 * requirement.  *removed (may be NULL) receives KONTA. */
int asohf_accidental_substructure(asohf_ctx *ctx, asohf_catalogue *cat, int nclus, int on_device,
                                  int32_t *removed);
/* RE_SORT_HALOES (haloes_particles.f:2-56), host arrays: the entries of
 * level ir (LOWH1 = SUM(NHALLEV(0:ir-1))+1 .. LOWH2 = SUM(NHALLEV(0:ir));
 * nhallev: host array of ir+1 counts) with REALCLUS = 0 are dropped, the
 * others moved down in order (CLUSRX/Y/Z, RADIO, MASA, LEVHAL, PATCHCLUS,
 * DMPCLUS, CLUSRX/Y/ZCM; the catalogue has no HALBORDERS), and a positive
 * REALCLUS inside the window renumbered to its entry's new position (0
 * when that entry was dropped; outside the window it is kept).
 * NHALLEV(ir) and NCLUS receive the counts.  keep (may be NULL; LOWH2 -
 * LOWH1 + 1 bytes) receives 1 for the kept entries, 0 for the dropped. */
int asohf_re_sort_haloes(asohf_ctx *ctx, asohf_catalogue *cat, int32_t *nhallev, int ir, uint8_t *keep);
/* OVERLAPPING (haloes_grids.f:27-201), called by the grid finder at the end
 * of each level (haloes_grids.f:577, 1081): over the haloes 1..lowh2, with
 * the new level lowh3..lowh2 (lowh3 = SUM(NHALLEV(0:ir-1))+1, lowh2 =
 * SUM(NHALLEV(0:ir)); nhallev: host array of ir+1 counts), pass 1 removes
 * the smaller of two nested spheres, pass 2 the smaller of two spheres
 * whose lens overlap exceeds vol_solap_low of the smaller volume, with the
 * Fortran's sequential order reproduced.  The reference's mesh, SOLAP,
 * CR0AMR and density arguments are not read by the routine and are not
 * taken.  *removed (may be NULL) receives COUNT(REALCLUS(lowh3:lowh2)==0),
 * the figure the routine prints. */
int asohf_overlapping(asohf_ctx *ctx, asohf_catalogue *cat, int ir, const int32_t *nhallev,
                      float vol_solap_low, int on_device, int32_t *removed);

/* HALOFIND_GRID at the base level (haloes_grids.f:287-582): the candidate
 * peaks of u1 (NX^3 column-major; a device pointer when u1_on_device,
 * else host) above
 * CONTRASTEC/6, taken from the densest, each grown in spherical shells to
 * the contrast CONTRASTEC unless a kept halo already covers its peak; then
 * OVERLAPPING at IR = 0.  radx: host RADX(0:NX+1).  cat's arrays are
 * device pointers when cat_on_device, else host.  The catalogue is reset
 * (NCLUS = 0) and receives REALCLUS = -1, LEVHAL = 0, PATCHCLUS = 0,
 * CLUSRX..Z, RADIO, MASA and CLUSRXCM..ZCM of every halo; *nhal receives
 * NHALLEV(0).  A mesh with patches (the recentering on the AMR levels,
 * haloes_grids.f:343-360) returns ASOHF_ERR_UNSUPPORTED; a radius past
 * BOUND returns ASOHF_ERR_NOT_CONVERGED (the reference's STOP 1). */
int asohf_halofind_grid_base(asohf_ctx *ctx, int nx, float dx, const float *u1, const float *radx,
                             float contrastec, float rote, float rete, float rodo, float re0, float bound,
                             float vol_solap_low, const asohf_mesh *mesh, asohf_catalogue *cat, int u1_on_device,
                             int cat_on_device, int32_t *nhal);

/* HALOFIND_PARTICLES (haloes_particles.f:578-1411) over haloes
 * lowh1..lowh2: recentering, SO growth, radial sort, unbinding, SO walk,
 * properties and bound-particle IDs (appended to the context's
 * PARTICLES_PER_HALO stream; INDCS_PARTICLES_PER_HALO in cat). */
int asohf_halofind_particles(asohf_ctx *ctx, const asohf_consts *k, const asohf_mesh *mesh,
                             asohf_catalogue *cat, int lowh1, int lowh2, int on_device);

/* SUBSTRUCTURE_PARTICLES (substructure.f:756-1697) over the subhaloes of
 * level ir; subs_lev: host array SUBS_LEV(0:NL) (mesh->nl+1 entries). */
int asohf_substructure_particles(asohf_ctx *ctx, const asohf_consts *k, const asohf_mesh *mesh,
                                 asohf_catalogue *cat, int ir, const int32_t *subs_lev,
                                 int on_device);

/* No counterpart in the reference.  The periodic base-grid deposit of
 * DENSITY (the same cloud terms as asohf_density's u1) for callers that
 * cannot allocate device memory while they run -- an application that gives
 * all GPU memory to its own pool up front and forbids later cudaMalloc, or
 * code that must avoid the device synchronisation cudaMalloc/cudaFree can
 * cause.  It allocates nothing and needs no context: x, y, z, m (n
 * particles) and u1 (nx^3, column-major) are the caller's device pointers,
 * cuda_stream a stream of the current device (0 for the default stream;
 * another device's stream is refused with ASOHF_ERR_INVALID).  Its float64
 * scratch is a fixed file-scope device array of ASOHF_NOALLOC_MAX_CELLS
 * cells (16 MiB); grids with more cells are refused with
 * ASOHF_ERR_CAPACITY.  Under CUDA's default lazy module loading that array
 * and the two kernels are placed on a device at the first call there, not
 * at library load: the first call on each device (n = 0 is enough) does this
 * set-up and is the only one that may need device memory, so make it before
 * the application reserves its device memory and before any stream capture.
 * The array then stays on that device until the process exits.  Every call
 * shares the array and clears the part it uses: calls that overlap on the
 * GPU (other streams, other host threads) race.  Without a usable device it
 * returns ASOHF_ERR_NO_DEVICE. */
#define ASOHF_NOALLOC_MAX_CELLS (128 * 128 * 128)
int asohf_density_base_noalloc(int nx, float lado0, float dx, float rote, float rete,
                               int interp_degree, int64_t n, const float *x, const float *y,
                               const float *z, const float *m, float *u1, void *cuda_stream);

/* PARTICLES_PER_HALO (particles.f:12): copies the ID stream (host out);
 * *n receives its length (the largest INDCS_PARTICLES_PER_HALO(2,.)). */
int asohf_get_particles_per_halo(asohf_ctx *ctx, int32_t *out, int64_t cap, int64_t *n,
                                 int on_device);

#ifdef __cplusplus
}
#endif
#endif /* ASOHF_GPU_H */
