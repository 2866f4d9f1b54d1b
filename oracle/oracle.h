/*
 * oracle.h -- CPU oracle of the ASOHF particle hot path.
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, the smoke check and the CPU
 * baseline leg of bench.py, as the checker.  The product library never links
 * or calls it.  Parity status: unpinned by the reference (no Fortran compiler
 * to build it, no reference tests or fixtures); pinned instead by analytic
 * known-answer tests and by golden vectors generated from this restatement.
 */
#ifndef ASOHF_ORACLE_H
#define ASOHF_ORACLE_H

#include <stdint.h>
#include "../include/asohf_types.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_FP32 = 0, ORC_FP64 = 1 };

typedef struct orc_cosmo {
  float pi, ache, rodo, re0, cgr, rote, rete, uv, um, contrastec, omegaz;
} orc_cosmo;

void orc_malla(int nx, float lado0, float *radx, float *dx_out);
void orc_cosmology(float hubble_h, float omega0, float zeta, orc_cosmo *c);
void orc_compute_kernels(int nl, int interp_degree, float *kernels);
void orc_density(int nx, float lado0, float dx, float rote, float rete,
                 const float *x, const float *y, const float *z,
                 const float *m, const int32_t *npart_esp,
                 const asohf_mesh *mesh, int interp_degree, int mode,
                 float *u1, float *u11);
void orc_renorm_density(int nx, const asohf_mesh *mesh, float fdm, float *u1, float *u11);
int orc_species_sort(int64_t n, float *x, float *y, float *z, float *vx,
                     float *vy, float *vz, float *m, int32_t *id, int nx,
                     float dx, float rodo, float re0, int32_t *npart_esp,
                     int32_t *species_out);
void orc_permute(int64_t n, const int64_t *idx, float *x, float *y, float *z,
                 float *vx, float *vy, float *vz, float *m, int32_t *id);
void orc_tsc_deposit(int nx, float lado0, float dx, const float *radx, float rote,
                     float rete, int64_t n, const float *x, const float *y,
                     const float *z, const float *m, const asohf_mesh *mesh,
                     int mode, float *u1, float *u11);
void orc_momento(int nx, float dx, float *kkk);
/* CREATE_MESH particle counts (grids.f:94-143, grids.f:341-380). */
void orc_mesh_base_counts(int64_t n, const float *x, const float *y, const float *z, int nx, float dx,
                          int refine_thr, int bor, const int32_t *npart_esp, int32_t *cr0);
/* COMPUTE_CR0AMR (grids.f:2076-2226) and VEINSGRID (grids.f:2229-2500): refinement and overlap masks. */
void orc_compute_cr0amr(int nx, float lado0, const asohf_mesh *m, int32_t *cr0amr, int32_t *cr0amr1);
void orc_veinsgrid(int ir, float dx, float radx1, const asohf_mesh *m, int32_t *solap);
/* VEINSGRID_REDUCED (grids.f:1771-2073) on one level's patches. */
int orc_veinsgrid_reduced(int ir, float dx, float radx1, int npatch, const int32_t *pnx, const int32_t *pny,
                          const int32_t *pnz, const float *prx, const float *pry, const float *prz, int max_nb,
                          int32_t *cr01, int32_t *conta11);
void orc_mesh_patch_counts(int64_t n, const float *x, const float *y, const float *z, int irpa, float dx,
                           int refine_thr, int boramr, const int32_t *npart_esp, int npatch,
                           const int32_t *pnx, const int32_t *pny, const int32_t *pnz, const float *prx,
                           const float *pry, const float *prz, int32_t *cr01);
void orc_poisson_fft(int nx, float dx, const float *u1, float *pot);
void orc_argsort(int64_t n, const float *a, int64_t *indx);
void orc_sort_x(int64_t n, float *x, float *y, float *z, float *vx, float *vy,
                float *vz, float *m, int32_t *id, int nx, float lado0,
                int32_t *ndmpart_x);

/* Halo side (oracle_halo.c). The particle arrays are the x-sorted store. */
typedef struct orc_store {
  int64_t n;
  const float *x, *y, *z, *vx, *vy, *vz, *m;
  const int32_t *id;
  const int32_t *ndmpart_x; /* NDMPART_X(0:NX) */
  float norma;              /* MAXVAL(MASAP) */
} orc_store;

void orc_find_particle_indices(float cx, float r, float xldom, float dx, int nmax,
                               const int32_t *ndmpart_x, int64_t *lowp1, int64_t *lowp2);
void orc_prune_poor_haloes(const orc_store *st, const asohf_consts *k,
                           asohf_catalogue *cat, int low1, int low2,
                           float facrad, int do_need_to_count);
/* CHECK_RUBISH (haloes_particles.f:259-318): a halo of the window
 * low1..low2 is removed (REALCLUS=0) when a live halo of a lower level is
 * closer than 1.01 times the smaller radius, with mass ratio above 0.2 and
 * relative speed difference below 3.  Returns the number removed. */
int orc_check_rubish(asohf_catalogue *cat, int nclus, int low1, int low2);
/* OVERLAPPING (haloes_grids.f:27-201) over halo indices 1..lowh2, the new level lowh3..lowh2. */
int orc_overlapping(asohf_catalogue *cat, int lowh3, int lowh2, float vol_solap_low);
/* ACCIDENTAL_SUBSTRUCTURE (haloes_particles.f:321-364): a confirmed halo
 * (REALCLUS=-1) lying wholly inside a confirmed halo of a lower level is
 * removed.  Returns the number removed. */
int orc_accidental_substructure(asohf_catalogue *cat, int nclus);
/* SEARCH_SUBSTRUCTURE_GRID (substructure.f:2-697) on AMR level ir; subs_lev[0..ir] in/out. */
int orc_search_substructure_grid(int ir, int nx, float dx, const float *u1, const float *radx,
                                 const asohf_mesh *m, const float *u11, const int32_t *cr0amr,
                                 const int32_t *cr0amr11, const int32_t *solap, float contrastec, float rote,
                                 float rete, float rodo, float re0, float um, int32_t *subs_lev,
                                 asohf_catalogue *cat);
/* HALOFIND_GRID on AMR level ir >= 1 (haloes_grids.f:586-1097), given the refinement and overlap masks. */
int orc_halofind_grid_amr(int ir, int nx, float dx, const float *u1, const float *radx, const asohf_mesh *m,
                          const float *u11, const int32_t *cr0amr, const int32_t *cr0amr11, const int32_t *solap,
                          float contrastec, float rote, float rete, float rodo, float re0, float bound,
                          float vol_solap_low, asohf_catalogue *cat);
/* HALOFIND_GRID at the base level (haloes_grids.f:287-582); mesh/u11 may be NULL (no AMR levels). */
int orc_halofind_grid_base(int nx, float dx, const float *u1, const float *radx, float contrastec, float rote,
                           float rete, float rodo, float re0, float bound, float vol_solap_low,
                           const asohf_mesh *mesh, const float *u11, asohf_catalogue *cat);
/* HALOFIND_PARTICLES for haloes low1..low2 (Fortran 1-based, inclusive).
 * The bound-particle ID stream is written to pph (capacity pph_cap) and the
 * total used length returned in *pph_len.  Returns a status code. */
/* Decision-margin counts (test instrumentation): rows4 receives, per
 * catalogue row, 4 counts of particle tests within a relative 1e-6 of their
 * threshold (sphere membership, overdensity, escape energy, velocity
 * dispersion), added by orc_halofind_particles and
 * orc_substructure_particles; NULL switches the counting off. */
void orc_set_margin_counts(int32_t *rows4, int64_t cap);
/* Seed of COMPUTE_EPOT's sampling estimator (default 1); the draws are
 * keyed by (seed, catalogue row, draw), as in the library. */
void orc_set_epot_seed(uint32_t seed);
int orc_halofind_particles(const orc_store *st, const asohf_consts *k,
                           const asohf_mesh *mesh, asohf_catalogue *cat,
                           int low1, int low2, int32_t *pph, int64_t pph_cap,
                           int64_t *pph_len, int nthreads);
/* SUBSTRUCTURE_PARTICLES for sub-level ir; subs_lev has nl+1 entries. */
int orc_substructure_particles(const orc_store *st, const asohf_consts *k,
                               const asohf_mesh *mesh, asohf_catalogue *cat,
                               int ir, const int32_t *subs_lev, int32_t *pph,
                               int64_t pph_cap, int64_t *pph_len, int nthreads);
void orc_diagonalise(const float *input_matrix, float *eigen_out);
void orc_sort_eigen(float *e, int n);

#ifdef __cplusplus
}
#endif
#endif
