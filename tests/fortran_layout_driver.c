/*
 * fortran_layout_driver.c -- calls libasohf_gpu.so the way the Fortran shim
 * (fortran/asohf_gpu.f) does, from C, with the Fortran driver's array
 * layouts: column-major grids with leading dimension NMAX, patch tables and
 * catalogue arrays declared longer than they are filled (NPALEV, MAXNCLUS),
 * NPATCH(0:NLEVELS), NDMPART_X(0:NMAX), particle arrays longer than N_DM,
 * and host pointers only (on_device = 0).  The order of the calls is
 * asohf.f's (asohf.f:418-746): species sort, DENSITY, RENORM_DENSITY,
 * SORT_DM_PARTICLES_X, then per level PRUNE_POOR_HALOES (counting),
 * RE_SORT_HALOES, HALOFIND_PARTICLES, PRUNE_POOR_HALOES, CHECK_RUBISH and
 * ACCIDENTAL_SUBSTRUCTURE, then SUBSTRUCTURE_PARTICLES per level, then the
 * PARTICLES_PER_HALO stream.  The permuting calls download the particle
 * arrays back, as the shim does, and DENSITY and SORT_DM_PARTICLES_X
 * upload them again.
 *
 * Test infrastructure: tests/test_gpu_fortran_layout.py writes the input
 * file, builds and runs this program, and compares its output file with
 * the oracle.  Usage: fortran_layout_driver IN OUT
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "asohf_gpu.h"

#define NLEVELS 9
#define NBINS ASOHF_NBINS

static FILE *fin, *fout;

static void rd(void *p, size_t sz, size_t n)
{
  if (n && fread(p, sz, n, fin) != n) { fprintf(stderr, "short input\n"); exit(3); }
}
static void wr(const void *p, size_t sz, size_t n)
{
  if (n && fwrite(p, sz, n, fout) != n) { fprintf(stderr, "short write\n"); exit(3); }
}
static void *zalloc(size_t n) { void *p = calloc(n ? n : 1, 1); if (!p) exit(4); return p; }

#define CHECK(call, what)                                                          \
  do {                                                                             \
    int rc_ = (call);                                                              \
    if (rc_ != 0) {                                                                \
      fprintf(stderr, "%s: status %d (%s)\n", what, rc_, asohf_strerror(rc_));     \
      exit(10 + rc_);                                                              \
    }                                                                              \
  } while (0)

/* The driver's catalogue: every array of MAXNCLUS (here `cap`) entries. */
typedef struct {
  asohf_catalogue c;
} Cat;

static void cat_alloc(asohf_catalogue *c, int cap)
{
  memset(c, 0, sizeof(*c));
  c->capacity = cap;
  float **f1[] = {&c->masa, &c->radio, &c->clusrx, &c->clusry, &c->clusrz, &c->clusrxcm,
                  &c->clusrycm, &c->clusrzcm, &c->msub, &c->rsub, &c->concentra, &c->vmaxclus,
                  &c->vx, &c->vy, &c->vz, &c->mean_vr, &c->vcmax, &c->mcmax, &c->rcmax,
                  &c->m200c, &c->r200c, &c->m500c, &c->r500c, &c->m2500c, &c->r2500c,
                  &c->m200m, &c->r200m, &c->m500m, &c->r500m, &c->m2500m, &c->r2500m,
                  &c->velocity_dispersion, &c->kinetic_e, &c->potential_e};
  for (size_t i = 0; i < sizeof(f1) / sizeof(f1[0]); i++) *f1[i] = zalloc(4 * (size_t)cap);
  int32_t **i1[] = {&c->patchclus, &c->realclus, &c->levhal, &c->dmpclus, &c->iplip};
  for (size_t i = 0; i < sizeof(i1) / sizeof(i1[0]); i++) *i1[i] = zalloc(4 * (size_t)cap);
  c->angularm = zalloc(12 * (size_t)cap);
  c->eigenval = zalloc(12 * (size_t)cap);
  c->inertia_tensor = zalloc(24 * (size_t)cap);
  c->profiles = zalloc(8 * NBINS * (size_t)cap);
  c->indcs = zalloc(8 * (size_t)cap);
}

/* RE_SORT_HALOES (haloes_particles.f:2-56) for the rows of level ir. */
static void re_sort_haloes(asohf_catalogue *c, int32_t *nhallev, int ir)
{
  int low1 = 1, low2 = 0;
  for (int q = 0; q < ir; q++) low1 += nhallev[q];
  for (int q = 0; q <= ir; q++) low2 += nhallev[q];
  int n = low2 - low1 + 1;
  if (n <= 0) return;
  int32_t *map = zalloc(4 * (size_t)n);
  int k = 0;
  for (int i = low1; i <= low2; i++)
    if (c->realclus[i - 1] != 0) map[i - low1] = low1 + k++;
  float *ff[] = {c->clusrx, c->clusry, c->clusrz, c->radio, c->masa, c->clusrxcm, c->clusrycm,
                 c->clusrzcm};
  int32_t *ii[] = {c->levhal, c->patchclus, c->dmpclus};
  int w = low1 - 1;
  for (int i = low1; i <= low2; i++) {
    int r = c->realclus[i - 1];
    if (r == 0) continue;
    for (size_t f = 0; f < sizeof(ff) / sizeof(ff[0]); f++) ff[f][w] = ff[f][i - 1];
    for (size_t f = 0; f < sizeof(ii) / sizeof(ii[0]); f++) ii[f][w] = ii[f][i - 1];
    if (r > 0 && r >= low1 && r <= low2) r = map[r - low1];
    c->realclus[w] = r;
    w++;
  }
  nhallev[ir] = k;
  c->nclus = low1 - 1 + k;
  free(map);
}

static void write_cat(const asohf_catalogue *c)
{
  int64_t n = c->nclus;
  wr(&n, 8, 1);
  /* the order of the ctypes catalogue's fields: scalar floats, scalar ints,
   * then the multi-valued arrays */
  const float *f1[] = {c->masa, c->radio, c->clusrx, c->clusry, c->clusrz, c->clusrxcm,
                       c->clusrycm, c->clusrzcm, c->msub, c->rsub, c->concentra, c->vmaxclus,
                       c->vx, c->vy, c->vz, c->mean_vr, c->vcmax, c->mcmax, c->rcmax,
                       c->m200c, c->r200c, c->m500c, c->r500c, c->m2500c, c->r2500c,
                       c->m200m, c->r200m, c->m500m, c->r500m, c->m2500m, c->r2500m,
                       c->velocity_dispersion, c->kinetic_e, c->potential_e};
  for (size_t i = 0; i < sizeof(f1) / sizeof(f1[0]); i++) wr(f1[i], 4, (size_t)n);
  const int32_t *i1[] = {c->patchclus, c->realclus, c->levhal, c->dmpclus, c->iplip};
  for (size_t i = 0; i < sizeof(i1) / sizeof(i1[0]); i++) wr(i1[i], 4, (size_t)n);
  wr(c->angularm, 12, (size_t)n);
  wr(c->profiles, 8 * NBINS, (size_t)n);
  wr(c->indcs, 8, (size_t)n);
  wr(c->eigenval, 12, (size_t)n);
  wr(c->inertia_tensor, 24, (size_t)n);
}

int main(int argc, char **argv)
{
  if (argc != 3) { fprintf(stderr, "usage: %s IN OUT\n", argv[0]); return 2; }
  fin = fopen(argv[1], "rb");
  if (!fin) return 2;
  int64_t h[16];
  float fh[16];
  rd(h, 8, 16);
  rd(fh, 4, 16);
  int64_t n = h[0];
  int nmax = (int)h[1], nl = (int)h[2], npt = (int)h[3], cap = (int)h[4];
  int ncand = (int)h[5], nsub = (int)h[6], deg = (int)h[7];
  int64_t parti = h[13];
  float lado0 = fh[0], dx = fh[1], rodo = fh[2], re0 = fh[3], rote = fh[4], rete = fh[5], fdm = fh[12];
  asohf_consts k;
  memset(&k, 0, sizeof(k));
  k.nx = nmax; k.lado0 = lado0; k.dx = dx; k.rote = rote; k.rete = rete;
  k.pi = fh[6]; k.cgr = fh[7]; k.um = fh[8]; k.uv = fh[9];
  k.contrastec = fh[10]; k.omegaz = fh[11]; k.fdm = fdm; k.zeta = fh[13];
  k.min_num_part = (int32_t)h[8]; k.do_compute_energies = (int32_t)h[9];
  k.max_part_dsum = (int32_t)h[10]; k.flag_wdm = (int32_t)h[11]; k.var = (int32_t)h[12];

  /* MODULE PARTICLES: arrays of PARTI entries, the first N_DM used */
  float *P[7];
  for (int a = 0; a < 7; a++) { P[a] = zalloc(4 * (size_t)parti); rd(P[a], 4, (size_t)n); }
  int32_t *oripa = zalloc(4 * (size_t)parti);
  rd(oripa, 4, (size_t)n);
  asohf_particles part = {n, P[0], P[1], P[2], P[3], P[4], P[5], P[6], oripa};

  /* the patch table: NPATCH(0:NLEVELS), per-patch arrays of NPALEV entries */
  int npalev = npt + 8;
  int32_t npatch[NLEVELS + 1];
  rd(npatch, 4, NLEVELS + 1);
  int32_t *pi32[7];
  float *pf[3];
  for (int a = 0; a < 6; a++) { pi32[a] = zalloc(4 * (size_t)npalev); rd(pi32[a], 4, (size_t)npt); }
  for (int a = 0; a < 3; a++) { pf[a] = zalloc(4 * (size_t)npalev); rd(pf[a], 4, (size_t)npt); }
  pi32[6] = zalloc(4 * (size_t)npalev);
  rd(pi32[6], 4, (size_t)npt);
  asohf_mesh mesh = {nl, npatch, pi32[0], pi32[1], pi32[2], pi32[3], pi32[4], pi32[5],
                     pf[0], pf[1], pf[2], pi32[6]};

  /* halo candidates per level, subhalo candidates per level */
  int32_t *clev = zalloc(4 * (size_t)(nl + 1)), *slev = zalloc(4 * (size_t)(nl + 1));
  rd(clev, 4, (size_t)nl + 1);
  float *cf[5];
  int32_t *ci[2];
  for (int a = 0; a < 5; a++) { cf[a] = zalloc(4 * (size_t)ncand); rd(cf[a], 4, (size_t)ncand); }
  for (int a = 0; a < 2; a++) { ci[a] = zalloc(4 * (size_t)ncand); rd(ci[a], 4, (size_t)ncand); }
  rd(slev, 4, (size_t)nl + 1);
  float *sf[4];
  int32_t *si[2];
  for (int a = 0; a < 4; a++) { sf[a] = zalloc(4 * (size_t)nsub); rd(sf[a], 4, (size_t)nsub); }
  for (int a = 0; a < 2; a++) { si[a] = zalloc(4 * (size_t)nsub); rd(si[a], 4, (size_t)nsub); }
  fclose(fin);

  asohf_ctx *ctx = NULL;
  CHECK(asohf_create(0, &ctx), "asohf_create");

  /* SORT_DM_PARTICLES_LOCALDENSITY: upload, sort, download */
  int32_t npart_esp[ASOHF_N_ESP];
  CHECK(asohf_upload_particles(ctx, &part, 0), "upload");
  CHECK(asohf_sort_dm_particles_localdensity(ctx, nmax, dx, rodo, re0, npart_esp), "species sort");
  CHECK(asohf_download_particles(ctx, &part, 0), "download");

  /* DENSITY into COMMON /VARIA/ U1(NMAX,NMAY,NMAZ), U11(32,32,32,NPALEV) */
  size_t g = (size_t)nmax * nmax * nmax;
  float *u1 = zalloc(4 * g);
  float *u11 = zalloc(4 * (size_t)npalev * 32768);
  CHECK(asohf_upload_particles(ctx, &part, 0), "upload");
  CHECK(asohf_density(ctx, nmax, lado0, dx, rote, rete, npart_esp, &mesh, deg, u1, u11, 0), "DENSITY");
  CHECK(asohf_renorm_density(ctx, nmax, &mesh, fdm, u1, u11, 0), "RENORM_DENSITY");

  /* SORT_DM_PARTICLES_X: NDMPART_X(0:NMAX) */
  int32_t *ndmpart_x = zalloc(4 * (size_t)(nmax + 1));
  CHECK(asohf_upload_particles(ctx, &part, 0), "upload");
  CHECK(asohf_sort_dm_particles_x(ctx, nmax, lado0, ndmpart_x), "SORT_DM_PARTICLES_X");
  CHECK(asohf_download_particles(ctx, &part, 0), "download");

  /* haloes, level by level */
  asohf_catalogue cat;
  cat_alloc(&cat, cap);
  int32_t nhallev[NLEVELS + 1];
  memset(nhallev, 0, sizeof(nhallev));
  int c0 = 0;
  for (int ir = 0; ir <= nl; ir++) {
    int nn = clev[ir];
    if (nn == 0) continue;
    int s0 = cat.nclus;
    for (int q = 0; q < nn; q++) {
      cat.clusrx[s0 + q] = cf[0][c0 + q];
      cat.clusry[s0 + q] = cf[1][c0 + q];
      cat.clusrz[s0 + q] = cf[2][c0 + q];
      cat.radio[s0 + q] = cf[3][c0 + q];
      cat.masa[s0 + q] = cf[4][c0 + q];
      cat.levhal[s0 + q] = ci[0][c0 + q];
      cat.patchclus[s0 + q] = ci[1][c0 + q];
      cat.realclus[s0 + q] = -1;
    }
    c0 += nn;
    cat.nclus = s0 + nn;
    nhallev[ir] = nn;
    re_sort_haloes(&cat, nhallev, ir);
    int low1 = 1, low2 = 0;
    for (int q = 0; q < ir; q++) low1 += nhallev[q];
    for (int q = 0; q <= ir; q++) low2 += nhallev[q];
    CHECK(asohf_prune_poor_haloes(ctx, &k, &cat, low1, low2, 1.0f, 1, 0), "PRUNE_POOR_HALOES");
    re_sort_haloes(&cat, nhallev, ir);
    low2 = low1 - 1 + nhallev[ir];
    if (nhallev[ir] == 0) continue;
    CHECK(asohf_halofind_particles(ctx, &k, &mesh, &cat, low1, low2, 0), "HALOFIND_PARTICLES");
    CHECK(asohf_prune_poor_haloes(ctx, &k, &cat, low1, low2, 1.0f, 0, 0), "PRUNE_POOR_HALOES");
    int32_t konta = 0;
    CHECK(asohf_check_rubish(ctx, &cat, cat.nclus, low1, low2, 0, &konta), "CHECK_RUBISH");
    CHECK(asohf_accidental_substructure(ctx, &cat, cat.nclus, 0, &konta), "ACCIDENTAL_SUBSTRUCTURE");
  }

  /* subhaloes, level by level: SUBS_LEV(0:NLEVELS) */
  int32_t subs_lev[NLEVELS + 1];
  memset(subs_lev, 0, sizeof(subs_lev));
  subs_lev[0] = cat.nclus;
  int s_0 = 0;
  for (int ir = 1; ir <= nl; ir++) {
    int nn = slev[ir];
    subs_lev[ir] = nn;
    if (nn == 0) continue;
    int s0 = cat.nclus;
    for (int q = 0; q < nn; q++) {
      cat.clusrx[s0 + q] = sf[0][s_0 + q];
      cat.clusry[s0 + q] = sf[1][s_0 + q];
      cat.clusrz[s0 + q] = sf[2][s_0 + q];
      cat.rsub[s0 + q] = sf[3][s_0 + q];
      cat.realclus[s0 + q] = si[0][s_0 + q];
      cat.levhal[s0 + q] = si[1][s_0 + q];
      cat.patchclus[s0 + q] = 0;
    }
    s_0 += nn;
    cat.nclus = s0 + nn;
    CHECK(asohf_substructure_particles(ctx, &k, &mesh, &cat, ir, subs_lev, 0), "SUBSTRUCTURE_PARTICLES");
  }

  /* PARTICLES_PER_HALO */
  int64_t npph = 0;
  CHECK(asohf_get_particles_per_halo(ctx, NULL, 0, &npph, 0), "PARTICLES_PER_HALO");
  int32_t *pph = zalloc(4 * (size_t)(npph + 1));
  CHECK(asohf_get_particles_per_halo(ctx, pph, npph, &npph, 0), "PARTICLES_PER_HALO");
  CHECK(asohf_destroy(ctx), "asohf_destroy");

  fout = fopen(argv[2], "wb");
  if (!fout) return 2;
  wr(npart_esp, 4, ASOHF_N_ESP);
  wr(u1, 4, g);
  wr(u11, 4, (size_t)npt * 32768);
  wr(ndmpart_x, 4, (size_t)nmax + 1);
  write_cat(&cat);
  wr(subs_lev, 4, NLEVELS + 1);
  wr(&npph, 8, 1);
  wr(pph, 4, (size_t)npph);
  fclose(fout);
  return 0;
}
