/*
 * oracle_halo.c -- CPU oracle (TEST INFRASTRUCTURE ONLY) for the per-halo
 * half of the ASOHF particle hot path: slab queries, pruning, density-peak
 * recentering, spherical-overdensity growth, radial sort, unbinding, the SO
 * walk, bound-particle properties and ID lists, and the subhalo variant.
 *
 * A statement-by-statement C restatement of haloes_particles.f,
 * substructure.f:756-1697 and num.f, keeping each Fortran statement's
 * precision (REAL*4 products and compares, REAL*8 accumulators, stores to
 * REAL*4 rounding at the assignment).  Work arrays keep the Fortran contents
 * beyond the active length (REORDENAR's in-place compaction leaves stale
 * tails; its sorting mode fills DISTA with 1e10), since a few statements read
 * past the active length.  Parity status: unpinned by the reference (see
 * oracle_grid.c).  Build with -ffp-contract=off.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"

#define NB ASOHF_NBINS

/* Decision margins (test instrumentation, off unless a buffer is set):
 * for each catalogue row, the number of particle tests whose two sides lie
 * within a relative 1e-6 of each other -- the particles whose decision a
 * last-bit difference in the arithmetic could flip.  Four counts per row:
 * [0] membership of the growth sphere (distance vs radius, final iteration),
 * [1] overdensity thresholds (FIND_IDX_VIR, the SO walk, the subhalo Jacobi
 *     estimate), [2] UNBINDING8's escape-energy test, [3] UNBINDING_SIGMA's
 * velocity-dispersion test.  Each row is refined by one thread, so the
 * counts need no atomics. */
#define MARGIN_REL 1e-6
static int32_t *g_margin = NULL;
static int64_t g_margin_cap = 0;
static _Thread_local int64_t g_row = -1;

void orc_set_margin_counts(int32_t *rows4, int64_t cap)
{
  g_margin = rows4;
  g_margin_cap = rows4 ? cap : 0;
}

static inline void margin_add(int kind, int64_t n)
{
  if (g_margin && g_row >= 0 && g_row < g_margin_cap && n) g_margin[g_row * 4 + kind] += (int32_t)n;
}

static inline int near_thr(double a, double thr)
{
  return fabs(a - thr) <= MARGIN_REL * fabs(thr);
}

/* FIND_PARTICLE_INDICES (haloes_particles.f:117-143).  lowp1/lowp2 are
 * 1-based inclusive positions in the x-sorted store. */
void orc_find_particle_indices(float cx, float r, float xldom, float dx, int nmax,
                               const int32_t *ndmpart_x, int64_t *lowp1, int64_t *lowp2)
{
  int pos1 = (int)(((cx - r) - xldom) / dx) + 1;
  int pos2 = (int)(((cx + r) - xldom) / dx) + 1;
  if (pos1 < 1) pos1 = 1;
  if (pos2 > nmax) pos2 = nmax;
  /* Out-of-range slabs (a query entirely outside the box) read outside
   * NDMPART_X in the Fortran; here they give an empty range. */
  if (pos1 > nmax + 1) pos1 = nmax + 1;
  if (pos2 < 0) pos2 = 0;
  *lowp1 = (int64_t)ndmpart_x[pos1 - 1] + 1;
  *lowp2 = (int64_t)ndmpart_x[pos2];
}

/* COUNT_PARTICLES_HALO (haloes_particles.f:147-182). */
static int count_particles_halo(const orc_store *st, const asohf_consts *k,
                                float cx, float cy, float cz, float r)
{
  int num = 0;
  float r2 = r * r;
  int64_t lo, hi;
  orc_find_particle_indices(cx, r, -k->lado0 / 2.0f, k->dx, k->nx, st->ndmpart_x, &lo, &hi);
  for (int64_t i = lo; i <= hi; i++) {
    float bx = st->x[i - 1] - cx;
    bx = bx * bx;
    if (bx > r2) continue;
    float by = st->y[i - 1] - cy;
    by = by * by;
    if (by > r2) continue;
    float bz = st->z[i - 1] - cz;
    bz = bz * bz;
    if (bz > r2) continue;
    float basr = bx + by + bz;
    if (basr < r2) num++;
  }
  return num;
}

/* PRUNE_POOR_HALOES (haloes_particles.f:185-256). low1/low2 Fortran 1-based. */
/* CHECK_RUBISH (haloes_particles.f:259-318), the Fortran loops in order.
 * A2 keeps its last value when one of the two speeds is zero (the Fortran
 * assigns it only otherwise); before any assignment it is taken as 0. */
int orc_check_rubish(asohf_catalogue *cat, int nclus, int low1, int low2)
{
  int konta = 0;
  float a2 = 0.0f;
  for (int i = 1; i <= nclus; i++) {
    if (cat->realclus[i - 1] == 0) continue;
    for (int j = low1; j <= low2; j++) {
      if (!(cat->realclus[j - 1] != 0 && cat->levhal[j - 1] > cat->levhal[i - 1])) continue;
      float dx = cat->clusrx[i - 1] - cat->clusrx[j - 1];
      float dy = cat->clusry[i - 1] - cat->clusry[j - 1];
      float dz = cat->clusrz[i - 1] - cat->clusrz[j - 1];
      float dis = sqrtf(dx * dx + dy * dy + dz * dz);
      float mi = cat->masa[i - 1], mj = cat->masa[j - 1];
      float a1 = (mi < mj ? mi : mj) / (mi > mj ? mi : mj);
      float v1 = sqrtf(cat->vx[i - 1] * cat->vx[i - 1] + cat->vy[i - 1] * cat->vy[i - 1] +
                       cat->vz[i - 1] * cat->vz[i - 1]);
      float v2 = sqrtf(cat->vx[j - 1] * cat->vx[j - 1] + cat->vy[j - 1] * cat->vy[j - 1] +
                       cat->vz[j - 1] * cat->vz[j - 1]);
      if ((v1 < v2 ? v1 : v2) != 0.0f) a2 = fabsf(v1 - v2) / (v1 > v2 ? v1 : v2);
      float ri = cat->radio[i - 1], rj = cat->radio[j - 1];
      float a3 = ri < rj ? ri : rj;
      if (dis < 1.01f * a3 && a1 > 0.2f && a2 < 3.0f) {
        cat->realclus[j - 1] = 0;
        konta++;
      }
    }
  }
  return konta;
}

/* ACCIDENTAL_SUBSTRUCTURE (haloes_particles.f:321-364), the Fortran loops in
 * order. */
int orc_accidental_substructure(asohf_catalogue *cat, int nclus)
{
  int konta = 0;
  for (int i = 1; i <= nclus; i++) {
    if (cat->realclus[i - 1] != -1) continue;
    for (int j = 1; j <= nclus; j++) {
      if (cat->realclus[j - 1] != -1) continue;
      float dx = cat->clusrx[i - 1] - cat->clusrx[j - 1];
      float dy = cat->clusry[i - 1] - cat->clusry[j - 1];
      float dz = cat->clusrz[i - 1] - cat->clusrz[j - 1];
      float dis = sqrtf(dx * dx + dy * dy + dz * dz);
      if (cat->levhal[j - 1] > cat->levhal[i - 1] && dis + cat->radio[j - 1] <= 1.0f * cat->radio[i - 1]) {
        cat->realclus[j - 1] = 0;
        konta++;
      }
    }
  }
  return konta;
}

/* OVERLAPPING (haloes_grids.f:27-201), the grid finder's overlap removal at
 * the end of level IR: lowh3 = SUM(NHALLEV(0:IR-1))+1, lowh2 =
 * SUM(NHALLEV(0:IR)).  Pass 1 removes the smaller of two spheres when one
 * lies inside the other (|R1-R2| >= DIST); pass 2 when the overlap volume
 * (two-sphere lens, in units of the smaller sphere) exceeds vol_solap_low.
 * The row halo's REALCLUS is read once per row (BASINT), so a removed row
 * halo still removes later partners.  Returns COUNT(REALCLUS(lowh3:lowh2)
 * == 0), the figure the routine prints. */
int orc_overlapping(asohf_catalogue *cat, int lowh3, int lowh2, float vol_solap_low)
{
  const float pi = (float)acos(-1.0);
  for (int pass = 1; pass <= 2; pass++) {
    for (int i = 1; i <= lowh2; i++) {
      if (cat->realclus[i - 1] == 0) continue;
      const float r1 = cat->radio[i - 1], x1 = cat->clusrx[i - 1], y1 = cat->clusry[i - 1],
                  z1 = cat->clusrz[i - 1];
      for (int j = (i + 1 > lowh3 ? i + 1 : lowh3); j <= lowh2; j++) {
        if (cat->realclus[j - 1] == 0) continue;
        const float r2 = cat->radio[j - 1];
        const float dx = x1 - cat->clusrx[j - 1], dy = y1 - cat->clusry[j - 1], dz = z1 - cat->clusrz[j - 1];
        const float dist = sqrtf(dx * dx + dy * dy + dz * dz);
        int imin = j;
        if (pass == 1) {
          if (!(fabsf(r1 - r2) >= dist)) continue;
          if (r2 > r1 && cat->levhal[j - 1] <= cat->levhal[i - 1]) imin = i;
        } else {
          const float s = r1 + r2, d = r1 - r2;
          const float bas = dist / s;
          if (!(bas < 1.0f)) continue;
          const float xi = bas, u = 1.0f - xi, m = fminf(r1, r2);
          float vint = pi / 12.0f * (s * s * s) * (u * u / xi) * (xi * xi + 2.0f * xi - 3.0f * (d * d) / (s * s));
          vint = vint / (4.0f * pi / 3.0f * (m * m * m));
          if (!(vint > vol_solap_low)) continue;
          if (r2 > 1.5f * r1 && cat->levhal[j - 1] <= cat->levhal[i - 1]) imin = i;
        }
        cat->realclus[imin - 1] = 0;
      }
    }
  }
  int n0 = 0;
  for (int j = lowh3; j <= lowh2; j++) n0 += cat->realclus[j - 1] == 0;
  return n0;
}

void orc_prune_poor_haloes(const orc_store *st, const asohf_consts *k,
                           asohf_catalogue *cat, int low1, int low2,
                           float facrad, int do_need_to_count)
{
  if (do_need_to_count == 1) {
#pragma omp parallel for schedule(dynamic)
    for (int i = low1; i <= low2; i++) {
      float rr = facrad * cat->radio[i - 1];
      int basint = count_particles_halo(st, k, cat->clusrx[i - 1], cat->clusry[i - 1],
                                        cat->clusrz[i - 1], rr);
      if (basint < k->min_num_part) cat->realclus[i - 1] = 0;
      cat->dmpclus[i - 1] = basint;
    }
  } else {
    for (int i = low1; i <= low2; i++)
      if (cat->dmpclus[i - 1] < k->min_num_part) cat->realclus[i - 1] = 0;
  }
}

/* ------------------------------------------------------------------ */
/* Growable int64 list. */
typedef struct { int64_t *v; int64_t n, cap; } ilist;
static void il_push(ilist *l, int64_t x)
{
  if (l->n == l->cap) {
    l->cap = l->cap ? 2 * l->cap : 1024;
    l->v = (int64_t *)realloc(l->v, sizeof(int64_t) * (size_t)l->cap);
  }
  l->v[l->n++] = x;
}

/* Particle test of the open cube (haloes_particles.f:405-407). */
static inline int in_cube(const orc_store *st, int64_t p, float cx, float cy, float cz, float r)
{
  return (cx - r < st->x[p] && st->x[p] < cx + r && cy - r < st->y[p] && st->y[p] < cy + r &&
          cz - r < st->z[p] && st->z[p] < cz + r);
}

/* RECENTER_DENSITY_PEAK_PARTICLES (haloes_particles.f:367-574).  Particle
 * indices are 0-based positions in the x-sorted store. */
static void recenter(const orc_store *st, const asohf_consts *k, float *pcx, float *pcy,
                     float *pcz, float r, float dxpamin)
{
  const int numpartmin = 32;
  float cx = *pcx, cy = *pcy, cz = *pcz;
  float xldom = -k->lado0 / 2.0f;
  float radio = fmaxf(0.05f * r, dxpamin);
  ilist lip = {0};
  float maxm, minm;
  for (;;) {
    lip.n = 0;
    int64_t lo, hi;
    orc_find_particle_indices(cx, radio, xldom, k->dx, k->nx, st->ndmpart_x, &lo, &hi);
    maxm = -1.e30f;
    minm = 1.e30f;
    for (int64_t i = lo; i <= hi; i++) {
      if (in_cube(st, i - 1, cx, cy, cz, radio)) {
        il_push(&lip, i - 1);
        maxm = fmaxf(maxm, st->m[i - 1]);
        minm = fminf(minm, st->m[i - 1]);
      }
    }
    if (lip.n > numpartmin) break;
    radio = radio * 1.2f;
  }
  const int nn = 4;
  double dens[64];
  float ddxx = 2.0f * radio / (float)nn;
  float xl = cx - radio, yl = cy - radio, zl = cz - radio;
  int flag_iter = 1;
  while (flag_iter == 1) {
    for (int c = 0; c < 64; c++) dens[c] = 0.0;
    if (maxm / minm < 8.0f) {
      for (int64_t i = 0; i < lip.n; i++) {
        int64_t ip = lip.v[i];
        int ix = (int)((st->x[ip] - xl) / ddxx) + 1;
        int jy = (int)((st->y[ip] - yl) / ddxx) + 1;
        int kz = (int)((st->z[ip] - zl) / ddxx) + 1;
        if (ix < 1) ix = 1;
        if (ix > nn) ix = nn;
        if (jy < 1) jy = 1;
        if (jy > nn) jy = nn;
        if (kz < 1) kz = 1;
        if (kz > nn) kz = nn;
        dens[((kz - 1) * nn + (jy - 1)) * nn + (ix - 1)] += (double)st->m[ip];
      }
    } else {
      for (int64_t i = 0; i < lip.n; i++) {
        int64_t ip = lip.v[i];
        int ix = (int)floorf((st->x[ip] - xl) / ddxx) + 1;
        int jy = (int)floorf((st->y[ip] - yl) / ddxx) + 1;
        int kz = (int)floorf((st->z[ip] - zl) / ddxx) + 1;
        int plev = (int)(logf(st->m[ip] / minm) / logf(8.0f));
        if (plev < 0) plev = 0;
        if (plev == 0) {
          if (ix < 1) ix = 1;
          if (ix > nn) ix = nn;
          if (jy < 1) jy = 1;
          if (jy > nn) jy = nn;
          if (kz < 1) kz = 1;
          if (kz > nn) kz = nn;
          dens[((kz - 1) * nn + (jy - 1)) * nn + (ix - 1)] += (double)st->m[ip];
        } else {
          int ksize = (int)(0.25f + 0.5f * (float)(1 << plev));
          int nden = ksize + 1;
          float bl = 1.0f / (float)nden;
          float norma = 1.0f / (float)(nden * nden * nden);
          int i1 = ix - ksize > 1 ? ix - ksize : 1, j1 = jy - ksize > 1 ? jy - ksize : 1,
              k1 = kz - ksize > 1 ? kz - ksize : 1;
          int i2 = ix + ksize < nn ? ix + ksize : nn, j2 = jy + ksize < nn ? jy + ksize : nn,
              k2 = kz + ksize < nn ? kz + ksize : nn;
          for (int kk = k1; kk <= k2; kk++)
            for (int jj = j1; jj <= j2; jj++)
              for (int ii = i1; ii <= i2; ii++) {
                float kx = 1.0f - bl * (float)abs(ii - ix);
                float ky = 1.0f - bl * (float)abs(jj - jy);
                float kzv = 1.0f - bl * (float)abs(kk - kz);
                float kern = kx * ky * kzv * norma;
                dens[((kk - 1) * nn + (jj - 1)) * nn + (ii - 1)] += (double)kern * (double)st->m[ip];
              }
        }
      }
    }
    /* MAXLOC: first maximum in column-major order */
    int best = 0;
    for (int c = 1; c < 64; c++)
      if (dens[c] > dens[best]) best = c;
    int ix = best % nn + 1, jy = (best / nn) % nn + 1, kz = best / (nn * nn) + 1;
    cx = xl + ((float)ix - 0.5f) * ddxx;
    cy = yl + ((float)jy - 0.5f) * ddxx;
    cz = zl + ((float)kz - 0.5f) * ddxx;
    radio = radio / 2.0f;
    xl = cx - radio;
    yl = cy - radio;
    zl = cz - radio;
    ddxx = ddxx / 2.0f;
    int64_t konta2 = 0;
    maxm = -1.e30f;
    minm = 1.e30f;
    for (int64_t i = 0; i < lip.n; i++) {
      int64_t ip = lip.v[i];
      if (in_cube(st, ip, cx, cy, cz, radio)) {
        lip.v[konta2++] = ip;
        maxm = fmaxf(maxm, st->m[ip]);
        minm = fminf(minm, st->m[ip]);
      }
    }
    lip.n = konta2;
    if (konta2 < numpartmin) flag_iter = 0;
  }
  double bas = 0.0, basx = 0.0, basy = 0.0, basz = 0.0;
  for (int64_t i = 0; i < lip.n; i++) {
    int64_t ip = lip.v[i];
    bas = bas + st->m[ip];
    basx = basx + (double)(st->x[ip] * st->m[ip]);
    basy = basy + (double)(st->y[ip] * st->m[ip]);
    basz = basz + (double)(st->z[ip] * st->m[ip]);
  }
  *pcx = (float)(basx / bas);
  *pcy = (float)(basy / bas);
  *pcz = (float)(basz / bas);
  free(lip.v);
}

/* ------------------------------------------------------------------ */
/* Per-halo work arrays with Fortran shapes: LIP(1:cap), CONTADM(1:cap),
 * DISTA(0:cap).  lip holds 0-based store positions (-1 for Fortran's 0). */
typedef struct {
  int64_t cap;
  int64_t *lip;
  int32_t *contadm;
  float *dista;
} hwork;

static void hw_alloc(hwork *w, int64_t cap)
{
  w->cap = cap;
  w->lip = (int64_t *)malloc(sizeof(int64_t) * (size_t)(cap + 2));
  w->contadm = (int32_t *)malloc(sizeof(int32_t) * (size_t)(cap + 2));
  w->dista = (float *)malloc(sizeof(float) * (size_t)(cap + 2));
  for (int64_t j = 0; j <= cap + 1; j++) { w->lip[j] = -1; w->contadm[j] = 1; w->dista[j] = 0.0f; }
}
static void hw_free(hwork *w) { free(w->lip); free(w->contadm); free(w->dista); }

static inline float dist3(const orc_store *st, int64_t p, float cx, float cy, float cz)
{
  float ax = st->x[p] - cx, ay = st->y[p] - cy, az = st->z[p] - cz;
  return sqrtf(ax * ax + ay * ay + az * az);
}

/* REORDENAR (haloes_particles.f:1632-1728). */
static void reordenar(const orc_store *st, int64_t konta, float cx, float cy, float cz,
                      hwork *w, int64_t *konta2, int do_sort, int64_t *idx_vir)
{
  if (do_sort == 1) {
    float *d = (float *)calloc((size_t)(konta + 1), sizeof(float));
    int64_t *quien = (int64_t *)malloc(sizeof(int64_t) * (size_t)(konta + 1));
    int64_t k2 = 0;
    for (int64_t j = 1; j <= konta; j++) {
      if (w->contadm[j] == 0) {
        k2++;
        int64_t jj = w->lip[j];
        d[k2] = dist3(st, jj, cx, cy, cz);
        quien[k2] = jj;
      }
    }
    int64_t *indice = (int64_t *)malloc(sizeof(int64_t) * (size_t)(k2 + 1));
    orc_argsort(k2, d + 1, indice + 1);
    for (int64_t j = 0; j <= w->cap + 1; j++) { w->dista[j] = 1.e10f; w->lip[j] = -1; }
    for (int64_t j = 1; j <= k2; j++) {
      int64_t jj = indice[j];
      w->dista[j] = d[jj];
      w->lip[j] = quien[jj];
    }
    *idx_vir = k2;
    *konta2 = k2;
    free(d);
    free(quien);
    free(indice);
  } else {
    int64_t k2 = 0;
    int reloc = 0;
    for (int64_t j = 1; j <= konta; j++) {
      if (w->contadm[j] == 0) {
        k2++;
        w->dista[k2] = w->dista[j];
        w->lip[k2] = w->lip[j];
        if (reloc == 0 && j >= *idx_vir) { reloc = 1; *idx_vir = k2; }
      }
    }
    if (reloc == 0) *idx_vir = k2;
    *konta2 = k2;
  }
  for (int64_t j = 1; j <= w->cap; j++) w->contadm[j] = 1;
  for (int64_t j = 1; j <= *konta2; j++) w->contadm[j] = 0;
}

/* FIND_IDX_VIR (haloes_particles.f:1453-1491).  Returns -1 on the
 * reference's STOP ("NOT PRE-FOUND VIRIAL RADIUS"). */
static int64_t find_idx_vir(const orc_store *st, const hwork *w, float rote, float rete,
                            float pi, float contrastec, int64_t idx_vir)
{
  double menc = 0.0;
  int64_t jjcore = idx_vir / 10 < 50 ? idx_vir / 10 : 50;
  for (int64_t j = 1; j <= jjcore; j++) menc = menc + (double)st->m[w->lip[j]];
  int64_t j;
  for (j = jjcore + 1; j <= idx_vir; j++) {
    menc = menc + (double)st->m[w->lip[j]];
    float d = w->dista[j];
    float den = rote * (rete * rete * rete) * (4.0f * pi / 3.0f) * (d * d * d);
    float delta = (float)(menc / (double)den);
    margin_add(1, near_thr(delta, contrastec));
    if (delta < contrastec) break;
  }
  if (j == idx_vir + 1) return -1;
  return j;
}

/* CENTROMASAS_PART (haloes_particles.f:1731-1824). */
static void centromasas(const orc_store *st, int64_t n, const hwork *w, float *cm, float *vcm,
                        float *masa)
{
  double c8[3] = {0, 0, 0}, v8[3] = {0, 0, 0}, m8 = 0.0;
  for (int64_t i = 1; i <= n; i++) {
    if (w->contadm[i] == 0) {
      int64_t j = w->lip[i];
      double bas = (double)st->m[j];
      c8[0] = c8[0] + (double)st->x[j] * bas;
      c8[1] = c8[1] + (double)st->y[j] * bas;
      c8[2] = c8[2] + (double)st->z[j] * bas;
      v8[0] = (double)st->vx[j] * bas + v8[0];
      v8[1] = (double)st->vy[j] * bas + v8[1];
      v8[2] = (double)st->vz[j] * bas + v8[2];
      m8 = m8 + bas;
    }
  }
  if (m8 > 0.0) {
    for (int a = 0; a < 3; a++) { c8[a] = c8[a] / m8; v8[a] = v8[a] / m8; }
  } else {
    for (int a = 0; a < 3; a++) { c8[a] = 0.0; v8[a] = 0.0; }
    m8 = 0.0;
  }
  for (int a = 0; a < 3; a++) { cm[a] = (float)c8[a]; vcm[a] = (float)v8[a]; }
  *masa = (float)m8;
}

/* Halo-level state that UNBINDING8/UNBINDING_SIGMA update through the
 * catalogue arrays (RADIO, MASA, CLUSR*CM, VX.., REALCLUS of halo I). */
typedef struct {
  float *radio, *masa, *cmx, *cmy, *cmz, *vx, *vy, *vz;
  int32_t *realclus;
} hstate;

static void unbind_result(hstate *h, int64_t konta3, const float *cm, const float *vcm, float mmm, float um)
{
  if (konta3 == 0) {
    *h->cmx = 0.0f; *h->cmy = 0.0f; *h->cmz = 0.0f;
    *h->vx = 0.0f; *h->vy = 0.0f; *h->vz = 0.0f;
    *h->masa = 0.0f; *h->radio = 0.0f;
    *h->realclus = 0;
  } else {
    *h->cmx = cm[0]; *h->cmy = cm[1]; *h->cmz = cm[2];
    *h->vx = vcm[0]; *h->vy = vcm[1]; *h->vz = vcm[2];
    *h->masa = mmm * um;
  }
}

/* UNBINDING8 (haloes_particles.f:1828-1983). */
static void unbinding8(const orc_store *st, const asohf_consts *k, int fac, float ref_max,
                       hwork *w, int64_t konta2, int64_t idx_vir, hstate *h)
{
  float cm[3] = {0, 0, 0}, vcm[3] = {0, 0, 0}, mmm = 0.0f;
  if (konta2 > 0) {
    double norma = (double)st->norma;
    double *pot = (double *)calloc((size_t)(konta2 + 2), sizeof(double));
    int64_t j;
    for (j = 1; j <= konta2; j++)
      if (w->dista[j] > 0.01f * ref_max) break;
    int64_t jj = j;
    double masa8 = 0.0;
    for (j = 1; j <= jj; j++) masa8 = masa8 + (double)st->m[w->lip[j]] / norma;
    for (j = 1; j <= jj; j++) pot[j] = masa8 / (double)w->dista[jj];
    for (j = jj + 1; j <= konta2; j++) {
      masa8 = masa8 + (double)st->m[w->lip[j]] / norma;
      double bas8;
      if (w->dista[j] != w->dista[j - 1]) bas8 = (double)(w->dista[j] - w->dista[j - 1]);
      else bas8 = 0.0;
      double dj = (double)w->dista[j];
      pot[j] = pot[j - 1] + masa8 * bas8 / (dj * dj);
    }
    double pot1 = pot[konta2] + masa8 / (double)ref_max;
    double aa8 = norma * (double)(k->cgr / k->rete);
    float bb = 2.0f;
    if (fac == 1) bb = 8.0f;
    if (fac == 2) bb = 4.0f;
    bb = bb * bb;
    for (j = 1; j <= konta2; j++) {
      float potok = (float)((pot[j] - pot1) * aa8);
      float vesc2 = 2.0f * fabsf(potok);
      int64_t p = w->lip[j];
      float ax = st->vx[p] - *h->vx, ay = st->vy[p] - *h->vy, az = st->vz[p] - *h->vz;
      float vvv2 = ax * ax + ay * ay + az * az;
      margin_add(2, near_thr(vvv2, bb * vesc2));
      if (vvv2 > bb * vesc2) w->contadm[j] = 1;
    }
    free(pot);
    centromasas(st, idx_vir, w, cm, vcm, &mmm);
  }
  int64_t konta3 = 0;
  for (int64_t j = 1; j <= konta2; j++) konta3 += (w->contadm[j] == 0);
  unbind_result(h, konta3, cm, vcm, mmm, k->um);
}

/* UNBINDING_SIGMA (haloes_particles.f:1987-2095). */
static void unbinding_sigma(const orc_store *st, const asohf_consts *k, int fac, hwork *w,
                            int64_t konta2, int64_t idx_vir, hstate *h)
{
  float bb = fmaxf(6.0f - 1.0f * (float)(fac - 1), 3.0f);
  bb = bb * bb;
  float cm[3] = {*h->cmx, *h->cmy, *h->cmz};
  float vcm[3] = {*h->vx, *h->vy, *h->vz};
  float mmm = 0.0f;
  if (konta2 > 0) {
    float *desv2 = (float *)malloc(sizeof(float) * (size_t)(konta2 + 1));
    double sigma2 = 0.0;
    for (int64_t j = 1; j <= konta2; j++) {
      int64_t p = w->lip[j];
      float ax = st->vx[p] - vcm[0], ay = st->vy[p] - vcm[1], az = st->vz[p] - vcm[2];
      float bas = ax * ax + ay * ay + az * az;
      desv2[j] = bas;
      if (j <= idx_vir) sigma2 = sigma2 + (double)bas;
    }
    if (idx_vir > 1) sigma2 = sigma2 / (double)(idx_vir - 1);
    for (int64_t j = 1; j <= konta2; j++) {
      margin_add(3, near_thr((double)desv2[j], (double)bb * sigma2));
      if ((double)desv2[j] > (double)bb * sigma2) w->contadm[j] = 1;
    }
    free(desv2);
    centromasas(st, idx_vir, w, cm, vcm, &mmm);
  }
  int64_t konta3 = 0;
  for (int64_t j = 1; j <= konta2; j++) konta3 += (w->contadm[j] == 0);
  unbind_result(h, konta3, cm, vcm, mmm, k->um);
}

/* Seed of the sampling estimator (orc_set_epot_seed; default 1). */
static uint32_t g_epot_seed = 1;

void orc_set_epot_seed(uint32_t seed) { g_epot_seed = seed; }

/* MurmurHash3's 32-bit finaliser and the chained mix of the draws. */
static inline uint32_t fmix32(uint32_t h)
{
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

static inline uint32_t mix2(uint32_t a, uint32_t b) { return fmix32(a ^ fmix32(b)); }

/* One draw J = 1 + FLOOR(U*KONTA) of the sampling branch, with U a REAL*4
 * of 24 random bits: U = (bits >> 8) * 2^-24, bits = mix(key_outer, inner +
 * 0x9E3779B9 * attempt).  Clamped to KONTA (U*KONTA can round up to KONTA
 * in REAL*4, where the reference would read past the list). */
static inline int64_t epot_draw(uint32_t key_outer, uint32_t inner, uint32_t attempt, int64_t konta)
{
  uint32_t bits = mix2(key_outer, inner + 0x9E3779B9u * attempt);
  float u = (float)(bits >> 8) * 5.9604644775390625e-8f;
  int64_t j = 1 + (int64_t)floorf(u * (float)konta);
  return j <= konta ? j : konta;
}

#define EPOT_MAX_ATTEMPTS 4096u

/* The sampling branch of COMPUTE_EPOT (haloes_particles.f:1568-1626),
 * statement by statement, with the reference's RANDOM_NUMBER stream (after
 * an unseeded RANDOM_SEED: irreproducible) replaced by epot_draw keyed by
 * (seed, catalogue row, outer draw): the draws of J and, for each J, of its
 * NSAMPLE partners K != J, rejecting unbound entries.  A draw that finds no
 * bound entry in EPOT_MAX_ATTEMPTS tries returns ASOHF_ERR_TIMEOUT (the
 * reference would loop on). */
static int compute_epot_sampled(const orc_store *st, int64_t konta, int64_t konta2, const hwork *w,
                                int max_part_dsum, float *epot, int64_t *most_bound)
{
  int64_t nsa = (int64_t)((float)max_part_dsum / 1.4f);
  int64_t nsb = (int64_t)(0.01f * (float)konta2);
  int64_t nsample = nsa > nsb ? nsa : nsb;
  int64_t npairs = 0;
  double epot8 = 0.0;
  float largest_energy = 1000000.0f;
  int64_t mb = w->lip[1];
  uint32_t key_row = mix2(g_epot_seed, (uint32_t)g_row);
  for (int64_t jjj = 1; jjj <= nsample; jjj++) {
    uint32_t ko = mix2(key_row, (uint32_t)jjj);
    int64_t j = -1;
    for (uint32_t a = 0; a < EPOT_MAX_ATTEMPTS; a++) {
      int64_t c = epot_draw(ko, 0u, a, konta);
      if (w->contadm[c] == 0) { j = c; break; }
    }
    if (j < 0) return ASOHF_ERR_TIMEOUT;
    int64_t jj = w->lip[j];
    float x1 = st->x[jj], y1 = st->y[jj], z1 = st->z[jj], m1 = st->m[jj];
    double bas = 0.0;
    for (int64_t kkk = 1; kkk <= nsample; kkk++) {
      int64_t kq = -1;
      for (uint32_t a = 0; a < EPOT_MAX_ATTEMPTS; a++) {
        int64_t c = epot_draw(ko, (uint32_t)kkk, a, konta);
        if (w->contadm[c] == 0 && c != j) { kq = c; break; }
      }
      if (kq < 0) return ASOHF_ERR_TIMEOUT;
      int64_t kk = w->lip[kq];
      float ax = x1 - st->x[kk], ay = y1 - st->y[kk], az = z1 - st->z[kk];
      float m2 = st->m[kk];
      npairs++;
      bas = bas - (double)(m1 * m2 / sqrtf(ax * ax + ay * ay + az * az));
    }
    epot8 = epot8 + bas;
    bas = bas / (double)m1;
    if (bas < (double)largest_energy) {
      largest_energy = (float)bas;
      mb = jj;
    }
  }
  int64_t npairs_total = konta * (konta - 1) / 2;
  epot8 = epot8 * (double)((float)npairs_total / (float)npairs);
  *epot = (float)epot8;
  *most_bound = mb;
  return 0;
}

/* COMPUTE_EPOT (haloes_particles.f:1494-1628): direct summation below
 * MAX_PART_DSUM bound entries, the seeded sampling estimator from there on. */
static int compute_epot(const orc_store *st, int64_t konta, int64_t konta2, const hwork *w,
                        int max_part_dsum, float *epot, int64_t *most_bound)
{
  if (!(konta2 < max_part_dsum))
    return compute_epot_sampled(st, konta, konta2, w, max_part_dsum, epot, most_bound);
  double epot8 = 0.0;
  double *ep = (double *)calloc((size_t)(konta + 1), sizeof(double));
  for (int64_t j = 1; j <= konta; j++) {
    if (w->contadm[j] == 1) continue;
    int64_t jj = w->lip[j];
    float x1 = st->x[jj], y1 = st->y[jj], z1 = st->z[jj], m1 = st->m[jj];
    for (int64_t q = j + 1; q <= konta; q++) {
      if (w->contadm[q] == 1) continue;
      int64_t kk = w->lip[q];
      float ax = x1 - st->x[kk], ay = y1 - st->y[kk], az = z1 - st->z[kk];
      float m2 = st->m[kk];
      double bas = (double)(-m1 * m2 / sqrtf(ax * ax + ay * ay + az * az));
      ep[j] = ep[j] + bas;
      ep[q] = ep[q] + bas;
      epot8 = epot8 + bas;
    }
  }
  int64_t best = 1;
  for (int64_t j = 1; j <= konta; j++) {
    if (w->contadm[j] == 1) ep[j] = 100000.0;
    else ep[j] = ep[j] / (double)st->m[w->lip[j]];
  }
  for (int64_t j = 2; j <= konta; j++)
    if (ep[j] < ep[best]) best = j;
  *most_bound = w->lip[best];
  *epot = (float)epot8;
  free(ep);
  return 0;
}

/* DIAGONALISE (num.f:2-116): Jacobi rotations in REAL*8.  input_matrix is
 * column-major 3x3 REAL*4. */
void orc_diagonalise(const float *in, float *eig)
{
  const int n = 3;
  double a[3][3], e[3], aux1[3], aux2[3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) a[i][j] = (double)in[j * 3 + i];
  for (int i = 0; i < n; i++) { aux1[i] = a[i][i]; e[i] = aux1[i]; aux2[i] = 0.0; }
  double sum_el = 0.0;
  for (int i = 0; i < n; i++)
    for (int j = i; j < n; j++) sum_el = sum_el + fabs(a[i][j]);
  for (int it = 1; it <= 100; it++) {
    double suma = 0.0;
    for (int i = 0; i < n - 1; i++)
      for (int j = i + 1; j < n; j++) suma = suma + fabs(a[i][j]);
    if (suma < (double)1.e-4f * sum_el) break;
    double upper = (it < 4) ? 0.2 * (suma * suma) : 0.0;
    for (int p = 0; p < n - 1; p++) {
      for (int q = p + 1; q < n; q++) {
        double var1 = 100.0 * fabs(a[p][q]);
        if (it > 4 && fabs(e[p]) + var1 == fabs(e[p]) && fabs(e[q]) + var1 == fabs(e[q])) {
          a[p][q] = 0.0;
        } else if (fabs(a[p][q]) > upper) {
          double var2 = e[q] - e[p], t;
          if (fabs(var2) + var1 == fabs(var2)) {
            t = a[p][q] / var2;
          } else {
            double th = 0.5 * var2 / a[p][q];
            t = 1.0 / (fabs(th) + sqrt(1.0 + th * th));
            if (th < 0.0) t = -t;
          }
          double c = 1.0 / sqrt(1.0 + t * t);
          double s = t * c;
          double tau = s / (1.0 + c);
          var2 = t * a[p][q];
          aux2[p] = aux2[p] - var2;
          aux2[q] = aux2[q] + var2;
          e[p] = e[p] - var2;
          e[q] = e[q] + var2;
          a[p][q] = 0.0;
          for (int j = 0; j < p; j++) {
            double v1 = a[j][p], v2 = a[j][q];
            a[j][p] = v1 - s * (v2 + v1 * tau);
            a[j][q] = v2 + s * (v1 - v2 * tau);
          }
          for (int j = p + 1; j < q; j++) {
            double v1 = a[p][j], v2 = a[j][q];
            a[p][j] = v1 - s * (v2 + v1 * tau);
            a[j][q] = v2 + s * (v1 - v2 * tau);
          }
          for (int j = q + 1; j < n; j++) {
            double v1 = a[p][j], v2 = a[q][j];
            a[p][j] = v1 - s * (v2 + v1 * tau);
            a[q][j] = v2 + s * (v1 - v2 * tau);
          }
        }
      }
    }
    for (int i = 0; i < n; i++) { aux1[i] = aux1[i] + aux2[i]; e[i] = aux1[i]; aux2[i] = 0.0; }
  }
  for (int i = 0; i < n; i++) eig[i] = (float)e[i];
}

/* SORT_EIGEN (num.f:119-147). */
void orc_sort_eigen(float *e, int n)
{
  for (int ii = 0; ii < n - 1; ii++) {
    int kk = ii;
    float valor = e[ii];
    for (int jj = ii + 1; jj < n; jj++)
      if (e[jj] >= valor) { kk = jj; valor = e[jj]; }
    if (kk != ii) { e[kk] = e[ii]; e[ii] = valor; }
  }
}

/* Bound-particle properties, profiles and ID list of one halo: the block
 * "GUARDAMOS LAS PARTICULAS LIGADAS" (haloes_particles.f:1187-1353 and
 * substructure.f:1478-1660).  `sym` selects the halo version, which copies
 * the lower triangle of the inertia tensor to the upper one. */
static int properties(const orc_store *st, const asohf_consts *k, asohf_catalogue *cat,
                      int I, hwork *w, int64_t konta, float rshell, float cx, float cy,
                      float cz, float cmx, float cmy, float cmz, int sym, ilist *ids)
{
  int i0 = I - 1;
  float norma = st->norma;
  int64_t konta2 = 0;
  double basmas = 0.0, vr = 0.0, basx = 0.0, basy = 0.0, basz = 0.0;
  double inertia8[3][3] = {{0}};
  double sigma_halo = 0.0, ekin = 0.0;
  cat->dmpclus[i0] = 0;
  float vcmx = cat->vx[i0], vcmy = cat->vy[i0], vcmz = cat->vz[i0];
  cat->vmaxclus[i0] = -1.0f;
  int64_t each_prof = konta / NB;
  if (each_prof == 0) each_prof = 1;
  for (int64_t j = 1; j <= konta; j++) {
    if (w->contadm[j] != 0) continue;
    int64_t jj = w->lip[j];
    float bv[3] = {st->x[jj] - cx, st->y[jj] - cy, st->z[jj] - cz};
    float aadm = sqrtf(bv[0] * bv[0] + bv[1] * bv[1] + bv[2] * bv[2]);
    if (aadm <= rshell) {
      konta2++;
      basmas = basmas + (double)(st->m[jj] / norma);
      if (j % each_prof == 0 && j / each_prof <= NB) {
        int64_t b = j / each_prof;
        cat->profiles[(size_t)i0 * 2 * NB + 0 * NB + (b - 1)] = aadm;
        cat->profiles[(size_t)i0 * 2 * NB + 1 * NB + (b - 1)] = (float)(basmas * norma * k->um);
      }
      float bc[3] = {st->x[jj] - cmx, st->y[jj] - cmy, st->z[jj] - cmz};
      float bvc[3] = {st->vx[jj] - vcmx, st->vy[jj] - vcmy, st->vz[jj] - vcmz};
      float vvv2 = bvc[0] * bvc[0] + bvc[1] * bvc[1] + bvc[2] * bvc[2];
      float mp = st->m[jj];
      sigma_halo = sigma_halo + (double)vvv2;
      ekin = ekin + (double)(mp * vvv2);
      basx = basx + (double)(mp * (bc[1] * bvc[2] - bc[2] * bvc[1]));
      basy = basy + (double)(mp * (bc[2] * bvc[0] - bc[0] * bvc[2]));
      basz = basz + (double)(mp * (bc[0] * bvc[1] - bc[1] * bvc[0]));
      for (int jy = 0; jy < 3; jy++)
        for (int ix = 0; ix < 3; ix++)
          inertia8[ix][jy] = inertia8[ix][jy] + (double)(mp * bc[ix] * bc[jy]);
      if (vvv2 > cat->vmaxclus[i0]) cat->vmaxclus[i0] = vvv2;
      if (aadm != 0.0f) {
        float aa = (bv[0] / aadm) * bvc[0] + (bv[1] / aadm) * bvc[1] + (bv[2] / aadm) * bvc[2];
        vr = vr + (double)(aa * mp);
      }
    } else {
      w->contadm[j] = 1;
    }
  }
  cat->dmpclus[i0] = (int32_t)konta2;
  if (konta2 < k->min_num_part) { cat->realclus[i0] = 0; return 0; }
  if (k->flag_wdm == 1 || k->var > 1) {
    for (int64_t j = 1; j <= konta; j++)
      if (w->contadm[j] == 0) il_push(ids, st->id[w->lip[j]]);
  }
  if (k->do_compute_energies == 1) {
    float epot;
    int64_t mb;
    int rc = compute_epot(st, konta, konta2, w, k->max_part_dsum, &epot, &mb);
    if (rc) return rc;
    double gcons = 4.301e-9f;
    epot = (float)((double)epot * (double)(k->um * k->um) * gcons);
    float ekin4 = (float)(0.5 * ekin * (double)k->um * (double)(k->uv * k->uv));
    cat->kinetic_e[i0] = ekin4;
    cat->potential_e[i0] = epot * (1.0f + k->zeta);
    cat->iplip[i0] = st->id[mb];
  } else {
    cat->potential_e[i0] = 0.0f;
    cat->iplip[i0] = st->id[w->lip[1]];
  }
  double den = basmas * (double)norma;
  cat->angularm[i0 * 3 + 0] = (float)(basx * (double)k->uv / den);
  cat->angularm[i0 * 3 + 1] = (float)(basy * (double)k->uv / den);
  cat->angularm[i0 * 3 + 2] = (float)(basz * (double)k->uv / den);
  cat->mean_vr[i0] = (float)(vr / den * (double)k->uv);
  float inertia[9]; /* column-major */
  for (int jy = 0; jy < 3; jy++)
    for (int ix = 0; ix < 3; ix++) inertia[jy * 3 + ix] = (float)(inertia8[ix][jy] / den);
  if (sym) {
    inertia[1 * 3 + 0] = inertia[0 * 3 + 1]; /* INERTIA(1,2)=INERTIA(2,1) */
    inertia[2 * 3 + 0] = inertia[0 * 3 + 2]; /* INERTIA(1,3)=INERTIA(3,1) */
    inertia[2 * 3 + 1] = inertia[1 * 3 + 2]; /* INERTIA(2,3)=INERTIA(3,2) */
  }
  float *it = cat->inertia_tensor + (size_t)i0 * 6;
  it[0] = inertia[0];         /* (1,1) */
  it[1] = inertia[1 * 3 + 0]; /* (1,2) */
  it[2] = inertia[2 * 3 + 0]; /* (1,3) */
  it[3] = inertia[1 * 3 + 1]; /* (2,2) */
  it[4] = inertia[2 * 3 + 1]; /* (2,3) */
  it[5] = inertia[2 * 3 + 2]; /* (3,3) */
  cat->velocity_dispersion[i0] = (float)(sqrt(sigma_halo / (double)(float)konta2) * (double)k->uv);
  cat->vmaxclus[i0] = sqrtf(cat->vmaxclus[i0]) * k->uv;
  float be[3] = {0.0f, 0.0f, 0.0f};
  if (cat->dmpclus[i0] >= k->min_num_part) {
    orc_diagonalise(inertia, be);
    orc_sort_eigen(be, 3);
  }
  for (int ii = 0; ii < 3; ii++) cat->eigenval[(size_t)i0 * 3 + ii] = sqrtf(5.0f * be[ii]);
  return 0;
}

/* Flags/outputs of the SO walk for one overdensity threshold. */
static inline void so_hit(int *flag, float delta2, float thr, float vol, float rote, float um,
                          float d, int64_t j, int64_t jjcore, float *mo, float *ro)
{
  if (*flag == 0) margin_add(1, near_thr(delta2, thr));
  if (*flag == 0 && delta2 <= thr) {
    *mo = delta2 * vol * rote * um;
    *ro = d;
    *flag = 1;
    if (j == jjcore + 1) { *mo = -1.0f; *ro = -1.0f; }
  }
}

/* One halo of HALOFIND_PARTICLES (haloes_particles.f:740-1353). */
static int halofind_one(const orc_store *st, const asohf_consts *k, const asohf_mesh *mesh,
                        asohf_catalogue *cat, int I, ilist *ids)
{
  int i0 = I - 1;
  g_row = i0;
  int kk_entero = cat->realclus[i0];
  if (kk_entero == 0) return 0;
  float pi = k->pi, rote = k->rote, rete = k->rete, fdm = k->fdm, um = k->um;
  float minoverdens = fminf(200.0f, k->contrastec) * fdm;
  float norma = st->norma;
  float xldom = -k->lado0 / 2.0f;
  /* level used for recentering */
  int ipatch = cat->patchclus[i0];
  int nl = mesh ? mesh->nl : 0;
  int irr, acc = mesh ? mesh->npatch[0] : 0;
  for (irr = 1; irr <= nl; irr++) {
    int lo = acc + 1, hi = acc + mesh->npatch[irr];
    acc = hi;
    if (lo <= ipatch && ipatch <= hi) break;
  }
  float cx = cat->clusrx[i0], cy = cat->clusry[i0], cz = cat->clusrz[i0];
  recenter(st, k, &cx, &cy, &cz, cat->radio[i0], k->dx / powf(2.0f, (float)irr));
  cat->clusrx[i0] = cx;
  cat->clusry[i0] = cy;
  cat->clusrz[i0] = cz;

  /* radius growth (haloes_particles.f:777-849) */
  float rclus = cat->radio[i0];
  float delta2 = 100.0f * minoverdens;
  double masadm = 0.0;
  ilist lip = {0};
  int64_t near_r = 0;
  while (delta2 > 0.99f * minoverdens) {
    lip.n = 0;
    masadm = 0.0;
    near_r = 0;
    float bas = -1.0f;
    int64_t lo, hi;
    orc_find_particle_indices(cx, rclus, xldom, k->dx, k->nx, st->ndmpart_x, &lo, &hi);
    for (int64_t j = lo; j <= hi; j++) {
      float aadm = dist3(st, j - 1, cx, cy, cz);
      near_r += near_thr(aadm, rclus);
      if (aadm < rclus) {
        il_push(&lip, j - 1);
        masadm = masadm + (double)st->m[j - 1];
        bas = fmaxf(bas, aadm);
      }
    }
    float den = rote * (rete * rete * rete) * (4.0f * pi / 3.0f) * (bas * bas * bas);
    delta2 = (float)(masadm / (double)den);
    if (delta2 > 0.9f * minoverdens) rclus = 1.25f * rclus;
  }
  margin_add(0, near_r);
  int64_t konta = lip.n;
  if (masadm <= 0.0 || konta == 0) {
    cat->realclus[i0] = 0;
    free(lip.v);
    return 0;
  }
  hwork w;
  hw_alloc(&w, konta > 12 ? konta : 12);
  for (int64_t j = 1; j <= konta; j++) { w.lip[j] = lip.v[j - 1]; w.contadm[j] = 0; }
  free(lip.v);
  int64_t konta2 = 0, idx_vir = 0;
  int64_t contaerr = konta;
  for (int64_t j = 0; j <= w.cap + 1; j++) w.dista[j] = 0.0f;
  reordenar(st, konta, cx, cy, cz, &w, &konta2, 1, &idx_vir);
  float ref_max = w.dista[konta2];
  cat->radio[i0] = rclus;
  cat->masa[i0] = (float)(masadm * (double)um);
  cat->dmpclus[i0] = (int32_t)konta;
  idx_vir = find_idx_vir(st, &w, rote, rete, pi, k->contrastec * fdm, idx_vir);
  if (idx_vir < 0) { hw_free(&w); return ASOHF_ERR_NOT_PREFOUND_VIRIAL; }

  float cm[3], vcm[3], masa2;
  centromasas(st, idx_vir, &w, cm, vcm, &masa2);
  cat->clusrxcm[i0] = cm[0]; cat->clusrycm[i0] = cm[1]; cat->clusrzcm[i0] = cm[2];
  cat->vx[i0] = vcm[0]; cat->vy[i0] = vcm[1]; cat->vz[i0] = vcm[2];
  hstate h = {&cat->radio[i0], &cat->masa[i0], &cat->clusrxcm[i0], &cat->clusrycm[i0],
              &cat->clusrzcm[i0], &cat->vx[i0], &cat->vy[i0], &cat->vz[i0], &cat->realclus[i0]};
  int fac = 0;
  while (contaerr > 0 || fac < 3) {
    fac++;
    int64_t prev = konta2;
    unbinding8(st, k, fac, ref_max, &w, konta2, idx_vir, &h);
    reordenar(st, konta, cx, cy, cz, &w, &konta2, 0, &idx_vir);
    ref_max = w.dista[konta2];
    contaerr = prev - konta2;
  }
  fac = 0;
  contaerr = konta2;
  while (contaerr > 0 || fac < 4) {
    fac++;
    int64_t prev = konta2;
    unbinding_sigma(st, k, fac, &w, konta2, idx_vir, &h);
    reordenar(st, konta, cx, cy, cz, &w, &konta2, 0, &idx_vir);
    ref_max = w.dista[konta2];
    contaerr = prev - konta2;
  }
  if (konta2 < k->min_num_part) {
    cat->realclus[i0] = 0;
    hw_free(&w);
    return 0;
  }
  /* SO walk (haloes_particles.f:973-1182) */
  double bas8 = 0.0, bvx = 0.0, bvy = 0.0, bvz = 0.0;
  float bas1 = -1.0f;
  int f2500c = 0, f500c = 0, f200c = 0, f2500m = 0, f500m = 0, f200m = 0, fvir = 0, salida = 0;
  int64_t ncapas = 0;
  float rshell = 0.0f;
  int64_t jjcore = (int64_t)fmaxf(10.0f, (float)konta2 / 100.0f);
  int64_t j;
  for (j = 1; j <= jjcore; j++) {
    int64_t jj = w.lip[j];
    float mn = st->m[jj] / norma;
    bas8 = bas8 + (double)mn;
    bvx = bvx + (double)(mn * st->vx[jj]);
    bvy = bvy + (double)(mn * st->vy[jj]);
    bvz = bvz + (double)(mn * st->vz[jj]);
  }
  float c2500 = 2500.0f / k->omegaz * fdm, c500 = 500.0f / k->omegaz * fdm, c200 = 200.0f / k->omegaz * fdm;
  float m2500 = 2500.0f * fdm, m500 = 500.0f * fdm, m200 = 200.0f * fdm;
  float cvir = k->contrastec * fdm;
  int64_t jvir_min = (int64_t)(0.1f * (float)konta2);
  for (j = jjcore + 1; j <= konta2; j++) {
    int64_t jj = w.lip[j];
    float d = w.dista[j];
    float dr = d * rete;
    float vol = pi * (4.0f / 3.0f) * (dr * dr * dr);
    float mn = st->m[jj] / norma;
    bas8 = bas8 + (double)mn;
    bvx = bvx + (double)(mn * st->vx[jj]);
    bvy = bvy + (double)(mn * st->vy[jj]);
    bvz = bvz + (double)(mn * st->vz[jj]);
    delta2 = (float)((double)norma * bas8 / (double)vol / (double)rote);
    float bas2 = (float)(bas8 / (double)d);
    if (bas2 > bas1) {
      cat->vcmax[i0] = bas2;
      cat->mcmax[i0] = (float)bas8;
      cat->rcmax[i0] = d;
      bas1 = bas2;
    }
    so_hit(&f2500c, delta2, c2500, vol, rote, um, d, j, jjcore, &cat->m2500c[i0], &cat->r2500c[i0]);
    so_hit(&f500c, delta2, c500, vol, rote, um, d, j, jjcore, &cat->m500c[i0], &cat->r500c[i0]);
    so_hit(&f200c, delta2, c200, vol, rote, um, d, j, jjcore, &cat->m200c[i0], &cat->r200c[i0]);
    so_hit(&f2500m, delta2, m2500, vol, rote, um, d, j, jjcore, &cat->m2500m[i0], &cat->r2500m[i0]);
    so_hit(&f500m, delta2, m500, vol, rote, um, d, j, jjcore, &cat->m500m[i0], &cat->r500m[i0]);
    so_hit(&f200m, delta2, m200, vol, rote, um, d, j, jjcore, &cat->m200m[i0], &cat->r200m[i0]);
    if (fvir == 0 && j > jvir_min) margin_add(1, near_thr(delta2, cvir));
    if (fvir == 0 && delta2 <= cvir && j > jvir_min) {
      salida = 1;
      fvir = 1;
      bas8 = bas8 - (double)mn;
      bvx = bvx - (double)(mn * st->vx[jj]);
      bvy = bvy - (double)(mn * st->vy[jj]);
      bvz = bvz - (double)(mn * st->vz[jj]);
      cat->masa[i0] = (float)(bas8 * (double)norma * (double)um);
      vol = (float)(((double)norma * bas8) / (double)(k->contrastec * fdm * rote));
      cat->radio[i0] = powf((3.0f * vol) / (4.0f * pi), 1.0f / 3.0f) / rete;
      cat->vx[i0] = (float)(bvx / bas8);
      cat->vy[i0] = (float)(bvy / bas8);
      cat->vz[i0] = (float)(bvz / bas8);
      ncapas = j - 1;
      rshell = cat->radio[i0];
    }
    if (salida == 1 && f200m == 1) break;
  }
  {
    float bas = cat->vcmax[i0] * norma * k->cgr / rete;
    cat->vcmax[i0] = sqrtf(bas) * k->uv;
    cat->mcmax[i0] = cat->mcmax[i0] * norma * um;
  }
  if (kk_entero == -1 && salida != 1) {
    salida = 1;
    fvir = 1;
    cat->masa[i0] = (float)(bas8 * (double)norma * (double)um);
    float vol = (float)(((double)norma * bas8) / (double)(k->contrastec * fdm * rote));
    cat->radio[i0] = powf((3.0f * vol) / (4.0f * pi), 1.0f / 3.0f) / rete;
    cat->vx[i0] = (float)(bvx / bas8);
    cat->vy[i0] = (float)(bvy / bas8);
    cat->vz[i0] = (float)(bvz / bas8);
    ncapas = j - 1;
    rshell = cat->radio[i0];
    if (f200m == 0) {
      cat->m200m[i0] = cat->masa[i0];
      cat->r200m[i0] = cat->radio[i0] * powf(k->contrastec / 200.0f, 1.0f / 3.0f);
    }
  }
  /* bound particles */
  konta = ncapas;
  if (konta < k->min_num_part) {
    cat->realclus[i0] = 0;
    hw_free(&w);
    return 0;
  }
  int rc = properties(st, k, cat, I, &w, konta, rshell, cx, cy, cz, cm[0], cm[1], cm[2], 1, ids);
  /* CMX.. of the property loop are the values CENTROMASAS_PART returned
   * before unbinding (haloes_particles.f:887-889): unbinding updates the
   * catalogue, not those locals. */
  hw_free(&w);
  return rc;
}

/* Concatenation of the per-halo ID lists in halo order
 * (haloes_particles.f:1377-1408). */
static int concat_ids(asohf_catalogue *cat, int low1, int low2, ilist *ids, int32_t *pph,
                      int64_t pph_cap, int64_t *pph_len)
{
  int64_t j = 0;
  for (int i = 1; i < low1; i++)
    if (cat->realclus[i - 1] != 0 && cat->indcs[(i - 1) * 2 + 1] > j) j = cat->indcs[(i - 1) * 2 + 1];
  int rc = 0;
  for (int i = low1; i <= low2; i++) {
    if (cat->realclus[i - 1] == 0) {
      cat->indcs[(i - 1) * 2] = -1;
      cat->indcs[(i - 1) * 2 + 1] = -1;
      continue;
    }
    cat->indcs[(i - 1) * 2] = (int32_t)(j + 1);
    ilist *l = &ids[i - low1];
    for (int64_t q = 0; q < l->n; q++) {
      if (j < pph_cap) pph[j] = (int32_t)l->v[q];
      else rc = ASOHF_ERR_CAPACITY;
      j++;
    }
    cat->indcs[(i - 1) * 2 + 1] = (int32_t)j;
  }
  *pph_len = j;
  return rc;
}

int orc_halofind_particles(const orc_store *st, const asohf_consts *k, const asohf_mesh *mesh,
                           asohf_catalogue *cat, int low1, int low2, int32_t *pph,
                           int64_t pph_cap, int64_t *pph_len, int nthreads)
{
  int nh = low2 - low1 + 1;
  if (nh <= 0) { *pph_len = 0; return 0; }
  ilist *ids = (ilist *)calloc((size_t)nh, sizeof(ilist));
  int rc = 0;
#pragma omp parallel for schedule(dynamic) num_threads(nthreads > 0 ? nthreads : 1)
  for (int i = low1; i <= low2; i++) {
    int r = halofind_one(st, k, mesh, cat, i, &ids[i - low1]);
    if (r) {
#pragma omp critical
      rc = r;
    }
  }
  int rc2 = 0;
  if (k->flag_wdm == 1 || k->var > 1) rc2 = concat_ids(cat, low1, low2, ids, pph, pph_cap, pph_len);
  else *pph_len = 0;
  for (int i = 0; i < nh; i++) free(ids[i].v);
  free(ids);
  return rc ? rc : rc2;
}

/* ------------------------------------------------------------------ */
/* Jacobi equation (substructure.f:1058-1092). */
static inline double eq_jacobi(double basx, double basy)
{
  double t = 1.0 - basx;
  return 1.0 / (t * t) - 1.0 - basy / (basx * basx) + (1.0 + basy) * basx;
}

/* One subhalo of SUBSTRUCTURE_PARTICLES (substructure.f:876-1660). */
static int substructure_one(const orc_store *st, const asohf_consts *k, const asohf_mesh *mesh,
                            asohf_catalogue *cat, int I, ilist *ids)
{
  int i0 = I - 1;
  g_row = i0;
  int kk_entero = cat->realclus[i0];
  if (kk_entero == 0) return 0;
  float pi = k->pi, rote = k->rote, rete = k->rete, um = k->um;
  float norma = st->norma;
  float xldom = -k->lado0 / 2.0f;
  int ipatch = cat->patchclus[i0];
  int nl = mesh ? mesh->nl : 0;
  int irr, acc = mesh ? mesh->npatch[0] : 0;
  for (irr = 1; irr <= nl; irr++) {
    int lo = acc + 1, hi = acc + mesh->npatch[irr];
    acc = hi;
    if (lo <= ipatch && ipatch <= hi) break;
  }
  float cx = cat->clusrx[i0], cy = cat->clusry[i0], cz = cat->clusrz[i0];
  recenter(st, k, &cx, &cy, &cz, cat->rsub[i0], k->dx / powf(2.0f, (float)irr));
  cat->clusrx[i0] = cx;
  cat->clusry[i0] = cy;
  cat->clusrz[i0] = cz;
  /* host characterisation (substructure.f:933-983) */
  int ih = cat->realclus[i0] - 1;
  float mhost = (cat->realclus[ih] == -1) ? cat->masa[ih] : cat->msub[ih];
  float hx = cat->clusrx[ih] - cx, hy = cat->clusry[ih] - cy, hz = cat->clusrz[ih] - cz;
  float disthost = sqrtf(hx * hx + hy * hy + hz * hz);
  const float *p1 = cat->profiles + (size_t)ih * 2 * NB;     /* PROFILES(:,1,host) */
  const float *p2 = p1 + NB;                                  /* PROFILES(:,2,host) */
  int nbp = NB;
  int jj;
  for (jj = 1; jj <= NB; jj++)
    if (p1[jj - 1] == 0.0f) { nbp = jj - 1; break; }
  for (jj = 1; jj <= nbp; jj++)
    if (p1[jj - 1] > disthost) break;
  if (jj == 1) {
    float q = disthost / p1[0];
    mhost = p2[0] * (q * q * q);
  } else if (jj <= nbp) {
    float a1 = p1[jj - 2], a2 = p1[jj - 1];
    mhost = p2[jj - 2] + (p2[jj - 1] - p2[jj - 2]) *
                             (disthost * disthost * disthost - a1 * a1 * a1) /
                             (a2 * a2 * a2 - a1 * a1 * a1);
  } else {
    mhost = p2[nbp - 1];
  }
  /* Jacobi radius (substructure.f:988-1127) */
  double masadm = 0.0;
  hwork w = {0};
  int64_t konta = 0, konta2 = 0, useless = 0;
  int flag_jacobi = 0;
  float rclus = 2.0f * cat->rsub[i0];
  int64_t near_r = 0, near_jac = 0;
  while (flag_jacobi == 0) {
    ilist lip = {0};
    int64_t lo, hi;
    near_r = 0;
    near_jac = 0;
    orc_find_particle_indices(cx, rclus, xldom, k->dx, k->nx, st->ndmpart_x, &lo, &hi);
    for (int64_t j = lo; j <= hi; j++) {
      float aadm = dist3(st, j - 1, cx, cy, cz);
      near_r += near_thr(aadm, rclus);
      if (aadm < rclus) il_push(&lip, j - 1);
    }
    konta = lip.n;
    if (w.lip) hw_free(&w);
    int64_t cap = konta;
    int64_t minj0 = 10 > konta / 50 ? 10 : konta / 50;
    if (cap < minj0 + 1) cap = minj0 + 1;
    hw_alloc(&w, cap);
    for (int64_t j = 1; j <= konta; j++) { w.lip[j] = lip.v[j - 1]; w.contadm[j] = 0; }
    free(lip.v);
    reordenar(st, konta, cx, cy, cz, &w, &konta2, 1, &useless);
    masadm = 0.0;
    int64_t j_jacobi = -1;
    int64_t minj = 10 > konta / 50 ? 10 : konta / 50;
    int64_t j;
    for (j = 1; j <= konta; j++) {
      masadm = masadm + (double)st->m[w.lip[j]];
      double mu = masadm * (double)um;
      double tid = pow(mu / (mu + (double)(3.0f * mhost)), (double)(1.0f / 3.0f));
      double eq = (double)(w.dista[j] / disthost) - tid;
      if (j > minj) near_jac += near_thr(tid + eq, tid);
      if (eq > 0.0 && j > minj) { j_jacobi = j; break; }
    }
    if (j_jacobi == -1) j_jacobi = konta;
    double basx = (double)(w.dista[j_jacobi] / disthost);
    double basy = masadm * (double)um / (double)mhost;
    double eq = eq_jacobi(basx, basy);
    int dir = -1;
    /* ABS(EQ_JACOBI_R).LT.0.D01 compares against 0.0D+01 = 0: never true */
    if (fabs(eq) < 0.0) {
      flag_jacobi = 1;
    } else {
      dir = -1;
      if (eq < 0.0) dir = 1;
      if (dir == 1) {
        for (j = j_jacobi + 1; j <= konta; j++) {
          basx = (double)(w.dista[j] / disthost);
          masadm = masadm + (double)st->m[w.lip[j]];
          basy = masadm * (double)um / (double)mhost;
          eq = eq_jacobi(basx, basy);
          if (eq > 0.0) { j_jacobi = j; flag_jacobi = 1; break; }
        }
      } else {
        for (j = j_jacobi - 1; j >= minj; j--) {
          basx = (double)(w.dista[j] / disthost);
          masadm = masadm - (double)st->m[w.lip[j + 1]];
          basy = masadm * (double)um / (double)mhost;
          eq = eq_jacobi(basx, basy);
          if (eq < 0.0) { j_jacobi = j; flag_jacobi = 1; break; }
        }
      }
    }
    if (flag_jacobi == 0) {
      if (dir == 1) rclus = 1.5f * rclus;
      else { j_jacobi = minj; flag_jacobi = 1; }
    }
    if (flag_jacobi == 1) {
      rclus = w.dista[j_jacobi];
      cat->rsub[i0] = rclus;
      cat->msub[i0] = (float)(masadm * (double)um);
      for (int64_t q = 1; q <= konta; q++) w.contadm[q] = 1;
      for (int64_t q = 1; q <= j_jacobi && q <= w.cap; q++) w.contadm[q] = 0;
      konta = j_jacobi;
    }
  }
  margin_add(0, near_r);
  margin_add(1, near_jac);
  if (masadm <= 0.0 || konta < k->min_num_part) {
    cat->realclus[i0] = 0;
    hw_free(&w);
    return 0;
  }
  for (int64_t q = 1; q <= konta; q++) w.contadm[q] = 0;
  float cm[3], vcm[3], masa2;
  centromasas(st, konta, &w, cm, vcm, &masa2);
  cat->clusrxcm[i0] = cm[0]; cat->clusrycm[i0] = cm[1]; cat->clusrzcm[i0] = cm[2];
  cat->vx[i0] = vcm[0]; cat->vy[i0] = vcm[1]; cat->vz[i0] = vcm[2];
  cat->rsub[i0] = rclus;
  cat->msub[i0] = (float)(masadm * (double)um);
  cat->dmpclus[i0] = (int32_t)konta;
  int64_t contaerr = konta;
  for (int64_t q = 0; q <= w.cap + 1; q++) w.dista[q] = 0.0f;
  reordenar(st, konta, cx, cy, cz, &w, &konta2, 1, &useless);
  float ref_max = w.dista[konta2];
  hstate h = {&cat->rsub[i0], &cat->msub[i0], &cat->clusrxcm[i0], &cat->clusrycm[i0],
              &cat->clusrzcm[i0], &cat->vx[i0], &cat->vy[i0], &cat->vz[i0], &cat->realclus[i0]};
  int fac = 0;
  while (contaerr > 0 || fac < 3) {
    fac++;
    int64_t prev = konta2;
    useless = konta2;
    unbinding8(st, k, fac, ref_max, &w, konta2, useless, &h);
    reordenar(st, konta, cx, cy, cz, &w, &konta2, 0, &useless);
    ref_max = w.dista[konta2];
    contaerr = prev - konta2;
  }
  if (konta2 < k->min_num_part) { cat->realclus[i0] = 0; hw_free(&w); return 0; }
  fac = 0;
  contaerr = konta2;
  while (contaerr > 0 || fac < 4) {
    fac++;
    int64_t prev = konta2;
    useless = konta2;
    unbinding_sigma(st, k, fac, &w, konta2, useless, &h);
    reordenar(st, konta, cx, cy, cz, &w, &konta2, 0, &useless);
    ref_max = w.dista[konta2];
    contaerr = prev - konta2;
  }
  if (konta2 < k->min_num_part) { cat->realclus[i0] = 0; hw_free(&w); return 0; }
  /* Jacobi correction after unbinding (substructure.f:1241-1264) */
  int64_t ncapas = 0; /* NCAPAS is a shared array zeroed on entry */
  float rshell = 0.0f;
  {
    double m8 = (double)(cat->msub[i0] / um);
    double basx = (double)(w.dista[konta2] / disthost);
    double basy = m8 * (double)um / (double)mhost;
    double eq = eq_jacobi(basx, basy);
    if (eq > 0.0) {
      int64_t j;
      for (j = konta2; j >= 1; j--) {
        m8 = m8 - (double)st->m[w.lip[j]];
        basx = (double)(w.dista[j] / disthost);
        basy = m8 * (double)um / (double)mhost;
        eq = eq_jacobi(basx, basy);
        if (eq < 0.0) break;
      }
      cat->rsub[i0] = w.dista[j + 1];
      cat->msub[i0] = (float)(m8 * (double)um);
      konta2 = j;
      ncapas = j;
      rshell = w.dista[j]; /* J.EQ.KONTA2 always holds here */
    }
  }
  if (konta2 < k->min_num_part) { cat->realclus[i0] = 0; hw_free(&w); return 0; }
  /* SO walk without early exit (substructure.f:1293-1463) */
  double bas8 = 0.0, bvx = 0.0, bvy = 0.0, bvz = 0.0;
  float bas1 = -1.0f;
  int f2500c = 0, f500c = 0, f200c = 0, f2500m = 0, f500m = 0, f200m = 0, fvir = 0;
  int64_t jjcore = (int64_t)fmaxf(10.0f, (float)konta2 / 100.0f);
  int64_t j;
  for (j = 1; j <= jjcore; j++) {
    int64_t jp = w.lip[j];
    float mn = st->m[jp] / norma;
    bas8 = bas8 + (double)mn;
    bvx = bvx + (double)(mn * st->vx[jp]);
    bvy = bvy + (double)(mn * st->vy[jp]);
    bvz = bvz + (double)(mn * st->vz[jp]);
  }
  float c2500 = 2500.0f / k->omegaz, c500 = 500.0f / k->omegaz, c200 = 200.0f / k->omegaz;
  int64_t jvir_min = (int64_t)(0.1f * (float)konta2);
  for (j = jjcore + 1; j <= konta2; j++) {
    int64_t jp = w.lip[j];
    float d = w.dista[j];
    float dr = d * rete;
    float vol = pi * (4.0f / 3.0f) * (dr * dr * dr);
    float mn = st->m[jp] / norma;
    bas8 = bas8 + (double)mn;
    bvx = bvx + (double)(mn * st->vx[jp]);
    bvy = bvy + (double)(mn * st->vy[jp]);
    bvz = bvz + (double)(mn * st->vz[jp]);
    float delta2 = (float)((double)norma * bas8 / (double)vol / (double)rote);
    float bas2 = (float)(bas8 / (double)d);
    if (bas2 > bas1) {
      cat->vcmax[i0] = bas2;
      cat->mcmax[i0] = (float)bas8;
      cat->rcmax[i0] = d;
      bas1 = bas2;
    }
    so_hit(&f2500c, delta2, c2500, vol, rote, um, d, j, jjcore, &cat->m2500c[i0], &cat->r2500c[i0]);
    so_hit(&f500c, delta2, c500, vol, rote, um, d, j, jjcore, &cat->m500c[i0], &cat->r500c[i0]);
    so_hit(&f200c, delta2, c200, vol, rote, um, d, j, jjcore, &cat->m200c[i0], &cat->r200c[i0]);
    so_hit(&f2500m, delta2, 2500.0f, vol, rote, um, d, j, jjcore, &cat->m2500m[i0], &cat->r2500m[i0]);
    so_hit(&f500m, delta2, 500.0f, vol, rote, um, d, j, jjcore, &cat->m500m[i0], &cat->r500m[i0]);
    so_hit(&f200m, delta2, 200.0f, vol, rote, um, d, j, jjcore, &cat->m200m[i0], &cat->r200m[i0]);
    if (fvir == 0 && j > jvir_min) margin_add(1, near_thr(delta2, k->contrastec));
    if (fvir == 0 && delta2 <= k->contrastec && j > jvir_min) {
      fvir = 1;
      cat->masa[i0] = delta2 * vol * rote * um;
      cat->radio[i0] = d;
    }
  }
  if (fvir == 0) { cat->radio[i0] = 0.0f; cat->masa[i0] = 0.0f; }
  if (f2500c == 0) { cat->m2500c[i0] = 0.0f; cat->r2500c[i0] = 0.0f; }
  if (f2500m == 0) { cat->m2500m[i0] = 0.0f; cat->r2500m[i0] = 0.0f; }
  if (f500c == 0) { cat->m500c[i0] = 0.0f; cat->r500c[i0] = 0.0f; }
  if (f500m == 0) { cat->m500m[i0] = 0.0f; cat->r500m[i0] = 0.0f; }
  if (f200c == 0) { cat->m200c[i0] = 0.0f; cat->r200c[i0] = 0.0f; }
  if (f200m == 0) { cat->m200m[i0] = 0.0f; cat->r200m[i0] = 0.0f; }
  cat->vx[i0] = (float)(bvx / bas8);
  cat->vy[i0] = (float)(bvy / bas8);
  cat->vz[i0] = (float)(bvz / bas8);
  {
    float bas = cat->vcmax[i0] * norma * k->cgr / rete;
    cat->vcmax[i0] = sqrtf(bas) * k->uv;
    cat->mcmax[i0] = cat->mcmax[i0] * norma * um;
  }
  int rc = properties(st, k, cat, I, &w, ncapas, rshell, cx, cy, cz, cm[0], cm[1], cm[2], 0, ids);
  hw_free(&w);
  return rc;
}

int orc_substructure_particles(const orc_store *st, const asohf_consts *k,
                               const asohf_mesh *mesh, asohf_catalogue *cat, int ir,
                               const int32_t *subs_lev, int32_t *pph, int64_t pph_cap,
                               int64_t *pph_len, int nthreads)
{
  int low1 = 1, low2 = 0;
  for (int q = 0; q < ir; q++) low1 += subs_lev[q];
  for (int q = 0; q <= ir; q++) low2 += subs_lev[q];
  int nh = low2 - low1 + 1;
  if (nh <= 0) { *pph_len = 0; return 0; }
  ilist *ids = (ilist *)calloc((size_t)nh, sizeof(ilist));
  int rc = 0;
#pragma omp parallel for schedule(dynamic) num_threads(nthreads > 0 ? nthreads : 1)
  for (int i = low1; i <= low2; i++) {
    int r = substructure_one(st, k, mesh, cat, i, &ids[i - low1]);
    if (r) {
#pragma omp critical
      rc = r;
    }
  }
  int rc2 = 0;
  if (k->flag_wdm == 1 || k->var > 1) rc2 = concat_ids(cat, low1, low2, ids, pph, pph_cap, pph_len);
  else *pph_len = 0;
  for (int i = 0; i < nh; i++) free(ids[i].v);
  free(ids);
  return rc ? rc : rc2;
}


/* Strict local maximum test of UBAS(ii, jj, kk) (1-based in the 6^3 block). */
static int ubas_peak(const float ub[6][6][6], int ii, int jj, int kk)
{
#define UB(i, j, k) ub[(k) - 1][(j) - 1][(i) - 1]
  const float c = UB(ii, jj, kk);
  const float dxp = UB(ii + 1, jj, kk) - c, dxm = c - UB(ii - 1, jj, kk);
  const float dyp = UB(ii, jj + 1, kk) - c, dym = c - UB(ii, jj - 1, kk);
  const float dzp = UB(ii, jj, kk + 1) - c, dzm = c - UB(ii, jj, kk - 1);
#undef UB
  return dxp < 0.0f && dyp < 0.0f && dzp < 0.0f && dxm > 0.0f && dym > 0.0f && dzm > 0.0f;
}

/* RECENTER_DENSITY_PEAK (haloes_grids.f:1099-1259): from level hlev+1 down,
 * the first patch of the level that strictly encloses the 6-cell box
 * around the current centre; in its 6^3 block the highest strict local
 * maximum among the inner 2^3 cells, then among the inner 4^3 (the second
 * scan always runs); the centre moves to that cell's RX/RY/RZ.  Stops at the
 * first level with no enclosing patch or no maximum.  *pipatch receives the
 * last patch used (1-based).  A block reaching outside the NAMRX^3 array
 * ends the descent (the Fortran would read past the patch there). */
static void recenter_grid_peak(float *c3, int hlev, const asohf_mesh *m, const float *u11, float dx, int *pipatch)
{
  const int bor = 2, na = ASOHF_NAMRX;
  const size_t pc = (size_t)na * na * na;
  const int32_t *pn[3] = {m->patchnx, m->patchny, m->patchnz};
  const float *pr[3] = {m->patchrx, m->patchry, m->patchrz};
  for (int ir = hlev + 1; ir <= m->nl; ir++) {
    const float dxpa = dx / powf(2.0f, (float)ir);
    float x1[3], x2[3], x3[3];
    for (int a = 0; a < 3; a++) {
      x1[a] = c3[a] - (1.0f + (float)bor) * dxpa;
      x2[a] = c3[a] + (1.0f + (float)bor) * dxpa;
    }
    int low1 = 0;
    for (int l = 0; l < ir; l++) low1 += m->npatch[l];
    const int low2 = low1 + m->npatch[ir];
    int found = -1;
    for (int i = low1; i < low2 && found < 0; i++) {
      int ok = 1;
      for (int a = 0; a < 3; a++) {
        const float lo = pr[a][i] - dxpa, hi = lo + (float)pn[a][i] * dxpa;
        ok &= lo < x1[a] && x2[a] < hi;
      }
      if (ok) found = i;
    }
    if (found < 0) break;
    int i1[3];
    int inside = 1;
    for (int a = 0; a < 3; a++) {
      x3[a] = pr[a][found] - dxpa;
      i1[a] = (int)((x1[a] - x3[a]) / dxpa + 0.5f) + 1;
      inside &= i1[a] >= 1 && i1[a] + 1 + 2 * bor <= na;
    }
    if (!inside) break;
    float ub[6][6][6];
    const float *u = u11 + (size_t)found * pc;
    for (int kk = 0; kk < 6; kk++)
      for (int jj = 0; jj < 6; jj++)
        for (int ii = 0; ii < 6; ii++)
          ub[kk][jj][ii] = u[((size_t)(i1[2] - 1 + kk) * na + (i1[1] - 1 + jj)) * na + (i1[0] - 1 + ii)];
    float cur = -100000.0f;
    int inmax[3] = {0, 0, 0};
    for (int pass = 0; pass < 2; pass++) {
      const int lo = pass == 0 ? 3 : 2, hi = pass == 0 ? 4 : 5;
      for (int kk = lo; kk <= hi; kk++)
        for (int jj = lo; jj <= hi; jj++)
          for (int ii = lo; ii <= hi; ii++)
            if (ubas_peak((const float(*)[6][6])ub, ii, jj, kk) && ub[kk - 1][jj - 1][ii - 1] > cur) {
              cur = ub[kk - 1][jj - 1][ii - 1];
              inmax[0] = ii;
              inmax[1] = jj;
              inmax[2] = kk;
            }
    }
    if (cur < 0.0f) break;
    for (int a = 0; a < 3; a++) {
      const int ix = i1[a] + inmax[a] - 1;
      c3[a] = (pr[a][found] - 0.5f * dxpa) + (float)(ix - 1) * dxpa;  /* RX(IX, I) */
    }
    *pipatch = found + 1;
  }
}

/* HALOFIND_GRID at the base level (haloes_grids.f:287-582).  With AMR levels
 * (mesh->nl > 0 and u11: NAMRX^3 per patch, patches in mesh order) each new
 * peak is first recentred on the finer levels (RECENTER_DENSITY_PEAK) and
 * dropped when the new centre lies inside a halo already found.  U1
 * (nx^3, IX fastest) is rho/rho_B; radx holds RADX(0..NX+1).  Peaks: cells
 * at least BOR=1 from the faces with U1 >= CONTRASTEC/6 that exceed their
 * six neighbours, taken in decreasing density (SORT_CELLS: ARGSORT of
 * 1/U1).  A peak not yet inside a halo (CONTA = 1) starts one and grows it
 * in spherical shells (R_EXT = 0.8 DX, then MAX(R_EXT + 0.2 DX, 1.05
 * R_EXT)) while its mean density exceeds CONTRASTEC*ROTE, zeroing CONTA
 * over its cells.  The shell sums are the sequential (K, J, I) order of the
 * reference's OpenMP reductions.  As in the reference, the centre-of-mass
 * numerators restart each shell from the box bound held in the same
 * variable (BASX = XCEN + R_EXT) while the denominator BASDELTA runs over
 * all shells.  OVERLAPPING (vol_solap_low) follows.  Returns the haloes
 * appended (NHALLEV(0)), -1 when a halo grows past BOUND (the reference
 * stops), -2 when the catalogue is full. */
int orc_halofind_grid_base(int nx, float dx, const float *u1, const float *radx, float contrastec, float rote,
                           float rete, float rodo, float re0, float bound, float vol_solap_low,
                           const asohf_mesh *mesh, const float *u11, asohf_catalogue *cat)
{
  const int amr = mesh && mesh->nl > 0 && u11;
  const int bor = 1;
  const float esp = 0.2f * dx, esp_log = 1.05f;
  const float peak_thr = contrastec / 6.0f;
  const size_t g = (size_t)nx * nx * nx;
#define U(i, j, k) u1[((size_t)((k) - 1) * nx + ((j) - 1)) * nx + ((i) - 1)]
  int32_t *conta = (int32_t *)calloc(g, sizeof(int32_t));
  if (!conta) return -2;
#define CONTA(i, j, k) conta[((size_t)((k) - 1) * nx + ((j) - 1)) * nx + ((i) - 1)]
  for (int k = 1 + bor; k <= nx - bor; k++)
    for (int j = 1 + bor; j <= nx - bor; j++)
      for (int i = 1 + bor; i <= nx - bor; i++) CONTA(i, j, k) = 1;
  /* candidates in (KZ, JY, IX) order */
  int64_t cap = 1024, ncand = 0;
  float *ddd = malloc(sizeof(float) * cap);
  int *dx3 = malloc(sizeof(int) * 3 * cap);
  for (int k = 1 + bor; k <= nx - bor; k++)
    for (int j = 1 + bor; j <= nx - bor; j++)
      for (int i = 1 + bor; i <= nx - bor; i++) {
        const float b = U(i, j, k);
        if (!(b >= peak_thr)) continue;
        if (!(U(i + 1, j, k) - b < 0.0f)) continue;
        if (!(U(i, j + 1, k) - b < 0.0f)) continue;
        if (!(U(i, j, k + 1) - b < 0.0f)) continue;
        if (!(b - U(i - 1, j, k) > 0.0f)) continue;
        if (!(b - U(i, j - 1, k) > 0.0f)) continue;
        if (!(b - U(i, j, k - 1) > 0.0f)) continue;
        if (ncand == cap) {
          cap *= 2;
          ddd = realloc(ddd, sizeof(float) * cap);
          dx3 = realloc(dx3, sizeof(int) * 3 * cap);
        }
        ddd[ncand] = b;
        dx3[3 * ncand] = i;
        dx3[3 * ncand + 1] = j;
        dx3[3 * ncand + 2] = k;
        ncand++;
      }
  /* SORT_CELLS: ARGSORT of 1/DDD */
  float *inv = calloc((size_t)(ncand > 0 ? ncand : 1), sizeof(float));
  int64_t *order = malloc(sizeof(int64_t) * (ncand > 0 ? ncand : 1));
  for (int64_t q = 0; q < ncand; q++) inv[q] = 1.0f / ddd[q];
  orc_argsort(ncand, inv, order);
  cat->nclus = 0;  /* IF (IR.EQ.0) NCLUS=0 */
  int rc = 0, added = 0;
  const float volcell = dx * dx * dx;
  for (int64_t l = 0; l < ncand && rc == 0; l++) {
    const int64_t q = order[l] - 1;
    const int ic = dx3[3 * q], jc = dx3[3 * q + 1], kc = dx3[3 * q + 2];
    if (CONTA(ic, jc, kc) != 1) continue;
    if (cat->nclus >= cat->capacity) { rc = -2; break; }
    float c3[3] = {radx[ic], radx[jc], radx[kc]};
    int ipatch = 0;
    if (amr) {
      recenter_grid_peak(c3, 0, mesh, u11, dx, &ipatch);
      int dup = 0;  /* the same halo found again after recentering */
      for (int q2 = 0; q2 < cat->nclus && !dup; q2++) {
        const float ex = c3[0] - cat->clusrx[q2], ey = c3[1] - cat->clusry[q2], ez = c3[2] - cat->clusrz[q2];
        dup = ex * ex + ey * ey + ez * ez < cat->radio[q2] * cat->radio[q2];
      }
      if (dup) continue;
    }
    const int h = cat->nclus++;
    added++;
    cat->realclus[h] = -1;
    cat->levhal[h] = 0;
    cat->patchclus[h] = ipatch;
    const float xc = c3[0], yc = c3[1], zc = c3[2];
    cat->clusrx[h] = xc;
    cat->clusry[h] = yc;
    cat->clusrz[h] = zc;
    float basx = 0.0f, basy = 0.0f, basz = 0.0f, basdelta = 0.0f, basmass = 0.0f, basvol = 0.0f;
    float r_int = 0.0f, r_ext = 0.8f * dx;
    float delta = 10.0f * contrastec * rote;
    int iter = 0;
    while (delta > contrastec * rote) {
      iter++;
      if (iter > 1) {
        if (r_ext <= bound) {
          r_int = r_ext;
          const float a = r_ext + esp, b = r_ext * esp_log;
          r_ext = a > b ? a : b;
        } else {
          rc = -1;
          break;
        }
      }
      int lo[3], hi[3];
      const float c3[3] = {xc, yc, zc};
      for (int a = 0; a < 3; a++) {
        float bb = c3[a] - r_ext;
        lo[a] = (int)(((bb - radx[1]) / dx) + 0.5f) + 1;
        if (lo[a] < 1) lo[a] = 1;
        bb = c3[a] + r_ext;
        hi[a] = (int)(((bb - radx[1]) / dx) + 0.5f) + 1;
        if (hi[a] > nx) hi[a] = nx;
      }
      /* BASX..BASZ hold the upper box bounds when the shell sums start */
      basx = xc + r_ext;
      basy = yc + r_ext;
      basz = zc + r_ext;
      float shell = 0.0f;
      for (int k = lo[2]; k <= hi[2]; k++)
        for (int j = lo[1]; j <= hi[1]; j++)
          for (int i = lo[0]; i <= hi[0]; i++) {
            const float ddx = radx[i] - xc, ddy = radx[j] - yc, ddz = radx[k] - zc;
            const float aa = sqrtf(ddx * ddx + ddy * ddy + ddz * ddz);
            if (!(aa >= r_int && aa < r_ext)) continue;
            CONTA(i, j, k) = 0;
            basvol = basvol + volcell;
            const float b = U(i, j, k) * volcell;
            shell = shell + b;
            basx = basx + radx[i] * b;
            basy = basy + radx[j] * b;
            basz = basz + radx[k] * b;
            basdelta = basdelta + b;
          }
      basmass = basmass + shell * rodo * (re0 * re0 * re0);
      if (basvol > 0.0f) delta = basmass / (basvol * (rete * rete * rete));
    }
    cat->radio[h] = r_ext;
    cat->masa[h] = basmass;
    cat->clusrxcm[h] = basx / basdelta;
    cat->clusrycm[h] = basy / basdelta;
    cat->clusrzcm[h] = basz / basdelta;
  }
  free(ddd);
  free(dx3);
  free(inv);
  free(order);
  free(conta);
#undef U
#undef CONTA
  if (rc) return rc;
  /* OVERLAPPING at IR = 0: LOWH3 = 1, LOWH2 = NHALLEV(0) */
  orc_overlapping(cat, 1, cat->nclus, vol_solap_low);
  return added;
}


/* HALOFIND_GRID on the AMR level ir >= 1 (haloes_grids.f:586-1097).  The
 * catalogue holds the haloes of the levels below (appended to).  cr0amr
 * (nx^3), cr0amr11 and solap (NAMRX^3 per patch, mesh order) are the
 * caller's refinement and overlap masks, 1 where a cell is not refined
 * further (CR0AMR, CR0AMR11) or is the master copy (SOLAP).  Steps:
 * CONTA1 = 1 on the level's patches, 0 inside any halo already found
 * (AA <= RADIO) and where SOLAP = 0 (CLEAN_OVERLAPS_INT); peaks as on the
 * base grid but inside BORAMR = 1 of the patch faces and with CONTA1 = 1,
 * in decreasing density (SORT_CELLS_AMR); a peak still at CONTA1 = 1 is
 * recentred on the finer levels when ir < NL (and dropped when inside a
 * halo found before), then grown from R_EXT = 0.87 DXPA by MAX(R_EXT + 0.2
 * DXPA, 1.05 R_EXT) up to MAX(BOUND/1.5^ir, 3): each shell sums the base
 * cells with CR0AMR = 1, the cells of the levels 1..ir-1 with CR0AMR11 = 1
 * and SOLAP = 1 and the level-ir cells with SOLAP = 1 (zeroing CONTA1
 * there), on the patches whose boxes meet the sphere's (PATCHES_SPHERE).
 * OVERLAPPING follows.  Returns NHALLEV(ir), -1 when a halo grows past the
 * bound, -2 when the catalogue is full. */
int orc_halofind_grid_amr(int ir, int nx, float dx, const float *u1, const float *radx, const asohf_mesh *m,
                          const float *u11, const int32_t *cr0amr, const int32_t *cr0amr11, const int32_t *solap,
                          float contrastec, float rote, float rete, float rodo, float re0, float bound,
                          float vol_solap_low, asohf_catalogue *cat)
{
  const int na = ASOHF_NAMRX, boramr = 1;
  const size_t pc = (size_t)na * na * na;
  const int32_t *pn[3] = {m->patchnx, m->patchny, m->patchnz};
  const float *pr[3] = {m->patchrx, m->patchry, m->patchrz};
  const float peak_thr = contrastec / 6.0f;
  int *lev_lo = malloc(sizeof(int) * (size_t)(m->nl + 2));
  {
    int acc = 0;
    for (int l = 0; l <= m->nl; l++) {
      lev_lo[l] = acc;  /* 0-based first patch of level l */
      acc += m->npatch[l];
    }
    lev_lo[m->nl + 1] = acc;
  }
  const int low1 = lev_lo[ir], low2 = lev_lo[ir + 1];
  const float dxpa = dx / powf(2.0f, (float)ir);
  /* RX(IX, I) = PATCHRX(I) - DXPA/2 + (IX-1) DXPA on level l */
#define RXL(a, ix, i, d) ((pr[a][i] - 0.5f * (d)) + (float)((ix) - 1) * (d))
  int32_t *conta1 = calloc((size_t)(low2 > low1 ? low2 - low1 : 1), pc * sizeof(int32_t));
#define C1(i, j, k, p) conta1[(size_t)((p) - low1) * pc + ((size_t)((k) - 1) * na + ((j) - 1)) * na + ((i) - 1)]
#define U11(i, j, k, p) u11[(size_t)(p) * pc + ((size_t)((k) - 1) * na + ((j) - 1)) * na + ((i) - 1)]
#define MASK(a, i, j, k, p) (a)[(size_t)(p) * pc + ((size_t)((k) - 1) * na + ((j) - 1)) * na + ((i) - 1)]
  for (int p = low1; p < low2; p++)
    for (int k = 1; k <= pn[2][p]; k++)
      for (int j = 1; j <= pn[1][p]; j++)
        for (int i = 1; i <= pn[0][p]; i++) C1(i, j, k, p) = 1;
  for (int p = low1; p < low2; p++) {
    float x1[3], x2[3];
    for (int a = 0; a < 3; a++) {
      x1[a] = pr[a][p] - dxpa;
      x2[a] = x1[a] + (float)pn[a][p] * dxpa;
    }
    for (int h = 0; h < cat->nclus; h++) {
      const float c3[3] = {cat->clusrx[h], cat->clusry[h], cat->clusrz[h]}, b = cat->radio[h];
      int meet = 1;
      for (int a = 0; a < 3; a++) meet &= x1[a] <= c3[a] + b && c3[a] - b <= x2[a];
      if (!meet) continue;
      for (int k = 1; k <= pn[2][p]; k++)
        for (int j = 1; j <= pn[1][p]; j++)
          for (int i = 1; i <= pn[0][p]; i++) {
            const float ex = RXL(0, i, p, dxpa) - c3[0], ey = RXL(1, j, p, dxpa) - c3[1],
                        ez = RXL(2, k, p, dxpa) - c3[2];
            if (sqrtf(ex * ex + ey * ey + ez * ez) <= b) C1(i, j, k, p) = 0;
          }
    }
    for (int k = 1; k <= pn[2][p]; k++)  /* CLEAN_OVERLAPS_INT */
      for (int j = 1; j <= pn[1][p]; j++)
        for (int i = 1; i <= pn[0][p]; i++) C1(i, j, k, p) = C1(i, j, k, p) * MASK(solap, i, j, k, p);
  }
  /* peaks, in (patch, KZ, JY, IX) order, then SORT_CELLS_AMR */
  int64_t cap = 1024, ncand = 0;
  float *ddd = malloc(sizeof(float) * cap);
  int *d4 = malloc(sizeof(int) * 4 * cap);
  for (int p = low1; p < low2; p++)
    for (int k = 1 + boramr; k <= pn[2][p] - boramr; k++)
      for (int j = 1 + boramr; j <= pn[1][p] - boramr; j++)
        for (int i = 1 + boramr; i <= pn[0][p] - boramr; i++) {
          const float b = U11(i, j, k, p);
          if (!(b >= peak_thr && C1(i, j, k, p) == 1)) continue;
          if (!(U11(i + 1, j, k, p) - b < 0.0f)) continue;
          if (!(U11(i, j + 1, k, p) - b < 0.0f)) continue;
          if (!(U11(i, j, k + 1, p) - b < 0.0f)) continue;
          if (!(b - U11(i - 1, j, k, p) > 0.0f)) continue;
          if (!(b - U11(i, j - 1, k, p) > 0.0f)) continue;
          if (!(b - U11(i, j, k - 1, p) > 0.0f)) continue;
          if (ncand == cap) {
            cap *= 2;
            ddd = realloc(ddd, sizeof(float) * cap);
            d4 = realloc(d4, sizeof(int) * 4 * cap);
          }
          ddd[ncand] = b;
          d4[4 * ncand] = i;
          d4[4 * ncand + 1] = j;
          d4[4 * ncand + 2] = k;
          d4[4 * ncand + 3] = p;
          ncand++;
        }
  float *inv = calloc((size_t)(ncand > 0 ? ncand : 1), sizeof(float));
  int64_t *order = malloc(sizeof(int64_t) * (size_t)(ncand > 0 ? ncand : 1));
  for (int64_t q = 0; q < ncand; q++) inv[q] = 1.0f / ddd[q];
  orc_argsort(ncand, inv, order);
  const int lowh3 = cat->nclus + 1;
  const float esp = 0.2f * dxpa, esp_log = 1.05f;
  const float b15 = bound / powf(1.5f, (float)ir);
  const float boundir = b15 > 3.0f ? b15 : 3.0f;
  int rc = 0, added = 0;
  for (int64_t l = 0; l < ncand && rc == 0; l++) {
    const int64_t q = order[l] - 1;
    const int ic = d4[4 * q], jc = d4[4 * q + 1], kc = d4[4 * q + 2];
    int ipatch = d4[4 * q + 3];
    if (C1(ic, jc, kc, ipatch) != 1) continue;
    float c3[3] = {RXL(0, ic, ipatch, dxpa), RXL(1, jc, ipatch, dxpa), RXL(2, kc, ipatch, dxpa)};
    int ipf = ipatch + 1;  /* 1-based, as PATCHCLUS */
    if (ir != m->nl) {
      recenter_grid_peak(c3, ir, m, u11, dx, &ipf);
      int dup = 0;
      for (int q2 = 0; q2 < cat->nclus; q2++) {
        const float ex = c3[0] - cat->clusrx[q2], ey = c3[1] - cat->clusry[q2], ez = c3[2] - cat->clusrz[q2];
        if (ex * ex + ey * ey + ez * ez < cat->radio[q2] * cat->radio[q2]) dup = 1;
      }
      if (dup) continue;
    }
    if (cat->nclus >= cat->capacity) { rc = -2; break; }
    const int h = cat->nclus++;
    added++;
    cat->realclus[h] = -1;
    cat->levhal[h] = ir;
    cat->patchclus[h] = ipf;
    cat->clusrx[h] = c3[0];
    cat->clusry[h] = c3[1];
    cat->clusrz[h] = c3[2];
    float bx = 0.0f, by = 0.0f, bz = 0.0f, basdelta = 0.0f, basmass = 0.0f, basvol = 0.0f;
    float r_int = 0.0f, r_ext = 0.87f * dxpa;
    float delta = 10.0f * contrastec * rote;
    int iter = 0;
    while (delta > contrastec * rote) {
      iter++;
      if (iter > 1) {
        if (r_ext <= boundir) {
          r_int = r_ext;
          const float a1 = r_ext + esp, a2 = r_ext * esp_log;
          r_ext = a1 > a2 ? a1 : a2;
        } else {
          rc = -1;
          break;
        }
      }
      int lo[3], hi[3];
      for (int a = 0; a < 3; a++) {
        float bb = c3[a] - r_ext;
        lo[a] = (int)(((bb - radx[1]) / dx) + 0.5f) + 1;
        if (lo[a] < 1) lo[a] = 1;
        bb = c3[a] + r_ext;
        hi[a] = (int)(((bb - radx[1]) / dx) + 0.5f) + 1;
        if (hi[a] > nx) hi[a] = nx;
      }
      /* BASX..BASZ hold the upper box bounds when the shell sums start */
      bx = c3[0] + r_ext;
      by = c3[1] + r_ext;
      bz = c3[2] + r_ext;
      float shell = 0.0f;
      float volcell = dx * dx * dx;
      for (int k = lo[2]; k <= hi[2]; k++)
        for (int j = lo[1]; j <= hi[1]; j++)
          for (int i = lo[0]; i <= hi[0]; i++) {
            if (cr0amr[((size_t)(k - 1) * nx + (j - 1)) * nx + (i - 1)] != 1) continue;
            const float ex = radx[i] - c3[0], ey = radx[j] - c3[1], ez = radx[k] - c3[2];
            const float aa = sqrtf(ex * ex + ey * ey + ez * ez);
            if (!(aa >= r_int && aa < r_ext)) continue;
            basvol = basvol + volcell;
            const float b = u1[((size_t)(k - 1) * nx + (j - 1)) * nx + (i - 1)] * volcell;
            shell = shell + b;
            bx = bx + radx[i] * b;
            by = by + radx[j] * b;
            bz = bz + radx[k] * b;
            basdelta = basdelta + b;
          }
      /* PATCHES_SPHERE: the patches of levels 1..ir whose boxes meet the sphere's */
      for (int irr = 1; irr <= ir; irr++) {
        const float d = dx / powf(2.0f, (float)irr);
        volcell = d * d * d;
        for (int p = lev_lo[irr]; p < lev_lo[irr + 1]; p++) {
          int meet = 1;
          for (int a = 0; a < 3; a++) {
            const float x3 = pr[a][p] - d, x4 = x3 + (float)pn[a][p] * d;
            meet &= c3[a] - r_ext <= x4 && x3 <= c3[a] + r_ext;
          }
          if (!meet) continue;
          for (int k = 1; k <= pn[2][p]; k++)
            for (int j = 1; j <= pn[1][p]; j++)
              for (int i = 1; i <= pn[0][p]; i++) {
                if (irr < ir && MASK(cr0amr11, i, j, k, p) != 1) continue;
                if (MASK(solap, i, j, k, p) != 1) continue;
                const float rx = RXL(0, i, p, d), ry = RXL(1, j, p, d), rz = RXL(2, k, p, d);
                const float ex = rx - c3[0], ey = ry - c3[1], ez = rz - c3[2];
                const float aa = sqrtf(ex * ex + ey * ey + ez * ez);
                if (!(aa >= r_int && aa < r_ext)) continue;
                if (irr == ir) C1(i, j, k, p) = 0;
                basvol = basvol + volcell;
                const float b = U11(i, j, k, p) * volcell;
                shell = shell + b;
                bx = bx + rx * b;
                by = by + ry * b;
                bz = bz + rz * b;
                basdelta = basdelta + b;
              }
        }
      }
      basmass = basmass + shell * rodo * (re0 * re0 * re0);
      if (basvol > 0.0f) delta = basmass / (basvol * (rete * rete * rete));
    }
    cat->radio[h] = r_ext;
    cat->masa[h] = basmass;
    cat->clusrxcm[h] = bx / basdelta;
    cat->clusrycm[h] = by / basdelta;
    cat->clusrzcm[h] = bz / basdelta;
  }
#undef RXL
#undef C1
#undef U11
#undef MASK
  free(ddd);
  free(d4);
  free(inv);
  free(order);
  free(conta1);
  free(lev_lo);
  if (rc) return rc;
  orc_overlapping(cat, lowh3, cat->nclus, vol_solap_low);
  return added;
}


/* FIND_HOST_HALO (substructure.f:1699-1747): from level ir-1 down to 0, the
 * entries of that level's range (SUBS_LEV) still alive whose sphere (RADIO
 * for haloes, RSUB for subhaloes) holds the point; the closest in units of
 * that radius at the first level with any.  0-based index, or -1. */
static int find_host_halo(const float *c3, int ir, const int32_t *subs_lev, const asohf_catalogue *cat)
{
  int host = -1;
  float mind = 100000.0f;
  for (int irr = ir - 1; irr >= 0; irr--) {
    int low1 = 0;
    for (int l = 0; l < irr; l++) low1 += subs_lev[l];
    const int low2 = low1 + subs_lev[irr];
    int flag = 0;
    for (int ii = low1; ii < low2; ii++) {
      if (cat->realclus[ii] == 0) continue;
      const float bas = cat->realclus[ii] == -1 ? cat->radio[ii] : cat->rsub[ii];
      const float ex = c3[0] - cat->clusrx[ii], ey = c3[1] - cat->clusry[ii], ez = c3[2] - cat->clusrz[ii];
      const float d = sqrtf(ex * ex + ey * ey + ez * ez) / bas;
      if (d < 1.0f) {
        flag = 1;
        if (d < mind) {
          mind = d;
          host = ii;
        }
      }
    }
    if (flag) break;
  }
  return host;
}

/* SEARCH_SUBSTRUCTURE_GRID (substructure.f:2-697) on AMR level ir: seeds
 * subhaloes at density peaks of the level's patches that lie inside a halo
 * or subhalo already found (CONTA1 = 1 within RADIO / RSUB, 0 within 2 DXPA
 * of any centre and where SOLAP = 0).  A peak is a cell at least BORAMR = 1
 * from the faces, with U11 >= CONTRASTEC/6 (CONTRASTEC from level 2 on) and
 * no lower than any of its 26 neighbours, taken in decreasing density.  It
 * is recentred on the finer levels when ir < NL (and dropped when inside a
 * subhalo of this call), given a host by FIND_HOST_HALO (none: dropped;
 * closer than 2 DXPA: dropped) and grown in shells as in HALOFIND_GRID
 * (base cells with CR0AMR = 1, patch cells of levels 1..ir with CR0AMR11 =
 * 1 and SOLAP = 1) until the Jacobi radius test R/DISTHOST >
 * (M/(M + 3 MHOST))^(1/3) holds with more than 15 cells; MHOST is the
 * host's profile mass interpolated at DISTHOST in r^3.  MASA and RADIO
 * take the first shell below the virial contrast, scaled by UM (RADIO too,
 * as in the reference), RSUB/MSUB the Jacobi shell.  subs_lev[ir] receives
 * the subhaloes found.  Returns that count, -2 when the catalogue is full,
 * -3 when a growth counts no cell in 100000 shells (the reference would
 * loop for ever). */
int orc_search_substructure_grid(int ir, int nx, float dx, const float *u1, const float *radx,
                                 const asohf_mesh *m, const float *u11, const int32_t *cr0amr,
                                 const int32_t *cr0amr11, const int32_t *solap, float contrastec, float rote,
                                 float rete, float rodo, float re0, float um, int32_t *subs_lev,
                                 asohf_catalogue *cat)
{
  const int na = ASOHF_NAMRX, boramr = 1, nb = ASOHF_NBINS;
  const size_t pc = (size_t)na * na * na;
  const int32_t *pn[3] = {m->patchnx, m->patchny, m->patchnz};
  const float *pr[3] = {m->patchrx, m->patchry, m->patchrz};
  float peak_thr = contrastec / 6.0f;
  if (ir >= 2) peak_thr = contrastec;
  const int nclus_ini = cat->nclus;
  int *lev_lo = malloc(sizeof(int) * (size_t)(m->nl + 2));
  {
    int acc = 0;
    for (int l = 0; l <= m->nl; l++) { lev_lo[l] = acc; acc += m->npatch[l]; }
    lev_lo[m->nl + 1] = acc;
  }
  const int ntot = lev_lo[m->nl + 1];
  const int low1 = lev_lo[ir], low2 = lev_lo[ir + 1];
  const float dxpa = dx / powf(2.0f, (float)ir);
#define RXL(a, ix, i, d) ((pr[a][i] - 0.5f * (d)) + (float)((ix) - 1) * (d))
#define U11(i, j, k, p) u11[(size_t)(p) * pc + ((size_t)((k) - 1) * na + ((j) - 1)) * na + ((i) - 1)]
#define MASK(a, i, j, k, p) (a)[(size_t)(p) * pc + ((size_t)((k) - 1) * na + ((j) - 1)) * na + ((i) - 1)]
  int32_t *conta1 = calloc((size_t)(ntot > 0 ? ntot : 1), pc * sizeof(int32_t));
#define C1(i, j, k, p) MASK(conta1, i, j, k, p)
  for (int p = low1; p < low2; p++) {
    float x1[3], x2[3];
    for (int a = 0; a < 3; a++) {
      x1[a] = pr[a][p] - dxpa;
      x2[a] = x1[a] + (float)pn[a][p] * dxpa;
    }
    for (int pass = 0; pass < 2; pass++)   /* inside a halo: 1; near a centre: 0 */
      for (int h = 0; h < cat->nclus; h++) {
        if (cat->realclus[h] == 0) continue;
        const float c3[3] = {cat->clusrx[h], cat->clusry[h], cat->clusrz[h]};
        const float b = pass == 0 ? (cat->realclus[h] == -1 ? cat->radio[h] : cat->rsub[h]) : 2.0f * dxpa;
        int meet = 1;
        for (int a = 0; a < 3; a++) meet &= x1[a] <= c3[a] + b && c3[a] - b <= x2[a];
        if (!meet) continue;
        for (int k = 1; k <= pn[2][p]; k++)
          for (int j = 1; j <= pn[1][p]; j++)
            for (int i = 1; i <= pn[0][p]; i++) {
              const float ex = RXL(0, i, p, dxpa) - c3[0], ey = RXL(1, j, p, dxpa) - c3[1],
                          ez = RXL(2, k, p, dxpa) - c3[2];
              if (sqrtf(ex * ex + ey * ey + ez * ez) <= b) C1(i, j, k, p) = pass == 0 ? 1 : 0;
            }
      }
  }
  for (int p = 0; p < ntot; p++)   /* CLEAN_OVERLAPS_INT over all levels */
    for (int k = 1; k <= pn[2][p]; k++)
      for (int j = 1; j <= pn[1][p]; j++)
        for (int i = 1; i <= pn[0][p]; i++) C1(i, j, k, p) = C1(i, j, k, p) * MASK(solap, i, j, k, p);
  /* peaks: no lower than the 3^3 neighbourhood */
  int64_t cap = 1024, ncand = 0;
  float *ddd = malloc(sizeof(float) * cap);
  int *d4 = malloc(sizeof(int) * 4 * cap);
  for (int p = low1; p < low2; p++)
    for (int k = 1 + boramr; k <= pn[2][p] - boramr; k++)
      for (int j = 1 + boramr; j <= pn[1][p] - boramr; j++)
        for (int i = 1 + boramr; i <= pn[0][p] - boramr; i++) {
          const float b = U11(i, j, k, p);
          if (!(b >= peak_thr && C1(i, j, k, p) == 1)) continue;
          float mx = -INFINITY;
          for (int kk = k - 1; kk <= k + 1; kk++)
            for (int jj = j - 1; jj <= j + 1; jj++)
              for (int ii = i - 1; ii <= i + 1; ii++) {
                const float v = U11(ii, jj, kk, p);
                if (v > mx || mx != mx) mx = v;
              }
          if (!(b >= mx)) continue;
          if (ncand == cap) {
            cap *= 2;
            ddd = realloc(ddd, sizeof(float) * cap);
            d4 = realloc(d4, sizeof(int) * 4 * cap);
          }
          ddd[ncand] = b;
          d4[4 * ncand] = i;
          d4[4 * ncand + 1] = j;
          d4[4 * ncand + 2] = k;
          d4[4 * ncand + 3] = p;
          ncand++;
        }
  float *inv = calloc((size_t)(ncand > 0 ? ncand : 1), sizeof(float));
  int64_t *order = malloc(sizeof(int64_t) * (size_t)(ncand > 0 ? ncand : 1));
  for (int64_t q = 0; q < ncand; q++) inv[q] = 1.0f / ddd[q];
  orc_argsort(ncand, inv, order);
  const float esp = 0.2f * dxpa, esp_log = 1.05f;
  int rc = 0;
  for (int64_t l = 0; l < ncand && rc == 0; l++) {
    const int64_t q = order[l] - 1;
    const int ic = d4[4 * q], jc = d4[4 * q + 1], kc = d4[4 * q + 2];
    const int ipatch = d4[4 * q + 3];
    if (C1(ic, jc, kc, ipatch) == 0) continue;
    float c3[3] = {RXL(0, ic, ipatch, dxpa), RXL(1, jc, ipatch, dxpa), RXL(2, kc, ipatch, dxpa)};
    int ipf = ipatch + 1;
    if (ir != m->nl) {
      recenter_grid_peak(c3, ir, m, u11, dx, &ipf);
      int dup = 0;
      for (int q2 = nclus_ini; q2 < cat->nclus && !dup; q2++) {
        const float ex = c3[0] - cat->clusrx[q2], ey = c3[1] - cat->clusry[q2], ez = c3[2] - cat->clusrz[q2];
        dup = ex * ex + ey * ey + ez * ez < cat->rsub[q2] * cat->rsub[q2];
      }
      if (dup) continue;
    }
    const int host = find_host_halo(c3, ir, subs_lev, cat);
    if (host < 0) continue;
    const float hx = c3[0] - cat->clusrx[host], hy = c3[1] - cat->clusry[host], hz = c3[2] - cat->clusrz[host];
    const float disthost = sqrtf(hx * hx + hy * hy + hz * hz);
    if (disthost < 2.0f * dxpa) continue;
    /* MHOST: the host's profile mass interpolated at DISTHOST in r^3 */
    const float *pr1 = cat->profiles + (size_t)host * 2 * nb, *pm = pr1 + nb;
    int nbp = nb;
    for (int jj = 1; jj <= nb; jj++)
      if (pr1[jj - 1] == 0.0f) { nbp = jj - 1; break; }
    int jj = 1;
    while (jj <= nbp && !(pr1[jj - 1] > disthost)) jj++;
    float mhost;
    if (jj == 1) {
      const float t = disthost / pr1[0];
      mhost = pm[0] * (t * t * t);
    } else if (jj <= nbp) {
      const float r1 = pr1[jj - 2], r2 = pr1[jj - 1];
      mhost = pm[jj - 2] + (pm[jj - 1] - pm[jj - 2]) * (disthost * disthost * disthost - r1 * r1 * r1) /
                               (r2 * r2 * r2 - r1 * r1 * r1);
    } else {
      mhost = pm[nbp - 1];
    }
    if (cat->nclus >= cat->capacity) { rc = -2; break; }
    const int h = cat->nclus++;
    cat->realclus[h] = host + 1;
    cat->levhal[h] = ir;
    cat->patchclus[h] = ipf;
    cat->clusrx[h] = c3[0];
    cat->clusry[h] = c3[1];
    cat->clusrz[h] = c3[2];
    float bx = 0.0f, by = 0.0f, bz = 0.0f, basdelta = 0.0f, basmass = 0.0f, basvol = 0.0f;
    float r_int = 0.0f, r_ext = 0.8f * dxpa;
    float delta = 10.0f * contrastec * rote;
    int iter = 0, cells = 0, flag_vir = 0;
    for (;;) {
      iter++;
      if (iter > 100000) { rc = -3; break; }  /* no cell ever counted: the reference loops for ever */
      if (iter > 1) {
        r_int = r_ext;
        const float a1 = r_ext + esp, a2 = r_ext * esp_log;
        r_ext = a1 > a2 ? a1 : a2;
      }
      int lo[3], hi[3];
      for (int a = 0; a < 3; a++) {
        float bb = c3[a] - r_ext;
        lo[a] = (int)(((bb - radx[1]) / dx) + 0.5f) + 1;
        if (lo[a] < 1) lo[a] = 1;
        bb = c3[a] + r_ext;
        hi[a] = (int)(((bb - radx[1]) / dx) + 0.5f) + 1;
        if (hi[a] > nx) hi[a] = nx;
      }
      bx = c3[0] + r_ext;  /* BASX..BASZ hold the upper box bounds when the sums start */
      by = c3[1] + r_ext;
      bz = c3[2] + r_ext;
      float shell = 0.0f, volcell = dx * dx * dx;
      for (int k = lo[2]; k <= hi[2]; k++)
        for (int j = lo[1]; j <= hi[1]; j++)
          for (int i = lo[0]; i <= hi[0]; i++) {
            if (cr0amr[((size_t)(k - 1) * nx + (j - 1)) * nx + (i - 1)] != 1) continue;
            const float ex = radx[i] - c3[0], ey = radx[j] - c3[1], ez = radx[k] - c3[2];
            const float aa = sqrtf(ex * ex + ey * ey + ez * ez);
            if (!(aa >= r_int && aa < r_ext)) continue;
            cells++;
            basvol = basvol + volcell;
            const float b = u1[((size_t)(k - 1) * nx + (j - 1)) * nx + (i - 1)] * volcell;
            shell = shell + b;
            bx = bx + radx[i] * b;
            by = by + radx[j] * b;
            bz = bz + radx[k] * b;
            basdelta = basdelta + b;
          }
      for (int irr = 1; irr <= ir; irr++) {   /* PATCHES_SPHERE up to level ir */
        const float d = dx / powf(2.0f, (float)irr);
        volcell = d * d * d;
        for (int p = lev_lo[irr]; p < lev_lo[irr + 1]; p++) {
          int meet = 1;
          for (int a = 0; a < 3; a++) {
            const float x3 = pr[a][p] - d, x4 = x3 + (float)pn[a][p] * d;
            meet &= c3[a] - r_ext <= x4 && x3 <= c3[a] + r_ext;
          }
          if (!meet) continue;
          for (int k = 1; k <= pn[2][p]; k++)
            for (int j = 1; j <= pn[1][p]; j++)
              for (int i = 1; i <= pn[0][p]; i++) {
                if (MASK(cr0amr11, i, j, k, p) != 1 || MASK(solap, i, j, k, p) != 1) continue;
                const float rx = RXL(0, i, p, d), ry = RXL(1, j, p, d), rz = RXL(2, k, p, d);
                const float ex = rx - c3[0], ey = ry - c3[1], ez = rz - c3[2];
                const float aa = sqrtf(ex * ex + ey * ey + ez * ez);
                if (!(aa >= r_int && aa < r_ext)) continue;
                cells++;
                basvol = basvol + volcell;
                const float b = U11(i, j, k, p) * volcell;
                shell = shell + b;
                bx = bx + rx * b;
                by = by + ry * b;
                bz = bz + rz * b;
                basdelta = basdelta + b;
                C1(i, j, k, p) = 0;
              }
        }
      }
      basmass = basmass + shell * rodo * (re0 * re0 * re0);
      if (basvol > 0.0f) delta = basmass / (basvol * (rete * rete * rete));
      if (flag_vir == 0 && delta < contrastec * rote) {
        flag_vir = 1;
        cat->masa[h] = basmass * um;
        cat->radio[h] = r_ext * um;
      }
      const float mm = basmass * um;
      const float eq = r_ext / disthost - powf(mm / (mm + 3.0f * mhost), 1.0f / 3.0f);
      if (eq > 0.0f && cells > 15) {
        cat->rsub[h] = r_ext;
        cat->msub[h] = basmass * um;
        break;
      }
    }
    cat->clusrxcm[h] = bx / basdelta;
    cat->clusrycm[h] = by / basdelta;
    cat->clusrzcm[h] = bz / basdelta;
  }
#undef RXL
#undef U11
#undef MASK
#undef C1
  free(ddd);
  free(d4);
  free(inv);
  free(order);
  free(conta1);
  free(lev_lo);
  if (rc) return rc;
  subs_lev[ir] = cat->nclus - nclus_ini;
  return subs_lev[ir];
}
