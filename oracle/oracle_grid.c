/*
 * oracle_grid.c -- CPU oracle (TEST INFRASTRUCTURE ONLY) for the mesh half of
 * the ASOHF particle hot path: grid constants, density kernels, the kernel
 * deposit, the true-TSC deposit, the FFT Poisson solve and the x-slab sort.
 *
 * This file is the checker, never the product: only tests/, the smoke check
 * and bench.py's CPU-baseline leg may load it.  It is a statement-by-statement
 * C restatement of the reference Fortran (dvallesp/ASOHF), keeping the
 * per-statement precision of the Fortran source (REAL*4 vs REAL*8, left to
 * right evaluation, INT truncation vs FLOOR).  Build with -ffp-contract=off.
 *
 * PARITY STATUS: unpinned by the reference.  The reference is Fortran, no
 * Fortran compiler is available to build it, and it ships no tests, golden
 * vectors or fixtures.  The pins are analytic known-answer tests (kernel
 * normalisation, mass conservation, single-mode Poisson) and the golden
 * vectors this project generated from this restatement (tests/golden/).
 *
 * Fortran column-major arrays A(i,j,k) of shape (n,n,n) are stored here as
 * a[(k-1)*n*n + (j-1)*n + (i-1)].
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"

/* ------------------------------------------------------------------ */
/* MALLA (grids.f:2509-2573) with LADO = LADO0 - LADO0/NX (asohf.f:323). */
void orc_malla(int nx, float lado0, float *radx, float *dx_out)
{
  float lado = lado0 - (lado0 / (float)nx);
  float a = -lado / 2.0f;
  float b = lado / 2.0f;
  float c = (b - a) / (float)(nx - 1);
  radx[1] = a;
  for (int i = 2; i <= nx; i++) radx[i] = radx[1] + (float)(i - 1) * c;
  radx[0] = radx[1] - c;
  radx[nx + 1] = radx[nx] + c;
  *dx_out = radx[2] - radx[1];
}

/* Background constants of the driver (asohf.f:347-364, 440-441) and
 * BRYAN_NORMAN_98 (haloes_grids.f:2-24).  REAL*4 variables assigned from
 * REAL*8 expressions are rounded at the assignment, as in Fortran. */
void orc_cosmology(float hubble_h, float omega0, float zeta, orc_cosmo *c)
{
  float pi = (float)acos(-1.0);
  float ache = (float)((double)hubble_h * 3.66e-3);
  float rodo = (float)((double)omega0 * 3.0 * (double)(ache * ache));
  float re0 = 1.0f / 10.98f;
  float cgr = (float)(1.0 / (8.0 * (double)pi));
  float onez = 1.0f + zeta;
  c->pi = pi;
  c->ache = ache;
  c->rodo = rodo;
  c->re0 = re0;
  c->cgr = cgr;
  c->rote = rodo * (onez * onez * onez);
  c->rete = re0 / onez;
  c->uv = 299792.458f;
  c->um = 9.1717e18f;
  /* BRYAN_NORMAN_98 */
  float omegalambda0 = 1.0f - omega0;
  float bas = omega0 * (onez * onez * onez);
  float omegaz = bas / (bas + omegalambda0);
  float x = omegaz - 1.0f;
  float contrastec = 18.0f * (pi * pi) + 82.0f * x - 39.0f * (x * x);
  c->contrastec = contrastec / omegaz;
  c->omegaz = omegaz;
}

/* COMPUTE_KERNELS (grids.f:997-1067).  kernels[(l)*(2*NMK+1) + (i+NMK)] for
 * i in [-2^l, 2^l].  The 3-D normalisation sum is accumulated in REAL*4 in
 * (I,J,K) loop order (single-thread order of the OMP reduction). */
void orc_compute_kernels(int nl, int interp_degree, float *kernels)
{
  const int W = 2 * ASOHF_NMAX_KERNELS + 1;
  memset(kernels, 0, sizeof(float) * (size_t)W * (ASOHF_NLEVELS + 1));
  for (int ir = 0; ir <= nl; ir++) {
    int n = 1 << ir;
    float h32 = (float)n + 0.5f;
    float h = 2.0f * h32 / 3.0f;
    float *k = kernels + (size_t)ir * W + ASOHF_NMAX_KERNELS;
    for (int i = -n; i <= n; i++) {
      if (interp_degree == 2) {
        float bas = (float)abs(i) / h;
        if (bas <= 0.5f) k[i] = 0.75f - bas * bas;
        else { float t = 1.5f - bas; k[i] = 0.5f * (t * t); }
      } else {
        float bas = (float)abs(i) / h32;
        k[i] = 1.0f - bas;
      }
    }
    float bas = 0.0f;
    for (int i = -n; i <= n; i++)
      for (int j = -n; j <= n; j++)
        for (int kk = -n; kk <= n; kk++)
          bas = bas + k[i] * k[j] * k[kk];
    bas = 1.0f / powf(bas, 1.0f / 3.0f);
    for (int i = -n; i <= n; i++) k[i] = bas * k[i];
  }
}

/* ------------------------------------------------------------------ */
/* DENSITY (grids.f:710-994).
 * mode ORC_FP32: the reference's REAL*4 accumulation, single-thread order.
 * mode ORC_FP64: identical arithmetic for every cloud term, accumulated in
 *                REAL*8 and rounded once: the FP64 oracle for error reports.
 * u1 is NX^3 (column-major); u11 is 32^3 per patch. */
void orc_density(int nx, float lado0, float dx, float rote, float rete,
                 const float *x, const float *y, const float *z,
                 const float *m, const int32_t *npart_esp,
                 const asohf_mesh *mesh, int interp_degree, int mode,
                 float *u1, float *u11)
{
  const int W = 2 * ASOHF_NMAX_KERNELS + 1;
  const int NA = ASOHF_NAMRX;
  float *kernels = (float *)malloc(sizeof(float) * (size_t)W * (ASOHF_NLEVELS + 1));
  int nl = mesh ? mesh->nl : 0;
  orc_compute_kernels(nl, interp_degree, kernels);
  int64_t ntot = 0;
  for (int s = 0; s < ASOHF_N_ESP; s++) ntot += npart_esp[s];
  size_t g = (size_t)nx * nx * nx;

  /* base grid, kernel of level 0 (N = 1) */
  const float *k0 = kernels + ASOHF_NMAX_KERNELS;
  float xl = -lado0 / 2.0f;
  if (mode == ORC_FP32) {
    for (size_t c = 0; c < g; c++) u1[c] = 0.0f;
  }
  double *acc = NULL;
  if (mode == ORC_FP64) acc = (double *)calloc(g, sizeof(double));
  for (int64_t ip = 0; ip < ntot; ip++) {
    float bas = m[ip];
    int ix = (int)((x[ip] - xl) / dx) + 1;
    int jy = (int)((y[ip] - xl) / dx) + 1;
    int kz = (int)((z[ip] - xl) / dx) + 1;
    for (int kk = -1; kk <= 1; kk++)
      for (int jj = -1; jj <= 1; jj++)
        for (int ii = -1; ii <= 1; ii++) {
          int i1 = ix + ii, j1 = jy + jj, k1 = kz + kk;
          if (i1 > nx) i1 -= nx;
          if (i1 < 1) i1 += nx;
          if (j1 > nx) j1 -= nx;
          if (j1 < 1) j1 += nx;
          if (k1 > nx) k1 -= nx;
          if (k1 < 1) k1 += nx;
          size_t c = ((size_t)(k1 - 1) * nx + (j1 - 1)) * nx + (i1 - 1);
          float t = bas * k0[ii] * k0[jj] * k0[kk];
          if (mode == ORC_FP32) u1[c] = u1[c] + t;
          else acc[c] += (double)t;
        }
  }
  float denbas = dx * dx * dx * rote * (rete * rete * rete);
  for (size_t c = 0; c < g; c++) {
    float v = (mode == ORC_FP32) ? u1[c] : (float)acc[c];
    u1[c] = v / denbas;
  }
  free(acc);

  /* AMR patches */
  float maxkernelext = dx;
  int ipatch0 = mesh ? mesh->npatch[0] : 0;
  for (int ir = 1; ir <= nl; ir++) {
    float dxpa = dx / powf(2.0f, (float)ir);
    float denbasp = dxpa * dxpa * dxpa * rote * (rete * rete * rete);
    int low1 = ipatch0, low2 = ipatch0 + mesh->npatch[ir];
    ipatch0 = low2;
#pragma omp parallel for schedule(dynamic)
    for (int ip = low1; ip < low2; ip++) {
      int n1 = mesh->patchnx[ip], n2 = mesh->patchny[ip], n3 = mesh->patchnz[ip];
      float *u = u11 + (size_t)ip * NA * NA * NA;
      double *a64 = NULL;
      for (int c = 0; c < NA * NA * NA; c++) u[c] = 0.0f;
      if (mode == ORC_FP64) a64 = (double *)calloc((size_t)NA * NA * NA, sizeof(double));
      float xlfix = mesh->patchrx[ip] - dxpa;
      float ylfix = mesh->patchry[ip] - dxpa;
      float zlfix = mesh->patchrz[ip] - dxpa;
      float pxl = xlfix, pyl = ylfix, pzl = zlfix;
      float pxr = pxl + (float)n1 * dxpa;
      float pyr = pyl + (float)n2 * dxpa;
      float pzr = pzl + (float)n3 * dxpa;
      pxl = pxl - maxkernelext; pxr = pxr + maxkernelext;
      pyl = pyl - maxkernelext; pyr = pyr + maxkernelext;
      pzl = pzl - maxkernelext; pzr = pzr + maxkernelext;
      int64_t lowp = 0;
      for (int irpart = 0; irpart < ASOHF_N_ESP; irpart++) {
        int irkern = ir - irpart;
        if (irkern < 0) irkern = 0;
        int n = 1 << irkern;
        const float *kern = kernels + (size_t)irkern * W + ASOHF_NMAX_KERNELS;
        int64_t lowp1 = lowp, lowp2 = lowp + npart_esp[irpart];
        lowp = lowp2;
        for (int64_t q = lowp1; q < lowp2; q++) {
          float xp = x[q];
          if (!(pxl < xp && xp < pxr)) continue;
          float yp = y[q];
          if (!(pyl < yp && yp < pyr)) continue;
          float zp = z[q];
          if (!(pzl < zp && zp < pzr)) continue;
          float bas = m[q];
          int ix = (int)floorf((xp - xlfix) / dxpa) + 1;
          int jy = (int)floorf((yp - ylfix) / dxpa) + 1;
          int kz = (int)floorf((zp - zlfix) / dxpa) + 1;
          int i1 = ix - n, i2 = ix + n, j1 = jy - n, j2 = jy + n, k1 = kz - n, k2 = kz + n;
          /* grids.f:925-927 tests J2 twice instead of K2; clipping follows */
          if (i1 > n1 || i2 < 1 || j1 > n2 || j2 < 1 || k1 > n3 || j2 < 1) continue;
          if (i1 < 1) i1 = 1;
          if (i2 > n1) i2 = n1;
          if (j1 < 1) j1 = 1;
          if (j2 > n2) j2 = n2;
          if (k1 < 1) k1 = 1;
          if (k2 > n3) k2 = n3;
          for (int kk = k1; kk <= k2; kk++)
            for (int jj = j1; jj <= j2; jj++)
              for (int ii = i1; ii <= i2; ii++) {
                float t = bas * kern[ii - ix] * kern[jj - jy] * kern[kk - kz];
                size_t c = ((size_t)(kk - 1) * NA + (jj - 1)) * NA + (ii - 1);
                if (mode == ORC_FP32) u[c] = u[c] + t;
                else a64[c] += (double)t;
              }
        }
      }
      for (int kz = 1; kz <= n3; kz++)
        for (int jy = 1; jy <= n2; jy++)
          for (int ix = 1; ix <= n1; ix++) {
            size_t c = ((size_t)(kz - 1) * NA + (jy - 1)) * NA + (ix - 1);
            float v = (mode == ORC_FP32) ? u[c] : (float)a64[c];
            u[c] = v / denbasp;
          }
      free(a64);
    }
  }
  free(kernels);
}

/* RENORM_DENSITY (grids.f:2668-2722). */
void orc_renorm_density(int nx, const asohf_mesh *mesh, float fdm, float *u1, float *u11)
{
  const int NA = ASOHF_NAMRX;
  size_t g = (size_t)nx * nx * nx;
  for (size_t c = 0; c < g; c++) u1[c] = u1[c] / fdm;
  if (!mesh) return;
  int ip0 = mesh->npatch[0];
  for (int ir = 1; ir <= mesh->nl; ir++) {
    for (int ip = ip0; ip < ip0 + mesh->npatch[ir]; ip++) {
      float *u = u11 + (size_t)ip * NA * NA * NA;
      for (int kz = 0; kz < mesh->patchnz[ip]; kz++)
        for (int jy = 0; jy < mesh->patchny[ip]; jy++)
          for (int ix = 0; ix < mesh->patchnx[ip]; ix++) {
            size_t c = ((size_t)kz * NA + jy) * NA + ix;
            u[c] = u[c] / fdm;
          }
    }
    ip0 += mesh->npatch[ir];
  }
}

/* ------------------------------------------------------------------ */
/* SORT_DM_PARTICLES_LOCALDENSITY (reader.f:140-336).  NGP mass grid summed
 * in REAL*4 in particle order (single-thread order of the OMP reduction),
 * species INT(LOG(rho)/LOG(8)) clamped to [0, N_ESP-1], then a stable
 * counting sort by species.  Arrays are permuted in place; species_out (may
 * be NULL) receives the species of each particle in the ORIGINAL order. */
int orc_species_sort(int64_t n, float *x, float *y, float *z, float *vx,
                     float *vy, float *vz, float *m, int32_t *id, int nx,
                     float dx, float rodo, float re0, int32_t *npart_esp,
                     int32_t *species_out)
{
  size_t g = (size_t)nx * nx * nx;
  float *dens = (float *)calloc(g, sizeof(float));
  float xmin = -((float)nx * dx) / 2.0f;
  int32_t *cell = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  for (int64_t i = 0; i < n; i++) {
    int ix = (int)((x[i] - xmin) / dx) + 1;
    int jy = (int)((y[i] - xmin) / dx) + 1;
    int kz = (int)((z[i] - xmin) / dx) + 1;
    if (ix < 1) ix = 1;
    if (ix > nx) ix = nx;
    if (jy < 1) jy = 1;
    if (jy > nx) jy = nx;
    if (kz < 1) kz = 1;
    if (kz > nx) kz = nx;
    size_t c = ((size_t)(kz - 1) * nx + (jy - 1)) * nx + (ix - 1);
    cell[i] = (int32_t)c;
    dens[c] = dens[c] + m[i];
  }
  float bas = dx * dx * dx * rodo * (re0 * re0 * re0);
  for (size_t c = 0; c < g; c++) dens[c] = dens[c] / bas;
  float log8 = logf(8.0f);
  int32_t *lev = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  for (int64_t i = 0; i < n; i++) {
    float b = dens[cell[i]];
    int l = 0;
    if (b > 0.0f) {
      l = (int)(logf(b) / log8);
      if (l > ASOHF_N_ESP - 1) l = ASOHF_N_ESP - 1;
      if (l < 0) l = 0;
    }
    lev[i] = l;
  }
  free(dens);
  free(cell);
  if (species_out) memcpy(species_out, lev, sizeof(int32_t) * (size_t)n);
  int64_t *indices = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
  int64_t conta = 0;
  for (int s = 0; s < ASOHF_N_ESP; s++) {
    int64_t before = conta;
    for (int64_t i = 0; i < n; i++)
      if (lev[i] == s) indices[conta++] = i;
    npart_esp[s] = (int32_t)(conta - before);
  }
  free(lev);
  if (conta != n) { free(indices); return ASOHF_ERR_WRONG_SORTING; }
  orc_permute(n, indices, x, y, z, vx, vy, vz, m, id);
  free(indices);
  return 0;
}

/* Applies dst[i] = src[idx[i]] to the 7 float arrays and the id array. */
void orc_permute(int64_t n, const int64_t *idx, float *x, float *y, float *z,
                 float *vx, float *vy, float *vz, float *m, int32_t *id)
{
  float *scr = (float *)malloc(sizeof(float) * (size_t)n);
  float *arrs[7] = {x, y, z, vx, vy, vz, m};
  for (int a = 0; a < 7; a++) {
    for (int64_t i = 0; i < n; i++) scr[i] = arrs[a][idx[i]];
    memcpy(arrs[a], scr, sizeof(float) * (size_t)n);
  }
  free(scr);
  int32_t *si = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  for (int64_t i = 0; i < n; i++) si[i] = id[idx[i]];
  memcpy(id, si, sizeof(int32_t) * (size_t)n);
  free(si);
}

/* ------------------------------------------------------------------ */
/* INTERPOLATE_DENSITY_TSC (grids.f:1070-1398): per-particle maximum level
 * PLEV (first containing patch with a 1-cell buffer, finest level first),
 * periodic TSC on the base grid, clipped TSC on the patches.  Same FP32/FP64
 * modes as orc_density. */
static inline void tsc_w(float xp, float r_m1, float r_0, float r_p1, float d, float *v)
{
  float bas = fabsf(xp - r_m1) / d;
  float t = 1.5f - bas;
  v[0] = 0.5f * (t * t);
  bas = fabsf(xp - r_0) / d;
  v[1] = 0.75f - bas * bas;
  bas = fabsf(xp - r_p1) / d;
  t = 1.5f - bas;
  v[2] = 0.5f * (t * t);
}

void orc_tsc_deposit(int nx, float lado0, float dx, const float *radx, float rote,
                     float rete, int64_t n, const float *x, const float *y,
                     const float *z, const float *m, const asohf_mesh *mesh,
                     int mode, float *u1, float *u11)
{
  const int NA = ASOHF_NAMRX;
  const int buf = 1;
  int nl = mesh ? mesh->nl : 0;
  int32_t *plev = (int32_t *)calloc((size_t)n, sizeof(int32_t));
  int *low = (int *)malloc(sizeof(int) * (nl + 2));
  low[0] = 0;
  if (mesh) {
    low[1] = mesh->npatch[0];
    for (int ir = 1; ir <= nl; ir++) low[ir + 1] = low[ir] + mesh->npatch[ir];
  }
  for (int ir = nl; ir >= 1; ir--) {
    float dxpa = dx / powf(2.0f, (float)ir);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
      if (plev[i] != 0) continue;
      for (int ip = low[ir]; ip < low[ir + 1]; ip++) {
        float xl = mesh->patchrx[ip] - (float)(1 + buf) * dxpa;
        float yl = mesh->patchry[ip] - (float)(1 + buf) * dxpa;
        float zl = mesh->patchrz[ip] - (float)(1 + buf) * dxpa;
        float xr = xl + (float)(mesh->patchnx[ip] + 2 * buf) * dxpa;
        float yr = yl + (float)(mesh->patchny[ip] + 2 * buf) * dxpa;
        float zr = zl + (float)(mesh->patchnz[ip] + 2 * buf) * dxpa;
        if (xl < x[i] && x[i] < xr && yl < y[i] && y[i] < yr && zl < z[i] && z[i] < zr) {
          plev[i] = ir;
          break;
        }
      }
    }
  }
  size_t g = (size_t)nx * nx * nx;
  double *acc = NULL;
  if (mode == ORC_FP64) acc = (double *)calloc(g, sizeof(double));
  else for (size_t c = 0; c < g; c++) u1[c] = 0.0f;
  float xl = -lado0 / 2.0f;
  for (int64_t i = 0; i < n; i++) {
    float xp = x[i], yp = y[i], zp = z[i];
    int ix = (int)((xp - xl) / dx) + 1;
    int jy = (int)((yp - xl) / dx) + 1;
    int kz = (int)((zp - xl) / dx) + 1;
    if (ix < 1) ix = 1;
    if (ix > nx) ix = nx;
    if (jy < 1) jy = 1;
    if (jy > nx) jy = nx;
    if (kz < 1) kz = 1;
    if (kz > nx) kz = nx;
    float vxw[3], vyw[3], vzw[3];
    tsc_w(xp, radx[ix - 1], radx[ix], radx[ix + 1], dx, vxw);
    tsc_w(yp, radx[jy - 1], radx[jy], radx[jy + 1], dx, vyw);
    tsc_w(zp, radx[kz - 1], radx[kz], radx[kz + 1], dx, vzw);
    for (int kk = -1; kk <= 1; kk++)
      for (int jj = -1; jj <= 1; jj++)
        for (int ii = -1; ii <= 1; ii++) {
          int i1 = ix + ii, j1 = jy + jj, k1 = kz + kk;
          if (i1 == nx + 1) i1 = 1;
          if (i1 == 0) i1 = nx;
          if (j1 == nx + 1) j1 = 1;
          if (j1 == 0) j1 = nx;
          if (k1 == nx + 1) k1 = 1;
          if (k1 == 0) k1 = nx;
          size_t c = ((size_t)(k1 - 1) * nx + (j1 - 1)) * nx + (i1 - 1);
          float t = m[i] * vxw[ii + 1] * vyw[jj + 1] * vzw[kk + 1];
          if (mode == ORC_FP32) u1[c] = u1[c] + t;
          else acc[c] += (double)t;
        }
  }
  float denbas = dx * dx * dx * rote * (rete * rete * rete);
  for (size_t c = 0; c < g; c++) {
    float v = (mode == ORC_FP32) ? u1[c] : (float)acc[c];
    u1[c] = v / denbas;
  }
  free(acc);
  for (int ir = 1; ir <= nl; ir++) {
    float dxpa = dx / powf(2.0f, (float)ir);
    float denbasp = dxpa * dxpa * dxpa * rote * (rete * rete * rete);
#pragma omp parallel for schedule(dynamic)
    for (int ip = low[ir]; ip < low[ir + 1]; ip++) {
      float *u = u11 + (size_t)ip * NA * NA * NA;
      double *a64 = NULL;
      for (int c = 0; c < NA * NA * NA; c++) u[c] = 0.0f;
      if (mode == ORC_FP64) a64 = (double *)calloc((size_t)NA * NA * NA, sizeof(double));
      float pxl = mesh->patchrx[ip] - (float)(1 + buf) * dxpa;
      float pyl = mesh->patchry[ip] - (float)(1 + buf) * dxpa;
      float pzl = mesh->patchrz[ip] - (float)(1 + buf) * dxpa;
      int n1 = mesh->patchnx[ip], n2 = mesh->patchny[ip], n3 = mesh->patchnz[ip];
      float pxr = pxl + (float)(n1 + 2 * buf) * dxpa;
      float pyr = pyl + (float)(n2 + 2 * buf) * dxpa;
      float pzr = pzl + (float)(n3 + 2 * buf) * dxpa;
      float mrx[NA + 6], mry[NA + 6], mrz[NA + 6]; /* MINIRADX(-2:NAMRX+3) */
      for (int ii = -2; ii <= n1 + 3; ii++) mrx[ii + 2] = mesh->patchrx[ip] + ((float)ii - 1.5f) * dxpa;
      for (int jj = -2; jj <= n2 + 3; jj++) mry[jj + 2] = mesh->patchry[ip] + ((float)jj - 1.5f) * dxpa;
      for (int kk = -2; kk <= n3 + 3; kk++) mrz[kk + 2] = mesh->patchrz[ip] + ((float)kk - 1.5f) * dxpa;
      for (int64_t i = 0; i < n; i++) {
        if (plev[i] < ir) continue;
        float xp = x[i], yp = y[i], zp = z[i];
        if (!(pxl < xp && xp < pxr)) continue;
        if (!(pyl < yp && yp < pyr)) continue;
        if (!(pzl < zp && zp < pzr)) continue;
        int ix = (int)((xp - pxl) / dxpa) + 1 - buf;
        int jy = (int)((yp - pyl) / dxpa) + 1 - buf;
        int kz = (int)((zp - pzl) / dxpa) + 1 - buf;
        float vxw[3], vyw[3], vzw[3];
        tsc_w(xp, mrx[ix - 1 + 2], mrx[ix + 2], mrx[ix + 1 + 2], dxpa, vxw);
        tsc_w(yp, mry[jy - 1 + 2], mry[jy + 2], mry[jy + 1 + 2], dxpa, vyw);
        tsc_w(zp, mrz[kz - 1 + 2], mrz[kz + 2], mrz[kz + 1 + 2], dxpa, vzw);
        for (int kk = -1; kk <= 1; kk++)
          for (int jj = -1; jj <= 1; jj++)
            for (int ii = -1; ii <= 1; ii++) {
              int i1 = ix + ii, j1 = jy + jj, k1 = kz + kk;
              if (i1 > 0 && i1 <= n1 && j1 > 0 && j1 <= n2 && k1 > 0 && k1 <= n3) {
                size_t c = ((size_t)(k1 - 1) * NA + (j1 - 1)) * NA + (i1 - 1);
                float t = m[i] * vxw[ii + 1] * vyw[jj + 1] * vzw[kk + 1];
                if (mode == ORC_FP32) u[c] = u[c] + t;
                else a64[c] += (double)t;
              }
            }
      }
      for (int kz = 1; kz <= n3; kz++)
        for (int jy = 1; jy <= n2; jy++)
          for (int ix = 1; ix <= n1; ix++) {
            size_t c = ((size_t)(kz - 1) * NA + (jy - 1)) * NA + (ix - 1);
            float v = (mode == ORC_FP32) ? u[c] : (float)a64[c];
            u[c] = v / denbasp;
          }
      free(a64);
    }
  }
  free(low);
  free(plev);
}

/* ------------------------------------------------------------------ */
/* MOMENTO (poisson.f:98-175): KKK = -(DX/2)^2 / sum_d sin^2(pi k_d / NX),
 * KKK(1,1,1) from the 1e30 denominator. */
void orc_momento(int nx, float dx, float *kkk)
{
  float pi = acosf(-1.0f);
  float consta = pi / (float)nx;
  float del2 = (dx * 0.5f) * (dx * 0.5f);
  int n2 = nx / 2 + 2;
  float *s2 = (float *)malloc(sizeof(float) * nx);
  for (int i = 1; i <= nx; i++) {
    int k = (i >= n2) ? i - nx - 1 : i - 1;
    float a = consta * (float)k;
    float s = sinf(a);
    s2[i - 1] = s * s;
  }
  for (int k = 1; k <= nx; k++)
    for (int j = 1; j <= nx; j++)
      for (int i = 1; i <= nx; i++) {
        size_t c = ((size_t)(k - 1) * nx + (j - 1)) * nx + (i - 1);
        kkk[c] = s2[i - 1] + s2[j - 1] + s2[k - 1];
      }
  kkk[0] = 1.0e30f;
  size_t g = (size_t)nx * nx * nx;
  for (size_t c = 0; c < g; c++) kkk[c] = -del2 / kkk[c];
  free(s2);
}

/* FOURN (poisson.f:252-333): Numerical-Recipes style in-place complex FFT,
 * REAL*4 data with REAL*8 trigonometric recurrences.  data is 1-based in the
 * Fortran; here data[0] is DATA(1). */
static void fourn(float *data, const int *nn, int ndim, int isign)
{
  float *d = data - 1; /* 1-based view */
  long ntot = 1;
  for (int idim = 0; idim < ndim; idim++) ntot *= nn[idim];
  long nprev = 1;
  for (int idim = 0; idim < ndim; idim++) {
    long n = nn[idim];
    long nrem = ntot / (n * nprev);
    long ip1 = 2 * nprev, ip2 = ip1 * n, ip3 = ip2 * nrem;
    long i2rev = 1;
    for (long i2 = 1; i2 <= ip2; i2 += ip1) {
      if (i2 < i2rev) {
        for (long i1 = i2; i1 <= i2 + ip1 - 2; i1 += 2)
          for (long i3 = i1; i3 <= ip3; i3 += ip2) {
            long i3rev = i2rev + i3 - i2;
            float tr = d[i3], ti = d[i3 + 1];
            d[i3] = d[i3rev];
            d[i3 + 1] = d[i3rev + 1];
            d[i3rev] = tr;
            d[i3rev + 1] = ti;
          }
      }
      long ibit = ip2 / 2;
      while (ibit >= ip1 && i2rev > ibit) {
        i2rev -= ibit;
        ibit /= 2;
      }
      i2rev += ibit;
    }
    long ifp1 = ip1;
    while (ifp1 < ip2) {
      long ifp2 = 2 * ifp1;
      double theta = (double)isign * 6.28318530717959 / (double)(ifp2 / ip1);
      double st = sin(0.5 * theta);
      double wpr = -2.0 * st * st;
      double wpi = sin(theta);
      double wr = 1.0, wi = 0.0;
      for (long i3 = 1; i3 <= ifp1; i3 += ip1) {
        for (long i1 = i3; i1 <= i3 + ip1 - 2; i1 += 2)
          for (long i2 = i1; i2 <= ip3; i2 += ifp2) {
            long k1 = i2, k2 = k1 + ifp1;
            float fwr = (float)wr, fwi = (float)wi;
            float tempr = fwr * d[k2] - fwi * d[k2 + 1];
            float tempi = fwr * d[k2 + 1] + fwi * d[k2];
            d[k2] = d[k1] - tempr;
            d[k2 + 1] = d[k1 + 1] - tempi;
            d[k1] = d[k1] + tempr;
            d[k1 + 1] = d[k1 + 1] + tempi;
          }
        double wtemp = wr;
        wr = wr * wpr - wi * wpi + wr;
        wi = wi * wpr + wtemp * wpi + wi;
      }
      ifp1 = ifp2;
    }
    nprev = n * nprev;
  }
}

/* POFFT3D (poisson.f:178-249) with KKK from MOMENTO.  Packing index
 * IJK=(I-1)*NY*NZ+(J-1)*NZ+K as in the Fortran. */
void orc_poisson_fft(int nx, float dx, const float *u1, float *pot)
{
  size_t g = (size_t)nx * nx * nx;
  float *kkk = (float *)malloc(sizeof(float) * g);
  orc_momento(nx, dx, kkk);
  float *data = (float *)malloc(sizeof(float) * 2 * g);
  for (int i = 1; i <= nx; i++)
    for (int j = 1; j <= nx; j++)
      for (int k = 1; k <= nx; k++) {
        size_t ijk = ((size_t)(i - 1) * nx + (j - 1)) * nx + k;
        size_t c = ((size_t)(k - 1) * nx + (j - 1)) * nx + (i - 1);
        data[2 * ijk - 2] = u1[c];
        data[2 * ijk - 1] = 0.0f;
      }
  int nnn[3] = {nx, nx, nx};
  fourn(data, nnn, 3, 1);
  for (int i = 1; i <= nx; i++)
    for (int j = 1; j <= nx; j++)
      for (int k = 1; k <= nx; k++) {
        size_t ijk = ((size_t)(i - 1) * nx + (j - 1)) * nx + k;
        size_t c = ((size_t)(k - 1) * nx + (j - 1)) * nx + (i - 1);
        data[2 * ijk - 2] = data[2 * ijk - 2] * kkk[c];
        data[2 * ijk - 1] = data[2 * ijk - 1] * kkk[c];
      }
  fourn(data, nnn, 3, -1);
  int nxyz = nx * nx * nx;
  for (int i = 1; i <= nx; i++)
    for (int j = 1; j <= nx; j++)
      for (int k = 1; k <= nx; k++) {
        size_t ijk = ((size_t)(i - 1) * nx + (j - 1)) * nx + k;
        size_t c = ((size_t)(k - 1) * nx + (j - 1)) * nx + (i - 1);
        pot[c] = data[2 * ijk - 2] / (float)nxyz;
      }
  free(data);
  free(kkk);
}

/* ------------------------------------------------------------------ */
/* ARGSORT (num.f:150-203): bottom-up merge sort of indices; on equal keys
 * the element of the right run is taken first (num.f:181).  indx receives
 * 1-based indices as in the Fortran. */
void orc_argsort(int64_t n, const float *a, int64_t *indx)
{
  for (int64_t i = 0; i < n; i++) indx[i] = i + 1;
  if (n <= 1) return;
  int64_t *tmp = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
  const float *A = a - 1;
  int64_t *I = indx - 1, *T = tmp - 1;
  int64_t delta = 1;
  while (delta < n) {
    for (int64_t iii = 1; iii <= n - delta; iii += delta * 2) {
      int64_t i1 = iii, i2 = iii + delta;
      int64_t kkk = (delta * 2 < n - iii + 1) ? delta * 2 : n - iii + 1;
      int64_t k = 1;
      while (i1 < iii + delta && i2 < iii + kkk) {
        if (A[I[i1]] < A[I[i2]]) T[k++] = I[i1++];
        else T[k++] = I[i2++];
      }
      if (i1 < iii + delta) {
        while (k <= kkk) T[k++] = I[i1++];
      } else {
        while (k <= kkk) T[k++] = I[i2++];
      }
      for (int64_t q = 1; q <= kkk; q++) I[iii + q - 1] = T[q];
    }
    delta *= 2;
  }
  free(tmp);
}

/* SORT_DM_PARTICLES_X (grids.f:2726-2838): ARGSORT by x, permute, and the
 * slab table NDMPART_X(0:NX) (ndmpart_x has nx+1 entries). */
void orc_sort_x(int64_t n, float *x, float *y, float *z, float *vx, float *vy,
                float *vz, float *m, int32_t *id, int nx, float lado0,
                int32_t *ndmpart_x)
{
  int64_t *idx = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
  orc_argsort(n, x, idx);
  for (int64_t i = 0; i < n; i++) idx[i] -= 1;
  orc_permute(n, idx, x, y, z, vx, vy, vz, m, id);
  free(idx);
  float xl = -lado0 / 2.0f;
  float dx = lado0 / (float)nx;
  float *radxr = (float *)malloc(sizeof(float) * (nx + 2));
  for (int i = 0; i <= nx; i++) radxr[i] = xl + (float)i * dx;
  radxr[nx + 1] = INFINITY; /* guards a particle beyond RADXR(NX) (out of bounds in the Fortran) */
  for (int i = 0; i <= nx; i++) ndmpart_x[i] = 0;
  int ix = 1;
  int64_t i;
  for (i = 1; i <= n; i++) {
    if (x[i - 1] > radxr[ix]) {
      if (ix <= nx) ndmpart_x[ix] = (int32_t)(i - 1);
      ix++;
      while (ix <= nx && x[i - 1] > radxr[ix]) {
        ndmpart_x[ix] = (int32_t)(i - 1);
        ix++;
      }
    }
  }
  for (int q = ix; q <= nx; q++) ndmpart_x[q] = (int32_t)(i - 1);
  free(radxr);
}


/* PLEV(I) of CREATE_MESH (grids.f:83-91): the species whose NPART_ESP range
 * holds the 0-based store index i, 0 past the last range. */
static int mesh_plev(int64_t i, const int32_t *npart_esp)
{
  int64_t acc = 0;
  for (int s = 0; s < ASOHF_N_ESP; s++) {
    acc += npart_esp[s];
    if (i < acc) return s;
  }
  return 0;
}

/* CREATE_MESH base-grid counts (grids.f:94-143): CONTA1 by NGP with
 * IX = INT((RXPA-XL)/DX)+1 clamped to 1..NX, weight 1 for PLEV 0 and
 * REFINE_THR otherwise, then zero within BOR cells of the faces; CR0 =
 * CONTA1, IX fastest.  A NaN offset takes the lower clamp. */
void orc_mesh_base_counts(int64_t n, const float *x, const float *y, const float *z, int nx, float dx,
                          int refine_thr, int bor, const int32_t *npart_esp, int32_t *cr0)
{
  const float xl = -((float)nx * dx / 2.0f);
  const int64_t g = (int64_t)nx * nx * nx;
  memset(cr0, 0, sizeof(int32_t) * (size_t)g);
  for (int64_t i = 0; i < n; i++) {
    const float v3[3] = {x[i], y[i], z[i]};
    int c3[3];
    for (int a = 0; a < 3; a++) {
      const float v = (v3[a] - xl) / dx;
      int ic;
      if (v >= (float)nx) ic = nx;            /* INT(v)+1 > NX */
      else if (v >= 1.0f) ic = (int)v + 1;    /* INT truncates toward zero */
      else ic = 1;                            /* INT(v)+1 <= 1, or NaN */
      c3[a] = ic;
    }
    const int w = mesh_plev(i, npart_esp) == 0 ? 1 : refine_thr;
    int64_t q = ((int64_t)(c3[2] - 1) * nx + (c3[1] - 1)) * nx + (c3[0] - 1);
    cr0[q] = (int32_t)((uint32_t)cr0[q] + (uint32_t)w);
  }
  for (int kz = 1; kz <= nx; kz++)
    for (int jy = 1; jy <= nx; jy++)
      for (int ix = 1; ix <= nx; ix++)
        if (ix <= bor || ix >= nx - bor + 1 || jy <= bor || jy >= nx - bor + 1 || kz <= bor || kz >= nx - bor + 1)
          cr0[((int64_t)(kz - 1) * nx + (jy - 1)) * nx + (ix - 1)] = 0;
}

/* CREATE_MESH counts on the patches of level IRPA (grids.f:341-380): per
 * patch, XL = PATCHRX - DXPA, IX = FLOOR((RXPA-XL)/DXPA)+1 kept when
 * 1 <= IX <= N1 (and the same in y, z), weight 1 for PLEV <= IRPA and
 * REFINE_THR otherwise, zero within BORAMR cells of the faces; each patch
 * NAMRX^3 cells, IX fastest, zero outside N1 x N2 x N3. */
void orc_mesh_patch_counts(int64_t n, const float *x, const float *y, const float *z, int irpa, float dx,
                           int refine_thr, int boramr, const int32_t *npart_esp, int npatch,
                           const int32_t *pnx, const int32_t *pny, const int32_t *pnz, const float *prx,
                           const float *pry, const float *prz, int32_t *cr01)
{
  const int na = ASOHF_NAMRX;
  const float dxpa = dx / powf(2.0f, (float)irpa);
#pragma omp parallel for schedule(dynamic)
  for (int ip = 0; ip < npatch; ip++) {
    int32_t *o = cr01 + (size_t)ip * na * na * na;
    memset(o, 0, sizeof(int32_t) * (size_t)na * na * na);
    const float xl = prx[ip] - dxpa, yl = pry[ip] - dxpa, zl = prz[ip] - dxpa;
    const int n1 = pnx[ip], n2 = pny[ip], n3 = pnz[ip];
    for (int64_t i = 0; i < n; i++) {
      const float vx = floorf((x[i] - xl) / dxpa);
      if (!(vx >= 0.0f && vx <= (float)(n1 - 1))) continue;
      const float vy = floorf((y[i] - yl) / dxpa);
      if (!(vy >= 0.0f && vy <= (float)(n2 - 1))) continue;
      const float vz = floorf((z[i] - zl) / dxpa);
      if (!(vz >= 0.0f && vz <= (float)(n3 - 1))) continue;
      const int w = mesh_plev(i, npart_esp) <= irpa ? 1 : refine_thr;
      const size_t q = ((size_t)vz * na + (size_t)vy) * na + (size_t)vx;
      o[q] = (int32_t)((uint32_t)o[q] + (uint32_t)w);
    }
    for (int kz = 1; kz <= n3; kz++)
      for (int jy = 1; jy <= n2; jy++)
        for (int ix = 1; ix <= n1; ix++)
          if (ix <= boramr || ix >= n1 - boramr + 1 || jy <= boramr || jy >= n2 - boramr + 1 || kz <= boramr ||
              kz >= n3 - boramr + 1)
            o[((size_t)(kz - 1) * na + (jy - 1)) * na + (ix - 1)] = 0;
  }
}


/* One axis of VEINSGRID_REDUCED's overlap corners (grids.f:1965-2026, the X
 * block; Y and Z are the same): the cells CORN1..CORN2 of patch I and
 * CORNN1..CORNN2 of patch J that face each other.  INT truncates toward
 * zero. */
static void veins_axis(float r1, float r2, float rr1, float rr2, float dxpa, int n, int nn, int *c1, int *c2,
                       int *cc1, int *cc2)
{
  if (rr1 >= r1 && rr2 <= r2) {
    *c1 = (int)(((rr1 - r1) / dxpa) + 0.5f) + 1;
    *c2 = (int)(((rr2 - r1) / dxpa) + 0.5f) + 1;
    *cc1 = 1;
    *cc2 = nn;
  }
  if (rr1 >= r1 && rr2 > r2) {
    *c1 = (int)(((rr1 - r1) / dxpa) + 0.5f) + 1;
    *c2 = n;
    *cc1 = 1;
    *cc2 = (int)(((r2 - rr1) / dxpa) + 0.5f) + 1;
  }
  if (rr2 <= r2 && rr1 < r1) {
    *c1 = 1;
    *c2 = (int)(((rr2 - r1) / dxpa) + 0.5f) + 1;
    *cc1 = (int)(((r1 - rr1) / dxpa) + 0.5f) + 1;
    *cc2 = nn;
  }
  if (rr1 < r1 && rr2 > r2) {
    *c1 = 1;
    *c2 = n;
    *cc1 = (int)(((r1 - rr1) / dxpa) + 0.5f) + 1;
    *cc2 = (int)(((r2 - rr1) / dxpa) + 0.5f) + 1;
  }
}

/* VEINSGRID_REDUCED (grids.f:1771-2073) on the npatch patches of level ir
 * (the slice LOW1..LOW2): neighbours are the other patches whose cell boxes
 * on the level's grid (origin RXFIX = RADX(1) - DX/2 + DXPA/2) intersect;
 * then, patch I in order and its neighbours J in order, when the overlap
 * covers more than 0.1 of J, every cell of J facing a cell of I not yet
 * marked is marked and its CR01 / CONTA11 zeroed.  Returns 0, or -1 when a
 * patch has more than max_nb neighbours (the reference's STOP).  Cells
 * outside the NAMRX^3 arrays are skipped. */
int orc_veinsgrid_reduced(int ir, float dx, float radx1, int npatch, const int32_t *pnx, const int32_t *pny,
                          const int32_t *pnz, const float *prx, const float *pry, const float *prz, int max_nb,
                          int32_t *cr01, int32_t *conta11)
{
  const int na = ASOHF_NAMRX;
  const size_t pc = (size_t)na * na * na;
  const float dxpa = dx / powf(2.0f, (float)ir);
  const float fix = radx1 - dx * 0.5f + 0.5f * dxpa;
  int *g1 = malloc(sizeof(int) * 3 * (size_t)(npatch > 0 ? npatch : 1));
  uint8_t *solap = calloc((size_t)(npatch > 0 ? npatch : 1), pc);
  int *nb = malloc(sizeof(int) * (size_t)(npatch > 0 ? npatch : 1));
  if (!g1 || !solap || !nb) { free(g1); free(solap); free(nb); return -2; }
  const float *pr[3] = {prx, pry, prz};
  const int32_t *pn[3] = {pnx, pny, pnz};
  for (int i = 0; i < npatch; i++)
    for (int a = 0; a < 3; a++)
      g1[3 * i + a] = (int)(((pr[a][i] - 0.5f * dxpa - fix) / dxpa) + 0.5f) + 1;
  int rc = 0;
  for (int i = 0; i < npatch && rc == 0; i++) {
    int nv = 0;
    for (int j = 0; j < npatch; j++) {
      if (j == i) continue;
      int ok = 1;
      for (int a = 0; a < 3; a++)
        ok &= g1[3 * i + a] <= g1[3 * j + a] + pn[a][j] - 1 && g1[3 * j + a] <= g1[3 * i + a] + pn[a][i] - 1;
      nv += ok;
    }
    if (nv > max_nb) rc = -1;
  }
  for (int i = 0; i < npatch && rc == 0; i++) {
    float r1[3], r2[3];
    for (int a = 0; a < 3; a++) {
      r1[a] = pr[a][i] - 0.5f * dxpa;
      r2[a] = pr[a][i] - 0.5f * dxpa + (float)(pn[a][i] - 1) * dxpa;
    }
    for (int j = 0; j < npatch; j++) {
      if (j == i) continue;
      int ok = 1;
      for (int a = 0; a < 3; a++)
        ok &= g1[3 * i + a] <= g1[3 * j + a] + pn[a][j] - 1 && g1[3 * j + a] <= g1[3 * i + a] + pn[a][i] - 1;
      if (!ok) continue;
      int c1[3], c2[3], cc1[3], cc2[3];
      for (int a = 0; a < 3; a++) {
        const float rr1 = pr[a][j] - 0.5f * dxpa;
        const float rr2 = pr[a][j] - 0.5f * dxpa + (float)(pn[a][j] - 1) * dxpa;
        c1[a] = c2[a] = cc1[a] = cc2[a] = 0;
        veins_axis(r1[a], r2[a], rr1, rr2, dxpa, pn[a][i], pn[a][j], &c1[a], &c2[a], &cc1[a], &cc2[a]);
      }
      int prod = (cc2[2] - cc1[2] + 1) * (cc2[1] - cc1[1] + 1) * (cc2[0] - cc1[0] + 1);
      float ov = fabsf((float)prod) / (float)pnx[j] / (float)pny[j] / (float)pnz[j];
      if (!(ov > 0.1f)) continue;
      for (int kk = cc1[2]; kk <= cc2[2]; kk++)
        for (int jj = cc1[1]; jj <= cc2[1]; jj++)
          for (int ii = cc1[0]; ii <= cc2[0]; ii++) {
            const int ix = ii - cc1[0] + c1[0], jy = jj - cc1[1] + c1[1], kz = kk - cc1[2] + c1[2];
            if (ii < 1 || ii > na || jj < 1 || jj > na || kk < 1 || kk > na || ix < 1 || ix > na || jy < 1 ||
                jy > na || kz < 1 || kz > na)
              continue;
            const size_t qi = (size_t)i * pc + ((size_t)(kz - 1) * na + (jy - 1)) * na + (ix - 1);
            const size_t qj = (size_t)j * pc + ((size_t)(kk - 1) * na + (jj - 1)) * na + (ii - 1);
            if (solap[qi] == 0) {
              solap[qj] = 1;
              cr01[qj] = 0;
              if (conta11) conta11[qj] = 0;
            }
          }
    }
  }
  free(g1);
  free(solap);
  free(nb);
  return rc;
}


/* COMPUTE_CR0AMR (grids.f:2076-2226): CR0AMR(IX,JY,KZ) = 0 for the base
 * cells under a level-1 patch (its odd cells' parents from PATCHX..Z),
 * CR0AMR1 = 0 for the cells of a patch under one of its children (parent
 * cells from PATCHX..Z in the parent's grid, PARE) and, on levels 1..NL-1,
 * for cells inside the cell-centre box of a next-level patch that is not
 * their child; 1 elsewhere.  cr0amr: nx^3; cr0amr1: NAMRX^3 per patch in
 * mesh order (patch q = Fortran index q+1).  Parent cells outside the
 * arrays are skipped. */
void orc_compute_cr0amr(int nx, float lado0, const asohf_mesh *m, int32_t *cr0amr, int32_t *cr0amr1)
{
  const int na = ASOHF_NAMRX;
  const size_t pc = (size_t)na * na * na;
  int ntot = 0;
  for (int l = 0; l <= m->nl; l++) ntot += m->npatch[l];
  for (size_t q = 0; q < (size_t)nx * nx * nx; q++) cr0amr[q] = 1;
  for (size_t q = 0; q < (size_t)ntot * pc; q++) cr0amr1[q] = 1;
  int *lo = malloc(sizeof(int) * (size_t)(m->nl + 2));
  int acc = 0;
  for (int l = 0; l <= m->nl; l++) { lo[l] = acc; acc += m->npatch[l]; }
  lo[m->nl + 1] = acc;
  if (m->nl >= 1)
    for (int i = lo[1]; i < lo[2]; i++)
      for (int kz = 1; kz <= m->patchnz[i]; kz += 2)
        for (int jy = 1; jy <= m->patchny[i]; jy += 2)
          for (int ix = 1; ix <= m->patchnx[i]; ix += 2) {
            const int c1 = m->patchx[i] - 1 + (ix + 1) / 2, c2 = m->patchy[i] - 1 + (jy + 1) / 2,
                      c3 = m->patchz[i] - 1 + (kz + 1) / 2;
            if (c1 < 1 || c1 > nx || c2 < 1 || c2 > nx || c3 < 1 || c3 > nx) continue;
            cr0amr[((size_t)(c3 - 1) * nx + (c2 - 1)) * nx + (c1 - 1)] = 0;
          }
  for (int ir = 2; ir <= m->nl; ir++)
    for (int i = lo[ir]; i < lo[ir + 1]; i++) {
      const int par = m->pare[i] - 1;
      if (par < 0 || par >= ntot) continue;
      for (int kz = 1; kz <= m->patchnz[i]; kz++)
        for (int jy = 1; jy <= m->patchny[i]; jy++)
          for (int ix = 1; ix <= m->patchnx[i]; ix++) {
            const int c1 = m->patchx[i] - 1 + (ix + 1) / 2, c2 = m->patchy[i] - 1 + (jy + 1) / 2,
                      c3 = m->patchz[i] - 1 + (kz + 1) / 2;
            if (c1 < 1 || c1 > na || c2 < 1 || c2 > na || c3 < 1 || c3 > na) continue;
            cr0amr1[(size_t)par * pc + ((size_t)(c3 - 1) * na + (c2 - 1)) * na + (c1 - 1)] = 0;
          }
    }
  const float dx = lado0 / (float)nx;
  for (int ir = 1; ir <= m->nl - 1; ir++) {
    const float dxpa = dx / powf(2.0f, (float)ir);
    for (int i = lo[ir]; i < lo[ir + 1]; i++)
      for (int kz = 1; kz <= m->patchnz[i]; kz++)
        for (int jy = 1; jy <= m->patchny[i]; jy++)
          for (int ix = 1; ix <= m->patchnx[i]; ix++) {
            int32_t *c = &cr0amr1[(size_t)i * pc + ((size_t)(kz - 1) * na + (jy - 1)) * na + (ix - 1)];
            if (*c != 1) continue;
            const float xx = m->patchrx[i] - 0.5f * dxpa + (float)(ix - 1) * dxpa;
            const float yy = m->patchry[i] - 0.5f * dxpa + (float)(jy - 1) * dxpa;
            const float zz = m->patchrz[i] - 0.5f * dxpa + (float)(kz - 1) * dxpa;
            for (int ii = lo[ir + 1]; ii < lo[ir + 2]; ii++) {
              if (m->pare[ii] == i + 1) continue;
              const float xx1 = m->patchrx[ii] - 0.5f * (dxpa * 0.5f);
              const float yy1 = m->patchry[ii] - 0.5f * (dxpa * 0.5f);
              const float zz1 = m->patchrz[ii] - 0.5f * (dxpa * 0.5f);
              const float xx2 = xx1 + (float)(m->patchnx[ii] - 1) * dxpa * 0.5f;
              const float yy2 = yy1 + (float)(m->patchny[ii] - 1) * dxpa * 0.5f;
              const float zz2 = zz1 + (float)(m->patchnz[ii] - 1) * dxpa * 0.5f;
              const float b1 = (xx - xx1) * (xx2 - xx), b2 = (yy - yy1) * (yy2 - yy), b3 = (zz - zz1) * (zz2 - zz);
              if (b1 >= 0.0f && b2 >= 0.0f && b3 >= 0.0f) {
                *c = 0;
                break;
              }
            }
          }
  }
  free(lo);
}

/* VEINSGRID (grids.f:2229-2500): SOLAP = 1 on the level's patches; then,
 * patch I in order and each neighbour J in order (the intersecting cell
 * boxes of VEINSGRID_REDUCED), for each pair of facing cells both still 1,
 * the cell of I is cleared when it lies on I's faces (IX = 1 or N1, ...),
 * else the cell of J.  solap: NAMRX^3 per patch in mesh order; only the
 * level's patches are written.  Cells outside the arrays are skipped. */
void orc_veinsgrid(int ir, float dx, float radx1, const asohf_mesh *m, int32_t *solap)
{
  const int na = ASOHF_NAMRX;
  const size_t pc = (size_t)na * na * na;
  int low1 = 0;
  for (int l = 0; l < ir; l++) low1 += m->npatch[l];
  const int low2 = low1 + m->npatch[ir];
  const float dxpa = dx / powf(2.0f, (float)ir);
  const float fix = radx1 - dx * 0.5f + 0.5f * dxpa;
  const int32_t *pn[3] = {m->patchnx, m->patchny, m->patchnz};
  const float *pr[3] = {m->patchrx, m->patchry, m->patchrz};
  for (int i = low1; i < low2; i++)
    for (size_t q = 0; q < pc; q++) solap[(size_t)i * pc + q] = 1;
  for (int i = low1; i < low2; i++) {
    int g1[3], n[3];
    float r1[3], r2[3];
    for (int a = 0; a < 3; a++) {
      n[a] = pn[a][i];
      g1[a] = (int)(((pr[a][i] - 0.5f * dxpa - fix) / dxpa) + 0.5f) + 1;
      r1[a] = pr[a][i] - 0.5f * dxpa;
      r2[a] = pr[a][i] - 0.5f * dxpa + (float)(n[a] - 1) * dxpa;
    }
    for (int j = low1; j < low2; j++) {
      if (j == i) continue;
      int ok = 1;
      for (int a = 0; a < 3; a++) {
        const int gj = (int)(((pr[a][j] - 0.5f * dxpa - fix) / dxpa) + 0.5f) + 1;
        ok &= g1[a] <= gj + pn[a][j] - 1 && gj <= g1[a] + n[a] - 1;
      }
      if (!ok) continue;
      int c1[3], c2[3], cc1[3], cc2[3];
      for (int a = 0; a < 3; a++) {
        const float rr1 = pr[a][j] - 0.5f * dxpa;
        const float rr2 = pr[a][j] - 0.5f * dxpa + (float)(pn[a][j] - 1) * dxpa;
        c1[a] = c2[a] = cc1[a] = cc2[a] = 0;
        veins_axis(r1[a], r2[a], rr1, rr2, dxpa, n[a], pn[a][j], &c1[a], &c2[a], &cc1[a], &cc2[a]);
      }
      for (int kk = cc1[2]; kk <= cc2[2]; kk++)
        for (int jj = cc1[1]; jj <= cc2[1]; jj++)
          for (int ii = cc1[0]; ii <= cc2[0]; ii++) {
            const int ix = ii - cc1[0] + c1[0], jy = jj - cc1[1] + c1[1], kz = kk - cc1[2] + c1[2];
            if (ii < 1 || ii > na || jj < 1 || jj > na || kk < 1 || kk > na || ix < 1 || ix > na || jy < 1 ||
                jy > na || kz < 1 || kz > na)
              continue;
            int32_t *si = &solap[(size_t)i * pc + ((size_t)(kz - 1) * na + (jy - 1)) * na + (ix - 1)];
            int32_t *sj = &solap[(size_t)j * pc + ((size_t)(kk - 1) * na + (jj - 1)) * na + (ii - 1)];
            if (*si == 1 && *sj == 1) {
              if (ix == 1 || ix == n[0] || jy == 1 || jy == n[1] || kz == 1 || kz == n[2]) *si = 0;
              else *sj = 0;
            }
          }
    }
  }
}
