/*
 * asohf_types.h -- plain-C data layouts shared by the B200 library
 * (libasohf_gpu.so) and its callers.
 *
 * Every array here is laid out exactly as the Fortran driver declares it
 * (asohf.f:47-107), so a Fortran ISO_C_BINDING shim can pass its own arrays
 * straight through: column-major, 1-based logical indices handed over as
 * 0-based pointers.  Halo I (Fortran) is element I-1 here.
 *
 *   ANGULARM(3,NMAXNCLUS)        -> angularm[(I-1)*3 + (j-1)]
 *   EIGENVAL(3,NMAXNCLUS)        -> eigenval[(I-1)*3 + (j-1)]
 *   INERTIA_TENSOR(6,NMAXNCLUS)  -> inertia_tensor[(I-1)*6 + (j-1)]
 *   PROFILES(NBINS,2,NMAXNCLUS)  -> profiles[(I-1)*2*NBINS + (k-1)*NBINS + (b-1)]
 *   INDCS_PARTICLES_PER_HALO(2,.)-> indcs[(I-1)*2 + (j-1)]
 *   U11(NAMRX,NAMRY,NAMRZ,NPALEV)-> u11[(ip-1)*32^3 + (k-1)*32^2 + (j-1)*32 + (i-1)]
 */
#ifndef ASOHF_TYPES_H
#define ASOHF_TYPES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Compile-time sizes of the reference (input_files/asohf_parameters.dat). */
#define ASOHF_NAMRX 32          /* max patch side (NAMRX=NAMRY=NAMRZ) */
#define ASOHF_NBINS 20          /* profile bins (NBINS) */
#define ASOHF_NLEVELS 9         /* max AMR levels (NLEVELS) */
#define ASOHF_N_ESP 9           /* particle species (N_ESP) */
#define ASOHF_NMAX_KERNELS 512  /* 2**NLEVELS */

/* Status codes returned by every entry point (0 = success).  Non-zero codes
 * stand for the reference's `STOP 1` exits; asohf_strerror() gives the text. */
enum {
  ASOHF_OK = 0,
  ASOHF_ERR_INVALID = 1,      /* bad argument (null pointer, size out of range) */
  ASOHF_ERR_CUDA = 2,         /* a CUDA runtime / cuFFT call failed */
  ASOHF_ERR_CAPACITY = 3,     /* a caller-provided output buffer is too small */
  ASOHF_ERR_TIMEOUT = 4,      /* a bounded device wait ran out */
  ASOHF_ERR_NOT_PREFOUND_VIRIAL = 5, /* haloes_particles.f:1483-1486 */
  ASOHF_ERR_WRONG_SORTING = 6,       /* reader.f:267-270 */
  ASOHF_ERR_NO_DEVICE = 7,    /* no usable CUDA device: the library never falls back to the CPU */
  ASOHF_ERR_UNSUPPORTED = 8,  /* option outside the implemented hot path */
  ASOHF_ERR_NOT_CONVERGED = 9 /* haloes_grids.f:482-488: growing not converged */
};

/* AMR patch table (the arrays CREATE_MESH fills, asohf.f:51-62).  Host
 * pointers.  npatch has nl+1 entries (NPATCH(0:NL)); the per-patch arrays
 * have sum(npatch) entries, patches of level ir being contiguous. */
typedef struct asohf_mesh {
  int32_t nl;
  const int32_t *npatch;
  const int32_t *patchnx, *patchny, *patchnz;
  const int32_t *patchx, *patchy, *patchz;
  const float *patchrx, *patchry, *patchrz;
  const int32_t *pare;
} asohf_mesh;

/* Particle store (MODULE PARTICLES, particles.f:1-14), SoA. */
typedef struct asohf_particles {
  int64_t n;
  float *x, *y, *z;       /* RXPA, RYPA, RZPA */
  float *vx, *vy, *vz;    /* U2DM, U3DM, U4DM */
  float *m;               /* MASAP */
  int32_t *id;            /* ORIPA */
} asohf_particles;

/* Scalars the hot path reads from COMMON blocks and the driver. */
typedef struct asohf_consts {
  int32_t nx;          /* NX = NMAX (cubic base grid) */
  float lado0;         /* LADO0, box side (cMpc) */
  float dx;            /* COMMON /ESPACIADO/ DX, as MALLA computes it */
  float rote, rete;    /* COMMON /BACK/ */
  float pi, cgr;       /* COMMON /CONS/ (single precision) */
  float um, uv;        /* mass and velocity units (asohf.f:360-361) */
  float contrastec;    /* BN98 virial contrast, CONTRASTEC */
  float omegaz;        /* OMEGAZ */
  float fdm;           /* fraction of DM mass (FDM) */
  float zeta;          /* redshift */
  int32_t min_num_part;
  int32_t do_compute_energies;
  int32_t max_part_dsum;
  int32_t flag_wdm;
  int32_t var;
} asohf_consts;

/* Halo catalogue: the driver's per-halo SoA arrays (asohf.f:77-107).
 * `capacity` is the declared length (MAXNCLUS = NMAXNCLUS). */
typedef struct asohf_catalogue {
  int32_t nclus;
  int32_t capacity;
  float *masa, *radio;
  float *clusrx, *clusry, *clusrz;
  float *clusrxcm, *clusrycm, *clusrzcm;
  float *msub, *rsub;
  int32_t *patchclus, *realclus, *levhal, *dmpclus;
  float *concentra;
  float *angularm;            /* [3*capacity] */
  float *vmaxclus;
  int32_t *iplip;
  float *vx, *vy, *vz, *mean_vr;
  float *vcmax, *mcmax, *rcmax;
  float *m200c, *r200c, *m500c, *r500c, *m2500c, *r2500c;
  float *m200m, *r200m, *m500m, *r500m, *m2500m, *r2500m;
  float *profiles;            /* [2*NBINS*capacity] */
  float *velocity_dispersion, *kinetic_e, *potential_e;
  int32_t *indcs;             /* INDCS_PARTICLES_PER_HALO, [2*capacity] */
  float *eigenval;            /* [3*capacity] */
  float *inertia_tensor;      /* [6*capacity] */
} asohf_catalogue;

#ifdef __cplusplus
}
#endif
#endif /* ASOHF_TYPES_H */
