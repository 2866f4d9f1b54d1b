! asohf_gpu_mod.f90 -- ISO_C_BINDING shim: same-name replacements of the
! particle hot-path subroutines of ASOHF that forward to libasohf_gpu.so.
!
! Include from asohf.f under `#if gpu == 1` in place of the Fortran bodies of
! DENSITY, RENORM_DENSITY, SORT_DM_PARTICLES_LOCALDENSITY,
! SORT_DM_PARTICLES_X, PRUNE_POOR_HALOES, CHECK_RUBISH,
! ACCIDENTAL_SUBSTRUCTURE, OVERLAPPING (haloes_grids.f:27),
! HALOFIND_PARTICLES and SUBSTRUCTURE_PARTICLES.
! The dummy argument lists are the reference's (grids.f:710, grids.f:2668,
! reader.f:140, grids.f:2726, haloes_particles.f:185,
! haloes_particles.f:259, haloes_particles.f:321, haloes_particles.f:578,
! substructure.f:756).
! Written against those declarations; not compiled in this repository (no
! Fortran compiler is available where it was written).

      MODULE ASOHF_GPU
       USE ISO_C_BINDING
       IMPLICIT NONE

       TYPE, BIND(C) :: ASOHF_MESH_T
        INTEGER(C_INT) :: NL
        TYPE(C_PTR) :: NPATCH, PATCHNX, PATCHNY, PATCHNZ
        TYPE(C_PTR) :: PATCHX, PATCHY, PATCHZ
        TYPE(C_PTR) :: PATCHRX, PATCHRY, PATCHRZ, PARE
       END TYPE

       TYPE, BIND(C) :: ASOHF_PARTICLES_T
        INTEGER(C_INT64_T) :: N
        TYPE(C_PTR) :: X, Y, Z, VX, VY, VZ, M, ID
       END TYPE

       TYPE, BIND(C) :: ASOHF_CONSTS_T
        INTEGER(C_INT) :: NX
        REAL(C_FLOAT) :: LADO0, DX, ROTE, RETE, PI, CGR, UM, UV
        REAL(C_FLOAT) :: CONTRASTEC, OMEGAZ, FDM, ZETA
        INTEGER(C_INT) :: MIN_NUM_PART, DO_COMPUTE_ENERGIES
        INTEGER(C_INT) :: MAX_PART_DSUM, FLAG_WDM, VAR
       END TYPE

       TYPE, BIND(C) :: ASOHF_CATALOGUE_T
        INTEGER(C_INT) :: NCLUS, CAPACITY
        TYPE(C_PTR) :: MASA, RADIO, CLUSRX, CLUSRY, CLUSRZ
        TYPE(C_PTR) :: CLUSRXCM, CLUSRYCM, CLUSRZCM, MSUB, RSUB
        TYPE(C_PTR) :: PATCHCLUS, REALCLUS, LEVHAL, DMPCLUS
        TYPE(C_PTR) :: CONCENTRA, ANGULARM, VMAXCLUS, IPLIP
        TYPE(C_PTR) :: VX, VY, VZ, MEAN_VR, VCMAX, MCMAX, RCMAX
        TYPE(C_PTR) :: M200C, R200C, M500C, R500C, M2500C, R2500C
        TYPE(C_PTR) :: M200M, R200M, M500M, R500M, M2500M, R2500M
        TYPE(C_PTR) :: PROFILES, VELOCITY_DISPERSION, KINETIC_E
        TYPE(C_PTR) :: POTENTIAL_E, INDCS, EIGENVAL, INERTIA_TENSOR
       END TYPE

       TYPE(C_PTR), SAVE :: CTX = C_NULL_PTR

       INTERFACE
        INTEGER(C_INT) FUNCTION ASOHF_CREATE(DEV, OUT)
     &   BIND(C, NAME='asohf_create')
         IMPORT :: C_INT, C_PTR
         INTEGER(C_INT), VALUE :: DEV
         TYPE(C_PTR) :: OUT
        END FUNCTION
        TYPE(C_PTR) FUNCTION ASOHF_STRERROR(CODE)
     &   BIND(C, NAME='asohf_strerror')
         IMPORT :: C_INT, C_PTR
         INTEGER(C_INT), VALUE :: CODE
        END FUNCTION
        INTEGER(C_INT) FUNCTION ASOHF_UPLOAD_PARTICLES(C, P, ONDEV)
     &   BIND(C, NAME='asohf_upload_particles')
         IMPORT :: C_INT, C_PTR, ASOHF_PARTICLES_T
         TYPE(C_PTR), VALUE :: C
         TYPE(ASOHF_PARTICLES_T) :: P
         INTEGER(C_INT), VALUE :: ONDEV
        END FUNCTION
        INTEGER(C_INT) FUNCTION ASOHF_DOWNLOAD_PARTICLES(C, P, ONDEV)
     &   BIND(C, NAME='asohf_download_particles')
         IMPORT :: C_INT, C_PTR, ASOHF_PARTICLES_T
         TYPE(C_PTR), VALUE :: C
         TYPE(ASOHF_PARTICLES_T) :: P
         INTEGER(C_INT), VALUE :: ONDEV
        END FUNCTION
        INTEGER(C_INT) FUNCTION ASOHF_SORT_LOCALDENSITY(C, NX, DX,
     &   RODO, RE0, NPART_ESP)
     &   BIND(C, NAME='asohf_sort_dm_particles_localdensity')
         IMPORT :: C_INT, C_PTR, C_FLOAT
         TYPE(C_PTR), VALUE :: C
         INTEGER(C_INT), VALUE :: NX
         REAL(C_FLOAT), VALUE :: DX, RODO, RE0
         INTEGER(C_INT) :: NPART_ESP(*)
        END FUNCTION
        INTEGER(C_INT) FUNCTION ASOHF_DENSITY_C(C, NX, LADO0, DX, ROTE,
     &   RETE, NPART_ESP, MESH, DEG, U1, U11, ONDEV)
     &   BIND(C, NAME='asohf_density')
         IMPORT :: C_INT, C_PTR, C_FLOAT, ASOHF_MESH_T
         TYPE(C_PTR), VALUE :: C
         INTEGER(C_INT), VALUE :: NX, DEG, ONDEV
         REAL(C_FLOAT), VALUE :: LADO0, DX, ROTE, RETE
         INTEGER(C_INT) :: NPART_ESP(*)
         TYPE(ASOHF_MESH_T) :: MESH
         REAL(C_FLOAT) :: U1(*), U11(*)
        END FUNCTION
        INTEGER(C_INT) FUNCTION ASOHF_RENORM_C(C, NX, MESH, FDM, U1,
     &   U11, ONDEV) BIND(C, NAME='asohf_renorm_density')
         IMPORT :: C_INT, C_PTR, C_FLOAT, ASOHF_MESH_T
         TYPE(C_PTR), VALUE :: C
         INTEGER(C_INT), VALUE :: NX, ONDEV
         TYPE(ASOHF_MESH_T) :: MESH
         REAL(C_FLOAT), VALUE :: FDM
         REAL(C_FLOAT) :: U1(*), U11(*)
        END FUNCTION
        INTEGER(C_INT) FUNCTION ASOHF_SORT_X_C(C, NX, LADO0, NDMPART_X)
     &   BIND(C, NAME='asohf_sort_dm_particles_x')
         IMPORT :: C_INT, C_PTR, C_FLOAT
         TYPE(C_PTR), VALUE :: C
         INTEGER(C_INT), VALUE :: NX
         REAL(C_FLOAT), VALUE :: LADO0
         INTEGER(C_INT) :: NDMPART_X(*)
        END FUNCTION
        INTEGER(C_INT) FUNCTION ASOHF_PRUNE_C(C, K, CAT, LOW1, LOW2,
     &   FACRAD, DOCOUNT, ONDEV) BIND(C, NAME='asohf_prune_poor_haloes')
         IMPORT :: C_INT, C_PTR, C_FLOAT, ASOHF_CONSTS_T,
     &             ASOHF_CATALOGUE_T
         TYPE(C_PTR), VALUE :: C
         TYPE(ASOHF_CONSTS_T) :: K
         TYPE(ASOHF_CATALOGUE_T) :: CAT
         INTEGER(C_INT), VALUE :: LOW1, LOW2, DOCOUNT, ONDEV
         REAL(C_FLOAT), VALUE :: FACRAD
        END FUNCTION
        INTEGER(C_INT) FUNCTION ASOHF_HALOFIND_C(C, K, MESH, CAT, LOW1,
     &   LOW2, ONDEV) BIND(C, NAME='asohf_halofind_particles')
         IMPORT :: C_INT, C_PTR, ASOHF_CONSTS_T, ASOHF_MESH_T,
     &             ASOHF_CATALOGUE_T
         TYPE(C_PTR), VALUE :: C
         TYPE(ASOHF_CONSTS_T) :: K
         TYPE(ASOHF_MESH_T) :: MESH
         TYPE(ASOHF_CATALOGUE_T) :: CAT
         INTEGER(C_INT), VALUE :: LOW1, LOW2, ONDEV
        END FUNCTION
        INTEGER(C_INT) FUNCTION ASOHF_SUBSTRUCTURE_C(C, K, MESH, CAT, IR,
     &   SUBS_LEV, ONDEV) BIND(C, NAME='asohf_substructure_particles')
         IMPORT :: C_INT, C_PTR, ASOHF_CONSTS_T, ASOHF_MESH_T,
     &             ASOHF_CATALOGUE_T
         TYPE(C_PTR), VALUE :: C
         TYPE(ASOHF_CONSTS_T) :: K
         TYPE(ASOHF_MESH_T) :: MESH
         TYPE(ASOHF_CATALOGUE_T) :: CAT
         INTEGER(C_INT), VALUE :: IR, ONDEV
         INTEGER(C_INT) :: SUBS_LEV(*)
        END FUNCTION
        INTEGER(C_INT) FUNCTION ASOHF_GET_PPH_C(C, OUT, CAP, N, ONDEV)
     &   BIND(C, NAME='asohf_get_particles_per_halo')
         IMPORT :: C_INT, C_PTR, C_INT64_T
         TYPE(C_PTR), VALUE :: C
         INTEGER(C_INT) :: OUT(*)
         INTEGER(C_INT64_T), VALUE :: CAP
         INTEGER(C_INT64_T) :: N
         INTEGER(C_INT), VALUE :: ONDEV
        END FUNCTION
        INTEGER(C_INT) FUNCTION ASOHF_CHECK_RUBISH_C(C, CAT, NCLUS, LOW1,
     &   LOW2, ONDEV, KONTA) BIND(C, NAME='asohf_check_rubish')
         IMPORT :: C_INT, C_PTR, ASOHF_CATALOGUE_T
         TYPE(C_PTR), VALUE :: C
         TYPE(ASOHF_CATALOGUE_T) :: CAT
         INTEGER(C_INT), VALUE :: NCLUS, LOW1, LOW2, ONDEV
         INTEGER(C_INT) :: KONTA
        END FUNCTION
        INTEGER(C_INT) FUNCTION ASOHF_ACCIDENTAL_C(C, CAT, NCLUS, ONDEV,
     &   KONTA) BIND(C, NAME='asohf_accidental_substructure')
         IMPORT :: C_INT, C_PTR, ASOHF_CATALOGUE_T
         TYPE(C_PTR), VALUE :: C
         TYPE(ASOHF_CATALOGUE_T) :: CAT
         INTEGER(C_INT), VALUE :: NCLUS, ONDEV
         INTEGER(C_INT) :: KONTA
        END FUNCTION
        INTEGER(C_INT) FUNCTION ASOHF_OVERLAPPING_C(C, CAT, IR, NHALLEV,
     &   VOLSOL, ONDEV, NREM) BIND(C, NAME='asohf_overlapping')
         IMPORT :: C_INT, C_PTR, C_FLOAT, ASOHF_CATALOGUE_T
         TYPE(C_PTR), VALUE :: C
         TYPE(ASOHF_CATALOGUE_T) :: CAT
         INTEGER(C_INT), VALUE :: IR, ONDEV
         INTEGER(C_INT) :: NHALLEV(*), NREM
         REAL(C_FLOAT), VALUE :: VOLSOL
        END FUNCTION
        INTEGER(C_INT) FUNCTION ASOHF_MESH_BASE_COUNTS_C(C, NX, DX,
     &   REFINE_THR, BOR, NPART_ESP, CR0, ONDEV)
     &   BIND(C, NAME='asohf_mesh_base_counts')
         IMPORT :: C_INT, C_PTR, C_FLOAT
         TYPE(C_PTR), VALUE :: C
         INTEGER(C_INT), VALUE :: NX, REFINE_THR, BOR, ONDEV
         REAL(C_FLOAT), VALUE :: DX
         INTEGER(C_INT) :: NPART_ESP(*), CR0(*)
        END FUNCTION
        INTEGER(C_INT) FUNCTION ASOHF_MESH_PATCH_COUNTS_C(C, NX, LADO0,
     &   DX, IRPA, REFINE_THR, BORAMR, NPART_ESP, NPATCH, PNX, PNY, PNZ,
     &   PRX, PRY, PRZ, CR01, ONDEV)
     &   BIND(C, NAME='asohf_mesh_patch_counts')
         IMPORT :: C_INT, C_PTR, C_FLOAT
         TYPE(C_PTR), VALUE :: C
         INTEGER(C_INT), VALUE :: NX, IRPA, REFINE_THR, BORAMR, NPATCH
         INTEGER(C_INT), VALUE :: ONDEV
         REAL(C_FLOAT), VALUE :: LADO0, DX
         INTEGER(C_INT) :: NPART_ESP(*), PNX(*), PNY(*), PNZ(*), CR01(*)
         REAL(C_FLOAT) :: PRX(*), PRY(*), PRZ(*)
        END FUNCTION
        INTEGER(C_INT) FUNCTION ASOHF_VEINSGRID_REDUCED_C(C, IR, DX,
     &   RADX1, NPATCH, PNX, PNY, PNZ, PRX, PRY, PRZ, MAXNB, CR01,
     &   CONTA11, ONDEV) BIND(C, NAME='asohf_veinsgrid_reduced')
         IMPORT :: C_INT, C_PTR, C_FLOAT
         TYPE(C_PTR), VALUE :: C
         INTEGER(C_INT), VALUE :: IR, NPATCH, MAXNB, ONDEV
         REAL(C_FLOAT), VALUE :: DX, RADX1
         INTEGER(C_INT) :: PNX(*), PNY(*), PNZ(*), CR01(*), CONTA11(*)
         REAL(C_FLOAT) :: PRX(*), PRY(*), PRZ(*)
        END FUNCTION
       END INTERFACE

      CONTAINS

       SUBROUTINE ASOHF_CHECK(RC, WHAT)
*       The reference's STOP 1 on a non-zero status.
        INTEGER(C_INT) :: RC
        CHARACTER(*) :: WHAT
        IF (RC.NE.0) THEN
         WRITE(*,*) 'ASOHF GPU error in ', WHAT, ': status', RC
         STOP 1
        END IF
       END SUBROUTINE

       SUBROUTINE ASOHF_ENSURE_CTX()
        IF (.NOT.C_ASSOCIATED(CTX)) THEN
         CALL ASOHF_CHECK(ASOHF_CREATE(0_C_INT, CTX), 'asohf_create')
        END IF
       END SUBROUTINE

      END MODULE ASOHF_GPU

! Replacement of SORT_DM_PARTICLES_X (grids.f:2726-2838): same dummies.
      SUBROUTINE SORT_DM_PARTICLES_X(N_DM,NDMPART_X,NX,LADO0)
       USE PARTICLES
       USE ASOHF_GPU
       IMPLICIT NONE
       INCLUDE 'input_files/asohf_parameters.dat'
       INTEGER N_DM,NDMPART_X(0:NMAX),NX
       REAL*4 LADO0
       TYPE(ASOHF_PARTICLES_T), TARGET :: P
       CALL ASOHF_ENSURE_CTX()
       P%N=N_DM
       P%X=C_LOC(RXPA); P%Y=C_LOC(RYPA); P%Z=C_LOC(RZPA)
       P%VX=C_LOC(U2DM); P%VY=C_LOC(U3DM); P%VZ=C_LOC(U4DM)
       P%M=C_LOC(MASAP); P%ID=C_LOC(ORIPA)
       CALL ASOHF_CHECK(ASOHF_UPLOAD_PARTICLES(CTX, P, 0_C_INT),
     &                  'upload')
       CALL ASOHF_CHECK(ASOHF_SORT_X_C(CTX, NX, LADO0, NDMPART_X),
     &                  'SORT_DM_PARTICLES_X')
       CALL ASOHF_CHECK(ASOHF_DOWNLOAD_PARTICLES(CTX, P, 0_C_INT),
     &                  'download')
      END SUBROUTINE

! Replacement of CHECK_RUBISH (haloes_particles.f:259-318): same dummies.
! Only the fields the test reads are bound; the rest stay C_NULL_PTR.
      SUBROUTINE CHECK_RUBISH(NCLUS,REALCLUS,CLUSRX,CLUSRY,CLUSRZ,VX,
     &                        VY,VZ,MASA,RADIO,LEVHAL,LOWH1,LOWH2)
       USE ASOHF_GPU
       IMPLICIT NONE
       INCLUDE 'input_files/asohf_parameters.dat'
       INTEGER NCLUS,LOWH1,LOWH2
       INTEGER, TARGET :: REALCLUS(MAXNCLUS),LEVHAL(MAXNCLUS)
       REAL*4, TARGET :: CLUSRX(MAXNCLUS),CLUSRY(MAXNCLUS),
     &                   CLUSRZ(MAXNCLUS),RADIO(MAXNCLUS),MASA(MAXNCLUS)
       REAL*4, TARGET :: VX(NMAXNCLUS),VY(NMAXNCLUS),VZ(NMAXNCLUS)
       TYPE(ASOHF_CATALOGUE_T) :: CAT
       INTEGER(C_INT) :: KONTA
       CALL ASOHF_ENSURE_CTX()
       CAT%NCLUS=NCLUS; CAT%CAPACITY=MAXNCLUS
       CAT%CLUSRX=C_LOC(CLUSRX); CAT%CLUSRY=C_LOC(CLUSRY)
       CAT%CLUSRZ=C_LOC(CLUSRZ); CAT%VX=C_LOC(VX); CAT%VY=C_LOC(VY)
       CAT%VZ=C_LOC(VZ); CAT%MASA=C_LOC(MASA); CAT%RADIO=C_LOC(RADIO)
       CAT%LEVHAL=C_LOC(LEVHAL); CAT%REALCLUS=C_LOC(REALCLUS)
       CALL ASOHF_CHECK(ASOHF_CHECK_RUBISH_C(CTX, CAT, NCLUS, LOWH1,
     &                  LOWH2, 0_C_INT, KONTA), 'CHECK_RUBISH')
       WRITE(*,*)'... Checking rubbish ----->', KONTA
      END SUBROUTINE

! Replacement of ACCIDENTAL_SUBSTRUCTURE (haloes_particles.f:321-364).
      SUBROUTINE ACCIDENTAL_SUBSTRUCTURE(NCLUS,REALCLUS,CLUSRX,CLUSRY,
     &                                   CLUSRZ,VX,VY,VZ,MASA,RADIO,
     &                                   LEVHAL)
       USE ASOHF_GPU
       IMPLICIT NONE
       INCLUDE 'input_files/asohf_parameters.dat'
       INTEGER NCLUS
       INTEGER, TARGET :: REALCLUS(MAXNCLUS),LEVHAL(MAXNCLUS)
       REAL*4, TARGET :: CLUSRX(MAXNCLUS),CLUSRY(MAXNCLUS),
     &                   CLUSRZ(MAXNCLUS),RADIO(MAXNCLUS),MASA(MAXNCLUS)
       REAL*4, TARGET :: VX(NMAXNCLUS),VY(NMAXNCLUS),VZ(NMAXNCLUS)
       TYPE(ASOHF_CATALOGUE_T) :: CAT
       INTEGER(C_INT) :: KONTA
       CALL ASOHF_ENSURE_CTX()
       CAT%NCLUS=NCLUS; CAT%CAPACITY=MAXNCLUS
       CAT%CLUSRX=C_LOC(CLUSRX); CAT%CLUSRY=C_LOC(CLUSRY)
       CAT%CLUSRZ=C_LOC(CLUSRZ); CAT%VX=C_LOC(VX); CAT%VY=C_LOC(VY)
       CAT%VZ=C_LOC(VZ); CAT%MASA=C_LOC(MASA); CAT%RADIO=C_LOC(RADIO)
       CAT%LEVHAL=C_LOC(LEVHAL); CAT%REALCLUS=C_LOC(REALCLUS)
       CALL ASOHF_CHECK(ASOHF_ACCIDENTAL_C(CTX, CAT, NCLUS, 0_C_INT,
     &                  KONTA), 'ACCIDENTAL_SUBSTRUCTURE')
       WRITE(*,*)'... Checking accidental substructure ----->', KONTA
      END SUBROUTINE

! Replacement of OVERLAPPING (haloes_grids.f:27-201): same dummies; the
! mesh, SOLAP, CR0AMR and density arguments are not read by the routine.
      SUBROUTINE OVERLAPPING(IR,NL,NX,NY,NZ,NPATCH,PATCHNX,PATCHNY,
     &                       PATCHNZ,PATCHX,PATCHY,PATCHZ,PATCHRX,
     &                       PATCHRY,PATCHRZ,PARE,NCLUS,MASA,RADIO,
     &                       CLUSRX,CLUSRY,CLUSRZ,REALCLUS,LEVHAL,
     &                       NHALLEV,BOUND,CONTRASTEC,RODO,SOLAP,
     &                       CR0AMR,CR0AMR11,VOL_SOLAP_LOW)
       USE ASOHF_GPU
       IMPLICIT NONE
       INCLUDE 'input_files/asohf_parameters.dat'
       INTEGER IR,NL,NX,NY,NZ
       INTEGER NPATCH(0:NLEVELS)
       INTEGER PATCHNX(NPALEV),PATCHNY(NPALEV),PATCHNZ(NPALEV)
       INTEGER PATCHX(NPALEV),PATCHY(NPALEV),PATCHZ(NPALEV)
       REAL PATCHRX(NPALEV),PATCHRY(NPALEV),PATCHRZ(NPALEV)
       INTEGER PARE(NPALEV)
       INTEGER NCLUS
       REAL, TARGET :: MASA(MAXNCLUS),RADIO(MAXNCLUS)
       REAL*4, TARGET :: CLUSRX(MAXNCLUS),CLUSRY(MAXNCLUS),
     &                   CLUSRZ(MAXNCLUS)
       INTEGER, TARGET :: REALCLUS(MAXNCLUS),LEVHAL(MAXNCLUS)
       INTEGER NHALLEV(0:NLEVELS)
       REAL BOUND,CONTRASTEC,RODO
       INTEGER SOLAP(NAMRX,NAMRY,NAMRZ,NPALEV)
       INTEGER CR0AMR(NMAX,NMAY,NMAZ)
       INTEGER CR0AMR11(NAMRX,NAMRY,NAMRZ,NPALEV)
       REAL VOL_SOLAP_LOW
       TYPE(ASOHF_CATALOGUE_T) :: CAT
       INTEGER(C_INT) :: NREM
       CALL ASOHF_ENSURE_CTX()
       CAT%NCLUS=NCLUS; CAT%CAPACITY=MAXNCLUS
       CAT%CLUSRX=C_LOC(CLUSRX); CAT%CLUSRY=C_LOC(CLUSRY)
       CAT%CLUSRZ=C_LOC(CLUSRZ); CAT%MASA=C_LOC(MASA)
       CAT%RADIO=C_LOC(RADIO); CAT%LEVHAL=C_LOC(LEVHAL)
       CAT%REALCLUS=C_LOC(REALCLUS)
       CALL ASOHF_CHECK(ASOHF_OVERLAPPING_C(CTX, CAT, IR, NHALLEV,
     &                  VOL_SOLAP_LOW, 0_C_INT, NREM), 'OVERLAPPING')
       WRITE(*,*) '... of these, overlapping: ', NREM
      END SUBROUTINE

! The other replacements (DENSITY, RENORM_DENSITY,
! SORT_DM_PARTICLES_LOCALDENSITY, PRUNE_POOR_HALOES, HALOFIND_PARTICLES,
! SUBSTRUCTURE_PARTICLES) follow the same pattern: fill ASOHF_MESH_T from
! NPATCH..PARE, ASOHF_CONSTS_T from the COMMON blocks (/ESPACIADO/, /BACK/,
! /CONS/) and the routine's dummies, ASOHF_CATALOGUE_T with C_LOC of the
! driver's catalogue arrays (NCLUS, MAXNCLUS), call the entry point with
! ONDEV=0, and after HALOFIND_PARTICLES / SUBSTRUCTURE_PARTICLES copy the
! ID stream into PARTICLES_PER_HALO with ASOHF_GET_PPH_C.
