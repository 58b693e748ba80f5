C  Replacements for source_code/mdprop.f, ldprop.f and mgprop.f that
C  run the propagation in libmolscat_gpu.so (sm_100a, FP64).  Same
C  argument lists and meanings as MDPROP (mdprop.f:1-4), LDPROP
C  (ldprop.f:1-4) and MGPROP with its MGISEL entry (mgprop.f:1-4,
C  144-156); same hidden inputs (module potential, /VLFLAG/,
C  /VLSAVE/, /PRPSCR/); same STOP messages on an inversion failure.
C
C  Build: add this file to the Makefile's object list in place of
C  mdprop.f, ldprop.f and mgprop.f and link with -L<dir>
C  -lmolscat_gpu.
C
C  What crosses the boundary: the R-dependent half of HAMMAT (POTENL,
C  the +-1E60 clamp, VCONST, SCAPOT, PERTRB, EP2RU, the 1/R**2 terms;
C  hammat.f:31-83) is user code, so HAMPVC evaluates the P vector SUMLAM
C  would receive at every radius the propagator visits, R = RSTART + K*H,
C  K = 0..2*NSTEP, accumulated as R=R+H like mdprop.f:117,203; the
C  library adds CENT/R**2, EINT, the confinement and -ERED on the device
C  as hammat.f:85-113 does.  Arguments pass by reference through plain
C  ISO_C_BINDING interface blocks (mgpu_mdprop_f / mgpu_ldprop_f in
C  include/molscat_gpu.h): no derived types and no C_LOC.
C
C  Not covered (the routine stops with a message): WAVE=.TRUE., the
C  ISCRU scratch file (IREAD/IWRITE), IVLU>0, and IVLFL>0 with a P
C  vector longer than NHAM.
C
      SUBROUTINE MDPROP(N,MXLAM,NHAM,
     1                  Y,VL,IV,EINT,CENT,
     2                  RSTART,RSTOP,NSTEP,DR,NODES,IREC,WAVE,
     3                  ERED,EP2RU,CM2RU,RSCALE,IPRINT)
      USE potential, ONLY: NCONST, NRSQ, NVLBLK, CONLEN
      IMPLICIT DOUBLE PRECISION (A-H,O-Z)
      LOGICAL WAVE
      DIMENSION Y(N,N),VL(*),IV(*),EINT(N),CENT(N)
      ALLOCATABLE :: RTAB(:),PTAB(:,:)
      COMMON /VLFLAG/ IVLFL
      COMMON /VLSAVE/ IVLU
      LOGICAL IREAD,IWRITE,IREADR,IWRITR
      COMMON /PRPSCR/ ESHIFT,ISCRU,ISCRUR,IREAD,IWRITE,IREADR,IWRITR
      INTERFACE
        SUBROUTINE MGPU_MDPROP_F(N,NHAM,NVLBLK,IVLFL,NCONST,NRSQ,
     1                           CONLEN,Y,VL,IV,EINT,CENT,NSTEP,DR,
     2                           RTAB,PTAB,ERED,NODES,KFAIL,ISTAT)
     3      BIND(C,NAME='mgpu_mdprop_f')
          USE ISO_C_BINDING, ONLY: C_INT, C_DOUBLE
          INTEGER(C_INT) N,NHAM,NVLBLK,IVLFL,NCONST,NRSQ,IV(*),NSTEP,
     1                   NODES,KFAIL,ISTAT
          REAL(C_DOUBLE) CONLEN,Y(*),VL(*),EINT(*),CENT(*),DR,
     1                   RTAB(*),PTAB(*),ERED
        END SUBROUTINE
      END INTERFACE
C
      CALL GPUCHK('MDPROP',WAVE,IREAD,IWRITE,IVLU,IVLFL,
     1            MXLAM+NCONST+NRSQ,NHAM)
      NP=MAX(NHAM,1)
      ALLOCATE (RTAB(2*NSTEP+1),PTAB(NP,2*NSTEP+1))
      CALL GPUTAB(RSTART,DR,NSTEP,RTAB,PTAB,NP,MXLAM,NHAM,EP2RU,CM2RU,
     1            RSCALE,IPRINT)
      CALL MGPU_MDPROP_F(N,NHAM,NVLBLK,IVLFL,NCONST,NRSQ,CONLEN,Y,VL,
     1                   IV,EINT,CENT,NSTEP,DR,RTAB,PTAB,ERED,NODES,
     2                   KFAIL,ISTAT)
      DEALLOCATE (RTAB,PTAB)
      IF (ISTAT.EQ.1 .OR. ISTAT.EQ.2) THEN
        WRITE(6,1000) KFAIL
        STOP
      ELSEIF (ISTAT.NE.0) THEN
        WRITE(6,1010) ISTAT
        STOP
      ENDIF
      RETURN
 1000 FORMAT(/' ***** MDPROP: MATRIX INVERSION ERROR AT STEP K = ',I6,
     &       '.  RUN HALTED.')
 1010 FORMAT(/' ***** MDPROP: libmolscat_gpu STATUS ',I3,
     &       ' (include/molscat_gpu.h).  RUN HALTED.')
      END
C
      SUBROUTINE LDPROP(N,MXLAM,NHAM,
     1                  Z,VL,IV,EINT,CENT,
     2                  RSTART,RSTOP,NSTEP,DR,NODES,
     3                  ERED,EP2RU,CM2RU,RSCALE,IPRINT)
      USE potential, ONLY: NCONST, NRSQ, NVLBLK, CONLEN
      IMPLICIT DOUBLE PRECISION (A-H,O-Z)
      LOGICAL NOWAVE
      DIMENSION Z(N,N),VL(*),IV(*),EINT(N),CENT(N)
      ALLOCATABLE :: RTAB(:),PTAB(:,:)
      COMMON /VLFLAG/ IVLFL
      COMMON /VLSAVE/ IVLU
      LOGICAL IREAD,IWRITE,IREADR,IWRITR
      COMMON /PRPSCR/ ESHIFT,ISCRU,ISCRUR,IREAD,IWRITE,IREADR,IWRITR
      INTERFACE
        SUBROUTINE MGPU_LDPROP_F(N,NHAM,NVLBLK,IVLFL,NCONST,NRSQ,
     1                           CONLEN,Z,VL,IV,EINT,CENT,NSTEP,DR,
     2                           RTAB,PTAB,ERED,NODES,KFAIL,ISTAT)
     3      BIND(C,NAME='mgpu_ldprop_f')
          USE ISO_C_BINDING, ONLY: C_INT, C_DOUBLE
          INTEGER(C_INT) N,NHAM,NVLBLK,IVLFL,NCONST,NRSQ,IV(*),NSTEP,
     1                   NODES,KFAIL,ISTAT
          REAL(C_DOUBLE) CONLEN,Z(*),VL(*),EINT(*),CENT(*),DR,
     1                   RTAB(*),PTAB(*),ERED
        END SUBROUTINE
      END INTERFACE
C
      NOWAVE=.FALSE.
      CALL GPUCHK('LDPROP',NOWAVE,IREAD,IWRITE,IVLU,IVLFL,
     1            MXLAM+NCONST+NRSQ,NHAM)
      NP=MAX(NHAM,1)
      ALLOCATE (RTAB(2*NSTEP+1),PTAB(NP,2*NSTEP+1))
      CALL GPUTAB(RSTART,DR,NSTEP,RTAB,PTAB,NP,MXLAM,NHAM,EP2RU,CM2RU,
     1            RSCALE,IPRINT)
      CALL MGPU_LDPROP_F(N,NHAM,NVLBLK,IVLFL,NCONST,NRSQ,CONLEN,Z,VL,
     1                   IV,EINT,CENT,NSTEP,DR,RTAB,PTAB,ERED,NODES,
     2                   KFAIL,ISTAT)
      DEALLOCATE (RTAB,PTAB)
      IF (ISTAT.EQ.1 .OR. ISTAT.EQ.2) THEN
        WRITE(6,901)
        STOP
      ELSEIF (ISTAT.NE.0) THEN
        WRITE(6,1010) ISTAT
        STOP
      ENDIF
      RETURN
  901 FORMAT(/' *** ERROR IN SYMINV CALLED FROM LDPROP - TERMINATING')
 1010 FORMAT(/' ***** LDPROP: libmolscat_gpu STATUS ',I3,
     &       ' (include/molscat_gpu.h).  RUN HALTED.')
      END
C
      SUBROUTINE MGPROP(N,MXLAM,NHAM,
     1                  Y,VL,IV,EINT,CENT,
     2                  RSTART,RSTOP,NSTEP,DR,NODES,
     3                  ERED,EP2RU,CM2RU,RSCALE,IPRINT)
C  IMGSEL (4: CS4, 5: MA5) as set through MGISEL; the stage radii
C  come from the library (mgpu_ldmg_radii), the P vectors from HAMPVC.
      USE potential, ONLY: NCONST, NRSQ, NVLBLK, CONLEN
      USE ISO_C_BINDING, ONLY: C_INT, C_DOUBLE
      IMPLICIT DOUBLE PRECISION (A-H,O-Z)
      LOGICAL NOWAVE
      DIMENSION Y(N,N),VL(*),IV(*),EINT(N),CENT(N)
      ALLOCATABLE :: RTAB(:),PTAB(:,:),P(:)
      COMMON /VLFLAG/ IVLFL
      COMMON /VLSAVE/ IVLU
      LOGICAL IREAD,IWRITE,IREADR,IWRITR
      COMMON /PRPSCR/ ESHIFT,ISCRU,ISCRUR,IREAD,IWRITE,IREADR,IWRITR
      COMMON /MGPUSL/ IMGSLC
      INTERFACE
        SUBROUTINE MGPU_MGPROP_F(IMGSEL,N,NHAM,NVLBLK,IVLFL,NCONST,
     1                           NRSQ,CONLEN,Y,VL,IV,EINT,CENT,NSTEP,
     2                           DR,RTAB,PTAB,ERED,NODES,KFAIL,ISTAT)
     3      BIND(C,NAME='mgpu_mgprop_f')
          USE ISO_C_BINDING, ONLY: C_INT, C_DOUBLE
          INTEGER(C_INT) IMGSEL,N,NHAM,NVLBLK,IVLFL,NCONST,NRSQ,IV(*),
     1                   NSTEP,NODES,KFAIL,ISTAT
          REAL(C_DOUBLE) CONLEN,Y(*),VL(*),EINT(*),CENT(*),DR,
     1                   RTAB(*),PTAB(*),ERED
        END SUBROUTINE
        INTEGER(C_INT) FUNCTION MGPU_LDMG_RADII(IPROP,RSTART,DR,
     1                                          NSTEP,RTAB)
     2      BIND(C,NAME='mgpu_ldmg_radii')
          USE ISO_C_BINDING, ONLY: C_INT, C_DOUBLE
          INTEGER(C_INT), VALUE :: IPROP,NSTEP
          REAL(C_DOUBLE), VALUE :: RSTART,DR
          REAL(C_DOUBLE) RTAB(*)
        END FUNCTION
      END INTERFACE
C
      NOWAVE=.FALSE.
      CALL GPUCHK('MGPROP',NOWAVE,IREAD,IWRITE,IVLU,IVLFL,
     1            MXLAM+NCONST+NRSQ,NHAM)
      IF (IMGSLC.NE.5) IMGSLC=4
      IPROP=80+IMGSLC
      NP=MAX(NHAM,1)
      NR=MAX(4*NSTEP+1,6*NSTEP)
      ALLOCATE (RTAB(NR),PTAB(NP,NR))
      ALLOCATE (P(MAX(MXLAM+NCONST+NRSQ,NHAM,1)))
      NR=MGPU_LDMG_RADII(IPROP,RSTART,DR,NSTEP,RTAB)
      DO K=1,NR
        P=0.D0
        CALL HAMPVC(RTAB(K),P,MXLAM,EP2RU,CM2RU,RSCALE,IPRINT)
        DO I=1,NHAM
          PTAB(I,K)=P(I)
        ENDDO
      ENDDO
      CALL MGPU_MGPROP_F(IMGSLC,N,NHAM,NVLBLK,IVLFL,NCONST,NRSQ,
     1                   CONLEN,Y,VL,IV,EINT,CENT,NSTEP,DR,RTAB,PTAB,
     2                   ERED,NODES,KFAIL,ISTAT)
      DEALLOCATE (RTAB,PTAB,P)
      IF (ISTAT.NE.0) THEN
        WRITE(6,1010) ISTAT,KFAIL
        STOP
      ENDIF
      RETURN
 1010 FORMAT(/' ***** MGPROP: libmolscat_gpu STATUS ',I3,
     &       ' IN SECTOR ',I6,' (include/molscat_gpu.h).  RUN HALTED.')
      END
C
      SUBROUTINE MGISEL(IMGSEL)
C  The MGPROP method: 4 (CS4) or 5 (MA5), as mgprop.f:144-156.
      COMMON /MGPUSL/ IMGSLC
      IF (IMGSEL.EQ.4 .OR. IMGSEL.EQ.5) THEN
        IMGSLC=IMGSEL
      ELSE
        WRITE(6,*) ' *** ERROR *** ONLY CS4 AND MA5 SYMPLECTIC '//
     1             'PROPAGATORS CODED AT THE MOMENT'
        STOP
      ENDIF
      RETURN
      END
C
      SUBROUTINE GPUCHK(NAME,WAVE,IREAD,IWRITE,IVLU,IVLFL,NPTOT,NHAM)
C  Stops on the inputs the library does not cover.
      CHARACTER(*) NAME
      LOGICAL WAVE,IREAD,IWRITE
      IF (WAVE) THEN
        WRITE(6,*) ' *** ',NAME,' (GPU): WAVE=.TRUE. NOT SUPPORTED'
        STOP
      ENDIF
      IF (IREAD .OR. IWRITE) THEN
        WRITE(6,*) ' *** ',NAME,' (GPU): ISCRU SCRATCH FILE NOT ',
     1             'SUPPORTED (ENERGIES SHARE U(C) ON THE DEVICE)'
        STOP
      ENDIF
      IF (IVLU.GT.0) THEN
        WRITE(6,*) ' *** ',NAME,' (GPU): IVLU>0 NOT SUPPORTED'
        STOP
      ENDIF
      IF (IVLFL.GT.0 .AND. NPTOT.GT.NHAM) THEN
        WRITE(6,*) ' *** ',NAME,' (GPU): IVLFL>0 NEEDS ',
     1             'MXLAM+NCONST+NRSQ <= NHAM'
        STOP
      ENDIF
      RETURN
      END
C
      SUBROUTINE GPUTAB(RSTART,DR,NSTEP,RTAB,PTAB,NP,MXLAM,NHAM,
     1                  EP2RU,CM2RU,RSCALE,IPRINT)
C  Radii R_K = RSTART + K*DR/2 (accumulated) and the P vectors there,
C  the first NHAM entries of each (the terms SUMLAM multiplies in).
      USE potential, ONLY: NCONST, NRSQ
      IMPLICIT DOUBLE PRECISION (A-H,O-Z)
      DIMENSION RTAB(2*NSTEP+1),PTAB(NP,2*NSTEP+1)
      ALLOCATABLE :: P(:)
      ALLOCATE (P(MAX(MXLAM+NCONST+NRSQ,NHAM,1)))
      H=DR/2.D0
      R=RSTART
      DO K=1,2*NSTEP+1
        IF (K.GT.1) R=R+H
        RTAB(K)=R
        P=0.D0
        CALL HAMPVC(R,P,MXLAM,EP2RU,CM2RU,RSCALE,IPRINT)
        DO I=1,NHAM
          PTAB(I,K)=P(I)
        ENDDO
      ENDDO
      DEALLOCATE (P)
      RETURN
      END
C
      SUBROUTINE HAMPVC(R,P,MXLAM,EP2RU,CM2RU,RSCALE,IPRINT)
C  The P vector HAMMAT hands to SUMLAM at radius R (hammat.f:31-83):
C  POTENL at R*RSCALE, values beyond +-1E60 clamped, the NCONST
C  constant terms VCONST/EP2CM appended, the SCAPOT and PERTRB hooks,
C  the conversion to reduced units, then NRSQ entries of
C  MIN(1/R**2, 1E16).
      USE potential, ONLY: NCONST, NRSQ, VCONST
      IMPLICIT DOUBLE PRECISION (A-H,O-Z)
      DIMENSION P(*),IDUM1(1)
      CALL POTENL(0,MXLAM,IDUM1,R*RSCALE,P,IDUM2,IPRINT)
      DO I=1,MXLAM
        IF (ABS(P(I)).GT.1.D60) P(I)=SIGN(1.D60,P(I))
      ENDDO
      EP2CM=EP2RU/CM2RU
      DO I=1,NCONST
        P(MXLAM+I)=VCONST(I)/EP2CM
      ENDDO
      CALL SCAPOT(P,MXLAM)
      CALL PERTRB(R*RSCALE,P,MXLAM+NCONST+NRSQ,0)
      DO I=1,MXLAM+NCONST
        P(I)=EP2RU*P(I)
      ENDDO
      IF (NRSQ.GT.0) THEN
        RSQ=MIN(1.D0/(R*R),1.D16)
        DO I=1,NRSQ
          P(MXLAM+NCONST+I)=RSQ
        ENDDO
      ENDIF
      RETURN
      END
