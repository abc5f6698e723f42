!##############################################################################
! module vacgpu -- program vac's hot path on the GPU through libsacgpu.so
!
! Preprocessed by the reference's vacpp.pl like its other .t files and built with
! them by sac_b200/fortran/host_build.py, which also rewrites a copy of src/vac.t
! so that its call sites call these routines instead of the CPU ones:
!   gpuini(w)       after startup, in place of the first getboundary (src/vac.t:54):
!                   creates the device context from the COMMON parameters, sets its
!                   grid and boundary regions, uploads w and fills the ghost cells
!   gpugetdt(w)     the dt block's dtpar / getdt_courant / getdt / getdt_special /
!                   dtcantgrow (src/vac.t:61-70)
!   gpuadvect(method,iws,idim^LIM)   advect in advance_expl (src/vac.t:317,323,329)
!   gpudownload(w)  before savefile (src/vac.t:57,112) and the residual (src/vac.t:90)
!   gpufinish       after the last save
! The state stays resident on the device between the calls; the host w is current
! only after gpudownload.  Every non-zero status goes to die() with the library's
! message.  The build is the reference's configured one (-d=33 -p=mhd -u=Slog):
! gravity grav1_..grav3_ and the hyperdiffusion coefficient nu_ are its eqpars.

!=============================================================================
subroutine gpucheck(ierr,what)

use sacgpu
include 'vacdef.f'

integer(c_int):: ierr
character(len=*):: what
!-----------------------------------------------------------------------------

if(ierr/=SAC_OK)call die('sacgpu '//what//': '//sac_error_text(vac_ctx))

return
end

!=============================================================================
subroutine gpuini(w)

use sacgpu
include 'vacdef.f'

double precision:: w(ixG^T,nw)
type(sac_params):: p
integer(c_int):: ierr,ixGh(3),ixMl(6),iB,idm
integer(c_int):: ixBl(ndim,nB,2),idimBl(nB),upperBl(nB),ipairBl(nB)
!-----------------------------------------------------------------------------

call sac_default_params(p)
p%gamma=eqpar(gamma_)
p%eta=eqpar(eta_)
p%grav(1)=eqpar(grav1_)
p%grav(2)=eqpar(grav2_)
p%grav(3)=eqpar(grav3_)
p%nu=eqpar(nu_)
p%courantpar=courantpar
p%dtpar=dtpar
p%dtdiffpar=dtdiffpar
p%dtcantgrow=merge(1,0,dtcantgrow)
call sac_set_name(p%typeadvance,typeadvance)
call sac_set_name(p%typepred,typepred1)
p%sourceunsplit=merge(1,0,sourceunsplit)
p%divbfix=merge(1,0,divbfix)
p%user=SAC_USR_SLOG
p%smallfix=merge(1,0,smallfix)
p%smallp=smallp
p%smallrho=smallrho
p%vacuumrho=vacuumrho
p%compactres=merge(1,0,compactres)
p%device=0
ierr=sac_create(p,vac_ctx)
if(ierr/=SAC_OK)call die('sacgpu: no device context (sac_create)')

ixGh=1; ixMl=1
{^D&ixGh(^D)=ixGhi^D; ixMl(^D)=ixMmin^D; ixMl(3+^D)=ixMmax^D;}
call gpucheck(sac_set_grid(vac_ctx,ndim,ndir,ixGh,ixMl,x,merge(1,0,fullgridini)),'set_grid')

! boundsetup has filled ixB^LIM for the default regions too; the library
! recognises those and resolves them in one pass
do iB=1,nB
   do idm=1,ndim
      ixBl(idm,iB,1)=ixBmin(idm,iB)
      ixBl(idm,iB,2)=ixBmax(idm,iB)
   end do
   idimBl(iB)=idimB(iB)
   upperBl(iB)=merge(1,0,upperB(iB))
   ipairBl(iB)=ipairB(iB)
end do
call gpucheck(sac_set_boundaries(vac_ctx,nB,typeB,ixBl,idimBl,upperBl,ipairBl),'set_boundaries')

call gpucheck(sac_upload(vac_ctx,w),'upload')
call gpucheck(sac_getboundary(vac_ctx,t),'getboundary')

return
end

!=============================================================================
subroutine gpugetdt(w)

use sacgpu
include 'vacdef.f'

double precision:: w(ixG^T,nw)
!-----------------------------------------------------------------------------

call gpucheck(sac_getdt(vac_ctx,dt,it),'getdt')

return
end

!=============================================================================
subroutine gpuadvect(method,iws,idim^LIM)

use sacgpu
include 'vacdef.f'

character*^LENTYPE :: method
integer:: iws(niw_),idim^LIM
!-----------------------------------------------------------------------------

call gpucheck(sac_advect(vac_ctx,trim(method)//c_null_char,iws,idimmin,idimmax,dt,t,it),'advect')

return
end

!=============================================================================
subroutine gpudownload(w)

use sacgpu
include 'vacdef.f'

double precision:: w(ixG^T,nw)
!-----------------------------------------------------------------------------

call gpucheck(sac_download(vac_ctx,w),'download')

return
end

!=============================================================================
subroutine gpufinish

use sacgpu
include 'vacdef.f'
!-----------------------------------------------------------------------------

call sac_destroy(vac_ctx)
vac_ctx=c_null_ptr

return
end
!=============================================================================
! end module vacgpu
!##############################################################################
