!ecg_gpu.f90 -- iso_c_binding layer between the reference's Fortran host and
!libecgb200.so (include/ecg_abi.h).  A maintainer adds this module to the
!reference's build and replaces the hot-path calls in workproc.f90 with the
!wrappers below, which keep the reference's routine names and arguments:
!
!   ComputeMatElem(Nmin,Nmax)          -> GPU_ComputeMatElem(Nmin,Nmax)
!   ComputeMatElemAndDeriv(Nmin,Nmax)  -> GPU_ComputeMatElemAndDeriv(Nmin,Nmax)
!   GHEPIIS(k,n,...)                   -> GPU_GHEPIIS(k,n,apprlambda,Tol,lambda,RelAcc,MaxIter,SpecifNorm,NumIter,ErrorCode)
!   EnergyIA / EnergyIAM               -> GPU_EnergyIA(Nmin,Nmax,AreMatElemNeeded,SpecifNorm,ErrorCode)
!   EnergyIB                           -> GPU_EnergyIB(Evalue,Gradient,AreMatElemNeeded,ErrorCode)
!   BasisEnlI trial loop (Kstep = 1)   -> GPU_EvalTrials(nfru,NTrials,ParSets,Energies,ErrorCodes)
!   EnergyIB of a new function, batched-> GPU_EvalTrialsGrad(nbase,NTrials,ParSets,Energies,Gradients,ErrorCodes)
!   EnergyGA / EnergyGAM               -> GPU_EnergyGA(Nmin,Nmax,AreMatElemNeeded,WantVector,ErrorCode)
!   EnergyGB                           -> GPU_EnergyGB(Evalue,Gradient,AreMatElemNeeded,ErrorCode)
!   ComputeOverlapPenalty(AndAddGradient) -> GPU_OverlapPenalty(AddGradient,TotalPenalty,Gradient)
!   ExpectationValuesG main loop       -> GPU_ExpcVals(SymmAdaptMethod,Evalue,NumCFGridPoints,CFGrid,
!   (src/workproc.f90:8159-8366)           NumDensGridPoints,DensGrid,MEkl_s,MEkl_e,CF,Dens)
!
!The Glob_* matrices live on the GPU inside the context; GPU_GetMatrices
!copies Glob_H/Glob_S/Glob_diagS/Glob_invD back where host code (pruning,
!expectation values, swap file) still reads them.  This file is not built in
!this repository (no Fortran compiler in its toolchain); the C ABI it binds
!is exercised from Python through ctypes in tests/.
module ecg_gpu
use iso_c_binding
use globvars
implicit none

type(c_ptr), save :: ecg_ctx = c_null_ptr

interface
  integer(c_int) function ecg_ctx_create(n, mass, charges, nterms, yhy, coeffs, ld, max_nfo, method, device, ctx) &
      bind(C, name='ecg_ctx_create')
    import :: c_int, c_double, c_char, c_ptr
    integer(c_int), value :: n, nterms, ld, max_nfo, device
    real(c_double), intent(in) :: mass(*), charges(*)
    integer(c_int), intent(in) :: yhy(*), coeffs(*)
    character(kind=c_char), value :: method
    type(c_ptr), intent(out) :: ctx
  end function
  integer(c_int) function ecg_ctx_destroy(ctx) bind(C, name='ecg_ctx_destroy')
    import :: c_int, c_ptr
    type(c_ptr), value :: ctx
  end function
  integer(c_int) function ecg_set_params(ctx, params, first, count) bind(C, name='ecg_set_params')
    import :: c_int, c_double, c_ptr
    type(c_ptr), value :: ctx
    real(c_double), intent(in) :: params(*)
    integer(c_int), value :: first, count
  end function
  integer(c_int) function ecg_compute_mat_elem(ctx, nmin, nmax, approx_energy) bind(C, name='ecg_compute_mat_elem')
    import :: c_int, c_double, c_ptr
    type(c_ptr), value :: ctx
    integer(c_int), value :: nmin, nmax
    real(c_double), value :: approx_energy
  end function
  integer(c_int) function ecg_compute_mat_elem_and_deriv(ctx, nmin, nmax, nfru, approx_energy) &
      bind(C, name='ecg_compute_mat_elem_and_deriv')
    import :: c_int, c_double, c_ptr
    type(c_ptr), value :: ctx
    integer(c_int), value :: nmin, nmax, nfru
    real(c_double), value :: approx_energy
  end function
  integer(c_int) function ecg_ghepiis(ctx, k, n, apprlambda, tol, max_iter, specif_norm, lambda, rel_acc, num_iter) &
      bind(C, name='ecg_ghepiis')
    import :: c_int, c_double, c_ptr
    type(c_ptr), value :: ctx
    integer(c_int), value :: k, n, max_iter, specif_norm
    real(c_double), value :: apprlambda, tol
    real(c_double), intent(out) :: lambda, rel_acc
    integer(c_int), intent(out) :: num_iter
  end function
  integer(c_int) function ecg_energy_ia(ctx, nmin, nmax, needed, approx_energy, tol, max_iter, specif_norm, &
      energy, num_iter) bind(C, name='ecg_energy_ia')
    import :: c_int, c_double, c_ptr
    type(c_ptr), value :: ctx
    integer(c_int), value :: nmin, nmax, needed, max_iter, specif_norm
    real(c_double), value :: approx_energy, tol
    real(c_double), intent(out) :: energy
    integer(c_int), intent(out) :: num_iter
  end function
  integer(c_int) function ecg_energy_ib_adjoint(ctx, nfru, nfa, needed, approx_energy, tol, max_iter, energy, &
      grad, num_iter) bind(C, name='ecg_energy_ib_adjoint')
    import :: c_int, c_double, c_ptr
    type(c_ptr), value :: ctx
    integer(c_int), value :: nfru, nfa, needed, max_iter
    real(c_double), value :: approx_energy, tol
    real(c_double), intent(out) :: energy
    real(c_double), intent(out) :: grad(*)
    integer(c_int), intent(out) :: num_iter
  end function
  integer(c_int) function ecg_eval_candidates(ctx, nbase, count, cand, approx_energy, tol, max_iter, energies, &
      errcodes, num_iter, rel_acc) bind(C, name='ecg_eval_candidates')
    import :: c_int, c_double, c_ptr
    type(c_ptr), value :: ctx
    integer(c_int), value :: nbase, count, max_iter
    real(c_double), intent(in) :: cand(*)
    real(c_double), value :: approx_energy, tol
    real(c_double), intent(out) :: energies(*), rel_acc(*)
    integer(c_int), intent(out) :: errcodes(*), num_iter(*)
  end function
  integer(c_int) function ecg_eval_candidates_grad(ctx, nbase, count, cand, approx_energy, tol, max_iter, &
      energies, errcodes, num_iter, rel_acc, grad) bind(C, name='ecg_eval_candidates_grad')
    import :: c_int, c_double, c_ptr
    type(c_ptr), value :: ctx
    integer(c_int), value :: nbase, count, max_iter
    real(c_double), intent(in) :: cand(*)
    real(c_double), value :: approx_energy, tol
    real(c_double), intent(out) :: energies(*), rel_acc(*), grad(*)
    integer(c_int), intent(out) :: errcodes(*), num_iter(*)
  end function
  integer(c_int) function ecg_energy_ga(ctx, nmin, nmax, needed, which, want_vector, energy, nfact) &
      bind(C, name='ecg_energy_ga')
    import :: c_int, c_double, c_ptr
    type(c_ptr), value :: ctx
    integer(c_int), value :: nmin, nmax, needed, which, want_vector
    real(c_double), intent(out) :: energy
    integer(c_int), intent(out) :: nfact
  end function
  integer(c_int) function ecg_energy_gb_adjoint(ctx, nfru, nfa, needed, which, energy, grad) &
      bind(C, name='ecg_energy_gb_adjoint')
    import :: c_int, c_double, c_ptr
    type(c_ptr), value :: ctx
    integer(c_int), value :: nfru, nfa, needed, which
    real(c_double), intent(out) :: energy
    real(c_double), intent(out) :: grad(*)
  end function
  integer(c_int) function ecg_overlap_penalty(ctx, nfru, nfa, maxpen, thr2, mode, total, grad) &
      bind(C, name='ecg_overlap_penalty')
    import :: c_int, c_double, c_ptr
    type(c_ptr), value :: ctx
    integer(c_int), value :: nfru, nfa, mode
    real(c_double), value :: maxpen, thr2
    real(c_double), intent(out) :: total
    real(c_double), intent(inout) :: grad(*)
  end function
  integer(c_int) function ecg_expectation_values(ctx, nbasis, masses, method, ny, ymats, ycoeffs, energy, c, &
      ncf, cfgrid, ndens, densgrid, vals, errs, cf, dens) bind(C, name='ecg_expectation_values')
    import :: c_int, c_double, c_ptr, c_double_complex
    type(c_ptr), value :: ctx
    integer(c_int), value :: nbasis, method, ny, ncf, ndens
    real(c_double), intent(in) :: masses(*), cfgrid(*), densgrid(*)
    integer(c_int), intent(in) :: ymats(*), ycoeffs(*)
    real(c_double), value :: energy
    complex(c_double_complex), intent(in) :: c(*)
    real(c_double), intent(out) :: vals(*), errs(*), cf(*), dens(*)
  end function
  integer(c_int) function ecg_get_matrices(ctx, n, H, S, ld, diagS, diagH, invD) bind(C, name='ecg_get_matrices')
    import :: c_int, c_double, c_ptr, c_double_complex
    type(c_ptr), value :: ctx
    integer(c_int), value :: n, ld
    complex(c_double_complex), intent(out) :: H(*), S(*), invD(*)
    real(c_double), intent(out) :: diagS(*), diagH(*)
  end function
  integer(c_int) function ecg_get_vectors(ctx, n, c, last) bind(C, name='ecg_get_vectors')
    import :: c_int, c_ptr, c_double_complex
    type(c_ptr), value :: ctx
    integer(c_int), value :: n
    complex(c_double_complex), intent(out) :: c(*), last(*)
  end function
end interface

contains

!Called once after ProgramDataInit (src/workproc.f90:575): the system
!constants and the Y^+Y terms move to the device.
subroutine GPU_Init(MaxBasisSize, MaxFuncToOpt)
  integer, intent(in) :: MaxBasisSize, MaxFuncToOpt
  real(c_double) :: charges(Glob_n+1)
  integer(c_int) :: st
  charges(1) = Glob_PseudoCharge0
  charges(2:Glob_n+1) = Glob_PseudoCharge(1:Glob_n)
  st = ecg_ctx_create(Glob_n, Glob_MassMatrix, charges, Glob_NumYHYTerms, Glob_YHYMatr, Glob_YHYCoeff, &
                      MaxBasisSize, MaxFuncToOpt, Glob_GSEPSolutionMethod, 0, ecg_ctx)
  if (st /= 0) stop 'GPU_Init: ecg_ctx_create failed'
end subroutine GPU_Init

!ComputeMatElem(Nmin,Nmax), src/matform.f90:119
subroutine GPU_ComputeMatElem(Nmin, Nmax)
  integer, intent(in) :: Nmin, Nmax
  integer(c_int) :: st
  st = ecg_set_params(ecg_ctx, Glob_NonlinParam, 1, Nmax)
  st = ecg_compute_mat_elem(ecg_ctx, Nmin, Nmax, Glob_ApproxEnergy)
  if (st /= 0) stop 'GPU_ComputeMatElem failed'
end subroutine GPU_ComputeMatElem

!ComputeMatElemAndDeriv(Nmin,Nmax), src/matform.f90:234
subroutine GPU_ComputeMatElemAndDeriv(Nmin, Nmax)
  integer, intent(in) :: Nmin, Nmax
  integer(c_int) :: st
  st = ecg_set_params(ecg_ctx, Glob_NonlinParam, 1, Nmax)
  st = ecg_compute_mat_elem_and_deriv(ecg_ctx, Nmin, Nmax, Glob_nfru, Glob_ApproxEnergy)
  if (st /= 0) stop 'GPU_ComputeMatElemAndDeriv failed'
end subroutine GPU_ComputeMatElemAndDeriv

!GHEPIIS on the context's Glob_H, Glob_invD, Glob_S, Glob_c, Glob_LastEigvector
!(src/linalg.f90:1781); ErrorCode as the reference returns it.
subroutine GPU_GHEPIIS(k, n, apprlambda, Tol, lambda, RelAcc, MaxIter, SpecifNorm, NumIter, ErrorCode)
  integer, intent(in) :: k, n, MaxIter, SpecifNorm
  real(dprec), intent(in) :: apprlambda, Tol
  real(dprec), intent(out) :: lambda, RelAcc
  integer, intent(out) :: NumIter, ErrorCode
  ErrorCode = ecg_ghepiis(ecg_ctx, k, n, apprlambda, Tol, MaxIter, SpecifNorm, lambda, RelAcc, NumIter)
end subroutine GPU_GHEPIIS

!EnergyIA (SpecifNorm=-1) / EnergyIAM (SpecifNorm=0), src/workproc.f90:1954
function GPU_EnergyIA(Nmin, Nmax, AreMatElemNeeded, SpecifNorm, ErrorCode)
  real(dprec) :: GPU_EnergyIA
  integer, intent(in) :: Nmin, Nmax, SpecifNorm
  logical, intent(in) :: AreMatElemNeeded
  integer, intent(out) :: ErrorCode
  integer(c_int) :: needed, it
  real(c_double) :: e
  needed = merge(1, 0, AreMatElemNeeded)
  if (AreMatElemNeeded) ErrorCode = ecg_set_params(ecg_ctx, Glob_NonlinParam, 1, Nmax)
  ErrorCode = ecg_energy_ia(ecg_ctx, Nmin, Nmax, needed, Glob_ApproxEnergy, Glob_EigvalTol, &
                            Glob_MaxIterForGHEPIIS, SpecifNorm, e, it)
  GPU_EnergyIA = e
  Glob_InvItTempCounter1 = Glob_InvItTempCounter1 + 1
  Glob_InvItTempCounter2 = Glob_InvItTempCounter2 + it
end function GPU_EnergyIA

!EnergyIB, src/workproc.f90:2063, through the fused adjoint pass
subroutine GPU_EnergyIB(Evalue, Gradient, AreMatElemNeeded, ErrorCode)
  real(dprec), intent(out) :: Evalue
  real(dprec), intent(out) :: Gradient(Glob_npt*Glob_nfo)
  logical, intent(in) :: AreMatElemNeeded
  integer, intent(out) :: ErrorCode
  integer(c_int) :: needed, it
  needed = merge(1, 0, AreMatElemNeeded)
  if (AreMatElemNeeded) ErrorCode = ecg_set_params(ecg_ctx, Glob_NonlinParam, 1, Glob_nfa)
  ErrorCode = ecg_energy_ib_adjoint(ecg_ctx, Glob_nfru, Glob_nfa, needed, Glob_ApproxEnergy, Glob_EigvalTol, &
                                    Glob_MaxIterForGHEPIIS, Evalue, Gradient, it)
  Glob_InvItTempCounter1 = Glob_InvItTempCounter1 + 1
  Glob_InvItTempCounter2 = Glob_InvItTempCounter2 + it
end subroutine GPU_EnergyIB

!The trial loop of BasisEnlI (src/workproc.f90:4054-4070) with Kstep = 1,
!all trials in one call: ParSets(1:npt,i) are the NTrials candidates drawn
!by GenerateTrialParam beforehand; Energies(i) and ErrorCodes(i) are what
!EnergyIA(nfru+1,nfru+1,.true.,ErrorCode) returns for candidate i.  The
!basis of nfru functions must be current on the device (as after the
!EnergyIA(1,nfru) that precedes the loop); it is left unchanged, so the
!chosen candidate is installed afterwards with GPU_EnergyIA(nfru+1,nfru+1,...)
!exactly as the reference does after its loop.
subroutine GPU_EvalTrials(nfru, NTrials, ParSets, Energies, ErrorCodes)
  integer, intent(in) :: nfru, NTrials
  real(dprec), intent(in) :: ParSets(Glob_npt, NTrials)
  real(dprec), intent(out) :: Energies(NTrials)
  integer, intent(out) :: ErrorCodes(NTrials)
  integer(c_int) :: st, codes(NTrials), iters(NTrials)
  real(c_double) :: relacc(NTrials)
  st = ecg_eval_candidates(ecg_ctx, nfru, NTrials, ParSets, Glob_ApproxEnergy, Glob_EigvalTol, &
                           Glob_MaxIterForGHEPIIS, Energies, codes, iters, relacc)
  if (st /= 0) stop 'GPU_EvalTrials: ecg_eval_candidates failed'
  ErrorCodes = codes
  Glob_InvItTempCounter1 = Glob_InvItTempCounter1 + NTrials
  Glob_InvItTempCounter2 = Glob_InvItTempCounter2 + sum(iters)
end subroutine GPU_EvalTrials

!The energy + gradient of a newly added function (EnergyIB with nfru = nbase,
!nfa = nbase+1, src/workproc.f90:2063-2154, as BasisEnlI's DRMNG loop calls
!it, :4137-4170) for NTrials candidate parameter sets at once: Energies(i),
!Gradients(1:npt,i) and ErrorCodes(i) are what EnergyIB returns once
!ParSets(1:npt,i) is function nbase+1.  The basis of nbase functions must be
!current on the device; it is left unchanged.
subroutine GPU_EvalTrialsGrad(nbase, NTrials, ParSets, Energies, Gradients, ErrorCodes)
  integer, intent(in) :: nbase, NTrials
  real(dprec), intent(in) :: ParSets(Glob_npt, NTrials)
  real(dprec), intent(out) :: Energies(NTrials), Gradients(Glob_npt, NTrials)
  integer, intent(out) :: ErrorCodes(NTrials)
  integer(c_int) :: st, codes(NTrials), iters(NTrials)
  real(c_double) :: relacc(NTrials)
  st = ecg_eval_candidates_grad(ecg_ctx, nbase, NTrials, ParSets, Glob_ApproxEnergy, Glob_EigvalTol, &
                                Glob_MaxIterForGHEPIIS, Energies, codes, iters, relacc, Gradients)
  if (st /= 0) stop 'GPU_EvalTrialsGrad: ecg_eval_candidates_grad failed'
  ErrorCodes = codes
  Glob_InvItTempCounter1 = Glob_InvItTempCounter1 + NTrials
  Glob_InvItTempCounter2 = Glob_InvItTempCounter2 + sum(iters)
end subroutine GPU_EvalTrialsGrad

!EnergyGA (WantVector=.false.) / EnergyGAM (.true.), src/workproc.f90:1697,
!for a context created with Glob_GSEPSolutionMethod='G': the
!Glob_WhichEigenvalue-th eigenvalue with ZHEGVX(RANGE='I') semantics; with
!WantVector, Glob_c (on the device) receives its eigenvector.
function GPU_EnergyGA(Nmin, Nmax, AreMatElemNeeded, WantVector, ErrorCode)
  real(dprec) :: GPU_EnergyGA
  integer, intent(in) :: Nmin, Nmax
  logical, intent(in) :: AreMatElemNeeded, WantVector
  integer, intent(out) :: ErrorCode
  integer(c_int) :: nf
  real(c_double) :: e
  if (AreMatElemNeeded) ErrorCode = ecg_set_params(ecg_ctx, Glob_NonlinParam, 1, Nmax)
  ErrorCode = ecg_energy_ga(ecg_ctx, Nmin, Nmax, merge(1, 0, AreMatElemNeeded), Glob_WhichEigenvalue, &
                            merge(1, 0, WantVector), e, nf)
  GPU_EnergyGA = e
  Glob_EnergyGACounter = Glob_EnergyGACounter + 1
end function GPU_EnergyGA

!EnergyGB, src/workproc.f90:1841, through the fused adjoint pass
subroutine GPU_EnergyGB(Evalue, Gradient, AreMatElemNeeded, ErrorCode)
  real(dprec), intent(out) :: Evalue
  real(dprec), intent(out) :: Gradient(Glob_npt*Glob_nfo)
  logical, intent(in) :: AreMatElemNeeded
  integer, intent(out) :: ErrorCode
  if (AreMatElemNeeded) ErrorCode = ecg_set_params(ecg_ctx, Glob_NonlinParam, 1, Glob_nfa)
  ErrorCode = ecg_energy_gb_adjoint(ecg_ctx, Glob_nfru, Glob_nfa, merge(1, 0, AreMatElemNeeded), &
                                    Glob_WhichEigenvalue, Evalue, Gradient)
  Glob_EnergyGBCounter = Glob_EnergyGBCounter + 1
end subroutine GPU_EnergyGB

!ComputeOverlapPenalty (AddGradient=.false.) and
!ComputeOverlapPenaltyAndAddGradient (.true.), src/workproc.f90:1491-1693,
!on the device's Glob_S: TotalPenalty, and with AddGradient the reference's
!penalty gradient added to the gradient the last GPU_EnergyIB/GB left on the
!device, returned in Gradient (npt * nfo).  Called where EnergyGA/GB call
!the reference routines (src/workproc.f90:1759,1824,1943).
subroutine GPU_OverlapPenalty(AddGradient, TotalPenalty, Gradient)
  logical, intent(in) :: AddGradient
  real(dprec), intent(out) :: TotalPenalty
  real(dprec), intent(inout) :: Gradient(*)
  integer(c_int) :: st
  st = ecg_overlap_penalty(ecg_ctx, Glob_nfru, Glob_nfa, Glob_MaxOverlapPenalty, Glob_OverlapPenaltyThreshold2, &
                           merge(1, 0, AddGradient), TotalPenalty, Gradient)
end subroutine GPU_OverlapPenalty

!The accumulation loop of ExpectationValuesG, src/workproc.f90:8159-8366,
!for functions 1..Glob_CurrBasisSize with the eigenvector Glob_c and
!Glob_CurrEnergy = Evalue: MEkl_s / MEkl_e (NumOfExpcVals = 6 np + 9 values,
!MEkl_e already times epsilon) and the CF / Dens sums, as the reference has
!them after its MPI_ALLREDUCE.  Glob_diagS must be current on the device
!(GPU_ComputeMatElem(1, Glob_CurrBasisSize) or GPU_EnergyGA).
subroutine GPU_ExpcVals(SymmAdaptMethod, Evalue, NumCFGridPoints, CFGrid, NumDensGridPoints, DensGrid, &
                        MEkl_s, MEkl_e, CF, Dens, ErrorCode)
  integer, intent(in) :: SymmAdaptMethod, NumCFGridPoints, NumDensGridPoints
  real(dprec), intent(in) :: Evalue, CFGrid(*), DensGrid(*)
  real(dprec), intent(out) :: MEkl_s(*), MEkl_e(*), CF(*), Dens(*)
  integer, intent(out) :: ErrorCode
  ErrorCode = ecg_expectation_values(ecg_ctx, Glob_CurrBasisSize, Glob_Mass, SymmAdaptMethod, Glob_NumYTerms, &
                                     Glob_YMatr, Glob_YCoeff, Evalue, Glob_c, NumCFGridPoints, CFGrid, &
                                     NumDensGridPoints, DensGrid, MEkl_s, MEkl_e, CF, Dens)
end subroutine GPU_ExpcVals

!Copy the device matrices and vectors back into the Glob_* host arrays for
!code that still reads them on the host.
subroutine GPU_GetMatrices(n)
  integer, intent(in) :: n
  integer(c_int) :: st
  st = ecg_get_matrices(ecg_ctx, n, Glob_H, Glob_S, Glob_HSLeadDim, Glob_diagS, Glob_diagH, Glob_invD)
  st = ecg_get_vectors(ecg_ctx, n, Glob_c, Glob_LastEigvector)
end subroutine GPU_GetMatrices

subroutine GPU_Finalize()
  integer(c_int) :: st
  if (c_associated(ecg_ctx)) st = ecg_ctx_destroy(ecg_ctx)
  ecg_ctx = c_null_ptr
end subroutine GPU_Finalize

end module ecg_gpu
