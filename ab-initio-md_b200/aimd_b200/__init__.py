"""
aimd_b200: the Hartree-Fock hot path of Ab-Initio-MD on one NVIDIA B200.

McMurchie-Davidson electron-repulsion integrals, the integral-direct J/K
Fock build of the RHF/UHF DIIS SCF and the integral-direct analytic nuclear
gradient, as hand-written sm_100a CUDA kernels behind a C ABI
(include/aimd_b200.h), with the reference's Python API on top:

  basis       build_basis, BasisSet                 (aimd.qc.basis)
  integrals   eri_tensor, jk, two_electron_gradient  (aimd.qc.integrals)
  scf         SCFOptions, SCFSolver, run_scf          (aimd.qc.scf)
  gradients   scf_gradient, gradient_terms            (aimd.qc.gradients)
  backend     ForceBackend, GradientResult, HFGPUBackend ("hf-gpu")
"""

from .basis import BasisSet, available_basis_sets, build_basis, normalize_basis_name

__all__ = ["BasisSet", "available_basis_sets", "build_basis", "normalize_basis_name"]

__version__ = "0.1.0"
