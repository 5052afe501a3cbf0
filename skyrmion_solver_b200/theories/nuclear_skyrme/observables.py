"""Host observables of the Nuclear Skyrme model with the reference's signatures
(skyrmion_solver th/nuclear_skyrme/observables.py: compute_energy, compute_skyrmion_number,
compute_center_of_mass, compute_rms_radius, compute_U_tensor, compute_V_tensor,
compute_W_tensor, compute_quadrupole_tensor, compute_D_term)."""
from ...core.observables import (BaryonObservable, CenterOfMassObservable, DTermObservable, EnergyObservable,
                                 QuadrupoleTensorObservable, RmsRadiusObservable, UTensorObservable,
                                 VTensorObservable, WTensorObservable)
from .kernels import THEORY_ID

compute_energy = EnergyObservable(THEORY_ID)
compute_skyrmion_number = BaryonObservable(THEORY_ID)
compute_center_of_mass = CenterOfMassObservable(THEORY_ID)
compute_rms_radius = RmsRadiusObservable(THEORY_ID)
compute_U_tensor = UTensorObservable(THEORY_ID)
compute_V_tensor = VTensorObservable(THEORY_ID)
compute_W_tensor = WTensorObservable(THEORY_ID)
compute_quadrupole_tensor = QuadrupoleTensorObservable(THEORY_ID)
compute_D_term = DTermObservable(THEORY_ID)
