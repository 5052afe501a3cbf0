"""Host observables of the Nuclear Skyrme model with the reference's signatures
(skyrmion_solver th/nuclear_skyrme/observables.py: compute_energy, compute_skyrmion_number,
compute_center_of_mass, compute_rms_radius)."""
from ...core.observables import (BaryonObservable, CenterOfMassObservable, EnergyObservable,
                                 RmsRadiusObservable)
from .kernels import THEORY_ID

compute_energy = EnergyObservable(THEORY_ID)
compute_skyrmion_number = BaryonObservable(THEORY_ID)
compute_center_of_mass = CenterOfMassObservable(THEORY_ID)
compute_rms_radius = RmsRadiusObservable(THEORY_ID)
