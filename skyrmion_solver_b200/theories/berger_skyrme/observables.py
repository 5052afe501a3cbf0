"""Host observables of the Berger Skyrme model with the reference's signatures
(skyrmion_solver th/berger_skyrme/observables.py: compute_energy, compute_skyrmion_number)."""
from ...core.observables import BaryonObservable, EnergyObservable
from .kernels import THEORY_ID

compute_energy = EnergyObservable(THEORY_ID)
compute_skyrmion_number = BaryonObservable(THEORY_ID)
