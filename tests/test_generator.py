"""The seeded system generator: properties its chains must have for the
dynamics to stay regular (CPU only)."""
import numpy as np

from md_nucleation_b200 import generate


def _angles_deg(spec):
    ion = spec.ion
    return np.degrees(spec.angle_coeff[ion.angles[:, 3], 1])


def _valence(spec):
    n = np.zeros(spec.ion.n, np.int64)
    for i, j, _ in spec.ion.bonds:
        n[i] += 1
        n[j] += 1
    return n


def test_chain_angles_stay_clear_of_180_degrees():
    """No equilibrium angle of a chain is near 180 degrees: the torsions
    through an atom on a collinear bond are singular (the reference's
    dihedral forces divide by the normals' lengths), which blew replicas up."""
    for spec in (generate.config1(0), generate.config2_replica(96), generate.config2_replica(4),
                 generate.config2_replica(7)):
        th = _angles_deg(spec)
        assert th.max() < 125.0, f"{spec.label}: equilibrium angle {th.max():.1f} deg"


def test_chain_atoms_are_at_most_tetravalent():
    for spec in (generate.config1(0), generate.config2_replica(96)):
        v = _valence(spec)
        assert v.max() <= 4, f"an atom with {v.max()} bonds"
        assert spec.ion.n == len(spec.ion.type)
