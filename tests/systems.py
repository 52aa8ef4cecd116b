"""Small seeded replicas shared by the parity tests.

The boxes are small and the gas dense so that every list (gas-ion, gas-vapor,
vapor-vapor) and every force term is populated at sizes the FP64 oracle and
the reference routines finish in milliseconds.
"""
from md_nucleation_b200 import abi
from md_nucleation_b200 import generate as g

NACL_N2_MEOH = dict(seed=11, gas="N2", vapor="methanol", ion="nacl", n_gas=3000, n_vap=40, box=260.0)
CHAIN_HE_WATER = dict(seed=12, gas="He", vapor="water", ion="chain", n_gas=3000, n_vap=60, box=250.0,
                      chain_atoms=45)
CHAIN_AR_MEOH_SHAKE = dict(seed=13, gas="Ar", vapor="methanol", ion="chain", n_gas=2500, n_vap=40,
                           box=250.0, chain_atoms=60, shake_h=True)
NACL_N2RIGID_WATER = dict(seed=14, gas="N2", vapor="water", ion="nacl", n_gas=2500, n_vap=50, box=250.0,
                          shake_h=True, rigid_gas=True)
NACL_N2MONO_MEOH = dict(seed=15, gas="N2monoatomic", vapor="methanol", ion="nacl", n_gas=2000, n_vap=30,
                        box=240.0)

ALL = {
    "nacl_n2_meoh": NACL_N2_MEOH,
    "chain_he_water": CHAIN_HE_WATER,
    "chain_ar_meoh_shake": CHAIN_AR_MEOH_SHAKE,
    "nacl_n2rigid_water": NACL_N2RIGID_WATER,
    "nacl_n2mono_meoh": NACL_N2MONO_MEOH,
}
NO_SHAKE = ["nacl_n2_meoh", "chain_he_water", "nacl_n2mono_meoh"]


def make(name, **over):
    kw = dict(ALL[name])
    kw.update(over)
    return g.small_system(**kw)


def with_terms(spec, extra=0, drop=0):
    spec.interactions = (spec.interactions | extra) & ~drop
    return spec
