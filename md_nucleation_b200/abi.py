"""ctypes mirror of include/mdn.h (the engine's C ABI) and of mdn_host.h.

Every structure here has the exact field order of its C counterpart; the
constants carry the same names without the MDN_ prefix.
"""
import ctypes as C

ABI_VERSION = 1

OK, ERR_ARG, ERR_CUDA, ERR_NO_DEVICE, ERR_CAPACITY, ERR_REPLICA = 0, -1, -2, -3, -4, -5

ST_SLAB_OVERFLOW = 0x0001
ST_CORE_OVERFLOW = 0x0002
ST_LIST_OVERFLOW = 0x0004
ST_SHAKE_NOCONV = 0x0008
ST_NONFINITE = 0x0010
ST_FIXED_OVERFLOW = 0x0020
ST_EVENT_OVERFLOW = 0x0040
ST_FATAL = ST_SLAB_OVERFLOW | ST_CORE_OVERFLOW | ST_LIST_OVERFLOW | ST_NONFINITE

I_GI = 0x0001
I_VI = 0x0002
I_VV = 0x0004
I_GV = 0x0008
I_GG = 0x0010
I_AMBER = 0x0020
I_BMH = 0x0040
I_GAS_INTRA = 0x0080
I_VAPOR_INTRA = 0x0100
I_EFIELD = 0x0200
I_SHAKE = 0x1000

Q_GV_GAS_COUNT = 0x01
Q_GAS_ROT_ZY = 0x02
Q_N2_ROT_VYVZ = 0x04
Q_ENERGY_BUCKETS = 0x08
Q_SHAKE_NO_VCORR = 0x10
Q_BLIND_INSERT = 0x20
Q_ALL = 0x2F  # Q_SHAKE_NO_VCORR is opt-in
INSERT_MIN_DIST = 2.0
INSERT_TRIES = 4

U_ION, U_GAS, U_VAP, U_GI, U_GG, U_VG, U_VI, U_VV = range(8)
ENERGY_NAMES = ("Uion", "Ugas", "Uvap", "Ugi", "Ugg", "Uvg", "Uvi", "Uvv")

GAS_HE, GAS_N2, GAS_N2MONO, GAS_AR = 1, 2, 3, 4
NVT_OFF, NVT_SCALE, NVT_NH = 0, 1, 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_ubp = C.POINTER(C.c_ubyte)


class Topology(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int), ("type", _ip), ("charge", _dp), ("x", _dp),
        ("n_bonds", C.c_int), ("bonds", _ip),
        ("n_rigid", C.c_int), ("rigid", _ip),
        ("n_angles", C.c_int), ("angles", _ip),
        ("n_dihedrals", C.c_int), ("dihedrals", _ip),
    ]


class ReplicaDesc(C.Structure):
    _fields_ = [
        ("n_atom_types", C.c_int), ("atom_mass", _dp), ("atom_eps", _dp), ("atom_sigma", _dp),
        ("n_bond_types", C.c_int), ("bond_coeff", _dp),
        ("n_angle_types", C.c_int), ("angle_coeff", _dp),
        ("n_dihedral_types", C.c_int), ("dihedral_multi", _ip), ("dihedral_coeff", _dp),
        ("ion", Topology), ("ion_v", _dp), ("ion_bmh_type", _ip),
        ("gas", Topology), ("gas_kind", C.c_int), ("gas_com_mass", C.c_double), ("gas_mb_mass", C.c_double),
        ("vapor", Topology), ("vapor_com_mass", C.c_double), ("vapor_mb_mass", C.c_double),
        ("n_gas", C.c_int), ("gas_x", _dp), ("gas_v", _dp),
        ("n_vapor", C.c_int), ("vapor_x", _dp), ("vapor_v", _dp),
        ("dt", C.c_double), ("temperature", C.c_double), ("box", C.c_double),
        ("cutoff", C.c_double), ("margin", C.c_double), ("r_inter", C.c_double), ("overlap", C.c_double),
        ("interactions", C.c_uint), ("nvt_mode", C.c_int), ("nvt_temperature", C.c_double),
        ("efield", C.c_double * 3), ("seed", C.c_ulonglong),
        ("pair_eps", C.POINTER(C.c_double)), ("pair_sigma", C.POINTER(C.c_double)),
    ]


class AdjointSpec(C.Structure):
    _fields_ = [
        ("n_steps", C.c_longlong), ("checkpoint_every", C.c_int), ("count_radius", C.c_double),
        ("count_width", C.c_double), ("w_energy", C.c_double), ("w_count", C.c_double),
    ]


class Options(C.Structure):
    _fields_ = [
        ("quirks", C.c_uint), ("force_mode", C.c_int), ("cluster_size", C.c_int),
        ("threads", C.c_int), ("steps_per_launch", C.c_int), ("use_graph", C.c_int),
        ("capacity_factor", C.c_double), ("device", C.c_int),
    ]


class ReplicaInfo(C.Structure):
    _fields_ = [
        ("n_ion", C.c_int), ("gas_atoms", C.c_int), ("vapor_atoms", C.c_int),
        ("n_gas", C.c_int), ("n_vapor", C.c_int),
        ("n_gas_in", C.c_int), ("n_vapor_in", C.c_int),
        ("loop_pair", C.c_int), ("loop_update", C.c_int), ("n_rebuilds", C.c_int),
        ("step", C.c_longlong), ("status", C.c_int),
        ("gi_pairs", C.c_int), ("gv_pairs", C.c_int), ("gg_pairs", C.c_int),
    ]


class State(C.Structure):
    _fields_ = [
        ("ion_x", _dp), ("ion_v", _dp), ("ion_f", _dp),
        ("mol_x", _dp), ("mol_v", _dp), ("region", _ubp),
        ("gas_ax", _dp), ("gas_av", _dp), ("gas_af", _dp),
        ("vap_ax", _dp), ("vap_av", _dp), ("vap_af", _dp), ("vap_w", _dp),
        ("loop_pair", C.c_int), ("loop_update", C.c_int),
        ("zeta", C.c_double), ("margin_length", C.c_double),
    ]


class PlaceDesc(C.Structure):
    _fields_ = [
        ("box", C.c_double), ("min_dist", C.c_double), ("n_ion", C.c_int), ("ion_x", _dp),
        ("n_gas", C.c_int), ("n_vapor", C.c_int), ("gas_sigma", C.c_double), ("vapor_sigma", C.c_double),
        ("seed", C.c_ulonglong),
    ]


class Event(C.Structure):
    _fields_ = [
        ("replica", C.c_int), ("molecule", C.c_int), ("kind", C.c_int), ("pad", C.c_int),
        ("step", C.c_longlong), ("dx", C.c_double * 3), ("dv", C.c_double * 3),
    ]


def ptr(a, ctype=C.c_double):
    """Pointer to a contiguous numpy array (None -> NULL)."""
    if a is None:
        return C.cast(None, C.POINTER(ctype))
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(C.POINTER(ctype))
