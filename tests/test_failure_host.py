"""Host-side failure handling of the C ABI, without a GPU: a malformed basis
description or bad options come back as an error code from tf_ctx_create before any
device call (Tonto's DIE/ENSURE convention, include/macros.in:339-367, maps a
non-zero status to an abort on the Fortran side).  Nothing here touches a device."""

import ctypes
import math

import numpy as np
import pytest

from tonto_b200.molecules import water_cluster

TF_EINVAL, TF_EUNSUPPORTED = -1, -4


def _basis_arrays(mol):
    sa, sl, sn, sf, ex, co = mol.flat_arrays()
    xyz = np.array(mol.xyz, dtype=np.float64, order="C", copy=True)
    return dict(xyz=xyz, sa=sa.copy(), sl=sl.copy(), sn=sn.copy(), sf=sf.copy(), ex=ex.copy(), co=co.copy())


def _create(a, n_atom, n_shell, spherical=1, opt=None):
    from tonto_b200.fock import _Basis, load_library
    L = load_library()
    dp = lambda x: x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
    ip = lambda x: x.ctypes.data_as(ctypes.POINTER(ctypes.c_int))     # noqa: E731
    b = _Basis(n_atom, dp(a["xyz"]), n_shell, ip(a["sa"]), ip(a["sl"]), ip(a["sn"]), ip(a["sf"]), dp(a["ex"]),
               dp(a["co"]), spherical)
    h = ctypes.c_void_p()
    rc = L.tf_ctx_create(ctypes.byref(b), ctypes.byref(opt) if opt is not None else None, ctypes.byref(h))
    assert not h.value, "no context may be returned on an error"
    return rc


@pytest.fixture(scope="module")
def mol():
    return water_cluster(2, seed=0)


def _corrupt(mol, what):
    a = _basis_arrays(mol)
    n_atom, n_shell = mol.n_atom, mol.n_shell
    if what == "no_shells":
        n_shell = 0
    elif what == "no_atoms":
        n_atom = 0
    elif what == "negative_l":
        a["sl"][3] = -1
    elif what == "atom_out_of_range":
        a["sa"][5] = mol.n_atom
    elif what == "zero_primitives":
        a["sn"][2] = 0
    elif what == "first_bf_gap":
        a["sf"][4] += 1
    elif what == "negative_exponent":
        a["ex"][7] = -a["ex"][7]
    elif what == "zero_exponent":
        a["ex"][0] = 0.0
    elif what == "nan_coefficient":
        a["co"][9] = math.nan
    elif what == "inf_exponent":
        a["ex"][1] = math.inf
    elif what == "nan_position":
        a["xyz"][1, 2] = math.nan
    else:
        raise ValueError(what)
    return a, n_atom, n_shell


@pytest.mark.parametrize("what", ["no_shells", "no_atoms", "negative_l", "atom_out_of_range", "zero_primitives",
                                  "first_bf_gap", "negative_exponent", "zero_exponent", "nan_coefficient",
                                  "inf_exponent", "nan_position"])
def test_malformed_basis_is_refused(mol, what):
    a, n_atom, n_shell = _corrupt(mol, what)
    assert _create(a, n_atom, n_shell) == TF_EINVAL


def test_angular_momentum_beyond_the_kernels_is_unsupported(mol):
    a = _basis_arrays(mol)
    a["sl"][-1] = 7                           # the last shell: no later first_bf moves
    assert _create(a, mol.n_atom, mol.n_shell) == TF_EUNSUPPORTED


def test_null_arrays_are_refused(mol):
    from tonto_b200.fock import _Basis, load_library
    L = load_library()
    b = _Basis(mol.n_atom, None, mol.n_shell, None, None, None, None, None, None, 1)
    h = ctypes.c_void_p()
    assert L.tf_ctx_create(ctypes.byref(b), None, ctypes.byref(h)) == TF_EINVAL
    assert L.tf_ctx_create(None, None, ctypes.byref(h)) == TF_EINVAL


@pytest.mark.parametrize("field,value", [("eri_schwarz_cutoff", 0.0), ("eri_schwarz_cutoff", -1e-9),
                                         ("eri_schwarz_cutoff", math.nan), ("eri_primitive_pair_cutoff", -1.0),
                                         ("mixed_fp32_cut", math.nan), ("device", -1), ("deterministic", 2),
                                         ("deterministic", -1)])
def test_bad_options_are_refused(mol, field, value):
    from tonto_b200.fock import default_options
    opt = default_options()
    setattr(opt, field, value)
    assert _create(_basis_arrays(mol), mol.n_atom, mol.n_shell, opt=opt) == TF_EINVAL


def test_batch_of_mixed_basis_kinds_is_refused():
    from tonto_b200.fock import _Basis, load_library
    L = load_library()
    keep = []
    structs = []
    for m in (water_cluster(2, seed=0), water_cluster(2, seed=1, spherical=False)):
        a = _basis_arrays(m)
        keep.append(a)
        dp = lambda x: x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
        ip = lambda x: x.ctypes.data_as(ctypes.POINTER(ctypes.c_int))     # noqa: E731
        structs.append(_Basis(m.n_atom, dp(a["xyz"]), m.n_shell, ip(a["sa"]), ip(a["sl"]), ip(a["sn"]), ip(a["sf"]),
                              dp(a["ex"]), dp(a["co"]), int(m.spherical)))
    arr = (_Basis * 2)(*structs)
    h = ctypes.c_void_p()
    assert L.tf_ctx_create_batch(arr, 2, None, ctypes.byref(h)) == TF_EINVAL


def test_failure_injection_rejects_a_negative_countdown():
    from tonto_b200.fock import load_library
    L = load_library()
    assert L.tf_debug_fail_alloc(-1) == TF_EINVAL
    assert L.tf_debug_fail_alloc(0) == 0
