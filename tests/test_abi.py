"""The C-ABI library loads on a machine without a GPU and exports every entry
point include/bd_b200.h declares.  No compute call is made here."""
import ctypes
import os
import subprocess

import numpy as np

import pytest

import bd_b200 as B


@pytest.fixture(scope="module")
def libpath():
    if not os.path.exists(B.LIB):
        B.build()
    return B.LIB


def test_header_declares_reference_entry_points():
    names = B.exported_symbols()
    for n in ("bd_create", "bd_destroy", "bd_bond_force", "bd_ev_force", "bd_coulomb_force",
              "bd_build_neighbors", "bd_check_verlet", "bd_calc_hi", "bd_update_hi",
              "bd_update_fd", "bd_get_noise", "bd_charge_hop", "bd_apply_pbc",
              "bd_update_lattice", "bd_step_reference"):
        assert n in names


def test_library_exports_every_declared_symbol(libpath):
    lib = ctypes.CDLL(libpath)
    missing = [n for n in B.exported_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True,
                         text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert set(B.exported_symbols()) <= exported


def test_default_grid_rule_matches_python(libpath):
    """bd_pme_default_grid (the grid bd_create picks) against the module's own
    statement of the rule, over boxes 10..200 and cutoffs 4..25 and the
    default cutoff; invalid boxes are rejected."""
    lib = ctypes.CDLL(libpath)
    lib.bd_pme_default_grid.argtypes = [ctypes.c_double, ctypes.c_double,
                                        ctypes.POINTER(ctypes.c_int)]
    K = ctypes.c_int()
    for L in np.linspace(10.0, 200.0, 39):
        for rc in [0.0] + list(np.linspace(4.0, min(25.0, 0.43 * L), 9)):
            assert lib.bd_pme_default_grid(L, rc, ctypes.byref(K)) == 0
            assert K.value == B.pme_default_grid(L, rc if rc > 0 else None), (L, rc)
    assert lib.bd_pme_default_grid(60.0, 12.1, ctypes.byref(K)) == 0 and K.value == 64
    assert lib.bd_pme_default_grid(0.0, 10.0, ctypes.byref(K)) != 0
    assert lib.bd_pme_default_grid(60.0, 1e-4, ctypes.byref(K)) != 0


def test_status_strings(libpath):
    lib = ctypes.CDLL(libpath)
    lib.bd_status_string.restype = ctypes.c_char_p
    assert lib.bd_status_string(0) == b"ok"
    assert b"overstretch" in lib.bd_status_string(4).lower()


def test_create_rejects_bad_params_without_touching_a_device(libpath):
    p = B.make_params(0, 0, 4, 10.0, 0.1, 5e-4)  # Nb = 0
    lib = B._lib()
    h = ctypes.c_void_p()
    assert lib.bd_create(ctypes.byref(p), ctypes.byref(h)) == 1  # BD_ERR_ARG
