"""The C-ABI library loads on a machine without a GPU and exports every entry
point include/bd_b200.h declares.  No compute call is made here."""
import ctypes
import os
import subprocess

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
