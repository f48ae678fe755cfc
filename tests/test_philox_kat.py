"""Philox4x32-10 against the published known-answer vectors.

The library draws its production noise (k_noise_philox) and the parallel
charge-hop sweep's proposals and uniforms from Philox4x32-10 (Salmon, Moraes,
Dror and Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11).  The
three vectors below are the philox4x32 / 10-round lines of the Random123
distribution's known-answer file (kat_vectors): counter, key, expected
output, all 32-bit words.

* CPU: oracle/hop_oracle.py's restatement (the model the GPU sweep is checked
  against) reproduces every vector.
* GPU: the device generator (bd_philox4x32_10, the same device function the
  noise and sweep kernels call) reproduces every vector, and agrees with the
  oracle on a few thousand seeded counters and keys.
"""
import ctypes

import numpy as np
import pytest

import bd_b200 as B
from hop_oracle import philox4x32_10

KAT = [
    ((0x00000000, 0x00000000, 0x00000000, 0x00000000), (0x00000000, 0x00000000),
     (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF), (0xFFFFFFFF, 0xFFFFFFFF),
     (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,out", KAT)
def test_oracle_philox_known_answers(ctr, key, out):
    assert tuple(philox4x32_10(ctr, key)) == out


def _device(ctr, key):
    lib = B._lib()
    u = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
    lib.bd_philox4x32_10.argtypes = [u, u, u, ctypes.c_int]
    ctr = np.ascontiguousarray(ctr, np.uint32).reshape(-1, 4)
    key = np.ascontiguousarray(key, np.uint32).reshape(-1, 2)
    out = np.zeros_like(ctr)
    s = lib.bd_philox4x32_10(ctr.reshape(-1), key.reshape(-1), out.reshape(-1), len(ctr))
    assert s == 0, lib.bd_status_string(s)
    return out


@pytest.mark.gpu
def test_device_philox_known_answers():
    got = _device([k[0] for k in KAT], [k[1] for k in KAT])
    assert [tuple(int(v) for v in row) for row in got] == [k[2] for k in KAT]


@pytest.mark.gpu
def test_device_philox_matches_oracle():
    r = np.random.default_rng(123)
    ctr = r.integers(0, 2 ** 32, size=(4096, 4), dtype=np.uint64).astype(np.uint32)
    key = r.integers(0, 2 ** 32, size=(4096, 2), dtype=np.uint64).astype(np.uint32)
    got = _device(ctr, key)
    for i in range(0, 4096, 7):
        ref = philox4x32_10(tuple(int(v) for v in ctr[i]), tuple(int(v) for v in key[i]))
        assert tuple(int(v) for v in got[i]) == tuple(ref)
