"""ctypes bindings for the test oracle.

TEST INFRASTRUCTURE ONLY: tests/, ``__graft_entry__.smoke()`` and bench.py's
cpu_baseline / reference arm may import this module; the product library never
does.  Two libraries are wrapped:

* ``liboracle.so`` -- the project's FP64 C restatement of the reference's
  step-loop routines (oracle/bd_oracle.c), always built;
* ``_ref/libref_{shear,ext}.so`` -- the unmodified reference simulator compiled
  from its own sources with a renamed ``main`` (oracle/ref_harness.c), present
  only where the reference sources were available at build time.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


# where the reference sources lie (only the recipe that compiles them reads
# this); override with the REF_ROOT environment variable
REF_ROOT = os.environ.get("REF_ROOT", "/root/reference")


def build(ref_root: str | None = REF_ROOT) -> None:
    """Compile liboracle.so and, when the reference sources exist, _ref/."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if ref_root and os.path.isdir(ref_root):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_ROOT={ref_root}"], check=True)


class Sys(C.Structure):
    _fields_ = [
        ("flow", C.c_int), ("N", C.c_int), ("Nb", C.c_int), ("Nc", C.c_int),
        ("L", C.c_double), ("edot", C.c_double), ("dt", C.c_double),
        ("tp", C.c_int), ("spring", C.c_int),
        ("kappas", C.c_double), ("qmax", C.c_double), ("qmax2", C.c_double),
        ("kappab", C.c_double), ("epsilon", C.c_double),
        ("rv", C.c_double), ("r2cut", C.c_double), ("rnew", C.c_double),
        ("lambda_b", C.c_double), ("lambda_d", C.c_double), ("kappa_d", C.c_double),
        ("barrier", C.c_double), ("barrier2", C.c_double), ("MStep", C.c_int),
        ("t", C.c_ulong),
        ("L1", C.c_double * 2), ("L2", C.c_double * 2),
        ("L1xp", C.c_double), ("L1yp", C.c_double), ("L2xp", C.c_double),
        ("L2yp", C.c_double), ("detL", C.c_double), ("theta", C.c_double),
        ("cth", C.c_double), ("sth", C.c_double), ("delx", C.c_double),
        ("nt_avg", C.c_int), ("nbx", C.c_int), ("nby", C.c_int), ("nbz", C.c_int),
        ("nhx", C.c_int), ("nhy", C.c_int), ("nhz", C.c_int), ("nbins", C.c_int),
        ("bsx", C.c_double), ("bsy", C.c_double), ("bsz", C.c_double),
        ("bin_size", C.c_double),
    ]


class Rng(C.Structure):
    _fields_ = [("idum", C.c_long), ("idum2", C.c_long), ("iy", C.c_long),
                ("iv", C.c_long * 32), ("iset", C.c_int), ("gset", C.c_float)]

    def state_words(self) -> np.ndarray:
        """idum, idum2, iy, iv[32], iset and the bits of gset as int64."""
        g = np.float32(self.gset).view(np.int32)
        return np.array([self.idum, self.idum2, self.iy, *self.iv, self.iset, int(g)], dtype=np.int64)


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(None)
        L = C.CDLL(path)
        sp, rp = C.POINTER(Sys), C.POINTER(Rng)
        L.bdo_init.argtypes = [sp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                               C.c_int, C.c_double, C.c_int, C.c_double, C.c_double, C.c_double,
                               C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int]
        L.bdo_lattice.argtypes = [sp, C.c_ulong]
        L.bdo_apply_pbc.argtypes = [sp, _dp, _dp, _dp]
        L.bdo_rotate.argtypes = [sp, _dp, _dp, C.c_int]
        L.bdo_nid.argtypes = [sp, _dp, _dp, _dp, C.c_int, C.c_int, _dp]
        L.bdo_nidbin.argtypes = [sp, _dp, _dp, _dp, C.c_int, C.c_int, _dp]
        L.bdo_binij.argtypes = [sp, _dp, _dp, _dp, C.c_int, C.c_int]
        L.bdo_bond.argtypes = [sp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.bdo_ev.argtypes = [sp, _dp, _dp, _dp, _ip, _ip, C.c_int, _dp, _dp, _dp, _dp]
        L.bdo_coulomb.argtypes = [sp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.bdo_verlet.argtypes = [sp, _dp, _dp, _dp, _ip, _ip, C.c_int]
        L.bdo_check_verlet.argtypes = [sp, _dp, _dp, _dp]
        L.bdo_calc_hi.argtypes = [sp, _dp, _dp, _dp, _dp, _dp]
        L.bdo_grid.argtypes = [sp, C.c_double, C.c_double, _dp, _ip]
        L.bdo_calc_hi_ewald.argtypes = [sp, _dp, _dp, _dp, _dp]
        L.bdo_grid_geom.argtypes = [sp, C.c_double, _ip]
        L.bdo_update_hi.argtypes = [sp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                    C.c_double, _dp]
        L.bdo_update_fd.argtypes = [sp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.bdo_rng_fresh.argtypes = [rp, C.c_long]
        L.bdo_ran1.argtypes = [rp]
        L.bdo_ran1.restype = C.c_float
        L.bdo_gasdev.argtypes = [rp]
        L.bdo_gasdev.restype = C.c_float
        L.bdo_noise.argtypes = [rp, _dp, C.c_int]
        L.bdo_charge_hop.argtypes = [sp, _dp, _dp, _dp, _ip, _ip, _ip, C.c_int, rp, _ip, C.c_int]
        L.bdo_dh_energy.argtypes = [sp, _dp, _dp, _dp, _ip, C.c_int]
        L.bdo_dh_energy.restype = C.c_double
        _lib = L
    return _lib


class Oracle:
    """Explicit-state FP64 restatement of one reference system."""

    def __init__(self, flow, Nb, Nc, L, edot, dt, nt_avg=8, bin_size=2.0, spring="FENE",
                 kappas=30.0, qmax=3.0, kappab=0.0, epsilon=1.0, lambda_b=2.0, lambda_d=5.0,
                 barrier=3.0, barrier2=3.0, MStep=100):
        self.s = Sys()
        lib().bdo_init(C.byref(self.s), int(flow), Nb, Nc, L, edot, dt, nt_avg, bin_size,
                       1 if spring == "FENE" else 0, kappas, qmax, kappab, epsilon,
                       lambda_b, lambda_d, barrier, barrier2, MStep)
        self.N = Nb * Nc

    def lattice(self, t):
        lib().bdo_lattice(C.byref(self.s), int(t))

    def apply_pbc(self, x, y, z):
        lib().bdo_apply_pbc(C.byref(self.s), x, y, z)

    def rotate(self, x, y, inverse):
        lib().bdo_rotate(C.byref(self.s), x, y, int(inverse))

    def nid(self, x, y, z, i, j):
        o = np.zeros(3)
        lib().bdo_nid(C.byref(self.s), x, y, z, i, j, o)
        return o

    def bond(self, x, y, z, f, stress):
        return lib().bdo_bond(C.byref(self.s), x, y, z, f[0], f[1], f[2], stress)

    def ev(self, x, y, z, counts, rows, f, stress):
        lib().bdo_ev(C.byref(self.s), x, y, z, counts, rows, rows.shape[1], f[0], f[1], f[2], stress)

    def coulomb(self, x, y, z, q, f):
        lib().bdo_coulomb(C.byref(self.s), x, y, z, np.ascontiguousarray(q, dtype=np.float64),
                          f[0], f[1], f[2])

    def verlet(self, x, y, z, maxnb=256):
        counts = np.zeros(self.N, np.int32)
        rows = np.zeros((self.N, maxnb), np.int32)
        if lib().bdo_verlet(C.byref(self.s), x, y, z, counts, rows, maxnb) != 0:
            raise RuntimeError("neighbour row overflow")
        return counts, rows

    def check_verlet(self, dx, dy, dz):
        return bool(lib().bdo_check_verlet(C.byref(self.s), dx, dy, dz))

    def calc_hi(self, x, y, z, grid):
        M = np.zeros(9 * self.N * self.N)
        lib().bdo_calc_hi(C.byref(self.s), x, y, z, np.ascontiguousarray(grid, dtype=np.float64), M)
        return M

    def calc_hi_ewald(self, x, y, z):
        M = np.zeros(9 * self.N * self.N)
        lib().bdo_calc_hi_ewald(C.byref(self.s), x, y, z, M)
        return M

    def grid(self, grid_dt=0.001, box_volume=None):
        """gridHI's table: (D[nt_avg, nbins*9], geom[8]) on gridHI's bin geometry."""
        bv = self.s.L ** 3 if box_volume is None else box_volume
        geom = np.zeros(8, np.int32)
        lib().bdo_grid_geom(C.byref(self.s), grid_dt, geom)
        D = np.zeros(self.s.nt_avg * int(geom[6]) * 9)
        lib().bdo_grid(C.byref(self.s), grid_dt, bv, D, geom)
        return D.reshape(self.s.nt_avg, -1), geom

    def update_hi(self, x, y, z, dv, f, R, M, beta, Ct):
        lib().bdo_update_hi(C.byref(self.s), x, y, z, dv[0], dv[1], dv[2], f[0], f[1], f[2],
                            R, M, beta, Ct)

    def update_fd(self, x, y, z, dv, f, R):
        lib().bdo_update_fd(C.byref(self.s), x, y, z, dv[0], dv[1], dv[2], f[0], f[1], f[2], R)

    def charge_hop(self, x, y, z, track, old, rng, logcap=None):
        nch = len(track)
        idx = track.copy()
        logcap = nch if logcap is None else logcap
        log = np.zeros(3 * max(logcap, 1), np.int32)
        nacc = lib().bdo_charge_hop(C.byref(self.s), x, y, z, track, idx, old, nch,
                                    C.byref(rng), log, logcap)
        return nacc, log.reshape(-1, 3)[:logcap]

    def dh_energy(self, x, y, z, beads):
        b = np.ascontiguousarray(beads, dtype=np.int32)
        return lib().bdo_dh_energy(C.byref(self.s), x, y, z, b, len(b))


def fresh_rng(seed: int) -> Rng:
    g = Rng()
    lib().bdo_rng_fresh(C.byref(g), seed)
    return g


# ---------------------------------------------------------------------------
# The reference itself (oracle/_ref), for pinning the restatement.


def ref_path(flow: int) -> str:
    return os.path.join(HERE, "_ref", "libref_shear.so" if flow == 0 else "libref_ext.so")


def ref_available(flow: int = 0) -> bool:
    return os.path.exists(ref_path(flow))


class RefSim:
    """The reference's own routines on its own globals (one per process)."""

    def __init__(self, flow, Nb, Nc, L, edot, dt, nt_avg=8, bin_size=2.0, spring="FENE",
                 kappas=30.0, qmax=3.0, kappab=0.0, epsilon=1.0, lambda_b=2.0, lambda_d=5.0,
                 Ncharges=0, barrier=3.0, barrier2=3.0, MStep=100, seed=830062920, threads=1):
        L_ = C.CDLL(ref_path(flow), mode=C.RTLD_LOCAL)
        self.lib = L_
        self.flow = flow
        L_.h_setup.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                               C.c_double, C.c_char_p, C.c_double, C.c_double, C.c_double,
                               C.c_double, C.c_double, C.c_double, C.c_int, C.c_double,
                               C.c_double, C.c_int, C.c_long, C.c_int]
        L_.h_setup(Nb, Nc, L, edot, dt, nt_avg, bin_size, spring.encode(), epsilon, kappab,
                   kappas, qmax, lambda_b, lambda_d, Ncharges, barrier, barrier2, MStep, seed,
                   threads)
        self.N = Nb * Nc
        self.Nb = Nb
        for name in ("h_set_pos", "h_get_pos", "h_set_dv", "h_get_dv", "h_set_force", "h_get_force"):
            getattr(L_, name).argtypes = [_dp, _dp, _dp]
        L_.h_set_t.argtypes = [C.c_ulong]
        L_.h_set_tstart.argtypes = [C.c_ulong]
        L_.h_set_strain.argtypes = [C.c_double]
        L_.h_update_lattice.argtypes = [C.c_ulong]
        L_.h_get_lattice.argtypes = [_dp]
        L_.h_nid.argtypes = [C.c_int, C.c_int, _dp]
        L_.h_nidbin.argtypes = [C.c_int, C.c_int, _dp]
        L_.h_binij.argtypes = [C.c_int, C.c_int]
        L_.h_get_stress.argtypes = [_dp]
        L_.h_get_verlet.argtypes = [_ip, _ip, C.c_int]
        L_.h_set_charges.argtypes = [_ip, C.c_int]
        L_.h_get_charges.argtypes = [_ip, _ip, _ip]
        L_.h_set_noise.argtypes = [_dp]
        L_.h_get_noise.argtypes = [_dp]
        L_.h_get_idum.restype = C.c_long
        L_.h_set_idum.argtypes = [C.c_long]
        L_.h_ran1.restype = C.c_float
        L_.h_gasdev.restype = C.c_float
        L_.h_bins.argtypes = [_ip]
        L_.h_bin_sizes.argtypes = [_dp]
        L_.h_set_grid.argtypes = [C.c_int, _dp]
        L_.h_set_tea.argtypes = [C.c_int, C.c_double, _dp]
        L_.h_get_M.argtypes = [_dp]
        L_.h_set_M.argtypes = [_dp]
        L_.h_hop_counters.argtypes = [_ip]
        L_.h_step_hi.argtypes = [C.c_ulong, C.c_int]
        L_.h_wtime.restype = C.c_double
        L_.h_tp.restype = C.c_ulong
        L_.h_ewald_bin.argtypes = [C.POINTER(C.c_double), _dp]
        L_.h_catea.argtypes = [C.c_double, C.c_char_p, _dp, _dp, _ip]
        for name in ("h_print_traj", "h_print_ext"):
            getattr(L_, name).argtypes = [C.c_char_p]
        L_.h_print_visc.argtypes = [C.c_char_p, C.c_int]
        L_.h_print_restart.argtypes = [C.c_char_p]
        L_.h_get_unwrapped.argtypes = [_dp, _dp, _dp]
        L_.h_msd.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_ulong, C.c_int, C.c_int,
                             C.c_double]
        self.Nb_, self.sbins = Nb, 20

    def __getattr__(self, name):
        return getattr(self.lib, "h_" + name)

    def pos(self):
        x, y, z = (np.zeros(self.N) for _ in range(3))
        self.lib.h_get_pos(x, y, z)
        return x, y, z

    def ewald_bin(self):
        eps = C.c_double()
        rs = np.zeros(3 * self.N)
        self.lib.h_ewald_bin(C.byref(eps), rs)
        return eps.value, rs

    def catea(self, strain, beta_path):
        brun = np.zeros(self.sbins + 1)
        crun = np.zeros((self.sbins + 1) * 3 * self.Nb_)
        gw = np.zeros(self.sbins + 1, np.int32)
        self.lib.h_catea(float(strain), beta_path.encode(), brun, crun, gw)
        return brun, crun.reshape(self.sbins + 1, 3 * self.Nb_), gw

    def set_pos(self, x, y, z):
        self.lib.h_set_pos(*(np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z)))

    def force(self):
        x, y, z = (np.zeros(self.N) for _ in range(3))
        self.lib.h_get_force(x, y, z)
        return np.stack([x, y, z])

    def dv(self):
        x, y, z = (np.zeros(self.N) for _ in range(3))
        self.lib.h_get_dv(x, y, z)
        return np.stack([x, y, z])

    def stress(self):
        o = np.zeros(3)
        self.lib.h_get_stress(o)
        return o

    def lattice(self):
        o = np.zeros(10)
        self.lib.h_get_lattice(o)
        return o

    def verlet_rows(self, maxnb=256):
        counts = np.zeros(self.N, np.int32)
        rows = np.zeros((self.N, maxnb), np.int32)
        if self.lib.h_get_verlet(counts, rows, maxnb) != 0:
            raise RuntimeError("neighbour row overflow")
        return counts, rows

    def charges(self, nch):
        tr, old = np.zeros(nch, np.int32), np.zeros(nch, np.int32)
        flags = np.zeros(self.N, np.int32)
        self.lib.h_get_charges(tr, old, flags)
        return tr, old, flags

    def M(self):
        o = np.zeros(9 * self.N * self.N)
        self.lib.h_get_M(o)
        return o

    def bins(self):
        o = np.zeros(7, np.int32)
        self.lib.h_bins(o)
        return o


class OracleSim:
    """The restated routines composed into the reference's hydrodynamic step
    (shear/src/main26.c:65-151, extensional/src/main14.c:68-171), without file
    output; mirrors ref_harness.c's h_begin_iteration/h_step_hi."""

    def __init__(self, orc: Oracle, x, y, z, charges, seed, grid, beta, C, MStep=100, srpy=100,
                 sbins=20, strain_ss=10.0, maxnb=256):
        self.o = orc
        self.N = orc.N
        self.x, self.y, self.z = (np.array(a, np.float64) for a in (x, y, z))
        self.dv = np.zeros((3, self.N))
        self.f = np.zeros((3, self.N))
        self.R = np.zeros(3 * self.N)
        self.track = np.array(charges, np.int32)
        self.old = self.track.copy()
        self.rng = fresh_rng(seed)
        self.grid = np.ascontiguousarray(grid, np.float64)
        self.beta, self.C = beta, C
        self.srpy, self.sbins = srpy, sbins
        self.strain_interval = strain_ss / sbins
        self.maxnb = maxnb
        self.tstart = 0
        self.M = None
        self.stress = np.zeros(3)
        orc.s.MStep = MStep

    def q(self):
        q = np.zeros(self.N)
        q[self.track] = 1.0
        return q

    def begin_iteration(self, tstart=0):
        o = self.o
        self.tstart = tstart
        o.lattice(tstart)
        if o.s.flow == 1:
            o.rotate(self.x, self.y, 0)
        o.apply_pbc(self.x, self.y, self.z)
        self.counts, self.rows = o.verlet(self.x, self.y, self.z, self.maxnb)
        self.dv[:] = 0
        if o.s.flow == 1:
            o.rotate(self.x, self.y, 1)

    def step_hi(self, t, with_hop=True):
        o, ext = self.o, self.o.s.flow == 1
        if ext:
            o.rotate(self.x, self.y, 0)
            o.rotate(self.x, self.y, 1)
        self.f[:] = 0
        self.stress[:] = 0
        strain = t * o.s.dt * o.s.edot
        o.lattice(t)
        if ext:
            o.rotate(self.x, self.y, 0)
        o.apply_pbc(self.x, self.y, self.z)
        if o.check_verlet(*self.dv):
            self.counts, self.rows = o.verlet(self.x, self.y, self.z, self.maxnb)
            self.dv[:] = 0
        if o.bond(self.x, self.y, self.z, self.f, self.stress):
            raise RuntimeError("FENE overstretch")
        o.ev(self.x, self.y, self.z, self.counts, self.rows, self.f, self.stress)
        o.coulomb(self.x, self.y, self.z, self.q(), self.f)
        lib().bdo_noise(C.byref(self.rng), self.R, 3 * self.N)
        if t % self.srpy == 0 or t == self.tstart:
            self.M = o.calc_hi(self.x, self.y, self.z, self.grid)
            sb = min(int(np.floor(strain / self.strain_interval)), self.sbins)
            self.bt = float(self.beta[sb])
            self.Ct = np.ascontiguousarray(np.tile(self.C[sb], o.s.Nc))
        o.update_hi(self.x, self.y, self.z, self.dv, self.f, self.R, self.M, self.bt, self.Ct)
        if with_hop:
            if ext:
                o.rotate(self.x, self.y, 0)
            o.charge_hop(self.x, self.y, self.z, self.track, self.old, self.rng)
            if ext:
                o.rotate(self.x, self.y, 1)


def ref_grid(flow, Nb, Nc, c_norm, edot, nt_avg, bin_size, workdir):
    """Runs the reference's gridHI main (one per process) in workdir and
    returns (D[nt_avg, nbins*9], bins[8], geom[7]) from its globals."""
    path = os.path.join(HERE, "_ref", "libref_grid_shear.so" if flow == 0 else "libref_grid_ext.so")
    lib_ = C.CDLL(path, mode=C.RTLD_LOCAL)
    os.makedirs(os.path.join(workdir, "mm"), exist_ok=True)
    cwd = os.getcwd()
    os.chdir(workdir)
    try:
        argv = ["gridHI", "-c", repr(c_norm), "-b", str(Nb), "-a", str(Nc), "-f", repr(edot),
                "-s", str(nt_avg), "-g", repr(bin_size), "-n", "1"]
        arr = (C.c_char_p * len(argv))(*[a.encode() for a in argv])
        lib_.grid_main.argtypes = [C.c_int, C.POINTER(C.c_char_p)]
        lib_.grid_main(len(argv), arr)
    finally:
        os.chdir(cwd)
    bins = np.zeros(8, np.int32)
    lib_.hg_bins.argtypes = [_ip]
    lib_.hg_bins(bins)
    geom = np.zeros(7)
    lib_.hg_geom.argtypes = [_dp]
    lib_.hg_geom(geom)
    lib_.hg_D.argtypes = [C.c_int, _dp]
    D = np.zeros((nt_avg, int(bins[6]) * 9))
    for nt in range(nt_avg):
        row = np.zeros(int(bins[6]) * 9)
        lib_.hg_D(nt, row)
        D[nt] = row
    return D, bins, geom


def full_mobility(M9, N):
    """The symmetric 3N x 3N matrix from the reference layout (upper blocks and
    the diagonal entries of the diagonal blocks filled): block (j, i) = block
    (i, j), whose 3x3 blocks are symmetric."""
    B = M9.reshape(N, N, 3, 3).copy()
    iu = np.triu_indices(N, 1)
    up = B[iu]
    B[(iu[1], iu[0])] = up
    for i in range(N):
        d = np.diag(B[i, i]).copy()
        B[i, i] = np.diag(d)
    return B.transpose(0, 2, 1, 3).reshape(3 * N, 3 * N)


def sqrtm_apply(Mfull, z):
    """sqrt(M) z by a dense eigendecomposition (numpy eigh), negative
    eigenvalues clamped to zero; also returns the smallest eigenvalue."""
    w, Q = np.linalg.eigh(Mfull)
    return Q @ (np.sqrt(np.clip(w, 0, None)) * (Q.T @ z)), float(w.min())
