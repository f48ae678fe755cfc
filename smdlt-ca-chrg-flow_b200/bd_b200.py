"""Python binding of the bd_b200 C ABI (include/bd_b200.h).

A thin ctypes layer over ``libbd_b200.so``: every method calls one exported C
function and raises :class:`BDError` on a non-zero status.  The library is
the CUDA implementation; there is no CPU path behind this module, and loading
fails loudly when the shared library has not been built.

Method names follow the reference's step-loop routines
(shear/src/main.h:7-65): ``bond_force`` is bondforce, ``ev_force`` is
LJforce, ``coulomb_force`` is coulombForce, ``build_neighbors`` is verletlist,
``calc_hi``/``update_hi``/``update_fd``/``charge_hop`` are calcHI, updateHI,
updateFD and chargeHop.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB = os.path.join(PKG, "libbd_b200.so")
INCLUDE = os.path.join(ROOT, "include")
SOURCES = ["bd_core.cu", "bd_neighbors.cu", "bd_mobility.cu", "bd_mc.cu", "bd_lanczos.cu",
           "bd_noalloc.cu", "bd_pme.cu", "bd_precond.cu", "bd_mpnn.cu", "bd_coulomb.cu",
           "bd_batch.cu", "bd_catea.cu", "bd_msd.cu", "bd_output.cu"]
CUDA_LIB = "/usr/local/cuda/lib64"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")

FLOW_SHEAR, FLOW_EXT = 0, 1
NOISE_RAN1, NOISE_PHILOX = 0, 1
SPRING_HOOKEAN, SPRING_FENE = 0, 1


def build(verbose: bool = False) -> str:
    """Compile libbd_b200.so for sm_100a with nvcc (in-tree)."""
    srcs = [os.path.join(PKG, "csrc", s) for s in SOURCES]
    cmd = ["nvcc", "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-shared",
           f"-I{INCLUDE}", "-o", LIB, *srcs, f"-L{CUDA_LIB}", "-lcufft",
           "-Xlinker", f"-rpath,{CUDA_LIB}"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return LIB


class BDError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        msg = _lib().bd_status_string(status).decode() if _LIB else str(status)
        if _LIB and status == 2:  # BD_ERR_CUDA: the failing call
            msg += " at " + _lib().bd_last_error_detail().decode()
        super().__init__(f"{where}: {msg} (status {status})")


class Params(C.Structure):
    _fields_ = [
        ("flow", C.c_int), ("Nb", C.c_int), ("Nc", C.c_int), ("L", C.c_double),
        ("box_volume", C.c_double), ("edot", C.c_double), ("dt", C.c_double),
        ("spring", C.c_int), ("kappas", C.c_double), ("qmax", C.c_double),
        ("kappab", C.c_double), ("epsilon", C.c_double), ("shear_kappas_override", C.c_int),
        ("lambda_b", C.c_double), ("lambda_d", C.c_double), ("Ncharges", C.c_int),
        ("barrier", C.c_double), ("barrier2", C.c_double), ("MStep", C.c_int),
        ("nt_avg", C.c_int), ("bin_size", C.c_double), ("srpy", C.c_int), ("sbins", C.c_int),
        ("strain_ss", C.c_double), ("max_neighbors", C.c_int), ("seed", C.c_long),
        ("noise", C.c_int), ("philox_seed", C.c_ulonglong),
        ("mobility", C.c_int), ("precision", C.c_int), ("lanczos_tol", C.c_double),
        ("lanczos_max", C.c_int), ("pme_grid", C.c_int), ("pme_order", C.c_int),
        ("pme_rc", C.c_double), ("pme_alpha", C.c_double), ("pme_max_pairs", C.c_int),
        ("coulomb", C.c_int), ("coulomb_beta", C.c_double), ("coulomb_rc", C.c_double),
        ("hop", C.c_int), ("hop_radius", C.c_double), ("noise_block", C.c_int),
    ]


class Ran1State(C.Structure):
    _fields_ = [("idum", C.c_long), ("idum2", C.c_long), ("iy", C.c_long),
                ("iv", C.c_long * 32), ("iset", C.c_int), ("gset", C.c_float)]

    def state_words(self) -> np.ndarray:
        g = np.float32(self.gset).view(np.int32)
        return np.array([self.idum, self.idum2, self.iy, *self.iv, self.iset, int(g)],
                        dtype=np.int64)


_LIB = None


def _lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB):
            raise OSError(f"{LIB} is not built; run __graft_entry__.build() (nvcc, sm_100a)")
        L = C.CDLL(LIB)
        vp = C.c_void_p
        L.bd_status_string.restype = C.c_char_p
        L.bd_status_string.argtypes = [C.c_int]
        L.bd_last_error_detail.restype = C.c_char_p
        L.bd_last_error_detail.argtypes = []
        L.bd_create.argtypes = [C.POINTER(Params), C.POINTER(vp)]
        L.bd_destroy.argtypes = [vp]
        L.bd_sync.argtypes = [vp]
        L.bd_device_bytes.argtypes = [vp]
        L.bd_device_bytes.restype = C.c_size_t
        for n in ("bd_upload_positions", "bd_download_positions", "bd_upload_displacements",
                  "bd_download_displacements", "bd_upload_forces", "bd_download_forces"):
            getattr(L, n).argtypes = [vp, _dp, _dp, _dp]
        L.bd_download_stress.argtypes = [vp, _dp]
        L.bd_reset_stress.argtypes = [vp]
        L.bd_upload_noise.argtypes = [vp, _dp]
        L.bd_download_noise.argtypes = [vp, _dp]
        L.bd_set_charges.argtypes = [vp, _ip, C.c_int]
        L.bd_download_charges.argtypes = [vp, _ip, _ip, _ip]
        L.bd_set_rng.argtypes = [vp, C.POINTER(Ran1State)]
        L.bd_get_rng.argtypes = [vp, C.POINTER(Ran1State)]
        L.bd_load_grid.argtypes = [vp, C.c_int, _dp]
        L.bd_grid_shape.argtypes = [vp, _ip]
        L.bd_build_grid.argtypes = [vp, C.c_double]
        L.bd_download_grid.argtypes = [vp, C.c_int, _dp]
        L.bd_set_tea.argtypes = [vp, C.c_int, C.c_double, _dp]
        L.bd_set_time.argtypes = [vp, C.c_ulong, C.c_ulong]
        L.bd_update_lattice.argtypes = [vp, C.c_ulong]
        L.bd_get_lattice.argtypes = [vp, _dp]
        for n in ("bd_apply_pbc", "bd_transform_coords", "bd_inverse_coords", "bd_reset_force",
                  "bd_build_neighbors", "bd_check_verlet", "bd_bond_force", "bd_ev_force",
                  "bd_coulomb_force", "bd_get_noise", "bd_calc_hi", "bd_update_hi",
                  "bd_update_fd", "bd_charge_hop"):
            getattr(L, n).argtypes = [vp]
        L.bd_download_neighbors.argtypes = [vp, _ip, _ip, C.c_int]
        L.bd_download_mobility.argtypes = [vp, _dp]
        L.bd_download_hop_log.argtypes = [vp, _ip]
        L.bd_download_hop_energies.argtypes = [vp, _dp]
        L.bd_step_reference.argtypes = [vp, C.c_ulong, C.c_int, C.c_int]
        L.bd_mobility_apply.argtypes = [vp, _dp, _dp]
        L.bd_mobility_apply_block.argtypes = [vp, C.c_int, _dp, _dp]
        L.bd_lanczos_sqrt.argtypes = [vp, _dp, _dp, C.POINTER(C.c_int)]
        L.bd_lanczos_stats.argtypes = [vp, np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")]
        L.bd_krylov_check_stats.argtypes = [vp, np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")]
        L.bd_set_device_krylov.argtypes = [vp, C.c_int]
        L.bd_noise_block_stats.argtypes = [vp, np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")]
        L.bd_noise_block_release.argtypes = [vp]
        L.bd_step_lanczos.argtypes = [vp, C.c_ulong, C.c_int, C.c_int]
        L.bd_profile_enable.argtypes = [vp, C.c_int]
        L.bd_profile_read.argtypes = [vp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_long)]
        L.bd_launch_count.argtypes = [vp]
        L.bd_launch_count.restype = C.c_longlong
        _fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
        _lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
        L.bd_set_preconditioner.argtypes = [vp, C.c_int, C.c_int]
        L.bd_enable_graphs.argtypes = [vp, C.c_int]
        L.bd_batch_create.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(vp)]
        L.bd_batch_step_lanczos.argtypes = [vp, C.c_ulong, C.c_int, C.c_int]
        L.bd_batch_destroy.argtypes = [vp]
        L.bd_autotune_pme_grid.argtypes = [C.c_double, C.c_int, C.POINTER(C.c_int)]
        L.bd_set_charge_values.argtypes = [vp, _dp]
        L.bd_ewald_bin.argtypes = [vp, C.POINTER(C.c_double), _dp]
        L.bd_catea.argtypes = [vp, C.c_double, C.POINTER(C.c_double)]
        L.bd_catea_averages.argtypes = [vp, _ip, _dp, _dp]
        L.bd_write_decomp.argtypes = [vp, C.c_char_p, C.c_ulong]
        L.bd_catea_apply.argtypes = [vp]
        L.bd_msd.argtypes = [_dp, C.c_int, C.c_int, C.c_int, _dp]
        L.bd_chain_props.argtypes = [vp, _dp, _dp, _dp, _dp]
        for n in ("bd_write_trajectory", "bd_write_restart"):
            getattr(L, n).argtypes = [vp, C.c_char_p, C.c_ulong]
        L.bd_write_ext.argtypes = [vp, C.c_char_p, C.c_ulong, C.c_double]
        L.bd_write_visc.argtypes = [vp, C.c_char_p, C.c_ulong, C.c_int]
        L.bd_coulomb_energy.argtypes = [vp, _dp]
        L.bd_set_precond_blocks.argtypes = [vp, _dp]
        L.bd_download_precond_blocks.argtypes = [vp, _dp, _dp, C.POINTER(C.c_int)]
        L.bd_precond_stats.argtypes = [vp, _lp]
        L.bd_lanczos_inv_sqrt.argtypes = [vp, _dp, _dp, C.POINTER(C.c_int)]
        L.bd_mpnn_param_count.restype = C.c_size_t
        L.bd_mpnn_param_count.argtypes = []
        L.bd_mpnn_set_params.argtypes = [vp, _fp]
        L.bd_mpnn_get_params.argtypes = [vp, _fp]
        L.bd_mpnn_features.argtypes = [vp]
        L.bd_mpnn_predict.argtypes = [vp, _dp]
        L.bd_mpnn_loss_grad.argtypes = [vp, _dp, _dp, C.POINTER(C.c_double), C.c_void_p]
        L.bd_mpnn_adam.argtypes = [vp, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int]
        _LIB = L
    return _LIB


def exported_symbols() -> list[str]:
    """Names declared in include/bd_b200.h (for the ABI export test)."""
    import re
    txt = open(os.path.join(INCLUDE, "bd_b200.h")).read()
    return sorted(set(re.findall(r"\b(bd_[a-z0-9_]+)\s*\(", txt)))


def _chk(status: int, where: str) -> None:
    if status != 0:
        raise BDError(status, where)


class Batch:
    """Independent replicas advanced concurrently (bd_batch_*); the contexts
    stay owned by the caller and must outlive the batch."""

    def __init__(self, contexts):
        self.L = _lib()
        self.ctxs = list(contexts)
        arr = (C.c_void_p * len(self.ctxs))(*[c.h.value for c in self.ctxs])
        h = C.c_void_p()
        _chk(self.L.bd_batch_create(arr, len(self.ctxs), C.byref(h)), "bd_batch_create")
        self.h = h

    def step_lanczos(self, t0, nsteps, with_hop=True):
        _chk(self.L.bd_batch_step_lanczos(self.h, int(t0), int(nsteps), int(bool(with_hop))),
             "bd_batch_step_lanczos")

    def close(self):
        if getattr(self, "h", None):
            self.L.bd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def msd(w, ncharges, Tmax, MSDstart=0):
    """calcMSD's rows {MSD, x, y, z} for lags 1..Tmax-MSDstart from the CH-file
    ordered displacement log w (Ncharges (Tmax+1) x 3)."""
    out = np.zeros(4 * (Tmax - MSDstart))
    _chk(_lib().bd_msd(np.ascontiguousarray(w, np.float64).reshape(-1), int(ncharges), int(Tmax),
                       int(MSDstart), out), "bd_msd")
    return out.reshape(-1, 4)


def autotune_pme_grid(L, precision="fp32"):
    K = C.c_int()
    _chk(_lib().bd_autotune_pme_grid(float(L), 1 if precision == "fp32" else 0, C.byref(K)),
         "bd_autotune_pme_grid")
    return K.value


def mpnn_param_count() -> int:
    return int(_lib().bd_mpnn_param_count())


# parameter layout of the learned preconditioner network (FP32):
# (name, shape) in storage order
MPNN_LAYOUT = [("W1", (64, 16)), ("b1", (64,)), ("W2", (64, 64)), ("b2", (64,)),
               ("W34", (64, 128)), ("b3", (64,)), ("wa", (64,)), ("ca", (1,)),
               ("wb", (64,)), ("cb", (1,))]


def mpnn_unpack(w):
    out, o = {}, 0
    for name, shp in MPNN_LAYOUT:
        n = int(np.prod(shp))
        out[name] = np.asarray(w[o:o + n]).reshape(shp)
        o += n
    return out


def mpnn_pack(d):
    return np.concatenate([np.asarray(d[name], np.float32).reshape(-1) for name, _ in MPNN_LAYOUT])


def mpnn_init(seed=0):
    """Seeded initial parameters: fan-in scaled Gaussian weights, zero heads
    (the initial blocks are the identity)."""
    r = np.random.default_rng(seed)
    d = {}
    for name, shp in MPNN_LAYOUT:
        if name.startswith("W"):
            d[name] = r.normal(0, 1 / np.sqrt(shp[1]), shp)
        else:
            d[name] = np.zeros(shp)
    return mpnn_pack(d)


def train_preconditioner(ctx, configs, steps_per_config=20, lr=3e-3, seed=0, step0=0):
    """Train the learned preconditioner network of ctx on the GPU.

    configs: iterable of (x, y, z, t) with positions in the frame bd_calc_hi
    reads them (PBC applied) at lattice step t.  For each configuration the
    mobility and the neighbour features are built; each training step draws
    z ~ N(0, I), forms the target M^-1/2 z by plain Lanczos and takes one Adam
    step on (1/N) sum_i |G_i z_i - (M^-1/2 z)_i|^2 (forward, backward and
    update are the library's own kernels).  ctx must have its network
    parameters set (bd_mpnn_set_params) and either no preconditioner active
    or the segment preconditioner, in which case the targets are
    (G M G^T)^-1/2 z and the network learns bead blocks to apply on top of
    the segment blocks (bd_set_preconditioner(LEARNED, segment)).
    Returns the per-step losses."""
    r = np.random.default_rng(seed)
    losses, step = [], step0
    for (x, y, z, t) in configs:
        ctx.set_positions(x, y, z)
        ctx.set_time(t, t)
        ctx.update_lattice(t)
        ctx.build_neighbors()
        ctx.calc_hi()
        ctx.mpnn_features()
        for _ in range(steps_per_config):
            zz = r.normal(size=3 * ctx.N)
            tgt, _ = ctx.lanczos_inv_sqrt(zz)
            losses.append(ctx.mpnn_loss_grad(zz, tgt))
            step += 1
            ctx.mpnn_adam(lr, step)
    return losses


def pme_default_grid(L, rc=None):
    """bd_create's default particle-mesh grid: the smallest 2^a 3^b 5^c at or
    above 12.9 L / rc (split parameter 4 / rc times spacing at most 0.31; cuFFT
    is markedly slower on sizes with a factor 7); rc defaults to the smaller of
    10 and 0.43 L, giving 1.29 L at rc = 10."""
    if rc is None:
        rc = min(10.0, 0.43 * L)
    K = int(np.ceil(12.9 * L / rc - 1e-9))
    while True:
        r = K
        for f in (2, 3, 5):
            while r % f == 0:
                r //= f
        if r == 1:
            return K
        K += 1


PME_CUTOFFS = (10.0, 11.1, 12.1, 13.6, 14.5, 15.5, 17.5)


def autotune_pme_cutoff(make_context, L, nrhs, candidates=PME_CUTOFFS, reps=4, seed=0):
    """Picks the particle-mesh cutoff, and with it the real-space cells and
    the grid (pme_default_grid: the accuracy rule fixes the grid spacing per
    cutoff), whose product of nrhs right-hand sides is fastest on this GPU
    for one configuration.  make_context(rc) returns a context with that
    cutoff and its mobility prepared (bd_calc_hi); each candidate's product
    is timed on the device (the BD_PROF_BLOCK events of
    bd_mobility_apply_block) after one untimed call, and the context is
    closed.  Candidates above 0.43 L (the minimum-image bound) are skipped.
    Returns (best cutoff, {cutoff: ms per product})."""
    times = {}
    for rc in candidates:
        if rc > 0.43 * L:
            continue
        c = make_context(rc)
        try:
            V = np.random.default_rng(seed).normal(size=(nrhs, 3 * c.N))
            c.mobility_apply_block(V)  # plans and first-touch allocations
            c.profile(True)
            for _ in range(reps):
                c.mobility_apply_block(V)
            ms, n = c.profile_read(Context.PROF_BLOCK)
            c.profile(False)
            times[rc] = ms / max(n, 1)
        finally:
            c.close()
    if not times:
        raise ValueError("autotune_pme_cutoff: no candidate cutoff fits the box")
    return min(times, key=times.get), times


def make_params(flow, Nb, Nc, L, edot, dt, *, spring="FENE", kappas=30.0, qmax=3.0, kappab=0.0,
                epsilon=1.0, lambda_b=2.0, lambda_d=5.0, Ncharges=0, barrier=3.0, barrier2=3.0,
                MStep=100, nt_avg=8, bin_size=2.0, srpy=100, sbins=20, strain_ss=10.0,
                max_neighbors=256, seed=None, shear_kappas_override=0, box_volume=0.0,
                noise="ran1", philox_seed=20261203, mobility="hybrid", precision="fp64",
                lanczos_tol=1e-6, lanczos_max=0, pme_grid=0, pme_order=0, pme_rc=0.0,
                pme_alpha=0.0, pme_max_pairs=0, coulomb="dh", coulomb_beta=0.0,
                coulomb_rc=0.0, hop="sequential", hop_radius=0.0, noise_block=1) -> Params:
    p = Params()
    p.flow, p.Nb, p.Nc, p.L, p.edot, p.dt = int(flow), Nb, Nc, L, edot, dt
    p.box_volume = box_volume
    p.spring = SPRING_FENE if spring == "FENE" else SPRING_HOOKEAN
    p.kappas, p.qmax, p.kappab, p.epsilon = kappas, qmax, kappab, epsilon
    p.shear_kappas_override = shear_kappas_override
    p.lambda_b, p.lambda_d, p.Ncharges = lambda_b, lambda_d, Ncharges
    p.barrier, p.barrier2, p.MStep = barrier, barrier2, MStep
    p.nt_avg, p.bin_size, p.srpy, p.sbins, p.strain_ss = nt_avg, bin_size, srpy, sbins, strain_ss
    p.max_neighbors = max_neighbors
    p.seed = (830062920 if flow == FLOW_SHEAR else 981272199) if seed is None else seed
    p.noise = NOISE_PHILOX if noise == "philox" else NOISE_RAN1
    p.philox_seed = philox_seed
    p.mobility = {"hybrid": 0, "ewald": 1, "pme": 2}[mobility]
    p.precision = 1 if precision == "fp32" else 0
    p.lanczos_tol, p.lanczos_max = lanczos_tol, lanczos_max
    p.pme_grid, p.pme_order, p.pme_rc = pme_grid, pme_order, pme_rc
    p.pme_alpha, p.pme_max_pairs = pme_alpha, pme_max_pairs
    p.coulomb = {"dh": 0, "ewald": 1}[coulomb]
    p.coulomb_beta, p.coulomb_rc = coulomb_beta, coulomb_rc
    p.hop = {"sequential": 0, "parallel": 1}[hop]
    p.hop_radius = hop_radius
    p.noise_block = noise_block
    return p


class Context:
    """Device-resident system; one CUDA stream per context."""

    def __init__(self, params: Params):
        self.L = _lib()
        self.p = params
        self.N = params.Nb * params.Nc
        h = C.c_void_p()
        _chk(self.L.bd_create(C.byref(params), C.byref(h)), "bd_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.bd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _call(self, name, *args):
        _chk(getattr(self.L, name)(self.h, *args), name)

    # state transfer
    def set_positions(self, x, y, z):
        self._call("bd_upload_positions", *(np.ascontiguousarray(a, np.float64) for a in (x, y, z)))

    def positions(self):
        a = [np.zeros(self.N) for _ in range(3)]
        self._call("bd_download_positions", *a)
        return a

    def set_displacements(self, x, y, z):
        self._call("bd_upload_displacements", *(np.ascontiguousarray(a, np.float64) for a in (x, y, z)))

    def displacements(self):
        a = [np.zeros(self.N) for _ in range(3)]
        self._call("bd_download_displacements", *a)
        return np.stack(a)

    def set_forces(self, x, y, z):
        self._call("bd_upload_forces", *(np.ascontiguousarray(a, np.float64) for a in (x, y, z)))

    def forces(self):
        a = [np.zeros(self.N) for _ in range(3)]
        self._call("bd_download_forces", *a)
        return np.stack(a)

    def stress(self):
        o = np.zeros(3)
        self._call("bd_download_stress", o)
        return o

    def set_noise(self, R):
        self._call("bd_upload_noise", np.ascontiguousarray(R, np.float64))

    def noise(self):
        o = np.zeros(3 * self.N)
        self._call("bd_download_noise", o)
        return o

    def set_charges(self, track):
        t = np.ascontiguousarray(track, np.int32)
        self._call("bd_set_charges", t, len(t))
        self.nch = len(t)

    def charges(self):
        n = getattr(self, "nch", 0)
        tr, old = np.zeros(max(n, 1), np.int32), np.zeros(max(n, 1), np.int32)
        fl = np.zeros(self.N, np.int32)
        self._call("bd_download_charges", tr, old, fl)
        return tr[:n], old[:n], fl

    def set_rng(self, state: Ran1State):
        self._call("bd_set_rng", C.byref(state))

    def rng(self) -> Ran1State:
        s = Ran1State()
        self._call("bd_get_rng", C.byref(s))
        return s

    def grid_shape(self):
        o = np.zeros(7, np.int32)
        self._call("bd_grid_shape", o)
        return o

    def load_grid(self, nt, D9):
        self._call("bd_load_grid", int(nt), np.ascontiguousarray(D9, np.float64))

    def build_grid(self, grid_dt=0.001):
        self._call("bd_build_grid", float(grid_dt))

    def grid(self, nt):
        o = np.zeros(int(self.grid_shape()[6]) * 9)
        self._call("bd_download_grid", int(nt), o)
        return o

    def set_tea(self, sbin, beta, c3nb):
        self._call("bd_set_tea", int(sbin), float(beta), np.ascontiguousarray(c3nb, np.float64))

    # step-loop routines
    def set_time(self, t, tstart=0):
        self._call("bd_set_time", int(t), int(tstart))

    def update_lattice(self, t):
        self._call("bd_update_lattice", int(t))

    def lattice(self):
        o = np.zeros(10)
        self._call("bd_get_lattice", o)
        return o

    def neighbors(self, maxnb=256):
        cnt = np.zeros(self.N, np.int32)
        rows = np.zeros((self.N, maxnb), np.int32)
        self._call("bd_download_neighbors", cnt, rows, maxnb)
        return cnt, rows

    def mobility(self):
        o = np.zeros(9 * self.N * self.N)
        self._call("bd_download_mobility", o)
        return o

    def hop_log(self):
        n = getattr(self, "nch", 0)
        o = np.zeros(3 * max(n, 1), np.int32)
        self._call("bd_download_hop_log", o)
        return o.reshape(-1, 3)[:n]

    def hop_energies(self):
        """Energy change each charge's trial of the last parallel sweep saw
        (NaN where the move was blocked)."""
        n = getattr(self, "nch", 0)
        o = np.zeros(max(n, 1))
        self._call("bd_download_hop_energies", o)
        return o[:n]

    def mobility_apply(self, v):
        out = np.zeros(3 * self.N)
        self._call("bd_mobility_apply", np.ascontiguousarray(v, np.float64), out)
        return out

    def mobility_apply_block(self, V):
        """M v_r for the rows v_r of V (k x 3N, bead-interleaved), through the
        noise blocks' multi-vector product where it applies."""
        V = np.ascontiguousarray(V, np.float64)
        out = np.zeros_like(V)
        self._call("bd_mobility_apply_block", V.shape[0], V.reshape(-1), out.reshape(-1))
        return out

    def lanczos_sqrt(self, z):
        out = np.zeros(3 * self.N)
        it = C.c_int()
        self._call("bd_lanczos_sqrt", np.ascontiguousarray(z, np.float64), out, C.byref(it))
        return out, it.value

    def lanczos_stats(self):
        o = np.zeros(4, np.int64)
        self._call("bd_lanczos_stats", o)
        return dict(calls=int(o[0]), iterations=int(o[1]), maxed=int(o[2]), negative=int(o[3]))

    def noise_block_stats(self):
        """Noise blocks of step_lanczos: block solves, block iterations run and
        the sum over those iterations of their right-hand sides."""
        o = np.zeros(3, np.int64)
        self._call("bd_noise_block_stats", o)
        return dict(blocks=int(o[0]), iterations=int(o[1]), rhs_iterations=int(o[2]))

    def noise_block_release(self):
        """Drops the noise block solved ahead; the generator rewinds to the
        per-step order."""
        self._call("bd_noise_block_release")

    def step_lanczos(self, t0, nsteps, with_hop=True):
        self._call("bd_step_lanczos", int(t0), int(nsteps), int(bool(with_hop)))

    def step_reference(self, t0, nsteps, with_hop=True):
        self._call("bd_step_reference", int(t0), int(nsteps), int(bool(with_hop)))

    def sync(self):
        self._call("bd_sync")

    PROF_MATVEC, PROF_HI_BUILD, PROF_HOP, PROF_FORCES, PROF_STEP, PROF_BLOCK = 0, 1, 2, 3, 4, 5

    def chain_props(self):
        Nc = self.p.Nc
        p, e, cm, rg = np.zeros(3 * self.N), np.zeros(Nc), np.zeros(3 * Nc), np.zeros(6 * Nc)
        self._call("bd_chain_props", p, e, cm, rg)
        return p.reshape(3, self.N), e, cm.reshape(Nc, 3), rg.reshape(Nc, 6)

    def write_trajectory(self, path, t):
        self._call("bd_write_trajectory", path.encode(), int(t))

    def write_restart(self, path, t):
        self._call("bd_write_restart", path.encode(), int(t))

    def write_ext(self, path, t, strain):
        self._call("bd_write_ext", path.encode(), int(t), float(strain))

    def write_visc(self, path, t, printperiod):
        self._call("bd_write_visc", path.encode(), int(t), int(printperiod))

    def ewald_bin(self):
        eps = C.c_double()
        rs = np.zeros(3 * self.N)
        self._call("bd_ewald_bin", C.byref(eps), rs)
        return eps.value, rs

    def catea(self, strain):
        b = C.c_double()
        self._call("bd_catea", float(strain), C.byref(b))
        return b.value

    def catea_averages(self, sbins=20):
        n = np.zeros(sbins + 1, np.int32)
        b = np.zeros(sbins + 1)
        Cc = np.zeros((sbins + 1) * 3 * self.p.Nb)
        self._call("bd_catea_averages", n, b, Cc)
        return n, b, Cc.reshape(sbins + 1, 3 * self.p.Nb)

    def write_decomp(self, path, t):
        self._call("bd_write_decomp", path.encode(), int(t))

    def catea_apply(self):
        self._call("bd_catea_apply")

    def enable_graphs(self, on=True):
        self._call("bd_enable_graphs", int(bool(on)))

    def set_charge_values(self, qk):
        self._call("bd_set_charge_values", np.ascontiguousarray(qk, np.float64))

    def coulomb_energy(self):
        o = np.zeros(4)
        self._call("bd_coulomb_energy", o)
        return dict(real=o[0], reciprocal=o[1], self=o[2], total=o[3])

    # Lanczos preconditioner
    PRECOND = {"none": 0, "segment": 1, "learned": 2, "blocks": 3}

    def set_preconditioner(self, kind, segment=0):
        self._call("bd_set_preconditioner", self.PRECOND[kind], int(segment))

    def set_precond_blocks(self, G9):
        self._call("bd_set_precond_blocks", np.ascontiguousarray(G9, np.float64).reshape(-1))

    def precond_blocks(self, S):
        n = (self.N // S) * 9 * S * S
        G, Gi, s = np.zeros(n), np.zeros(n), C.c_int()
        self._call("bd_download_precond_blocks", G, Gi, C.byref(s))
        assert s.value == S
        return G.reshape(self.N // S, 3 * S, 3 * S), Gi.reshape(self.N // S, 3 * S, 3 * S)

    def precond_stats(self):
        o = np.zeros(4, np.int64)
        self._call("bd_precond_stats", o)
        return dict(calls=int(o[0]), iterations=int(o[1]), fallbacks=int(o[2]),
                    identity_blocks=int(o[3]))

    def lanczos_inv_sqrt(self, z):
        out = np.zeros(3 * self.N)
        it = C.c_int()
        self._call("bd_lanczos_inv_sqrt", np.ascontiguousarray(z, np.float64), out, C.byref(it))
        return out, it.value

    # learned preconditioner network
    def mpnn_set_params(self, w):
        self._call("bd_mpnn_set_params", np.ascontiguousarray(w, np.float32))

    def mpnn_params(self):
        w = np.zeros(mpnn_param_count(), np.float32)
        self._call("bd_mpnn_get_params", w)
        return w

    def mpnn_features(self):
        self._call("bd_mpnn_features")

    def mpnn_predict(self):
        G = np.zeros(9 * self.N)
        self._call("bd_mpnn_predict", G)
        return G.reshape(self.N, 3, 3)

    def mpnn_loss_grad(self, z, t, want_grad=False):
        loss = C.c_double()
        g = np.zeros(mpnn_param_count(), np.float32) if want_grad else None
        self._call("bd_mpnn_loss_grad", np.ascontiguousarray(z, np.float64),
                   np.ascontiguousarray(t, np.float64), C.byref(loss),
                   g.ctypes.data_as(C.c_void_p) if want_grad else None)
        return (loss.value, g) if want_grad else loss.value

    def mpnn_adam(self, lr, step, beta1=0.9, beta2=0.999, eps=1e-8):
        self._call("bd_mpnn_adam", float(lr), float(beta1), float(beta2), float(eps), int(step))

    def profile(self, on=True):
        """True / 1: every event slot (noise-block products timed one by one,
        which runs the host-checked Krylov loop); 2: every slot but the
        block products (the device-checked loop); False: off."""
        self._call("bd_profile_enable", 2 if on == 2 else int(bool(on)))

    def set_device_krylov(self, on=True):
        self._call("bd_set_device_krylov", int(bool(on)))

    def krylov_check_stats(self):
        o = np.zeros(2, np.int64)
        self._call("bd_krylov_check_stats", o)
        return dict(device_solves=int(o[0]), host_fallbacks=int(o[1]))

    def profile_read(self, slot):
        ms, n = C.c_double(), C.c_long()
        self._call("bd_profile_read", int(slot), C.byref(ms), C.byref(n))
        return ms.value, n.value

    def launches(self) -> int:
        return int(self.L.bd_launch_count(self.h))

    def device_bytes(self) -> int:
        return int(self.L.bd_device_bytes(self.h))


for _n in ("apply_pbc", "transform_coords", "inverse_coords", "reset_force", "build_neighbors",
           "check_verlet", "bond_force", "ev_force", "coulomb_force", "get_noise", "calc_hi",
           "update_hi", "update_fd", "charge_hop"):
    setattr(Context, _n, (lambda name: lambda self: self._call("bd_" + name))(_n))


# ---------------------------------------------------------------------------
# synthetic inputs


def random_chains(Nb, Nc, L, seed, bond=2.0, min_sep=0.0, max_tries=200, max_restarts=200):
    """Seeded random-walk chains of bond length ``bond`` in a cubic box of edge L
    centred at the origin, returned as three float64 arrays (unwrapped along
    each chain).  With min_sep > 0 every bead keeps at least min_sep from all
    earlier beads under cubic periodicity: a bead is redrawn up to max_tries
    times, and a chain that gets stuck is regrown from a new start, as the
    reference's own initialiser does (shear/src/main26.c:398-474)."""
    rng = np.random.default_rng(seed)
    N = Nb * Nc
    r = np.zeros((N, 3))
    cell = max(min_sep, 1e-9)
    nc = max(1, int(np.floor(L / cell)))
    grid: dict = {}

    def key(p):
        q = np.floor((p - L * np.round(p / L) + L / 2) / L * nc).astype(int) % nc
        return int(q[0]), int(q[1]), int(q[2])

    def clear(p):
        if min_sep <= 0:
            return True
        kx, ky, kz = key(p)
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for b in grid.get(((kx + dx) % nc, (ky + dy) % nc, (kz + dz) % nc), ()):
                        d = r[b] - p
                        d -= L * np.round(d / L)
                        if d @ d < min_sep * min_sep:
                            return False
        return True

    for c in range(Nc):
        for _ in range(max_restarts):
            placed = []
            ok = True
            for b in range(Nb):
                a = c * Nb + b
                for _ in range(max_tries):
                    if b == 0:
                        p = rng.uniform(-L / 2, L / 2, 3)
                    else:
                        v = rng.normal(size=3)
                        p = r[a - 1] + bond * v / np.linalg.norm(v)
                    if clear(p):
                        break
                else:
                    ok = False
                    break
                r[a] = p
                grid.setdefault(key(p), []).append(a)
                placed.append(a)
            if ok:
                break
            for a in placed:
                grid[key(r[a])].remove(a)
        else:
            raise RuntimeError("could not place chain %d without overlaps" % c)
    return [np.ascontiguousarray(r[:, k]) for k in range(3)]


def lab_frame(flow, x, y):
    """Rotate chains generated in a cubic box into the lab frame of the flow.

    In extension the t = 0 cell is the cube rotated by theta = atan(L1y/L1x)
    = 31.7 degrees, so chains built with cubic periodicity are rotated by theta
    as the reference does after building them (extensional/src/main14.c:483-490).
    Shear needs no rotation."""
    if flow == FLOW_SHEAR:
        return x, y
    th = np.deg2rad(90.0 - (45.0 + 31.7))
    l1x, l1y = np.cos(th) + np.sin(th), -np.sin(th) + np.cos(th)
    t = np.arctan(l1y / l1x)
    c, s = np.cos(t), np.sin(t)
    return np.ascontiguousarray(x * c - y * s), np.ascontiguousarray(x * s + y * c)


def random_charges(Nb, Nc, frac, seed):
    """A seeded random subset of each chain's beads (frac of them) as bead indices."""
    rng = np.random.default_rng(seed)
    out = []
    k = int(round(frac * Nb))
    for c in range(Nc):
        out.extend(sorted(c * Nb + rng.choice(Nb, size=k, replace=False)))
    return np.array(out, np.int32)
