#!/usr/bin/env python
"""Benchmark: BSE time-to-spectrum of the B200 path on the synthetic plain-method workload.

One step = the whole BSE=T + SPEC=T path for one deck: bands on the k-mesh, velocities,
single-particle table, BSE kernel build, dense FP64 solve + oscillator strengths, and the
broadened eps(omega) of the BSE and single-particle spectra.

  value  device time of one step with the model resident in HBM (sum of the CUDA-event
         times of the stages, inputs already on the device), seconds (lower is better)
  e2e    the same step end to end through the deck-level C entry wtb_run (libwtbdriver.so):
         deck parse, params-file read, host->device model upload, every device stage, the
         device->host reads and all output files written
  roofline  the dominant kernel (the Hermitian matrix-vector product of the
         tridiagonalisation) timed per launch with CUDA events inside the timed steps
  cpu_baseline  the CPU oracle (numpy restatement of the reference, LAPACK ZHEEV with the
         reference's minimum workspace) on bounded samples of the same workload, scaled
  fast_form  the same deck's time-to-spectrum by the fast form (block Davidson on the
         split-BF16 tensor-core product with an FP64 polish to residual 1e-6 eV for the 32
         lowest excitons, Haydock recursion for eps(omega)), with its error against the plain
         FP64 step of the same run (lowest-32 energies in meV, eps2 at its peaks) and the
         roofline of the tensor-core product

Multi-GPU: the dense solve of one deck does not shard; --gpus N runs N independent
replicas (one per rank) and reports the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from wantibexos_b200 import synth, wtbgpu  # noqa: E402
from wantibexos_b200 import build as wbuild  # noqa: E402

WORKLOADS = {
    # name: (model, mesh n, nv, nc, r0, cshift, ebsef, nespec)
    "c2": dict(model="c2", n=48, nv=4, nc=4, r0=30.0, cshift=0.03, ebsef=6.0, nespec=2001,
               desc="config 2: w=24, 91 cells, 48x48x1 mesh, nv=nc=4, N=36864, V2DRK r0=30, eps 0-6 eV x2001"),
    "c5": dict(model="c4_w16", n=60, nv=2, nc=2, r0=35.0, cshift=0.03, ebsef=6.0, nespec=2001,
               desc="config 5 size: w=16, 61 cells, 60x60x1 mesh, nv=nc=2, N=14400, V2DRK r0=35"),
    "c1": dict(model="c1", n=12, nv=2, nc=2, r0=40.0, cshift=0.05, ebsef=5.0, nespec=1001,
               desc="config 1: w=8, 37 cells, 12x12x1 mesh, nv=nc=2, N=576, V2DRK r0=40, eps 0-5 eV x1001"),
    # smaller meshes of the config-2 model, for profiling captures
    "c2s": dict(model="c2", n=12, nv=4, nc=4, r0=30.0, cshift=0.03, ebsef=6.0, nespec=2001,
                desc="config-2 model on a 12x12x1 mesh, nv=nc=4, N=2304"),
    "c2m": dict(model="c2", n=24, nv=4, nc=4, r0=30.0, cshift=0.03, ebsef=6.0, nespec=2001,
                desc="config-2 model on a 24x24x1 mesh, nv=nc=4, N=9216"),
}

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")


def deck_text(wl, workdir, extra=""):
    return f"""{extra}BSE= T
SPEC= T
NGX= {wl['n']}
NGY= {wl['n']}
NGZ= 1
NBANDSV= {wl['nv']}
NBANDSC= {wl['nc']}
COULOMB_POT= V2DRK
R_0= {wl['r0']}
EDIEL_T= 1
EDIEL= 1
EDIEL_B= 1
EDIEL_Z= 1
W_COUL= 0
LC= 1
KTOL= 0.001
CSHIFT= {wl['cshift']}
ENSPECI= 0
ENSPECF= {wl['ebsef']}
NESPEC= {wl['nespec']}
DTDIAG= F
CPOL= F
RNMD= T
SYSDIM= "2D"
OUTPUT= "{workdir}/"
CALC_DATA= "{workdir}/"
PARAMS_FILE= "{workdir}/tb_synthetic.dat"
"""


# ----------------------------------------------------------------------------- host helpers
def recvec(rlat):
    pi32 = float(np.float32(np.pi))
    a1, a2, a3 = rlat
    v23, v31, v12 = np.cross(a2, a3), np.cross(a3, a1), np.cross(a1, a2)
    vol = abs(a1 @ v23)
    s = (2.0 * pi32) / vol
    return s * v23, s * v31, s * v12


def kmesh(n, rlat):
    b1, b2, b3 = recvec(rlat)
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    k = (b1[None, None, :] / n) * i[..., None] + (b2[None, None, :] / n) * j[..., None]
    return k.reshape(-1, 3)


def vcell3d(rlat):
    return abs(np.cross(rlat[0], rlat[1]) @ rlat[2])


def f154(x):
    """The value read back from an F15.4 field (the reference's file round trip)."""
    return np.array([float(f"{v:15.4f}") for v in np.ravel(x)]).reshape(np.shape(x))


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        if shutil.which("nvidia-smi") is None:
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                      "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        loaded = sorted(sm)[len(sm) // 2:] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons), "samples": len(rows)}


# ----------------------------------------------------------------------------- device step
def device_step(ctx, model, kpt, wl, c, keep=None):
    """One step with the model resident; returns device seconds per stage (and, when `keep`
    is a dict, stores the lowest 32 exciton energies and the BSE eps2_xx there)."""
    t = {}
    ctx.bands(kpt, wl["nv"], wl["nc"], want_vectors=False)
    t["bands"] = ctx.last_ms
    h = ctx.velocity(wl["cshift"], want=False)
    t["velocity"] = ctx.last_ms
    sp = ctx.sp_table()
    t["sp_table"] = ctx.last_ms
    ctx.bse_build(c)
    t["build"] = ctx.last_ms
    W, act = ctx.bse_solve(False, False)
    t["solve"] = ctx.last_ms
    E = f154(W)
    F = f154(act[:, :6])
    ng = [wl["n"], wl["n"], 1]
    _, eps = ctx.spectrum(E, F, ng, vcell3d(model.rlat), 0.0, wl["ebsef"], float(wl["nespec"]), wl["cshift"], True,
                          2.0)
    t["spectrum_bse"] = ctx.last_ms
    if keep is not None:
        keep["W32"] = W[:32].copy()
        keep["eps2"] = eps[:, 1, 0].astype(np.float64)
    Es = f154(sp[:, 6].astype(np.float64))
    Fs = f154(sp[:, 7:13].astype(np.float64))
    ctx.spectrum(Es, Fs, ng, vcell3d(model.rlat), 0.0, wl["ebsef"], float(wl["nespec"]), wl["cshift"], True, 2.0)
    t["spectrum_sp"] = ctx.last_ms
    return {k: v / 1e3 for k, v in t.items()}


def fast_step(ctx, model, kpt, wl, c):
    """The fast form of the same step: bands, velocities, build, block Davidson for the 32
    lowest excitons (tensor-core product, FP64 polish to residual 1e-6 eV), the highest
    exciton (residual 1e-3 eV, it only sets the broadening rule), and eps(omega) by the Haydock
    recursion (150 steps). Returns (device seconds per stage, W32, eps2_xx, Davidson stats)."""
    t = {}
    ctx.bands(kpt, wl["nv"], wl["nc"], want_vectors=False)
    t["bands"] = ctx.last_ms
    ctx.velocity(wl["cshift"], want=False)
    t["velocity"] = ctx.last_ms
    ctx.bse_build(c)
    t["build"] = ctx.last_ms
    ctx.set_fast_product(1)
    try:
        W, _, _, it, res = ctx.bse_davidson(32, nb=40, tol=1e-6, want_act=False)
        t["davidson"] = ctx.last_ms
        st = ctx.stats()
        dav = {"iters": it, "tensor_core_iters": st["dav_fast_iters"], "fp64_iters": st["dav_fp64_iters"],
               "max_residual_eV": res}
        top = ctx.bse_davidson(1, nb=8, largest=True, tol=1e-3, want_act=False)[0][0]
        t["davidson_top"] = ctx.last_ms
        _, eps = ctx.bse_spectrum_fast(150, W[0], top, [wl["n"], wl["n"], 1], vcell3d(model.rlat), 0.0, wl["ebsef"],
                                       float(wl["nespec"]), wl["cshift"], True, 2.0)
        t["haydock"] = ctx.last_ms
    finally:
        ctx.set_fast_product(0)
    return {k: v / 1e3 for k, v in t.items()}, W, eps[:, 1, 0].astype(np.float64), dav


def config4_leg(device=0):
    """Config-4 exciton band structure: w = 16 model, 30x30 mesh, nv = nc = 3 (N = 8100), 64 Q on
    Gamma-M-K-Gamma (22 points per segment with the float32 fraction of kpathbse, the two repeated
    junction points dropped), V2DRK r0 = 35 A, eps_env = 2.5, all Q in one wtbg_bse_q_batch call
    (after one sizing call on the first Q)."""
    model = synth.config_model("c4_w16")
    n, nv, nc, npts = 30, 3, 3, 22
    b1, b2, b3 = recvec(model.rlat)
    nodes = [(0, 0, 0), (0.5, 0, 0), (0.5, 0, 0), (1 / 3, 1 / 3, 0), (1 / 3, 1 / 3, 0), (0, 0, 0)]
    cart = [u[0] * b1 + u[1] * b2 + u[2] * b3 for u in nodes]
    qs = []
    for j in range(3):
        for i in range(npts):
            if j > 0 and i == 0:
                continue
            t = float(np.float32(i) / np.float32(npts - 1))
            q = cart[2 * j] + (cart[2 * j + 1] - cart[2 * j]) * t
            qs.append([0.0, q[0], q[1], q[2]])
    qs = np.array(qs)
    k = kmesh(n, model.rlat)
    kqs = [k + q[1:][None, :] for q in qs]
    c = wtbgpu.coulomb_params("V2DRK", [n, n, 1], 1e-3, [2.5] * 3, 1.0, 1.0, 0.0, 35.0)
    ctx = wtbgpu.Context(device)
    ctx.set_model(model)
    ctx.bands(k, nv, nc, want_vectors=False)
    ctx.bse_q_batch(kqs[:1], qs[:1], c, graph=False)
    t0 = time.perf_counter()
    W, ms = ctx.bse_q_batch(kqs, qs, c, graph=False)
    wall = time.perf_counter() - t0
    ctx.close()
    return {"workload": "config 4: w=16, 61 cells, 30x30 mesh, nv=nc=3, N=8100, 64 Q on Gamma-M-K-Gamma, "
                        "V2DRK r0=35, eps_env=2.5", "n_q": int(qs.shape[0]), "N": int(W.shape[1]),
            "device_s": float(ms.sum() / 1e3), "ms_per_q": float(ms.sum() / qs.shape[0]), "wall_s": wall,
            "lowest_exciton_eV": [float(W[:, 0].min()), float(W[:, 0].max())]}


def learned_leg(device=0, evaluated=16, judged=4):
    """Config-5 learned warm start, bounded for the bench: w = 16 model, 60x60 mesh, nv = nc = 2
    (N = 14400), 256 seeded (Q, r0, eps_env) points, the network trained on the first 192 against
    the 32 lowest block-Davidson eigenvectors (residual 1e-6 eV), then on `evaluated` held-out
    points cold start against learned start (iterations and device ms to residual 1e-6 eV, FP64
    and tensor-core products), the first `judged` of them checked against the dense FP64 solve."""
    from wantibexos_b200 import warmstart_sweep as ws
    a = ws.parser().parse_args(["--model", "c4_w16", "--n", "60", "--points", "256", "--train", "192",
                                "--targets", "davidson", "--eval", str(evaluated), "--judge", str(judged)])
    t0 = time.perf_counter()
    summ = ws.sweep(a, device)
    mi, ms = summ["mean_iters"], summ["mean_ms"]
    return {"protocol": "256 points (Q <= 0.05 b, r0 in [10, 60] A, eps_env in [1, 5]), 192 trained, "
                        f"{evaluated} held out evaluated, {judged} judged by the dense FP64 solve",
            "N": summ["N"], "heldout_loss_before_after": summ["heldout_loss"],
            "mean_capture_learned": summ["mean_capture_learned"], "mean_iters": mi, "mean_device_ms": ms,
            "gain_fp64_product": 1.0 - ms["fp64_learned"] / ms["fp64_cold"],
            "gain_tensor_core_product": 1.0 - ms["fast_learned"] / ms["fast_cold"],
            "max_final_err_meV_vs_dense": summ["max_final_err_meV"], "wall_s": time.perf_counter() - t0}


def peak_rel_error(ref, x):
    """max |x - ref| at the local maxima of ref, relative to max |ref|."""
    pk = np.where((ref[1:-1] > ref[:-2]) & (ref[1:-1] >= ref[2:]))[0] + 1
    if len(pk) == 0:
        pk = np.array([int(np.argmax(ref))])
    return float(np.abs(x[pk] - ref[pk]).max() / np.abs(ref).max())


FAST_DECK = "GPU_SOLVER= DAVIDSON\nGPU_PRECISION= BF16X3\nGPU_NEV= 32\nGPU_TOL= 1e-6\n"


def e2e_run(workdir, wl, device=0, extra=""):
    lib = C.CDLL(wbuild.DRIVER_LIB)

    class Timings(C.Structure):
        _fields_ = [(n, C.c_double) for n in ("bands", "sp", "build", "solve", "write_opt", "spectrum", "total")]

    lib.wtb_run.restype = C.c_int
    lib.wtb_run.argtypes = [C.c_char_p, C.c_int, C.POINTER(Timings), C.c_char_p, C.c_int]
    tm = Timings()
    err = C.create_string_buffer(1024)
    t0 = time.perf_counter()
    rc = lib.wtb_run(deck_text(wl, workdir, extra).encode(), device, C.byref(tm), err, 1024)
    t1 = time.perf_counter()
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return t1 - t0, {n: getattr(tm, n) for n, _ in Timings._fields_}


# ----------------------------------------------------------------------------- CPU baseline
ZHEEV_FIT_SIZES = (1152, 1536, 2304)


def zheev_fit(sizes=ZHEEV_FIT_SIZES, seed=0):
    """Dense ZHEEV('V','U') with the reference's minimum workspace (LWORK = 2N-1) timed at a few
    sizes on the host cores: the least-squares N^3 coefficient (weighted to the largest sizes,
    where the matrix no longer fits in cache) and the free power-law fit with its R^2."""
    import scipy.linalg.lapack as lapack
    rng = np.random.default_rng(seed)
    ts = []
    for n in sizes:
        X = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        H = np.asfortranarray(X + X.conj().T)
        t0 = time.perf_counter()
        lapack.zheev(H, compute_v=1, lower=0, lwork=max(2 * n - 1, 1))
        ts.append(time.perf_counter() - t0)
    n3 = np.array(sizes, dtype=float) ** 3
    t = np.array(ts)
    coef = float((t * n3).sum() / (n3 * n3).sum())
    lx, ly = np.log(np.array(sizes, dtype=float)), np.log(t)
    p, c0 = np.polyfit(lx, ly, 1)
    pred = p * lx + c0
    r2 = float(1.0 - ((ly - pred) ** 2).sum() / max(((ly - ly.mean()) ** 2).sum(), 1e-300))
    return {"sizes": list(sizes), "seconds": [float(x) for x in ts], "coef_n3": coef,
            "power_law_exponent": float(p), "power_law_r2": r2}


def c1_full_run(repeats=5):
    """The oracle port's whole config-1 run (bands, velocities, build, ZHEEV, oscillators,
    bsedielraw), median of `repeats` runs: a full measurement, nothing extrapolated."""
    from oracle import wtb_oracle as O
    from oracle.deck import parse_deck
    wl = WORKLOADS["c1"]
    m = synth.config_model("c1")
    d = parse_deck(deck_text(wl, ".").replace('OUTPUT= "./"', "").replace('CALC_DATA= "./"', ""))
    ts = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        r = O.run_bse(m, d)
        E = O.roundtrip_f154(r["W"])
        F = O.roundtrip_f154(r["act"][:, :6])
        O.bsedielraw(m.systype, m.rlat, r["ngrid"], E, F, d["ebse0"], d["ebsef"], d["numbse"], d["cshift"], True)
        ts.append(time.perf_counter() - t0)
    return float(np.median(ts))


def cpu_baseline(wl, model, fit=None):
    """Time the CPU oracle on bounded samples of the workload and scale to the full step; the
    dense ZHEEV comes from `fit` (zheev_fit), measured once per run."""
    from oracle import wtb_oracle as O
    n = wl["n"]
    nk = n * n
    nv, nc = wl["nv"], wl["nc"]
    N = nk * nc * nv
    kpts = O.monkhorst_pack(n, n, 1, [0, 0, 0], model.rlat)
    parts = {}
    # bands: eigsys on a sample of k-points
    ks = min(nk, 48)
    t0 = time.perf_counter()
    eigv, vec, nocp, _ = O.bands(model, kpts[:ks], nv, nc)
    parts["bands"] = (time.perf_counter() - t0) * nk / ks
    # velocities: the reference recomputes hlm for every (c, v, k) state
    t0 = time.perf_counter()
    O.optsp_all(model, kpts[:8], eigv[:8], vec[:8], nv, nc, wl["cshift"])
    parts["velocity"] = (time.perf_counter() - t0) * nk / 8 * 1.0
    # BSE build: a block of rows against all columns, scaled to the upper triangle
    kb = min(nk, 64)
    eig_all, vec_all, _, _ = O.bands(model, kpts[:kb], nv, nc)
    p = O.CoulombParams("V2DRK", 1e-3, [1, 1, 1], 1.0, 1.0, 0.0, wl["r0"], [n, n, 1], model.rlat)
    t0 = time.perf_counter()
    O.bse_matrix(p, kpts[:kb], eig_all, vec_all, nv, nc)
    tb = time.perf_counter() - t0
    parts["build"] = tb * (N / (kb * nc * nv)) ** 2
    # dense ZHEEV (minimum workspace): N^3 law fitted at a few sizes (measured at N itself when
    # N is not above them)
    rng = np.random.default_rng(0)
    if fit is None:
        fit = zheev_fit(sizes=(N,) if N <= ZHEEV_FIT_SIZES[-1] else ZHEEV_FIT_SIZES)
    parts["zheev"] = fit["coef_n3"] * N ** 3
    # oscillators: N^2 complex MACs per component (3 components), from a sample
    s = min(N, 1152)
    A = np.asfortranarray(rng.standard_normal((s, s)) + 1j * rng.standard_normal((s, s)))
    hv = rng.standard_normal(s) + 1j * rng.standard_normal(s)
    t0 = time.perf_counter()
    for _ in range(3):
        O.dielbsev(A, hv)
    parts["oscillators"] = (time.perf_counter() - t0) * (N / s) ** 2
    # spectrum: a slice of the photon grid, scaled (BSE + SP spectra)
    E = np.sort(rng.uniform(0.5, 6, N))
    F = rng.uniform(0, 1, (N, 6))
    om = O.omega_grid(0.0, wl["ebsef"], float(wl["nespec"]))[:50]
    t0 = time.perf_counter()
    for c in range(6):
        O.optdiel_grid(1, vcell3d(model.rlat), [n, n, 1], om, E, F[:, c], wl["cshift"])
    parts["spectrum"] = 2 * (time.perf_counter() - t0) * wl["nespec"] / 50
    total = sum(parts.values())
    return total, parts, fit


# ----------------------------------------------------------------------------- main
def solve_breakdown(st, nsteps):
    """Per-step CUDA-event times of the dense solve's parts (profiling mode): the mat-vec, the
    trailing rank-2k updates (with their FP64 tensor rate against the nominal 40 TFLOP/s: no
    measured FP64 peak exists for this GPU), the rest of the reduction (column kernels), and
    the tridiagonal eigenvalues + oscillators."""
    if not st["tri_ms"]:
        return None
    her2k_tf = st["her2k_flops"] / (st["her2k_ms"] / 1e3) / 1e12 if st["her2k_ms"] else None
    if st.get("stage1_ms"):
        hemm_tf = st["hemm_flops"] / (st["hemm_ms"] / 1e3) / 1e12 if st["hemm_ms"] else None
        return {"reduction": "two-stage", "tridiagonalise": st["tri_ms"] / 1e3 / nsteps,
                "stage1_dense_to_band": st["stage1_ms"] / 1e3 / nsteps,
                "panel_qr": st["panel_ms"] / 1e3 / nsteps,
                "hemm": st["hemm_ms"] / 1e3 / nsteps, "hemm_tflops": hemm_tf,
                "her2k": st["her2k_ms"] / 1e3 / nsteps, "her2k_tflops": her2k_tf,
                "stage1_other": (st["stage1_ms"] - st["panel_ms"] - st["hemm_ms"] - st["her2k_ms"]) / 1e3 / nsteps,
                "stage2_band_to_tridiagonal": st["stage2_ms"] / 1e3 / nsteps,
                "tridiagonal_solve": st["tdsolve_ms"] / 1e3 / nsteps}
    return {"tridiagonalise": st["tri_ms"] / 1e3 / nsteps, "hemv": st["hemv_ms"] / 1e3 / nsteps,
            "her2k": st["her2k_ms"] / 1e3 / nsteps,
            "column_kernels_and_gaps": (st["tri_ms"] - st["hemv_ms"] - st["her2k_ms"]) / 1e3 / nsteps,
            "tridiagonal_solve": st["tdsolve_ms"] / 1e3 / nsteps,
            "her2k_tflops": her2k_tf, "her2k_frac_of_nominal_fp64_40": (her2k_tf / 40.0) if her2k_tf else None}


def dgemm_peak(device=0, n=8192, reps=5):
    """cuBLAS DGEMM rate on this GPU in this run (torch.matmul float64, n^3, best of reps, CUDA
    events): the FP64 tensor-core denominator (the measured-peaks file has no FP64 figure)."""
    import torch
    dev = torch.device("cuda", device)
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    best = 1e30
    for i in range(reps + 1):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        if i > 0:
            best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best / 1e3) / 1e12


def max_over_ranks(values, dist):
    """Element-wise max of per-rank timings over the process group (the whole job ends when
    its slowest replica ends)."""
    import torch
    tt = torch.tensor(list(values), dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return [float(x) for x in tt]


def ncu_launch_summary(path: str) -> str:
    """Per-kernel launches, total device time and share from an ncu CSV launch list
    (``ncu --metrics gpu__time_duration.sum --csv --log-file path``)."""
    import csv
    import collections
    scale = {"nsecond": 1e-6, "ns": 1e-6, "usecond": 1e-3, "us": 1e-3, "msecond": 1.0, "ms": 1.0, "second": 1e3, "s": 1e3}
    agg = collections.OrderedDict()
    hdr = None
    with open(path, newline="") as f:
        for r in csv.reader(f):
            if r and r[0] == "ID":
                hdr = r
                continue
            if hdr is None or len(r) != len(hdr):
                continue
            d = dict(zip(hdr, r))
            if d.get("Metric Name") != "gpu__time_duration.sum":
                continue
            name = d["Kernel Name"].split("(")[0].replace("void ", "").replace("<unnamed>::", "")
            ms = float(d["Metric Value"].replace(",", "")) * scale.get(d.get("Metric Unit", "ns"), 1e-6)
            a = agg.setdefault(name, [0, 0.0])
            a[0] += 1
            a[1] += ms
    tot = sum(a[1] for a in agg.values())
    lines = [f"{'kernel':48s} {'launches':>9s} {'total ms':>11s} {'avg us':>10s} {'share':>7s}"]
    for name, (n, t) in sorted(agg.items(), key=lambda x: -x[1][1]):
        lines.append(f"{name[:48]:48s} {n:9d} {t:11.3f} {1e3 * t / n:10.1f} {100 * t / max(tot, 1e-30):6.2f}%")
    lines.append(f"{'total':48s} {sum(a[0] for a in agg.values()):9d} {tot:11.3f}")
    return "\n".join(lines)


def main():
    if len(sys.argv) == 3 and sys.argv[1] == "--ncu-summary":
        print(ncu_launch_summary(sys.argv[2]))
        return
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=os.environ.get("WTB_BENCH_WORKLOAD", "c2"), choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--form", default="both", choices=["both", "plain", "fast"],
                    help="plain FP64 path (the headline), the fast form, or both (default)")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned warm-start and config-4 legs")
    ap.add_argument("--reduction", default="auto", choices=["auto", "one", "two", "two-warp"],
                    help="tridiagonal reduction of the dense solve: automatic (two-stage for N >= 2048), "
                         "one-stage or two-stage")
    ap.add_argument("--device-only", action="store_true",
                    help="only the device-resident steps (no e2e run, no CPU baseline): profiling captures")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist  # plumbing only: barrier + max over ranks
        dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=1800))

    metric = "BSE time-to-spectrum (s) at <=0.5 meV vs FP64"
    unit = "s"
    cfg = {"workload": wl["desc"], "nk": wl["n"] ** 2, "N_bse": wl["n"] ** 2 * wl["nv"] * wl["nc"],
           "precision": "fp64 plain method", "parallelism": f"replicas{args.gpus}",
           "l2": "inputs larger than L2 (BSE matrix %.1f GB)" % ((wl["n"] ** 2 * wl["nv"] * wl["nc"]) ** 2 * 16 / 1e9)}
    model = synth.config_model(wl["model"])

    if args.impl == "reference":
        if rank != 0:
            return
        cores = os.cpu_count()
        vals = []
        N = cfg["N_bse"]
        fit = zheev_fit(sizes=(N,) if N <= ZHEEV_FIT_SIZES[-1] else ZHEEV_FIT_SIZES)
        for _ in range(args.warmup):
            cpu_baseline(wl, model, fit)
        parts = None
        for _ in range(max(1, args.steps)):
            v, parts, _ = cpu_baseline(wl, model, fit)
            vals.append(v)
        val = float(np.median(vals))
        parts = dict(parts, zheev_fit=fit)
        sample = (f"oracle port (numpy restatement, vectorised per stage: the reference is Fortran and no "
                  f"Fortran compiler exists on these machines) on samples: bands 48 k-points, velocities 8 "
                  f"k-points, BSE build 64 k-point row/column block, oscillators, spectrum 50 photon energies, "
                  f"each scaled to the full workload (N^2 for build/oscillators); ZHEEV(lwork=2N-1, scipy "
                  f"OpenBLAS) timed once at N={fit['sizes']} and scaled by the least-squares N^3 law "
                  f"(free power-law exponent {fit['power_law_exponent']:.2f}, R^2 {fit['power_law_r2']:.4f})")
        print(json.dumps({"impl": "reference", "metric": metric, "value": val, "unit": unit, "n_gpus": args.gpus,
                          "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
                          "cpu_baseline": {"value": val, "unit": unit, "cores": cores, "kind": "port",
                                           "sample": sample, "parts_s": parts},
                          "e2e": {"value": val, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    wbuild.build()
    ctx = wtbgpu.Context(local)   # one replica per GPU (LOCAL_RANK)
    ctx.set_reduction({"auto": 0, "one": 1, "two": 2, "two-warp": 3}[args.reduction])
    ctx.set_model(model)
    kpt = kmesh(wl["n"], model.rlat)
    c = wtbgpu.coulomb_params("V2DRK", [wl["n"], wl["n"], 1], 1e-3, [1, 1, 1], 1.0, 1.0, 0.0, wl["r0"])
    for _ in range(args.warmup if args.form != "fast" else 0):
        device_step(ctx, model, kpt, wl, c)
    if dist:
        dist.barrier()
    clocks = Clocks(local)
    clocks.start()
    ctx.reset_stats()
    ctx.set_profiling(True)
    steps = []
    keep = {}
    if args.form != "fast":
        for _ in range(args.steps):
            steps.append(device_step(ctx, model, kpt, wl, c, keep))
    ctx.set_profiling(False)
    st = ctx.stats()
    ck = clocks.stop()
    per_step = [sum(s.values()) for s in steps] or [float("nan")]
    t_dev = float(np.mean(per_step))
    fast = None
    if args.form != "plain":
        # fast form: untimed warm-up steps, then the timed steps with the product timed per launch
        for _ in range(max(1, args.warmup)):
            fast_step(ctx, model, kpt, wl, c)
        ctx.reset_stats()
        ctx.set_profiling(True)
        fsteps = []
        for _ in range(args.steps):
            fsteps.append(fast_step(ctx, model, kpt, wl, c))
        ctx.set_profiling(False)
        fst = ctx.stats()
        t_fast = float(np.mean([sum(s[0].values()) for s in fsteps]))
        _, W32, eps2, dav = fsteps[-1]
        hbm = float(json.load(open(PEAKS_PATH)).get("hbm_gbs", 6650.0)) if os.path.exists(PEAKS_PATH) else 6650.0
        fgbs = fst["fast_bytes"] / (fst["fast_ms"] / 1e3) / 1e9 if fst["fast_ms"] > 0 else None
        fast = {"time_to_spectrum_s": t_fast, "stages_s": fsteps[-1][0], "davidson": dav,
                "gpu_launches": int(fst["launches"] / max(1, args.steps)),
                "roofline": {"kernel": "split-BF16 tensor-core product Y = H X (k_fastprod)", "bound": "hbm",
                             "achieved": fgbs, "peak": hbm, "unit": "GB/s", "frac": (fgbs / hbm) if fgbs else None,
                             "algorithmic_bytes": "8 B x N^2 per product (bf16 hi/lo planes of Re H and Im H)",
                             # 1.05 x algorithmic in the ncu capture at N = 9216 (X planes, FP64 sums)
                             "traffic": 1.05 * fst["fast_bytes"] / max(1, fst["fast_launches"]),
                             "launches": fst["fast_launches"],
                             "avg_launch_ms": fst["fast_ms"] / max(1, fst["fast_launches"])}}
        if keep:
            fast["speedup_vs_plain_fp64"] = t_dev / t_fast
            fast["dW32_meV"] = float(np.abs(W32 - keep["W32"]).max() * 1e3)
            fast["eps2_peak_rel_err"] = peak_rel_error(keep["eps2"], eps2)
    ctx.close()
    if args.device_only:
        print(json.dumps({"metric": metric, "value": t_dev, "unit": unit, "stages_s": steps[-1] if steps else None,
                          "solve_breakdown_s": solve_breakdown(st, max(1, len(steps))),
                          "hemv_gbs": (st["hemv_bytes"] / (st["hemv_ms"] / 1e3) / 1e9) if st["hemv_ms"] else None,
                          "fast_form": fast, "config": cfg, "device_only": True}))
        return
    # e2e through the deck-level C entry (host buffers, files)
    workdir = tempfile.mkdtemp(prefix="wtb_bench_")
    synth.write_params(model, os.path.join(workdir, "tb_synthetic.dat"))
    e2e_times = []
    e2e_parts = None
    for _ in range(max(1, min(args.steps, 2))):
        t, e2e_parts = e2e_run(workdir, wl, local)
        e2e_times.append(t)
    t_e2e = float(np.mean(e2e_times))
    fast_e2e = None
    if fast is not None:
        # the fast form end to end: the same deck with GPU_SOLVER= DAVIDSON, GPU_PRECISION= BF16X3
        fe = []
        fparts = None
        for _ in range(max(1, min(args.steps, 2))):
            t, fparts = e2e_run(workdir, wl, local, FAST_DECK)
            fe.append(t)
        fast_e2e = {"value": float(np.mean(fe)), "unit": unit, "stages_s": fparts,
                    "path": "wtb_run with GPU_SOLVER= DAVIDSON, GPU_PRECISION= BF16X3 (files written; eps from the "
                            "Haydock recursion, bse_opt_diel.dat with the 32 lowest excitons)"}
        fast["e2e"] = fast_e2e
    shutil.rmtree(workdir, ignore_errors=True)
    if dist:
        t_dev, t_e2e = max_over_ranks([t_dev, t_e2e], dist)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    peaks = json.load(open(PEAKS_PATH)) if os.path.exists(PEAKS_PATH) else {}
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    hemv_gbs = st["hemv_bytes"] / (st["hemv_ms"] / 1e3) / 1e9 if st["hemv_ms"] > 0 else None
    build_gbs = st["build_bytes"] / (st["build_ms"] / 1e3) / 1e9 if st["build_ms"] > 0 else None
    N = cfg["N_bse"]
    nk = cfg["nk"]
    build_rf = {"achieved": build_gbs, "frac": (build_gbs / hbm) if build_gbs else None,
                "algorithmic_bytes": "16 B x N(N+1)/2 (lower triangle written once)"}
    if st.get("stage1_ms"):
        # two-stage reduction: the dominant kernels are the FP64 tensor-core products of stage 1
        dg = dgemm_peak(local)
        fl = st["hemm_flops"] + st["her2k_flops"]
        ms = st["hemm_ms"] + st["her2k_ms"]
        tf = fl / (ms / 1e3) / 1e12 if ms > 0 else None
        nl = 2 * st["her2k_launches"]
        roofline = {"kernel": "two-stage reduction, stage-1 FP64 tensor-core products (k_hemm2: X = A22 V; "
                              "k_her2k: A22 -= V W^H + W V^H; mma.sync m16n8k16 f64)",
                    "bound": "tensor", "achieved": tf, "peak": dg, "unit": "TFLOP/s",
                    "frac": (tf / dg) if tf else None,
                    "peak_source": "measured in this run: cuBLAS DGEMM (torch.matmul float64, 8192^3, best of 5); "
                                   "the measured-peaks file holds no FP64 figure",
                    "traffic": None,
                    "algorithmic_flops": "per panel (m = trailing order, 32 columns): 8 m^2 32 (k_hemm2) + "
                                         "16 m(m+1)/2 32 (k_her2k)",
                    "launches": nl, "avg_launch_ms": ms / max(1, nl),
                    "per_kernel": {"k_hemm2_tflops": (st["hemm_flops"] / (st["hemm_ms"] / 1e3) / 1e12)
                                   if st["hemm_ms"] else None,
                                   "k_her2k_tflops": (st["her2k_flops"] / (st["her2k_ms"] / 1e3) / 1e12)
                                   if st["her2k_ms"] else None},
                    "build_kernel": build_rf}
    else:
        roofline = {"kernel": "tridiagonalisation Hermitian mat-vec (k_hemv)", "bound": "hbm",
                    "achieved": hemv_gbs, "peak": hbm, "unit": "GB/s",
                    "frac": (hemv_gbs / hbm) if hemv_gbs else None,
                    # DRAM bytes per launch: 1.05 x the algorithmic bytes in the ncu capture of
                    # k_hemv at N = 9216 (read + write, three launches), scaled to the mean launch
                    "traffic": (1.05 * st["hemv_bytes"] / st["hemv_launches"]) if st["hemv_launches"] else None,
                    "peak_source": "measured" if peaks else "fallback",
                    "algorithmic_bytes": "16 B x (n'(n'+1)/2) per launch, n' = trailing order",
                    "launches": st["hemv_launches"], "avg_launch_ms": st["hemv_ms"] / max(1, st["hemv_launches"]),
                    "build_kernel": build_rf}
    out = {
        "metric": metric, "value": t_dev, "unit": unit, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_dev * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded hexagonal Wannier model)",
        "config": cfg,
        "stages_s": {k: float(np.mean([s[k] for s in steps])) for k in steps[0]},
        "e2e": {"value": t_e2e, "unit": unit,
                "h2d_bytes_per_step": int(model.hre.size * 16 + model.rvec.size * 4 + nk * 24 + N * 7 * 8 * 2),
                "d2h_bytes_per_step": int(nk * (wl["nv"] + wl["nc"]) * 8 + N * 5 * 16 + N * 15 * 4 + N * 8 * 9
                                          + wl["nespec"] * (8 + 48) * 2),
                "stages_s": e2e_parts, "path": "wtb_run (libwtbdriver.so) -> libwtbgpu.so C-ABI, files written"},
        "roofline": roofline,
        "solve_breakdown_s": solve_breakdown(st, max(1, len(steps))),
        "gpu_launches": int(st["launches"] / max(1, args.steps)),
        "clocks": ck,
        "fast_form": fast,
    }
    if not args.no_learned and args.form != "plain":
        out["learned_warm_start"] = learned_leg(local)
    if not args.no_learned:
        out["config4_q_batch"] = config4_leg(local)
    if not args.no_cpu_baseline:
        fit = zheev_fit(sizes=(N,) if N <= ZHEEV_FIT_SIZES[-1] else ZHEEV_FIT_SIZES)
        v, parts, _ = cpu_baseline(wl, model, fit)
        out["cpu_baseline"] = {"value": v, "unit": unit, "cores": os.cpu_count(), "kind": "port",
                               "sample": f"oracle port (numpy restatement, vectorised per stage; the reference is "
                                         f"Fortran and cannot be compiled here) on samples (bands 48 k, velocity 8 k, "
                                         f"build 64-k block, oscillators, 50 photon energies) scaled to the full "
                                         f"workload; ZHEEV(lwork=2N-1) timed at N={fit['sizes']}, N^3 law "
                                         f"(power-law exponent {fit['power_law_exponent']:.2f}, "
                                         f"R^2 {fit['power_law_r2']:.4f})",
                               "parts_s": dict(parts, zheev_fit=fit),
                               "c1_full_run_s": c1_full_run(),
                               "c1_full_run_note": "config 1 (N = 576) run in full by the oracle port, median of 5"}
    print(json.dumps(out))
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
