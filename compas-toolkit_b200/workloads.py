"""Seeded synthetic workloads for the compas-toolkit simulation hot path.

The reference quotes no public dataset (its examples use Shepp-Logan phantoms
from ImagePhantoms.jl, not vendored); these generators stand in for it with the
shapes, sizes and value distributions of the five benchmark configurations:

* ``fisp_small``     – 64×64 voxels, FISP 400 TRs, 8 EPG states, 1 slice
  position, 1 unit coil, Cartesian 400×64 (the reference's CPU-runnable case).
* ``mrstat``         – 224×224 voxels, FISP 1120 TRs, 25 states, 35 slice
  positions, 4 Gaussian-bump coils, Cartesian 1120×224 (MR-STAT scale).
* ``jacobian``       – as ``mrstat`` with 8 coils, random v [4][V] and residual
  r [8][1120][224] drawn from CN(0,1).
* ``pssfp_job`` / ``spiral_traj`` – pSSFP sequences (Gaussian RF of n_RF
  samples, 35 z positions) and variable-density Archimedean spirals used by
  the batched and served workloads.

All arrays use the reference's C++ layouts: tissue float32 [9][V] in the order
T1, T2, B1, B0, rho_x, rho_y, x, y, z; complex64 echos [R][V]; coils [C][V].
Times are seconds, B0 in Hz, positions in cm, RF in degrees.
"""
from __future__ import annotations

import math

import numpy as np

FIELDS = ("T1", "T2", "B1", "B0", "rho_x", "rho_y", "x", "y", "z")


def tissue(rng: np.random.Generator, n_side: int, fov: float) -> np.ndarray:
    """T1 logU[0.1,4] s, T2 logU[0.01,0.5] s with T2<T1, B1 U[0.8,1.2], B0 N(0,20 Hz),
    rho = U[0.5,1]·e^{iU[0,2π)}, (x, y) on a LinRange(-FOV/2, FOV/2, n) grid, z = 0."""
    nv = n_side * n_side
    T1 = np.exp(rng.uniform(np.log(0.1), np.log(4.0), nv))
    T2 = np.exp(rng.uniform(np.log(0.01), np.log(0.5), nv))
    bad = T2 >= T1
    while bad.any():
        T2[bad] = np.exp(rng.uniform(np.log(0.01), np.log(0.5), bad.sum()))
        bad = T2 >= T1
    B1 = rng.uniform(0.8, 1.2, nv)
    B0 = rng.normal(0.0, 20.0, nv)
    mag = rng.uniform(0.5, 1.0, nv)
    ph = rng.uniform(0.0, 2 * np.pi, nv)
    lin = np.linspace(-fov / 2, fov / 2, n_side)
    X, Y = np.meshgrid(lin, lin, indexing="ij")  # x varies slowest (Julia column-major vec of x-major grid)
    p = np.zeros((9, nv), np.float32)
    p[0], p[1], p[2], p[3] = T1, T2, B1, B0
    p[4], p[5] = mag * np.cos(ph), mag * np.sin(ph)
    p[6], p[7] = X.T.ravel(), Y.T.ravel()
    return p


def tissue_voxels(rng: np.random.Generator, nv: int, fov: float) -> np.ndarray:
    """`tissue` for an arbitrary voxel count: the first nv points of a ceil(√nv)² grid."""
    side = max(1, math.ceil(math.sqrt(nv)))
    return np.ascontiguousarray(tissue(rng, side, fov)[:, :nv])


def cartesian(nr: int, ns: int, fov: float, dt: float, nlines: int) -> dict:
    """k_start[r] = -S/2·Δkx + i·py[r]·Δky with py cycling -nlines/2 .. nlines/2-1; Δk = 2π/FOV."""
    dk = 2 * np.pi / fov
    py = np.arange(-(nlines // 2), nlines - nlines // 2)
    k_start = (-ns / 2 * dk + 1j * py[np.arange(nr) % nlines] * dk).astype(np.complex64)
    return {"kind": "cartesian", "nr": nr, "ns": ns, "dt": float(dt), "k_start": k_start, "dk": float(dk)}


def spiral(rng: np.random.Generator, ninterleaves: int, ns: int, fov: float, dt: float) -> dict:
    """Variable-density Archimedean spiral: interleave r starts at the spiral's first
    point rotated by 2πr/R; the per-sample step Δk[r] is the tangent at that start,
    scaled to the Nyquist step 2π/FOV (the reference models each readout as a
    linear k-step per sample, compas/trajectories/spiral.h:14-31)."""
    dkn = 2 * np.pi / fov
    k0 = 0.5 * dkn * rng.uniform(0.5, 1.5)
    ang = 2 * np.pi * np.arange(ninterleaves) / ninterleaves
    k_start = (k0 * np.exp(1j * ang)).astype(np.complex64)
    tangent = np.exp(1j * (ang + np.pi / 2)) * 0.7 + np.exp(1j * ang) * 0.3
    dkv = (dkn * tangent / np.abs(tangent)).astype(np.complex64)
    return {"kind": "spiral", "nr": ninterleaves, "ns": ns, "dt": float(dt), "k_start": k_start, "dk": dkv}


def gaussian_coils(nc: int, params: np.ndarray, fov: float) -> np.ndarray:
    """exp(-|r-r_c|²/(2(FOV/3)²))·e^{iφ_c}, centres on a circle of radius FOV/3, φ_c = 2πc/C."""
    x, y = params[6].astype(np.float64), params[7].astype(np.float64)
    out = np.zeros((nc, x.size), np.complex64)
    for c in range(nc):
        a = 2 * np.pi * c / nc
        cx, cy = fov / 3 * np.cos(a), fov / 3 * np.sin(a)
        out[c] = np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * (fov / 3) ** 2)) * np.exp(1j * a)
    return out


def fisp_sequence(rf_deg: np.ndarray, slices: np.ndarray, TR: float, TE: float, TI: float, max_state: int,
                  uf: int = 1, reps: int = 1, TW: float = 0.0) -> dict:
    return {"rf": np.asarray(rf_deg, np.complex64), "slices": np.asarray(slices, np.complex64), "TR": TR, "TE": TE,
            "TI": TI, "TW": TW, "max_state": int(max_state), "uf": int(uf), "reps": int(reps), "inversion": 1,
            "wait_spoil": 1}


def smooth_flip_train(rng: np.random.Generator, ntr: int, nknots: int = 15, lo: float = 0.0,
                      hi: float = 70.0) -> np.ndarray:
    """Cubic interpolation of `nknots` seeded knots ~U[lo,hi] degrees, clipped to [lo,hi]."""
    from scipy.interpolate import CubicSpline

    knots = rng.uniform(lo, hi, nknots)
    spl = CubicSpline(np.linspace(0, ntr - 1, nknots), knots)
    return np.clip(spl(np.arange(ntr)), lo, hi)


def gaussian_slice_profile(P: int, ntr: int) -> np.ndarray:
    p = np.arange(P)
    prof = np.exp(-((p - (P - 1) / 2) ** 2) / (2 * 8.0 ** 2))
    return np.repeat(prof[:, None], ntr, axis=1).astype(np.complex64)


def pssfp_sequence(rng: np.random.Generator, ntr: int, nrf: int = 15, nz: int = 35) -> dict:
    """Gaussian RF waveform of nRF samples normalised to 1° (γΔtRF in rad), constant
    40° flip train with 0-π phase cycling, z in LinRange(-1,1,nz); time intervals and
    slice-select gradients follow the reference examples (examples/common.jl:44-58)."""
    TR, dur = 0.010, 0.001
    i = np.arange(1, nrf + 1)
    g = np.exp(-((i - nrf / 2) ** 2) / nrf)
    gdtrf = (np.pi / 180) * g / np.abs(g).sum()
    rf = np.full(ntr, 40.0) * rng.uniform(0.9, 1.1)
    rf[1::2] *= -1
    return {"rf": rf.astype(np.complex64), "TR": TR, "gdtrf": gdtrf.astype(np.complex64),
            "dt": (dur / nrf, 10.0, (TR - dur) / 2), "gz": (0.002 / nrf, 0.0, -0.01),
            "z": np.linspace(-1, 1, nz).astype(np.float32)}


def cn(rng: np.random.Generator, shape) -> np.ndarray:
    """complex normal CN(0,1)."""
    return ((rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / math.sqrt(2)).astype(np.complex64)


# ------------------------------------------------------------------------------------------------
# Named configurations
# ------------------------------------------------------------------------------------------------

def fisp_small(seed: int = 1) -> dict:
    """64×64 voxels, FISP 400 TRs (60°·|sin(πn/400)|), TR 8.7 ms, TE 4.35 ms, TI 25 ms,
    8 states, 1 slice position, 1 unit coil, Cartesian 400×64 (FOV 25.6 cm, Δt 10 µs)."""
    rng = np.random.default_rng(seed)
    n, fov, ntr = 64, 25.6, 400
    params = tissue(rng, n, fov)
    rf = 60.0 * np.abs(np.sin(np.pi * np.arange(1, ntr + 1) / ntr))
    seq = fisp_sequence(rf, np.ones((1, ntr)), 8.7e-3, 4.35e-3, 25e-3, 8)
    traj = cartesian(ntr, 64, fov, 1e-5, 64)
    coils = np.ones((1, n * n), np.complex64)
    return {"name": "fisp_small", "params": params, "seq": seq, "traj": traj, "coils": coils, "fov": fov}


def mrstat(seed: int = 2, ncoils: int = 4, n_side: int = 224, ntr: int = 1120, P: int = 35,
           max_state: int = 25) -> dict:
    """224×224 voxels, FISP 1120 TRs (smooth random 0–70° train), 25 states, 35 Gaussian
    slice positions, `ncoils` Gaussian-bump coils, Cartesian 1120×224 (FOV 22.4 cm, Δt 5 µs)."""
    rng = np.random.default_rng(seed)
    fov = 22.4
    params = tissue(rng, n_side, fov)
    rf = smooth_flip_train(rng, ntr)
    seq = fisp_sequence(rf, gaussian_slice_profile(P, ntr), 8.7e-3, 4.35e-3, 25e-3, max_state)
    traj = cartesian(ntr, n_side, fov, 5e-6, n_side)
    coils = gaussian_coils(ncoils, params, fov)
    return {"name": "mrstat", "params": params, "seq": seq, "traj": traj, "coils": coils, "fov": fov}


def jacobian_inputs(seed: int = 3, ncoils: int = 8, n_side: int = 224, ntr: int = 1120) -> dict:
    """Jacobian products at MR-STAT scale: random complex echos / ∂echos (product-only
    timing), v ~ CN(0,1) [4][V], residual r ~ CN(0,1) [C][R][S]."""
    rng = np.random.default_rng(seed)
    fov = 22.4
    params = tissue(rng, n_side, fov)
    nv = n_side * n_side
    traj = cartesian(ntr, n_side, fov, 5e-6, n_side)
    coils = gaussian_coils(ncoils, params, fov)
    echo = cn(rng, (ntr, nv)) * 0.1
    dT1 = cn(rng, (ntr, nv)) * 0.05
    dT2 = cn(rng, (ntr, nv)) * 0.5
    v = cn(rng, (4, nv))
    r = cn(rng, (ncoils, ntr, n_side))
    return {"name": "jacobian", "params": params, "traj": traj, "coils": coils, "echo": echo, "dT1": dT1,
            "dT2": dT2, "v": v, "r": r, "fov": fov}


def tiny(seed: int = 7, n_side: int = 6, ntr: int = 13, ns: int = 7, nc: int = 3, P: int = 3,
         max_state: int = 5) -> dict:
    """Small ragged case (sizes that are multiples of no tile) for exhaustive parity."""
    rng = np.random.default_rng(seed)
    fov = 20.0
    params = tissue(rng, n_side, fov)
    nv = n_side * n_side
    params[8] = rng.uniform(-0.5, 0.5, nv)
    rf = rng.uniform(5, 80, ntr) * np.exp(1j * rng.uniform(-0.3, 0.3, ntr))
    slices = (rng.uniform(0.5, 1.0, (P, ntr)) * np.exp(1j * rng.uniform(-0.1, 0.1, (P, ntr))))
    seq = fisp_sequence(rf, slices, 8.7e-3, 4.35e-3, 20e-3, max_state)
    traj = cartesian(ntr, ns, fov, 1e-5, ns)
    coils = cn(rng, (nc, nv))
    return {"name": "tiny", "params": params, "seq": seq, "traj": traj, "coils": coils, "fov": fov}


def batch_jobs(seed: int = 4, njobs: int = 256, vmin: int = 1000, vmax: int = 64000, ntr_min: int = 400,
               ntr_max: int = 1120, cmax: int = 16, ns_spiral: int = 1000, P: int = 35, max_state: int = 25,
               nz: int = 35, nrf: int = 15) -> list:
    """Uneven independent jobs: V ~ logU[vmin, vmax], nTR ~ U{ntr_min..ntr_max}, C ~ U{1..cmax};
    50/50 FISP (max_state states, P Gaussian slice positions, smooth random 0–70° train) vs pSSFP
    (nz z positions, Gaussian RF of nrf samples); 50/50 Cartesian (S = round(√V), nTR readouts)
    vs variable-density spiral (nTR interleaves × ns_spiral samples). FOV 22.4 cm."""
    rng = np.random.default_rng(seed)
    fov = 22.4
    jobs = []
    for i in range(njobs):
        nv = int(round(math.exp(rng.uniform(math.log(vmin), math.log(vmax)))))
        ntr = int(rng.integers(ntr_min, ntr_max + 1))
        nc = int(rng.integers(1, cmax + 1))
        jrng = np.random.default_rng([seed, i])
        params = tissue_voxels(jrng, nv, fov)
        if rng.uniform() < 0.5:
            kind = "fisp"
            seq = fisp_sequence(smooth_flip_train(jrng, ntr), gaussian_slice_profile(P, ntr), 8.7e-3, 4.35e-3,
                                25e-3, max_state)
        else:
            kind = "pssfp"
            seq = pssfp_sequence(jrng, ntr, nrf=nrf, nz=nz)
        if rng.uniform() < 0.5:
            ns = max(2, int(round(math.sqrt(nv))))
            traj = cartesian(ntr, ns, fov, 5e-6, ns)
        else:
            traj = spiral(jrng, ntr, ns_spiral, fov, 4e-6)
        coils = gaussian_coils(nc, params, fov)
        jobs.append({"kind": kind, "params": params, "seq": seq, "traj": traj, "coils": coils,
                     "nvoxels": nv, "ntr": ntr, "ncoils": nc})
    return jobs


def serve_requests(seed: int = 5, n: int = 12, vmin: int = 4000, vmax: int = 200000, cmin: int = 4,
                   cmax: int = 16, **kw) -> list:
    """Distinct reconstruction requests for the served stream: the uneven jobs of `batch_jobs`
    with voxels logU[vmin, vmax] and coils U{cmin..cmax}, each with measured data
    y ~ 0.05·CN(0,1) of shape [C][R][S]."""
    jobs = batch_jobs(seed=seed, njobs=n, vmin=vmin, vmax=vmax, **kw)
    rng = np.random.default_rng([seed, 99])
    for j in jobs:
        c = int(rng.integers(cmin, cmax + 1))
        j["ncoils"] = c
        j["coils"] = gaussian_coils(c, j["params"], 22.4)
        j["data"] = cn(rng, (c, j["traj"]["nr"], j["traj"]["ns"])) * 0.05
    return jobs
