"""Seeded synthetic time-ordered data for the destriping benchmarks and tests.

The reference ships no data sets; its tests build toy inputs in numpy
(python/tests/test_libmadam.py:86-118).  The benchmark workloads are ring scans:
the boresight spins at 1 rpm at an opening angle of 85 deg around a spin axis
that precesses at 1 deg/day in the x-y plane.  Pixels come from the HEALPix
NESTED scheme (Gorski et al. 2005, ApJ 622, 759; the same mapping as
healpix_routines.f90:36-131 of the reference), weights are [1, cos 2psi,
sin 2psi], the sky is Gaussian (I rms 100 uK, Q/U rms 10 uK per pixel) and the
noise is white + 1/f with PSD = sigma^2/fs * (1 + (f/fknee)^alpha).

Everything is computed with torch so the same code runs on the CPU (small test
cases) and on a GPU (the full-size benchmark workloads, generated directly in
HBM).  Outputs use the reference ABI dtypes: float64 timestamps and signal,
int32 pixels, float32 weights (python/libmadam_wrapper/__init__.py:15-19).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

_HALFPI = 0.5 * math.pi


def ang2pix_nest(nside: int, theta: torch.Tensor, phi: torch.Tensor) -> torch.Tensor:
    """HEALPix NESTED pixel index of (theta, phi) [radians], int64.

    Equatorial zone |z| <= 2/3 uses the two edge-line indices; the polar caps
    use the sqrt(3(1-|z|)) rings; the face-local (ix, iy) are bit-interleaved.
    """
    z = torch.cos(theta)
    za = z.abs()
    tt = torch.remainder(phi, 2 * math.pi) / _HALFPI  # in [0, 4)
    tt = torch.where(tt >= 4.0, tt - 4.0, tt)
    ns = nside
    # equatorial
    temp1 = ns * (0.5 + tt)
    temp2 = ns * (z * 0.75)
    jp = torch.floor(temp1 - temp2).to(torch.int64)
    jm = torch.floor(temp1 + temp2).to(torch.int64)
    ifp = torch.div(jp, ns, rounding_mode="floor")
    ifm = torch.div(jm, ns, rounding_mode="floor")
    face_eq = torch.where(ifp == ifm, ifp | 4, torch.where(ifp < ifm, ifp, ifm + 8))
    ix_eq = jm & (ns - 1)
    iy_eq = ns - (jp & (ns - 1)) - 1
    # polar
    ntt = torch.clamp(tt.floor().to(torch.int64), max=3)
    tp = tt - ntt.to(tt.dtype)
    tmp = ns * torch.sqrt(torch.clamp(3.0 * (1.0 - za), min=0.0))
    jp2 = torch.clamp(torch.floor(tp * tmp).to(torch.int64), max=ns - 1)
    jm2 = torch.clamp(torch.floor((1.0 - tp) * tmp).to(torch.int64), max=ns - 1)
    north = z > 0
    face_p = torch.where(north, ntt, ntt + 8)
    ix_p = torch.where(north, ns - jm2 - 1, jp2)
    iy_p = torch.where(north, ns - jp2 - 1, jm2)
    eq = za <= 2.0 / 3.0
    face = torch.where(eq, face_eq, face_p)
    ix = torch.where(eq, ix_eq, ix_p)
    iy = torch.where(eq, iy_eq, iy_p)
    # interleave bits: ix -> even bit positions, iy -> odd
    ipf = torch.zeros_like(ix)
    nbits = max(1, int(ns).bit_length() - 1)
    for b in range(nbits):
        ipf |= ((ix >> b) & 1) << (2 * b)
        ipf |= ((iy >> b) & 1) << (2 * b + 1)
    return face * (ns * ns) + ipf


def pix2ang_nest(nside: int, pix: torch.Tensor):
    """Centre (theta, phi) of HEALPix NESTED pixels (inverse of ang2pix_nest)."""
    ns = nside
    npface = ns * ns
    face = torch.div(pix, npface, rounding_mode="floor")
    ipf = pix - face * npface
    ix = torch.zeros_like(pix)
    iy = torch.zeros_like(pix)
    nbits = max(1, int(ns).bit_length() - 1)
    for b in range(nbits):
        ix |= ((ipf >> (2 * b)) & 1) << b
        iy |= ((ipf >> (2 * b + 1)) & 1) << b
    jrll = torch.tensor([2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4], device=pix.device)
    jpll = torch.tensor([1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7], device=pix.device)
    jr = jrll[face] * ns - ix - iy - 1  # ring number in [1, 4ns-1]
    nl4 = 4 * ns
    # ring -> z, nr, kshift
    north = jr < ns
    south = jr > 3 * ns
    nr_n = jr
    nr_s = nl4 - jr
    z_n = 1.0 - (nr_n.double() ** 2) / (3.0 * npface)
    z_s = -(1.0 - (nr_s.double() ** 2) / (3.0 * npface))
    z_e = (2 * ns - jr).double() * 2.0 / (3.0 * ns)
    nr = torch.where(north, nr_n, torch.where(south, nr_s, torch.full_like(jr, ns)))
    z = torch.where(north, z_n, torch.where(south, z_s, z_e))
    kshift = torch.where(north | south, torch.zeros_like(jr), (jr - ns) & 1)
    jp = (jpll[face] * nr + ix - iy + 1 + kshift) // 2
    jp = torch.where(jp > nl4, jp - nl4, jp)
    jp = torch.where(jp < 1, jp + nl4, jp)
    phi = (jp.double() - (kshift + 1).double() * 0.5) * (_HALFPI / nr.double())
    theta = torch.acos(torch.clamp(z, -1.0, 1.0))
    return theta, phi


@dataclass
class ScanConfig:
    """One synthetic destriping workload."""

    nside: int = 64
    nside_submap: int = 16
    ndet: int = 4
    nobs: int = 1
    nsamp_obs: int = 1 << 20
    fsample: float = 10.0
    sigma: float = 1e-3          # white noise rms [K]
    fknee: float = 0.1           # [Hz]
    alpha: float = -1.0
    base_first: float = 1.0      # [s]
    sky_i_rms: float = 100e-6
    sky_qu_rms: float = 10e-6
    psi_deg: tuple = (0.0, 45.0, 90.0, 135.0)
    det_offset_deg: float = 0.2  # cross-scan offset between detector groups
    npsdbin: int = 1000
    seed: int = 1001
    temperature_only: bool = False
    fknee_range: tuple = ()      # (lo, hi): per-detector fknee drawn uniformly
    extra_pars: dict = field(default_factory=dict)

    @property
    def nsamp(self) -> int:
        return self.nobs * self.nsamp_obs


def config1() -> ScanConfig:
    """Plain destripe, CPU-runnable: nside 64, 4 dets x 2^20 samples @ 10 Hz."""
    return ScanConfig(
        nside=64, nside_submap=16, ndet=4, nobs=1, nsamp_obs=1 << 20, fsample=10.0,
        fknee=0.1, alpha=-1.0, base_first=1.0, seed=1001,
        extra_pars=dict(precond_width_min=20, precond_width_max=20, iter_max=100,
                        cglimit=1e-12),
    )


def config2() -> ScanConfig:
    """Plain destripe on one B200: nside 512, 16 dets x 4 obs x 2^23 @ 100 Hz."""
    return ScanConfig(
        nside=512, nside_submap=16, ndet=16, nobs=4, nsamp_obs=1 << 23,
        fsample=100.0, fknee=0.05, alpha=-1.5, base_first=0.5, seed=1002,
        extra_pars=dict(cglimit=1e-12),
    )


def config3() -> ScanConfig:
    """Precision form: nside 1024, 64 dets x 2^24 @ 100 Hz (1.07e9 samples),
    fknee 0.1 Hz, alpha -1, base_first 1 s; float32 TOD in destripe_fp32."""
    return ScanConfig(
        nside=1024, nside_submap=16, ndet=64, nobs=1, nsamp_obs=1 << 24,
        fsample=100.0, fknee=0.1, alpha=-1.0, base_first=1.0, seed=1003,
        extra_pars=dict(cglimit=1e-12),
    )


def config4() -> ScanConfig:
    """Batched Monte Carlo form: nside 512, 32 dets x 2^22 @ 100 Hz sharing
    one pointing, fknee per detector uniform in 0.02-0.2 Hz, alpha -1."""
    return ScanConfig(
        nside=512, nside_submap=16, ndet=32, nobs=1, nsamp_obs=1 << 22,
        fsample=100.0, fknee=0.1, fknee_range=(0.02, 0.2), alpha=-1.0, base_first=1.0,
        seed=1004, extra_pars=dict(cglimit=1e-12),
    )


def small_config(ndet=4, nsamp_obs=1 << 14, nobs=2, nside=16, seed=7, **kw) -> ScanConfig:
    """A few-second case for parity tests."""
    base = dict(nside=nside, nside_submap=4, ndet=ndet, nobs=nobs, nsamp_obs=nsamp_obs,
                fsample=10.0, fknee=0.1, alpha=-1.0, base_first=1.0, seed=seed,
                extra_pars=dict(iter_max=200, cglimit=1e-12))
    base.update(kw)
    return ScanConfig(**base)


def pars_for(cfg: ScanConfig) -> dict:
    """Madam parameter dictionary for the workload (dict2parstring input)."""
    pars = dict(
        nside_map=cfg.nside, nside_cross=cfg.nside, nside_submap=cfg.nside_submap,
        fsample=cfg.fsample, base_first=cfg.base_first, kfilter=True,
        temperature_only=cfg.temperature_only, info=0,
        write_map=False, write_binmap=False, write_hits=False,
    )
    pars.update(cfg.extra_pars)
    return pars


def _generator(seed: int, device) -> torch.Generator:
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    return g


def _boresight(cfg: ScanConfig, t: torch.Tensor, open_deg: float, psi_det: float):
    """Pointing (theta, phi, psi) of one detector at times t [s]."""
    lam = math.radians(1.0) * t / 86400.0          # spin axis longitude
    spin = 2 * math.pi / 60.0 * t                   # 1 rpm
    sx, sy = torch.cos(lam), torch.sin(lam)         # spin axis s = (sx, sy, 0)
    # basis of the plane orthogonal to s: u = z, v = s x z = (sy, -sx, 0)
    a = math.radians(open_deg)
    ca, sa = math.cos(a), math.sin(a)
    cs, ss = torch.cos(spin), torch.sin(spin)
    bx = ca * sx + sa * ss * sy
    by = ca * sy - sa * ss * sx
    bz = sa * cs
    # scan direction d = db/dspin (unit length up to sa)
    dx = sa * cs * sy
    dy = -sa * cs * sx
    dz = -sa * ss
    dn = torch.sqrt(dx * dx + dy * dy + dz * dz)
    dx, dy, dz = dx / dn, dy / dn, dz / dn
    theta = torch.acos(torch.clamp(bz, -1.0, 1.0))
    phi = torch.atan2(by, bx)
    # local frame: e_theta (south), e_phi (east)
    st = torch.sin(theta).clamp(min=1e-12)
    ct = torch.cos(theta)
    cp, sp = torch.cos(phi), torch.sin(phi)
    eth = (ct * cp, ct * sp, -st)
    eph = (-sp, cp, torch.zeros_like(sp))
    # polarisation direction: scan direction rotated by psi_det about b
    c2, s2 = math.cos(psi_det), math.sin(psi_det)
    # d2 = b x d
    d2x = by * dz - bz * dy
    d2y = bz * dx - bx * dz
    d2z = bx * dy - by * dx
    ex = c2 * dx + s2 * d2x
    ey = c2 * dy + s2 * d2y
    ez = c2 * dz + s2 * d2z
    psi = torch.atan2(ex * eph[0] + ey * eph[1] + ez * eph[2],
                      -(ex * eth[0] + ey * eth[1] + ez * eth[2]))
    return theta, phi, psi


def det_fknee(cfg: ScanConfig) -> np.ndarray:
    """Knee frequency of every detector: cfg.fknee, or seeded draws from
    cfg.fknee_range."""
    if not cfg.fknee_range:
        return np.full(cfg.ndet, cfg.fknee)
    rng = np.random.default_rng(cfg.seed + 4242)
    return rng.uniform(cfg.fknee_range[0], cfg.fknee_range[1], cfg.ndet)


def psd_model(cfg: ScanConfig, f: np.ndarray, fknee=None) -> np.ndarray:
    """Noise PSD sigma^2/fs (1 + (f/fknee)^alpha) at frequencies f > 0."""
    fk = cfg.fknee if fknee is None else fknee
    return cfg.sigma ** 2 / cfg.fsample * (1.0 + (f / fk) ** cfg.alpha)


def noise_realisations(cfg: ScanConfig, nreal: int, device="cuda", seed0=0):
    """nreal noise-only TODs [nreal, ndet, nsamp] (float64): white + 1/f with
    each detector's knee frequency, seeded per (realisation, detector)."""
    fk = det_fknee(cfg)
    out = torch.empty((nreal, cfg.ndet, cfg.nsamp), dtype=torch.float64, device=device)
    for r in range(nreal):
        for d in range(cfg.ndet):
            g = _generator(cfg.seed * 7 + 100003 * (seed0 + r) + d, torch.device(device))
            out[r, d] = _noise(cfg, cfg.nsamp, g, device, fknee=fk[d])
    return out


def _noise(cfg: ScanConfig, nsamp: int, gen: torch.Generator, device,
           fknee=None) -> torch.Tensor:
    """White + 1/f noise realisation of length nsamp (float64)."""
    n = 1
    while n < nsamp:
        n *= 2
    white = torch.randn(n, generator=gen, device=device, dtype=torch.float64)
    spec = torch.fft.rfft(white)
    f = torch.fft.rfftfreq(n, d=1.0 / cfg.fsample, device=device).to(torch.float64)
    f[0] = f[1]
    shape = torch.sqrt(1.0 + (f / (cfg.fknee if fknee is None else fknee)) ** cfg.alpha)
    shape[0] = 0.0
    out = torch.fft.irfft(spec * shape, n=n)[:nsamp]
    return out * cfg.sigma


def generate(cfg: ScanConfig, device="cpu", nnz=None, with_signal=True):
    """Build the destripe() inputs for a workload.

    Returns a dict of torch tensors on `device` (timestamps f64 [nsamp],
    pixels i32 [ndet, nsamp], pixweights f32 [ndet, nsamp, nnz], signal f64
    [ndet, nsamp]) plus numpy arrays for periods / PSDs / detector weights and
    the parameter dictionary.
    """
    device = torch.device(device)
    nnz = nnz if nnz is not None else (1 if cfg.temperature_only else 3)
    nsamp = cfg.nsamp
    g = _generator(cfg.seed, device)
    t0 = 1.0e6
    t = t0 + torch.arange(nsamp, device=device, dtype=torch.float64) / cfg.fsample
    npix = 12 * cfg.nside ** 2
    gs = _generator(cfg.seed + 7919, device)
    sky_i = torch.randn(npix, generator=gs, device=device, dtype=torch.float64) * cfg.sky_i_rms
    sky_q = torch.randn(npix, generator=gs, device=device, dtype=torch.float64) * cfg.sky_qu_rms
    sky_u = torch.randn(npix, generator=gs, device=device, dtype=torch.float64) * cfg.sky_qu_rms
    pixels = torch.empty((cfg.ndet, nsamp), dtype=torch.int32, device=device)
    weights = torch.empty((cfg.ndet, nsamp, nnz), dtype=torch.float32, device=device)
    signal = torch.empty((cfg.ndet, nsamp), dtype=torch.float64, device=device) if with_signal else None
    npsi = len(cfg.psi_deg)
    chunk = 1 << 24
    for d in range(cfg.ndet):
        psi_det = math.radians(cfg.psi_deg[d % npsi])
        grp = d // npsi
        open_deg = 85.0 + cfg.det_offset_deg * (grp - 0.5 * ((cfg.ndet - 1) // npsi))
        for s0 in range(0, nsamp, chunk):
            s1 = min(nsamp, s0 + chunk)
            theta, phi, psi = _boresight(cfg, t[s0:s1] - t0, open_deg, psi_det)
            pix = ang2pix_nest(cfg.nside, theta, phi)
            pixels[d, s0:s1] = pix.to(torch.int32)
            c2, s2 = torch.cos(2 * psi), torch.sin(2 * psi)
            weights[d, s0:s1, 0] = 1.0
            if nnz == 3:
                weights[d, s0:s1, 1] = c2.to(torch.float32)
                weights[d, s0:s1, 2] = s2.to(torch.float32)
            if with_signal:
                sig = sky_i[pix]
                if nnz == 3:
                    sig = sig + sky_q[pix] * c2.to(torch.float32).double() \
                        + sky_u[pix] * s2.to(torch.float32).double()
                signal[d, s0:s1] = sig
            del theta, phi, psi, pix
        if with_signal:
            gn = _generator(cfg.seed * 1000 + d, device)
            signal[d] += _noise(cfg, nsamp, gn, device, fknee=det_fknee(cfg)[d])
    periods = np.arange(cfg.nobs, dtype=np.int64) * cfg.nsamp_obs
    npsd = np.ones(cfg.ndet, dtype=np.int64)
    psdfreqs = np.logspace(-5, math.log10(cfg.fsample / 2), cfg.npsdbin)
    psdvals = np.concatenate([psd_model(cfg, psdfreqs, fk) for fk in det_fknee(cfg)])
    psdstarts = np.zeros(cfg.ndet, dtype=np.float64)
    detweights = np.full(cfg.ndet, 1.0 / cfg.sigma ** 2)
    dets = ["det{:03d}".format(d) for d in range(cfg.ndet)]
    return dict(
        timestamps=t, pixels=pixels, pixweights=weights, signal=signal,
        periods=periods, npsd=npsd, psdstarts=psdstarts, psdfreqs=psdfreqs,
        psdvals=psdvals, detweights=detweights, dets=dets, pars=pars_for(cfg),
        nnz=nnz, sky=(sky_i, sky_q, sky_u),
    )


def to_numpy(data: dict) -> dict:
    """Host (numpy) copy of generate()'s tensors."""
    out = dict(data)
    for k in ("timestamps", "pixels", "pixweights", "signal"):
        if out.get(k) is not None and isinstance(out[k], torch.Tensor):
            out[k] = out[k].cpu().numpy()
    out.pop("sky", None)
    return out
