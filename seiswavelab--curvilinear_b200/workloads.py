"""Seeded synthetic workloads in the reference's parameter vocabulary.

Each function returns a parameter dictionary for ``session.Simulation2D`` / ``Simulation3D``
(and for the reference's own CPU solver, which reads the same keys).  All randomness comes from
NumPy PCG64 generators with fixed seeds, so every run sees bit-identical inputs; the arrays'
SHA-256 digests are reported by ``digest``.

* ``plain_small``       500x200 2D elastic, flat surface, three layers, surface force, CFS-PML
* ``curvilinear_large`` 5001x2001 2D elastic, seeded terrain (6 sinusoids + 2 gullies, 60 m
                        relief, blend depth 300 m), five layers with a low-velocity top,
                        explosive source, 30-cell CFS-PML, 2000 steps, 1000 receivers
* ``gsls_medium``       2001x801 2D GSLS (3 mechanisms, Qs = Qp/2), sinusoidal terrain, CFS-PML
* ``elastic_3d``        400x288x200 3D, Gaussian-random-field DEM terrain, three layers,
                        explosive source, 20-cell sponge, 40x40 areal receivers
* ``serving_mix``       a stream of shot requests (2D elastic / GSLS and 3D) with Poisson arrivals
"""
from __future__ import annotations

import hashlib

import numpy as np


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def digest(params: dict) -> str:
    h = hashlib.sha256()
    for k in sorted(params):
        h.update(k.encode())
        h.update(np.ascontiguousarray(params[k], dtype=np.float64).tobytes())
    return h.hexdigest()


def terrain_profile(span: float, relief: float, seed: int, dx: float = 1.0, gullies: int = 2) -> np.ndarray:
    """Elevation samples (x, H) every dx over [0, span]: six sinusoids with log-uniform
    wavelengths in 200-4000 m and uniform phases plus Gaussian gullies (depth 10-30 m, sigma
    20-80 m, centres in the middle 60 %), rescaled so max |H| equals `relief`."""
    r = _rng(seed)
    x = np.arange(0.0, span + 0.5 * dx, dx)
    lam = np.exp(r.uniform(np.log(200.0), np.log(4000.0), 6))
    phase = r.uniform(0, 2 * np.pi, 6)
    amp = r.uniform(0.3, 1.0, 6)
    h = sum(a * np.sin(2 * np.pi * x / l + p) for a, l, p in zip(amp, lam, phase))
    h = h / np.max(np.abs(h)) * 0.6 * relief
    for _ in range(gullies):
        depth, sigma, c = r.uniform(10, 30), r.uniform(20, 80), r.uniform(0.2, 0.8) * span
        h = h - depth * np.exp(-0.5 * ((x - c) / sigma) ** 2)
    h = h / np.max(np.abs(h)) * relief
    return np.stack([x, h], axis=1)


def plain_small(precision: int = 0, steps: int = 4000, cfl: float = 0.442) -> dict:
    """500x200 FP64 elastic, h=2, flat surface; layers with interfaces at 80 m and 200 m;
    30 Hz vertical surface force at the midpoint; 20-cell external CFS-PML; receivers at every
    surface node.  cfl=0.442 gives dt ~0.25 ms (the reference rule at its default 0.8 gives 0.45 ms)."""
    return dict(precision=precision, nx=500, nz=200, spacing=2.0, relief=0.0, frequency=30.0, cfl=cfl,
                duration=1.0, maxSteps=steps, sourceX=250, sourceZ=0, sourceKind=0, sourceDirection=[0, 0, 1],
                absorbing=1, absorber=1, spongeX=20, spongeZ=20, externalAbsorption=1,
                receiverStart=0, receiverCount=500, receiverStride=1, receiverDepth=0,
                layered=1, layers=[80, 800, 400, 1600, 100, 60, 120, 1500, 800, 1900, 100, 60,
                                   0, 2500, 1400, 2200, 100, 60])


def _layers_2d(seed: int, n: int, top=(500.0, 250.0, 1500.0), vp_max=3500.0, q=None) -> list:
    r = _rng(seed)
    vps = np.concatenate([[top[0]], np.sort(r.uniform(900.0, vp_max, n - 2)), [vp_max]])
    thick = np.concatenate([[r.uniform(10, 30)], r.uniform(60, 400, n - 2), [0.0]])
    rows = []
    for i, vp in enumerate(vps):
        vs = top[1] if i == 0 else vp / r.uniform(1.75, 2.0)
        rho = top[2] if i == 0 else 1700 + 600 * (i / (n - 1))
        qp = q[i] if q is not None else 100.0
        rows += [float(thick[i]), float(vp), float(vs), float(rho), float(qp), float(qp / 2)]
    return rows


def curvilinear_large(precision: int = 0, steps: int = 2000, nx: int = 5001, nz: int = 2001) -> dict:
    """5001x2001 2D elastic curvilinear shot (seed 2).  The explosive source sits 5 nodes
    (10 m) below the surface: the reference requires an isotropic-moment centre at least five
    nodes deep, so the 4 m of the workload description is not representable."""
    h = 2.0
    span = (nx - 1) * h
    surf = terrain_profile(span, 60.0, seed=2)
    return dict(precision=precision, nx=nx, nz=nz, spacing=h, importedSurface=1, surfaceDatum=0.0,
                surface=surf.ravel().tolist(), flattenDepth=300.0, frequency=30.0, cfl=0.8, duration=1.0,
                maxSteps=steps, sourceX=nx // 2, sourceZ=5, sourceKind=1, absorbing=1, absorber=1,
                spongeX=30, spongeZ=30, externalAbsorption=1, receiverStart=3,
                receiverCount=min(1000, (nx - 4) // 5 + 1), receiverStride=5, receiverDepth=0,
                layered=1, layers=_layers_2d(2, 5))


def gsls_medium(precision: int = 1, steps: int = 6000, nx: int = 2001, nz: int = 801) -> dict:
    """2001x801 GSLS (3 mechanisms fitted over 5-60 Hz, reference 25 Hz), four layers with
    Qp in 30-100 and Qs = Qp/2 (seed 3), sinusoidal terrain of 40 m amplitude, 25 Hz Ricker."""
    r = _rng(3)
    qp = r.uniform(30, 100, 4)
    return dict(precision=precision, nx=nx, nz=nz, spacing=2.0, relief=40.0, wavelength=float(r.uniform(600, 1200)),
                frequency=25.0, cfl=0.8, duration=2.0, maxSteps=steps, sourceX=nx // 2, sourceZ=10, sourceKind=0,
                sourceDirection=[0, 0, 1], absorbing=1, absorber=1, spongeX=30, spongeZ=30, externalAbsorption=1,
                receiverStart=1, receiverCount=min(1000, (nx - 2) // 2), receiverStride=2, receiverDepth=0,
                attenuation=1, mechanisms=3, qMinFrequency=5.0, qMaxFrequency=60.0, qReferenceFrequency=25.0,
                layered=1, layers=_layers_2d(3, 4, top=(800.0, 400.0, 1700.0), vp_max=3000.0, q=qp))


def grf_dem(nx: int, ny: int, spacing: float, correlation: float, relief: float, seed: int) -> np.ndarray:
    """Gaussian random field on a DEM lattice: white noise smoothed by a Gaussian of the given
    correlation length (FFT), rescaled so max |elevation - mean| equals `relief`."""
    r = _rng(seed)
    noise = r.standard_normal((ny, nx))
    ky = np.fft.fftfreq(ny, d=spacing)[:, None]
    kx = np.fft.fftfreq(nx, d=spacing)[None, :]
    filt = np.exp(-0.5 * (2 * np.pi) ** 2 * (kx ** 2 + ky ** 2) * correlation ** 2)
    field = np.real(np.fft.ifft2(np.fft.fft2(noise) * filt))
    field -= field.mean()
    return field / np.max(np.abs(field)) * relief


def elastic_3d(precision: int = 0, steps: int = 1500, nx: int = 400, ny: int = 288, nz: int = 200,
               receivers: int = 40, relief: float = 150.0, flatten_depth: float = 800.0, absorber: int = 0,
               mechanisms: int = 0) -> dict:
    """400x288x200 3D elastic, h=10 m, DEM terrain (seed 4, correlation 500 m, relief 150 m on a
    25 m lattice), blend depth 800 m, layers 200 m / 600 m / basement below the surface, 15 Hz
    explosive source 5 nodes deep, 20-cell sponge, 40x40 areal surface receivers.  Reduced grids
    need a smaller relief and blend depth (the blend must fit the model depth and exceed 2.6 times
    the relief).  `absorber` 1: 20-cell CFS-PML slabs instead of the sponge; `mechanisms` > 0: GSLS
    viscoelasticity with that many mechanisms (Qp 100, Qs 60 over 2.5-37.5 Hz, referenced at 15 Hz)."""
    h = 10.0
    dem_dx = 25.0
    dnx = int(np.ceil((nx - 1) * h / dem_dx)) + 1
    dny = int(np.ceil((ny - 1) * h / dem_dx)) + 1
    elev = grf_dem(dnx, dny, dem_dx, 500.0, relief, seed=4)
    sx = max(1, (nx - 2) // receivers)
    sy = max(1, (ny - 2) // receivers)
    return dict(precision=precision, nx=nx, ny=ny, nz=nz, spacing=h, frequency=15.0, cfl=0.8, duration=2.0,
                maxSteps=steps, sourceX=nx // 2, sourceY=ny // 2, sourceZ=5, sourceKind=1,
                demShape=[dnx, dny, dem_dx, 0.0, 0.0, 0.0], demElevations=elev.ravel().tolist(),
                flattenDepth=float(flatten_depth), layered=1, layerDepthMode=1,
                layers=[200, 1200, 600, 1800, 600, 2400, 1300, 2100, 0, 3800, 2200, 2400],
                absorbing=1, absorbingCells=[20, 20, 20], absorbingStrength=3.0, absorber=int(absorber),
                receiverArray=[3, (nx - (receivers - 1) * sx) // 2, (ny - (receivers - 1) * sy) // 2, 0,
                               receivers, receivers, sx, sy],
                receiverLimit=receivers * receivers,
                **(dict(attenuation=1, mechanisms=int(mechanisms), qMinFrequency=2.5, qMaxFrequency=37.5,
                        qReferenceFrequency=15.0, qp=100.0, qs=60.0) if mechanisms > 0 else {}))


def serving_mix(n: int = 256, rate: float = 20.0, seed: int = 5, scale: float = 1.0, steps_scale: float = 1.0) -> list:
    """Shot requests with Poisson arrivals (mean `rate` per second): 80 % 2D elastic or GSLS
    (grids 300x150 .. 2001x801, h in {1, 2, 4} m, seeded terrain, 3-6 layers, Ricker 10-40 Hz,
    nt 1000-6000), 20 % 3D elastic (128^3 .. 256x256x160), all FP32.  `scale` shrinks grid edges
    and `steps_scale` step counts for bounded benchmark runs."""
    r = _rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += r.exponential(1.0 / rate)
        if r.uniform() < 0.8:
            nx = int(r.integers(300, 2002) * scale) or 16
            nz = int(r.integers(150, 802) * scale) or 16
            nx, nz = max(nx, 40), max(nz, 30)
            h = float(r.choice([1.0, 2.0, 4.0]))
            f = float(r.uniform(10, 40))
            nl = int(r.integers(3, 7))
            gsls = bool(r.uniform() < 0.5)
            relief = float(min(r.uniform(5, 40), 0.1 * (nz - 1) * h))
            p = dict(precision=1, nx=nx, nz=nz, spacing=h, importedSurface=1, surfaceDatum=0.0,
                     surface=terrain_profile((nx - 1) * h, relief, seed=1000 + i, dx=h).ravel().tolist(),
                     frequency=f, cfl=0.8, duration=10.0, maxSteps=max(10, int(r.integers(1000, 6001) * steps_scale)),
                     sourceX=nx // 2, sourceZ=6, sourceKind=int(r.uniform() < 0.5), absorbing=1, absorber=1,
                     spongeX=min(20, nx // 4), spongeZ=min(20, nz // 4), externalAbsorption=1, receiverStart=2,
                     receiverCount=min(1000, (nx - 4) // 2), receiverStride=2, receiverDepth=0,
                     layered=1, layers=_layers_2d(2000 + i, nl, vp_max=float(r.uniform(2500, 4000)),
                                                  q=r.uniform(30, 100, nl)),
                     attenuation=int(gsls), mechanisms=3, qMinFrequency=max(0.5, f / 6), qMaxFrequency=f * 2.5,
                     qReferenceFrequency=f)
            out.append({"arrival": t, "dim": 2, "params": p})
        else:
            nx = max(24, int(r.integers(128, 257) * scale))
            ny = max(24, int(r.integers(128, 257) * scale))
            nz = max(24, int(r.integers(128, 161) * scale))
            p = dict(precision=1, nx=nx, ny=ny, nz=nz, spacing=10.0, frequency=float(r.uniform(8, 15)), cfl=0.8,
                     duration=10.0, maxSteps=max(10, int(r.integers(1000, 6001) * steps_scale / 4)),
                     sourceX=nx // 2, sourceY=ny // 2, sourceZ=6, sourceKind=1, relief=float(r.uniform(5, 20)),
                     wavelength=float(r.uniform(400, 800)), absorbing=1, absorbingCells=[10, 10, 10],
                     receiverArray=[1, 2, ny // 2, 0, min(nx - 4, 200), 1, 1, 1], receiverLimit=4096,
                     layered=1, layerDepthMode=1, layers=[50, 1200, 600, 1800, 150, 2400, 1300, 2100, 0, 3800, 2200, 2400])
            out.append({"arrival": t, "dim": 3, "params": p})
    return out
