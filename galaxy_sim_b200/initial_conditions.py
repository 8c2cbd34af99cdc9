"""Seeded initial conditions for the gravity path.

Follows the algorithm of galaxy-sim's ``src/physics/InitialConditions.js``
(``galaxyDisk`` :83-276, ``uniformSphere`` :278-299, ``twoGalaxyCollision``
:301-363, ``kroupaIMF`` :18-37, ``sampleStar`` :56-62) with three deliberate
differences, all taken from the benchmark workloads this package is measured
on:

* every draw comes from a seeded counter-based generator (Philox) instead of
  ``Math.random``, so each workload is reproducible bit for bit;
* dynamical masses follow the Kroupa IMF rescaled to a total stellar mass
  (the reference gives every star mass 1.0), and the stellar record keeps the
  unscaled IMF mass in solar masses exactly as the reference does;
* the disk is an exponential disk (scale length ``Rd``, truncated at
  ``rmax * Rd``) with a sech^2 vertical profile (scale height ``z0``), a
  Hernquist bulge, log-spiral arm members drawn from the same exponential
  profile, and an optional central black-hole particle; rotation and
  dispersion come from the measured enclosed mass, Toomre Q and asymmetric
  drift as in the reference.

Particle layout (InitialConditions.js:1): ``[x, y, z, m, vx, vy, vz, pad]`` with
``pad = 0`` for stars and ``-1`` for gas. Stellar layout (:2):
``[stellarMass (Msun, -1 = gas), birthMyr, seed, dust]``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(seed))


def kroupa_imf(rng: np.random.Generator, n: int, m_max: float = 100.0) -> np.ndarray:
    """Kroupa (2001) inverse CDF, InitialConditions.js:18-37 (vectorised)."""
    low_int = (0.08 ** -0.3 - 0.5 ** -0.3) / 0.3
    hi_cut = max(min(m_max, 100.0), 0.5001)
    k2 = 0.5 ** (-1.3 + 2.3)
    hi_int = k2 * (0.5 ** -1.3 - hi_cut ** -1.3) / 1.3
    p_low = low_int / (low_int + hi_int)
    u = rng.random(n)
    v = rng.random(n)
    a, b = 0.08 ** -0.3, 0.5 ** -0.3
    low = (a - v * (a - b)) ** (-1.0 / 0.3)
    a2, b2 = 0.5 ** -1.3, hi_cut ** -1.3
    high = (a2 - v * (a2 - b2)) ** (-1.0 / 1.3)
    return np.where(u < p_low, low, high)


@dataclass
class Galaxy:
    """A generated particle set plus the physics parameters it was built for."""

    particles: np.ndarray            # (N, 8) float32
    stellar: np.ndarray              # (N, 4) float32
    halo_mass: float = 0.0           # per halo (Params.haloMass)
    halo_a: float = 1.0
    halo_centers: list = field(default_factory=list)
    central: tuple = (-1, -1)        # tracked black-hole particle indices
    sf_density: float = 1e9          # Params.sfDensity (particle-count density)

    @property
    def N(self) -> int:
        return self.particles.shape[0]


def galaxy_disk(N: int, seed: int, *, Rd: float = 1.0, rmax: float = 6.0, z0: float = 0.1,
                bulge_frac: float = 0.15, bulge_a: float = 0.2, arm_frac: float = 0.15,
                arms: int = 2, arm_tightness: float = 0.5, Q: float = 1.5,
                halo_factor: float = 5.0, halo_a: float = 3.0, gas_frac: float = 0.0,
                central_mass: float = 0.0, total_mass: float = 1.0, G: float = 1.0,
                sf_threshold: float = 2.5) -> Galaxy:
    """Equilibrium disk galaxy following InitialConditions.js:83-276.

    ``bulge_frac`` of the particles form the Hernquist bulge; the rest form the
    exponential disk, of which ``arm_frac`` (of all particles) are log-spiral
    arm members. ``gas_frac`` of the disk particles are gas. A central mass > 0
    adds a black-hole particle at index 0 (stellar mass 0), as the reference
    always does.
    """
    rng = _rng(seed)
    R = rmax * Rd
    has_bh = central_mass > 0.0
    i0 = 1 if has_bh else 0
    ns = N - i0
    n_bulge = int(math.floor(ns * bulge_frac))
    n_arm = int(math.floor(ns * arm_frac))
    comp = np.full(ns, 2, np.int8)              # 0 bulge, 1 arm, 2 disk
    comp[:n_bulge] = 0
    comp[n_bulge:n_bulge + n_arm] = 1

    m_imf = kroupa_imf(rng, ns)
    mass = m_imf / m_imf.sum() * total_mass

    # 1. radii (InitialConditions.js:114-137)
    radii = np.empty(ns)
    todo = np.flatnonzero(comp == 0)
    while todo.size:                             # Hernquist inverse CDF, rejection past R/2
        s = np.sqrt(rng.random(todo.size))
        r = bulge_a * s / np.maximum(1.0 - s, 1e-6)
        ok = r <= R * 0.5
        radii[todo[ok]] = r[ok]
        todo = todo[~ok]
    for c, rmin in ((1, 0.5 * Rd), (2, 0.02 * R)):
        todo = np.flatnonzero(comp == c)
        guard = 0
        while todo.size and guard < 64:           # Gamma(2, Rd) = exponential surface density
            r = -Rd * np.log(np.maximum(rng.random(todo.size), 1e-300) *
                             np.maximum(rng.random(todo.size), 1e-300))
            ok = (r <= R) & (r >= rmin)
            radii[todo[ok]] = r[ok]
            todo = todo[~ok]
            guard += 1
        if todo.size:
            radii[todo] = np.clip(-Rd * np.log(rng.random(todo.size)), rmin, R)

    # 2. measured mass profile on a radial grid (:140-163)
    NB = 256
    dr = R / NB
    b = np.minimum((radii / dr).astype(np.int64), NB - 1)
    counts = np.bincount(b, weights=mass, minlength=NB)
    m_enc = np.cumsum(counts)
    r_mid = (np.arange(NB) + 0.5) * dr
    sigma = counts / (2 * np.pi * r_mid * dr)
    sigma_s = np.array([sigma[max(0, k - 2):min(NB - 1, k + 2) + 1].mean() for k in range(NB)])

    # 3. rotation curve, epicyclic frequency, dispersions (:166-190)
    m_disk = mass[comp != 0].sum()
    halo_mass = halo_factor * m_disk
    m_halo = halo_mass * r_mid ** 2 / (r_mid + halo_a) ** 2
    vc = np.sqrt(G * (central_mass + m_enc + m_halo) / r_mid)
    omega = vc / r_mid
    k = np.arange(NB)
    b0 = np.maximum(0, k - 1)
    b1 = np.minimum(NB - 1, k + 1)
    dlnv = (np.log(vc[b1]) - np.log(vc[b0])) / np.log((b1 + 0.5) / np.maximum(b0 + 0.5, 0.01))
    kappa = np.sqrt(np.maximum(2 * omega ** 2 * (1 + dlnv), 0.1 * omega ** 2))
    sig_r = np.minimum(Q * 3.36 * G * sigma_s / kappa, 0.6 * vc)
    sig_phi = sig_r * kappa / (2 * omega)
    drift2 = sig_r ** 2 * (2 * r_mid / Rd)
    v_phi_mean = np.sqrt(np.maximum(vc ** 2 - drift2, 0.01 * vc ** 2))

    # 4. place particles (:195-266)
    g = lambda n: rng.standard_normal(n)  # noqa: E731
    theta = rng.random(ns) * 2 * np.pi
    arm_idx = np.flatnonzero(comp == 1)
    if arm_idx.size:
        arm = (np.arange(arm_idx.size) % arms)
        scatter = 0.04 + 0.09 * (radii[arm_idx] / R)
        theta[arm_idx] = (np.log(radii[arm_idx] / (0.08 * R)) / arm_tightness
                          + arm * (2 * np.pi / arms) + g(arm_idx.size) * scatter)
    cos_t, sin_t = np.cos(theta), np.sin(theta)
    x, y = radii * cos_t, radii * sin_t
    z = np.empty(ns)
    vx = np.empty(ns)
    vy = np.empty(ns)
    vz = np.empty(ns)
    gb = b.copy()

    bul = comp == 0
    nb = int(bul.sum())
    z[bul] = g(nb) * bulge_a * 0.55
    s_b = np.sqrt(G * (central_mass + m_enc[gb[bul]] * 0.5) / (3 * (radii[bul] + bulge_a)))
    v_rot = 0.35 * vc[gb[bul]]
    vx[bul] = -v_rot * sin_t[bul] + g(nb) * s_b
    vy[bul] = v_rot * cos_t[bul] + g(nb) * s_b
    vz[bul] = g(nb) * s_b * 0.8

    dsk = ~bul
    nd = int(dsk.sum())
    is_gas = np.zeros(ns, bool)
    is_gas[dsk] = rng.random(nd) < gas_frac
    u = np.clip(rng.random(nd), 1e-6, 1 - 1e-6)
    cold = np.where(is_gas[dsk], 0.5, 1.0)
    z[dsk] = z0 * np.arctanh(2 * u - 1) * np.where(is_gas[dsk], 0.6, 1.0)
    sr = sig_r[gb[dsk]] * cold
    v_r = g(nd) * sr
    v_phi = v_phi_mean[gb[dsk]] + g(nd) * sig_phi[gb[dsk]] * cold
    vx[dsk] = v_r * cos_t[dsk] - v_phi * sin_t[dsk]
    vy[dsk] = v_r * sin_t[dsk] + v_phi * cos_t[dsk]
    vz[dsk] = g(nd) * 0.5 * sr

    # stellar population (:245-256, sampleStar :56-62)
    age = np.where(comp == 0, rng.uniform(8000, 12000, ns),
                   np.where(comp == 1, rng.uniform(0, 50, ns), rng.uniform(0, 10000, ns)))
    seeds = rng.random(ns)
    dust_w = np.exp(-np.abs(z) / max(z0, 0.1))
    st = np.empty((ns, 4))
    st[:, 0] = np.where(is_gas, -1.0, m_imf)
    st[:, 1] = np.where(is_gas, 0.0, -age)
    st[:, 2] = seeds
    st[:, 3] = np.where(is_gas, 0.3 + 0.7 * dust_w, 0.0)

    P = np.zeros((N, 8), np.float32)
    S = np.zeros((N, 4), np.float32)
    P[i0:, 0], P[i0:, 1], P[i0:, 2], P[i0:, 3] = x, y, z, mass
    P[i0:, 4], P[i0:, 5], P[i0:, 6] = vx, vy, vz
    P[i0:, 7] = np.where(is_gas, -1.0, 0.0)
    S[i0:] = st
    if has_bh:                                  # particle 0 (:268-273)
        P[0, 3] = central_mass
    sf_density = sf_threshold * N / (math.pi * R * R * 2 * z0)
    return Galaxy(P, S, halo_mass=float(np.float32(halo_mass)), halo_a=halo_a,
                  halo_centers=[[0.0, 0.0, 0.0]], central=(0 if has_bh else -1, -1),
                  sf_density=float(np.float32(sf_density)))


def _rotate_x(P: np.ndarray, angle: float) -> None:
    c, s = math.cos(angle), math.sin(angle)
    for off in (0, 4):                       # position then velocity
        yy = P[:, off + 1].astype(np.float64)
        zz = P[:, off + 2].astype(np.float64)
        P[:, off + 1] = yy * c - zz * s
        P[:, off + 2] = yy * s + zz * c


def two_galaxy_collision(N: int, seed: int, *, separation: float = 30.0,
                         pericentre: float = 3.0, incl=(30.0, 60.0), bh_mass: float = 0.01,
                         G: float = 1.0, scale: float = 1.0, **disk_kw) -> Galaxy:
    """Two disks on a parabolic orbit, following InitialConditions.js:301-363.

    Each disk carries its own Hernquist halo (``halo_mass`` per halo) centred on
    the smoothed track of its central black hole (indices 0 and N/2). The
    relative orbit is the point-mass parabola with the given pericentre,
    started ``separation`` apart.
    """
    half = N // 2
    A = galaxy_disk(half, seed * 2 + 1, central_mass=bh_mass, G=G, **disk_kw)
    B = galaxy_disk(N - half, seed * 2 + 2, central_mass=bh_mass, G=G, **disk_kw)
    PA, PB = A.particles.copy(), B.particles.copy()
    _rotate_x(PA, math.radians(incl[0]))
    _rotate_x(PB, math.radians(incl[1]))
    m_gal = float(PA[:, 3].astype(np.float64).sum()) + A.halo_mass
    M = 2.0 * m_gal
    r0, q = separation * scale, pericentre * scale
    v = math.sqrt(2 * G * M / r0)
    vt = math.sqrt(2 * G * M * q) / r0
    vr = -math.sqrt(max(v * v - vt * vt, 0.0))
    rel_v = np.array([vr, vt, 0.0])
    for P, sgn in ((PA, -1.0), (PB, 1.0)):
        P[:, 0] = P[:, 0].astype(np.float64) * scale + sgn * r0 / 2
        P[:, 1] = P[:, 1].astype(np.float64) * scale
        P[:, 2] = P[:, 2].astype(np.float64) * scale
        for k in range(3):
            P[:, 4 + k] = P[:, 4 + k].astype(np.float64) + sgn * rel_v[k] / 2
    P = np.concatenate([PA, PB]).astype(np.float32)
    S = np.concatenate([A.stellar, B.stellar]).astype(np.float32)
    centers = [P[0, :3].astype(np.float64).tolist(), P[half, :3].astype(np.float64).tolist()]
    return Galaxy(P, S, halo_mass=A.halo_mass, halo_a=A.halo_a * scale, halo_centers=centers,
                  central=(0, half), sf_density=A.sf_density)


def hernquist_sphere(N: int, seed: int, *, a: float = 1.0, rtrunc: float = 20.0,
                     total_mass: float = 1.0) -> Galaxy:
    """Cold Hernquist sphere (zero velocities, like uniformSphere :278-299)."""
    rng = _rng(seed)
    r = np.empty(N)
    todo = np.arange(N)
    while todo.size:
        s = np.sqrt(rng.random(todo.size))
        rr = a * s / np.maximum(1.0 - s, 1e-9)
        ok = rr <= rtrunc * a
        r[todo[ok]] = rr[ok]
        todo = todo[~ok]
    cz = rng.uniform(-1, 1, N)
    ph = rng.uniform(0, 2 * np.pi, N)
    sz = np.sqrt(1 - cz * cz)
    m_imf = kroupa_imf(rng, N)
    P = np.zeros((N, 8), np.float32)
    P[:, 0], P[:, 1], P[:, 2] = r * sz * np.cos(ph), r * sz * np.sin(ph), r * cz
    P[:, 3] = m_imf / m_imf.sum() * total_mass
    S = np.zeros((N, 4), np.float32)
    S[:, 0] = m_imf
    S[:, 1] = -rng.uniform(0, 5000, N)
    S[:, 2] = rng.random(N)
    return Galaxy(P, S, halo_mass=0.0, halo_a=1.0, halo_centers=[], central=(-1, -1))


# ---- the benchmark workloads ------------------------------------------------------------

def disk_16k(seed: int = 0) -> Galaxy:
    """Single disk N=16384: Q=1.5, 2 arms, no gas (eps 0.05, theta 0.5, dt 0.005)."""
    return galaxy_disk(16384, seed, Q=1.5, arms=2, gas_frac=0.0)


def disk_512k(seed: int = 1, N: int = 524288) -> Galaxy:
    """Single disk N=524288: Q=1.2, 4 arms, 30% gas with drag and star formation."""
    return galaxy_disk(N, seed, Q=1.2, arms=4, gas_frac=0.3)


def collision_2x256k(seed: int = 2, N: int = 524288) -> Galaxy:
    """Two disks of N/2 with 0.01 black holes, 30 Rd apart, pericentre 3 Rd."""
    return two_galaxy_collision(N, seed, Q=1.5, arms=2, gas_frac=0.0)
