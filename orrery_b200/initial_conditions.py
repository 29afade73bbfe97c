"""Seeded initial conditions for the workloads (synthetic inputs).

Vectorised NumPy samplers for the configurations the backend is measured on.
They restate the published sampling methods the reference's generators use
(src/initial_conditions/plummer.cpp:43-128, disc_galaxy.cpp:63-327,
galaxy_collision.cpp:59-119), with NumPy's PCG64 generator in place of the
reference's mt19937_64, so a seed gives the same distribution, not the same
bits. Units: G = 1 (include/orrery/core/units.hpp:38). All arrays FP64.

The two-disc collision uses a Hernquist bulge (the reference's generator has a
Plummer bulge); a force evaluation does not depend on which profile the
particles were drawn from.
"""
from __future__ import annotations

import math

import numpy as np


def _unit_vectors(rng, n):
    # Uniform on the sphere: height uniform in [-1, 1], azimuth in [0, 2 pi)
    # (src/core/random.cpp:31-47).
    h = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * math.pi, n)
    r = np.sqrt(1.0 - h * h)
    return np.stack([r * np.cos(phi), r * np.sin(phi), h], axis=1)


def _centre_of_mass_frame(pos, vel, m):
    mt = m.sum()
    pos -= (pos * m[:, None]).sum(axis=0) / mt
    vel -= (vel * m[:, None]).sum(axis=0) / mt
    return pos, vel


def plummer_sphere(n: int, total_mass: float = 1.0, scale_radius: float = 1.0,
                   seed: int = 20260811, cutoff: float = 0.999) -> dict:
    """Plummer sphere: radius by inverting the enclosed-mass fraction, speed by
    rejection from the distribution function q^2 (1 - q^2)^{7/2} under an
    envelope of 0.1 (plummer.cpp:43-87), isotropic directions, centre-of-mass
    frame. Returns dict x y z vx vy vz m."""
    rng = np.random.default_rng(seed)
    if n == 0:
        z = np.zeros(0)
        return dict(x=z, y=z, z=z, vx=z, vy=z, vz=z, m=z)
    frac = rng.uniform(0.0, cutoff, n)
    frac = np.maximum(frac, np.finfo(np.float64).tiny)
    r = scale_radius / np.sqrt(frac ** (-2.0 / 3.0) - 1.0)
    q = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        cand = rng.uniform(0.0, 1.0, todo.size)
        c = 1.0 - cand * cand
        g = cand * cand * c ** 3.5
        keep = 0.1 * rng.uniform(0.0, 1.0, todo.size) < g
        q[todo[keep]] = cand[keep]
        todo = todo[~keep]
    vesc = np.sqrt(2.0 * total_mass / np.sqrt(r * r + scale_radius * scale_radius))
    pos = r[:, None] * _unit_vectors(rng, n)
    vel = (q * vesc)[:, None] * _unit_vectors(rng, n)
    m = np.full(n, total_mass / n)
    pos, vel = _centre_of_mass_frame(pos, vel, m)
    return dict(x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=pos[:, 2].copy(),
                vx=vel[:, 0].copy(), vy=vel[:, 1].copy(), vz=vel[:, 2].copy(), m=m)


def _rotate(v, inclination, position_angle):
    # Tilt about x by the inclination, then turn about z by the position angle
    # (disc_galaxy.cpp:108-122).
    ci, si = math.cos(inclination), math.sin(inclination)
    ca, sa = math.cos(position_angle), math.sin(position_angle)
    y = v[:, 1] * ci - v[:, 2] * si
    z = v[:, 1] * si + v[:, 2] * ci
    return np.stack([v[:, 0] * ca - y * sa, v[:, 0] * sa + y * ca, z], axis=1)


def _exponential_radius(u):
    # Invert 1 - (1 + x) e^{-x} = u by Newton iteration (disc_galaxy.cpp:63-95
    # bisects; the root is the same).
    x = np.where(u < 0.5, np.sqrt(2.0 * u), -np.log1p(-u) + 1.0)
    for _ in range(60):
        f = 1.0 - (1.0 + x) * np.exp(-x) - u
        df = x * np.exp(-x)
        x = np.maximum(x - f / np.maximum(df, 1e-300), 1e-12)
    return x


def disc_galaxy(n: int, mass: float, bulge_fraction: float = 0.2, scale_length: float = 1.0,
                scale_height: float = 0.1, bulge_radius: float = 0.2, softening: float = 0.0,
                inclination: float = 0.0, position_angle: float = 0.0, cutoff: float = 0.99,
                rng=None) -> dict:
    """Exponential disc (radius from the enclosed-mass fraction, exponential
    vertical profile) with a Hernquist bulge; disc particles on circular orbits
    at the speed the enclosed mass supports under the softened force
    (disc_galaxy.cpp:154-181, 232-246), bulge velocities isotropic with the
    Hernquist Jeans dispersion. Returns dict x y z vx vy vz m."""
    rng = rng if rng is not None else np.random.default_rng(0)
    n_disc = max(1, min(n, int(round((1.0 - bulge_fraction) * n)))) if n else 0
    n_bulge = n - n_disc
    pm = mass / n if n else 0.0
    disc_mass = n_disc * pm
    bulge_mass = n_bulge * pm
    # Disc positions.
    rd = scale_length * _exponential_radius(rng.uniform(0.0, cutoff, n_disc))
    ang = rng.uniform(0.0, 2.0 * math.pi, n_disc)
    sign = np.where(rng.uniform(0.0, 1.0, n_disc) < 0.5, -1.0, 1.0)
    hz = -scale_height * np.log1p(-rng.uniform(0.0, 1.0, n_disc)) * sign
    disc = np.stack([rd * np.cos(ang), rd * np.sin(ang), hz], axis=1)
    # Hernquist bulge: M(<r) = M r^2 / (r + a)^2, so r = a sqrt(u) / (1 - sqrt(u)).
    a = bulge_radius
    u = rng.uniform(0.0, 0.995, n_bulge)
    su = np.sqrt(u)
    rb = a * su / (1.0 - su)
    bulge = rb[:, None] * _unit_vectors(rng, n_bulge)
    # Isotropic Jeans dispersion of a Hernquist sphere in its own potential,
    # sigma^2(r) = (1 / rho) int_r^inf rho G M(r') / r'^2 dr', tabulated.
    if n_bulge:
        grid = np.geomspace(1e-4 * a, 1e4 * a, 4000)
        rho = 1.0 / (grid * (grid + a) ** 3)
        integrand = rho * bulge_mass * grid ** 2 / (grid + a) ** 2 / grid ** 2
        seg = 0.5 * (integrand[1:] + integrand[:-1]) * np.diff(grid)
        tail = np.concatenate([np.cumsum(seg[::-1])[::-1], [0.0]])
        sigma2 = tail / rho
        s = np.sqrt(np.interp(rb, grid, sigma2))
        bvel = rng.standard_normal((n_bulge, 3)) * s[:, None]
    else:
        bvel = np.zeros((0, 3))
    pos = np.concatenate([_rotate(disc, inclination, position_angle), bulge], axis=0)
    vel = np.concatenate([np.zeros((n_disc, 3)), bvel], axis=0)
    m = np.full(n, pm)
    pos, vel = _centre_of_mass_frame(pos, vel, m)
    # Circular speeds of the disc about its spin axis.
    axis = _rotate(np.array([[0.0, 0.0, 1.0]]), inclination, position_angle)[0]
    p = pos[:n_disc]
    off = p - np.outer(p @ axis, axis)
    rad = np.linalg.norm(off, axis=1)
    frac_enc = np.minimum((1.0 - (1.0 + rad / scale_length) * np.exp(-rad / scale_length)) /
                          cutoff, 1.0)
    m_enc = disc_mass * frac_enc + bulge_mass * rad ** 2 / (rad + a) ** 2
    soft = np.sqrt(rad * rad + softening * softening)
    vc = np.sqrt(m_enc * rad * rad / np.maximum(soft ** 3, 1e-300))
    direction = np.cross(axis, off) / np.maximum(rad, 1e-300)[:, None]
    vel[:n_disc] = direction * vc[:, None]
    pos, vel = _centre_of_mass_frame(pos, vel, m)
    return dict(x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=pos[:, 2].copy(),
                vx=vel[:, 0].copy(), vy=vel[:, 1].copy(), vz=vel[:, 2].copy(), m=m)


def collision_impact_parameter(m_total: float, separation: float, approach_speed: float,
                               pericentre: float) -> float:
    """Impact parameter b giving a point-mass two-body pericentre of
    ``pericentre`` for the encounter geometry of galaxy_collision.cpp:59-85:
    separation vector (s, b, 0), relative velocity (-f v_esc, 0, 0) with
    v_esc = sqrt(2 M / |r|). Solved by bisection."""

    def peri(b):
        r = math.hypot(separation, b)
        v = approach_speed * math.sqrt(2.0 * m_total / r)
        energy = 0.5 * v * v - m_total / r
        ang = b * v
        e = math.sqrt(max(0.0, 1.0 + 2.0 * energy * ang * ang / (m_total * m_total)))
        return ang * ang / (m_total * (1.0 + e))

    lo, hi = 0.0, separation
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if peri(mid) < pericentre:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def galaxy_collision(n: int, total_mass: float = 1.0, mass_ratio: float = 1.0 / 3.0,
                     separation: float = 20.0, approach_speed: float = 0.8,
                     pericentre_scale_lengths: float = 3.0, secondary_inclination_deg=30.0,
                     softening: float = 0.02, seed: int = 20260812) -> dict:
    """Two disc galaxies with bulges, masses split by ``mass_ratio`` (secondary
    / primary) into equal-mass particles, the secondary's lengths scaled by
    sqrt(ratio) (src/sim/assembly.cpp:175-202), the secondary's disc tilted by
    ``secondary_inclination_deg``, on a bound orbit (approach speed below escape)
    whose point-mass pericentre is ``pericentre_scale_lengths`` primary scale
    lengths. Returns dict x y z vx vy vz m."""
    rng = np.random.default_rng(seed)
    n_primary = int(round(n / (1.0 + mass_ratio)))
    n_secondary = n - n_primary
    m_primary = total_mass / (1.0 + mass_ratio)
    m_secondary = total_mass * mass_ratio / (1.0 + mass_ratio)
    size = math.sqrt(mass_ratio)
    g1 = disc_galaxy(n_primary, m_primary, softening=softening, rng=rng)
    g2 = disc_galaxy(n_secondary, m_secondary, scale_length=size, scale_height=0.1 * size,
                     bulge_radius=0.2 * size, softening=softening,
                     inclination=math.radians(secondary_inclination_deg), rng=rng)
    b = collision_impact_parameter(total_mass, separation, approach_speed,
                                   pericentre_scale_lengths * 1.0)
    r = math.hypot(separation, b)
    vrel = approach_speed * math.sqrt(2.0 * total_mass / r)
    sep = np.array([separation, b, 0.0])
    rel = np.array([-vrel, 0.0, 0.0])
    out = {}
    for k, axis in (("x", 0), ("y", 1), ("z", 2)):
        out[k] = np.concatenate([g1[k] + sep[axis] * (-m_secondary / total_mass),
                                 g2[k] + sep[axis] * (m_primary / total_mass)])
        vk = "v" + k
        out[vk] = np.concatenate([g1[vk] + rel[axis] * (-m_secondary / total_mass),
                                  g2[vk] + rel[axis] * (m_primary / total_mass)])
    out["m"] = np.concatenate([g1["m"], g2["m"]])
    pos = np.stack([out["x"], out["y"], out["z"]], axis=1)
    vel = np.stack([out["vx"], out["vy"], out["vz"]], axis=1)
    pos, vel = _centre_of_mass_frame(pos, vel, out["m"])
    for a, k in enumerate(("x", "y", "z")):
        out[k] = pos[:, a].copy()
        out["v" + k] = vel[:, a].copy()
    return out


def _require_bound_orbit(primary_mass, secondary_mass, semi_major_axis, eccentricity):
    # src/initial_conditions/kepler.cpp:24-39: comparisons written so that NaN fails.
    if not (primary_mass > 0) or not (secondary_mass > 0):
        raise ValueError("A Kepler orbit needs two positive masses")
    if not (semi_major_axis > 0):
        raise ValueError("A Kepler orbit needs a positive semi-major axis")
    if not (eccentricity >= 0) or not (eccentricity < 1):
        raise ValueError("A bound Kepler orbit needs an eccentricity in [0, 1)")


def kepler_orbit(primary_mass: float = 1.0, secondary_mass: float = 1.0,
                 semi_major_axis: float = 1.0, eccentricity: float = 0.0) -> dict:
    """Two bodies on a bound Kepler orbit, at periapsis on the x axis and moving
    along y, in the centre-of-mass frame: make_kepler_orbit
    (src/initial_conditions/kepler.cpp:51-80), with the same operations in the
    same order, so the state is the reference's bit for bit."""
    _require_bound_orbit(primary_mass, secondary_mass, semi_major_axis, eccentricity)
    total = primary_mass + secondary_mass
    separation = semi_major_axis * (1 - eccentricity)           # kepler_periapsis_distance
    speed = math.sqrt(total * (1 + eccentricity) / separation)  # vis-viva at periapsis, G = 1
    primary_fraction = primary_mass / total
    secondary_fraction = secondary_mass / total
    return dict(x=np.array([-secondary_fraction * separation, primary_fraction * separation]),
                y=np.zeros(2), z=np.zeros(2), vx=np.zeros(2),
                vy=np.array([-secondary_fraction * speed, primary_fraction * speed]),
                vz=np.zeros(2), m=np.array([float(primary_mass), float(secondary_mass)]))


def kepler_period(primary_mass: float = 1.0, secondary_mass: float = 1.0,
                  semi_major_axis: float = 1.0, eccentricity: float = 0.0) -> float:
    """The orbital period 2 pi sqrt(a^3 / (G M)) (src/initial_conditions/kepler.cpp:82-88)."""
    _require_bound_orbit(primary_mass, secondary_mass, semi_major_axis, eccentricity)
    axis = semi_major_axis
    return 2 * math.pi * math.sqrt(axis * axis * axis / (primary_mass + secondary_mass))
