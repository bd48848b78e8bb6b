"""Seeded synthetic inputs for the ionosphere potential solve.

The polar-cap workload: a colatitude-longitude node grid per hemisphere,
theta-major with longitude contiguous (the layout of
nonorthogonal/src/nonorthogonal/nonorthogonal_mi.h:74-83), colatitude 0 to
``max_colatitude_deg``.  Pedersen conductance is a seeded smooth field in
[2, 20] S plus a Gaussian ridge along an auroral oval; Hall conductance is a
multiple of it; the field-aligned current is a Region-1/Region-2 pattern of
amplitude 1 uA/m^2 plus seeded uniform noise.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import abi
from .abi import MiSolverConfig

NORTH = 1
SOUTH = -1


@dataclass
class MiCase:
    config: MiSolverConfig
    fac: np.ndarray          # A/m^2, (nt, np)
    pedersen: np.ndarray     # S, (nt, np)
    hall: np.ndarray         # S, (nt, np)
    potential: np.ndarray    # V, (nt, np) initial guess


def mi_config(longitudes: int, colatitudes: int, max_colatitude_deg: float = 45.0,
              hemisphere: int = NORTH, pedersen_siemens: float = 5.0,
              hall_siemens: float = 0.0, radius_m: float = 6.371e6,
              low_latitude_potential_v: float = 0.0, max_iterations: int = 20000,
              rel_tol: float = 1e-8, abs_tol: float = 0.0) -> MiSolverConfig:
    c = MiSolverConfig()
    c.longitude_count = longitudes
    c.colatitude_count = colatitudes
    c.maximum_colatitude = math.radians(max_colatitude_deg)
    c.ionosphere_radius_m = radius_m
    c.pedersen_siemens = pedersen_siemens
    c.hall_siemens = hall_siemens
    c.low_latitude_potential_v = low_latitude_potential_v
    c.hemisphere = hemisphere
    c.maximum_iterations = max_iterations
    c.relative_tolerance = rel_tol
    c.absolute_tolerance = abs_tol
    return c


def mi_case(longitudes: int = 361, colatitudes: int = 181, seed: int = 7,
            hemisphere: int = NORTH, max_colatitude_deg: float = 45.0,
            hall_ratio: float = 1.5, **config_kw) -> MiCase:
    """Region-1/2 currents over an auroral-oval conductance (seeded)."""
    rng = np.random.default_rng(seed + (0 if hemisphere == NORTH else 1000003))
    nt, npl = colatitudes, longitudes
    theta = np.linspace(0.0, math.radians(max_colatitude_deg), nt)[:, None]
    phi = (2.0 * math.pi / npl) * np.arange(npl)[None, :]
    # Smooth seeded background: low-order Fourier modes in longitude with a
    # slow colatitude envelope, mapped into [2, 14] S.
    smooth = np.zeros((nt, npl))
    for m in range(0, 5):
        for q in range(1, 4):
            a = rng.uniform(-1.0, 1.0) / (1.0 + m + q)
            ph = rng.uniform(0.0, 2.0 * math.pi)
            smooth += a * np.cos(m * phi + ph) * np.sin(q * math.pi * theta /
                                                        (2.0 * theta[-1, 0]) + ph)
    smooth = (smooth - smooth.min()) / max(smooth.max() - smooth.min(), 1e-30)
    oval = math.radians(20.0) + math.radians(3.0) * np.cos(phi)
    width = math.radians(2.5)
    ridge = np.exp(-((theta - oval) / width) ** 2)
    pedersen = np.clip(2.0 + 12.0 * smooth + 8.0 * ridge, 2.0, 20.0)
    hall = hall_ratio * pedersen
    r1 = np.exp(-((theta - (oval - math.radians(1.5))) / math.radians(1.2)) ** 2)
    r2 = np.exp(-((theta - (oval + math.radians(1.5))) / math.radians(1.2)) ** 2)
    fac = 1e-6 * np.sin(phi) * (r1 - r2)
    fac = fac + 0.05e-6 * rng.uniform(-1.0, 1.0, size=(nt, npl))
    cfg = mi_config(npl, nt, max_colatitude_deg, hemisphere, **config_kw)
    potential = np.zeros((nt, npl))
    return MiCase(cfg, np.ascontiguousarray(fac), np.ascontiguousarray(pedersen),
                  np.ascontiguousarray(hall), potential)


def mi_dipole_config(azimuth=192, colatitude=22, shell=1, max_iterations=4000):
    """The reference Earth driver's coupling configuration
    (cubedsphere/tests/test_cubedsphere_dipole_background.c:512-518):
    192 x 22 per hemisphere, FAC shell 1, R_I = 1 R_E, 5 S, 10 s cadence,
    Earth normalisation (1 R_E, 100 km/s, 1 proton cm^-3), rel. tol. 1e-8."""
    c = abi.MiDipoleConfig()
    c.azimuth_points = azimuth
    c.colatitude_points = colatitude
    c.current_shell = shell
    c.ionosphere_radius_re = 1.0
    c.pedersen_siemens = 5.0
    c.coupling_interval_s = 10.0
    c.length_norm_m = 6371000.0
    c.speed_norm_m_s = 100000.0
    c.mass_density_norm_kg_m3 = 1.67262192369e-21
    c.maximum_iterations = max_iterations
    c.relative_tolerance = 1e-8
    return c


def earth_startup():
    """Earth startup of the reference driver
    (test_cubedsphere_dipole_background.c:282-294): inner radius 2.5 R_E,
    n = 5, V = 4 (400 km/s), Mach 10, front at x = -30, dipole cut at
    16 +- 8 R_E, moment (0, 0, -6761.73) (0.31 G equatorial surface field)."""
    s = abi.EarthStartup()
    s.inner_radius = 2.5
    s.density = 5.0
    s.speed = 4.0
    s.mach = 10.0
    s.gamma = 5.0 / 3.0
    s.ambient_density = 1.0
    s.ambient_pressure = 0.001
    s.front_x = -30.0
    s.front_width = 1.5
    s.cut_radius = 16.0
    s.cut_length = 8.0
    s.dipole.moment.value[2] = -6761.730688424097
    return s
