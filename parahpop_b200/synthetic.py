"""Seeded synthetic environment and object populations in ParaHPOP's file formats.

The reference ships no environment data (its ``data/local`` tree is not
distributed), so every run here uses files generated by this module.  They are
written in exactly the formats the reference loaders read, so the same files
feed the reference CPU backend, the CPU oracle and this package:

* ``gravity.tab``   PDS-SHA text table, header ``R, GM, sigmaGM, N, N, 1, 0, 0``
                    then rows ``n, m, C, S, 0, 0`` for n >= 1 (no n = 0 row);
                    read by ``IF/config/model/sphericalharmonics/Coefficients.h:241-362``.
* ``bodies.brie``   CBOR layout 1 ``{"layout":1,"core":[unit...]}`` with Type-2
                    Chebyshev position units (``brie/states/metadata/EphUnit.h:55-86``);
                    data ``[radius, starts..., X..., Y..., Z...]``, coefficient j of
                    interval k at ``k + j*n`` (``brie/core/Type2BodyUnit.h:47-60``).
* ``earth.brot2``   CBOR layout 1 with one unit_type 4 (IERS2000 model + Lagrange
                    tables) unit for target 3001 (``brie/orientations/metadata/EphUnit.cpp:148-167``,
                    ``brie/orientations/detail/LagrangeInterp.h:88-110``).
* ``SW-All.txt``    CelesTrak space-weather rows (``Nrlmsise00Atmosphere.h:168-189``).
* ``EOP-All.txt``   HPOP EOP rows ``Y M D MJD xp yp UT1-UTC LOD dpsi deps dx dy TAI-UTC``
                    (``earthcorrections/EarthCorrections.h:142-177``).
* ``constants.json`` the reference's constants schema (``data/constants.json``).

Workload shapes follow the benchmark configurations: seeded Keplerian LEO /
MEO / GEO populations, a Kaula-rule degree/order 70 or 120 field, Sun / Moon /
Jupiter two-body Chebyshev ephemerides, constant EOP and space weather.
"""
from __future__ import annotations

import json
import math
import os
import struct
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

MU_ELEMENTS = 398600.4418  # km^3/s^2, element -> state conversion only
R_EARTH = 6378.137
EPOCH0 = 4035.0            # MJD2000 TDB, 2011-01-18
TAI_UTC_2011 = 34.0
AU_KM = 149597870.7
SECONDS_PER_DAY = 86400.0


# --------------------------------------------------------------------------
# Minimal CBOR encoder (RFC 8949 subset: maps, arrays, ints, doubles, text)
# --------------------------------------------------------------------------
def _cbor_head(major: int, value: int) -> bytes:
    if value < 24:
        return bytes([(major << 5) | value])
    if value < 256:
        return bytes([(major << 5) | 24, value])
    if value < 65536:
        return bytes([(major << 5) | 25]) + struct.pack(">H", value)
    if value < 2 ** 32:
        return bytes([(major << 5) | 26]) + struct.pack(">I", value)
    return bytes([(major << 5) | 27]) + struct.pack(">Q", value)


def cbor_dumps(obj) -> bytes:
    if isinstance(obj, bool):
        return bytes([0xF5 if obj else 0xF4])
    if isinstance(obj, (int, np.integer)):
        v = int(obj)
        return _cbor_head(0, v) if v >= 0 else _cbor_head(1, -1 - v)
    if isinstance(obj, (float, np.floating)):
        return b"\xfb" + struct.pack(">d", float(obj))
    if isinstance(obj, str):
        b = obj.encode()
        return _cbor_head(3, len(b)) + b
    if isinstance(obj, np.ndarray):
        obj = obj.tolist()
    if isinstance(obj, (list, tuple)):
        return _cbor_head(4, len(obj)) + b"".join(cbor_dumps(x) for x in obj)
    if isinstance(obj, dict):
        out = [_cbor_head(5, len(obj))]
        for k, v in obj.items():
            out.append(cbor_dumps(k))
            out.append(cbor_dumps(v))
        return b"".join(out)
    raise TypeError(type(obj))


# --------------------------------------------------------------------------
# Time helpers
# --------------------------------------------------------------------------
def mjd2000_to_et(mjd: float) -> float:
    """MJD2000 -> SPICE ET seconds (``IF/util/TimeConversion.h:30-33``)."""
    return mjd * SECONDS_PER_DAY - 43200.0


def calendar(mjd_full: float):
    """Modified Julian Date -> (year, month, day) (Fliegel-Van Flandern)."""
    jd = int(math.floor(mjd_full)) + 2400001
    l = jd + 68569
    n = 4 * l // 146097
    l = l - (146097 * n + 3) // 4
    i = 4000 * (l + 1) // 1461001
    l = l - 1461 * i // 4 + 31
    j = 80 * l // 2447
    d = l - 2447 * j // 80
    l = j // 11
    m = j + 2 - 12 * l
    y = 100 * (n - 49) + i + l
    return y, m, d


# --------------------------------------------------------------------------
# Keplerian elements -> Cartesian states
# --------------------------------------------------------------------------
def kepler_to_state(a, e, inc, raan, argp, M, mu=MU_ELEMENTS):
    """Vectorised element -> ICRF state conversion (km, km/s)."""
    a, e, inc, raan, argp, M = map(np.asarray, (a, e, inc, raan, argp, M))
    E = M.copy()
    for _ in range(50):
        E = E - (E - e * np.sin(E) - M) / (1.0 - e * np.cos(E))
    cE, sE = np.cos(E), np.sin(E)
    fac = np.sqrt(1.0 - e * e)
    r = a * (1.0 - e * cE)
    x_p = a * (cE - e)
    y_p = a * fac * sE
    n = np.sqrt(mu / a ** 3)
    vx_p = -a * n * sE / (1.0 - e * cE)
    vy_p = a * n * fac * cE / (1.0 - e * cE)
    cO, sO = np.cos(raan), np.sin(raan)
    cw, sw = np.cos(argp), np.sin(argp)
    ci, si = np.cos(inc), np.sin(inc)
    R11 = cO * cw - sO * sw * ci
    R12 = -cO * sw - sO * cw * ci
    R21 = sO * cw + cO * sw * ci
    R22 = -sO * sw + cO * cw * ci
    R31 = sw * si
    R32 = cw * si
    pos = np.stack([R11 * x_p + R12 * y_p, R21 * x_p + R22 * y_p, R31 * x_p + R32 * y_p], -1)
    vel = np.stack([R11 * vx_p + R12 * vy_p, R21 * vx_p + R22 * vy_p, R31 * vx_p + R32 * vy_p], -1)
    del r
    return np.concatenate([pos, vel], -1)


# --------------------------------------------------------------------------
# Populations
# --------------------------------------------------------------------------
@dataclass
class Population:
    """Seeded object set in the reference's target schema."""
    ids: np.ndarray
    epochs: np.ndarray           # MJD2000 TDB
    states: np.ndarray           # (n, 6) km, km/s
    mass: np.ndarray             # kg
    drag_area: np.ndarray        # m^2
    srp_area: np.ndarray         # m^2
    cd: np.ndarray
    cr: np.ndarray
    duration: np.ndarray | None = None   # s, per object (mixed populations)
    step: np.ndarray | None = None       # s, per object (mixed populations)
    seed: int = 0
    note: str = ""

    def __len__(self):
        return len(self.ids)

    def subset(self, idx):
        idx = np.asarray(idx)
        pick = lambda a: None if a is None else a[idx]
        return Population(self.ids[idx], self.epochs[idx], self.states[idx], self.mass[idx],
                          self.drag_area[idx], self.srp_area[idx], self.cd[idx], self.cr[idx],
                          pick(self.duration), pick(self.step), self.seed, self.note)

    def targets_json(self) -> dict:
        out = []
        for i in range(len(self)):
            t = {"id": int(self.ids[i]), "epoch_mjd2000_tdb": float(self.epochs[i]),
                 "state_km_km_s": [float(x) for x in self.states[i]],
                 "mass_kg": float(self.mass[i]), "drag_area_m2": float(self.drag_area[i]),
                 "srp_area_m2": float(self.srp_area[i]), "cd": float(self.cd[i]), "cr": float(self.cr[i])}
            if self.duration is not None:
                t["duration_seconds"] = float(self.duration[i])
            if self.step is not None:
                t["step_seconds"] = float(self.step[i])
            out.append(t)
        return {"description": self.note, "targets": out}


def _loguniform(rng, lo, hi, n):
    return np.exp(rng.uniform(math.log(lo), math.log(hi), n))


# Rough thermosphere (F10.7 = 150) for screening decay: (altitude km, density
# kg/m^3, scale height km).  Only used to keep objects that would re-enter
# during the run out of the population: the reference driver rejects a run in
# which any object ends non-finite ("Nonfinite final state").
_ATM = [(150, 2.0e-9, 22), (200, 2.8e-10, 37), (250, 7.2e-11, 45), (300, 2.4e-11, 53), (350, 9.5e-12, 53),
        (400, 4.0e-12, 58), (450, 1.8e-12, 60), (500, 8.5e-13, 63), (600, 2.2e-13, 71), (700, 6.5e-14, 88),
        (800, 2.2e-14, 124), (900, 9.5e-15, 181), (1000, 5.0e-15, 268)]


def _density(h):
    h = np.asarray(h, dtype=float)
    out = np.zeros_like(h)
    for k in range(len(_ATM)):
        lo = _ATM[k][0]
        hi = _ATM[k + 1][0] if k + 1 < len(_ATM) else 1e9
        m = (h >= lo) & (h < hi)
        out[m] = _ATM[k][1] * np.exp(-(h[m] - lo) / _ATM[k][2])
    out[h < _ATM[0][0]] = _ATM[0][1]
    return out


def decay_km(a_km, e, cd, area_m2, mass_kg, duration_s):
    """Semi-major-axis decay estimate (km) over ``duration_s`` at perigee density."""
    hp = a_km * (1 - e) - R_EARTH
    B = cd * area_m2 / mass_kg
    a = a_km * 1e3
    per_rev = 2 * np.pi * B * _density(hp) * a * a
    revs = duration_s / (2 * np.pi * np.sqrt(a ** 3 / (MU_ELEMENTS * 1e9)))
    return per_rev * revs * 1e-3


def _screen_decay(rng, a, e, mass, area, srp, cd, duration, limit_km=25.0):
    """Redraw mass and areas of objects whose decay over ``duration`` would
    exceed ``limit_km`` (they would re-enter and end non-finite)."""
    for _ in range(100):
        bad = decay_km(a, e, cd, area, mass, duration) > limit_km
        if not bad.any():
            break
        k = int(bad.sum())
        mass[bad] = _loguniform(rng, 100.0, 8000.0, k)
        area[bad] = _loguniform(rng, 1.0, 50.0, k)
        srp[bad] = _loguniform(rng, 1.0, 50.0, k)
    bad = decay_km(a, e, cd, area, mass, duration) > limit_km
    mass[bad], area[bad] = 8000.0, 1.0
    return mass, area, srp


def population_central(n=1024, seed=0):
    """Central-gravity population: a = R + U(300,1200) km, e ~ U(0,0.01)."""
    rng = np.random.default_rng(seed)
    a = R_EARTH + rng.uniform(300.0, 1200.0, n)
    e = rng.uniform(0.0, 0.01, n)
    inc = np.radians(rng.uniform(0.0, 180.0, n))
    raan, argp, M = (np.radians(rng.uniform(0.0, 360.0, n)) for _ in range(3))
    st = kepler_to_state(a, e, inc, raan, argp, M)
    return Population(np.arange(1, n + 1), np.full(n, EPOCH0), st, np.full(n, 1000.0),
                      np.full(n, 10.0), np.full(n, 10.0), np.full(n, 2.2), np.full(n, 1.3),
                      seed=seed, note=f"central LEO population, n={n}, seed={seed}")


def population_leo(n=10000, seed=1, alt=(300.0, 2000.0), screen_duration=86400.0):
    """Full-force LEO population with log-uniform mass and areas; objects that
    would decay more than 25 km within ``screen_duration`` get new mass and
    areas (see ``_screen_decay``)."""
    rng = np.random.default_rng(seed)
    a = R_EARTH + rng.uniform(alt[0], alt[1], n)
    e = rng.uniform(0.0, 0.01, n)
    # keep perigee above 200 km so no object re-enters within a day
    e = np.minimum(e, np.maximum(0.0, 1.0 - (R_EARTH + 200.0) / a))
    inc = np.radians(rng.uniform(0.0, 180.0, n))
    raan, argp, M = (np.radians(rng.uniform(0.0, 360.0, n)) for _ in range(3))
    st = kepler_to_state(a, e, inc, raan, argp, M)
    mass = _loguniform(rng, 100.0, 8000.0, n)
    ad = _loguniform(rng, 1.0, 50.0, n)
    asrp = _loguniform(rng, 1.0, 50.0, n)
    if screen_duration:
        mass, ad, asrp = _screen_decay(rng, a, e, mass, ad, asrp, np.full(n, 2.2), screen_duration)
    return Population(np.arange(1, n + 1), np.full(n, EPOCH0), st, mass, ad, asrp,
                      np.full(n, 2.2), np.full(n, 1.3), seed=seed,
                      note=f"full-force LEO population, n={n}, seed={seed}")


def population_lunar(n=16, seed=17, epoch=4035.0):
    """Objects on low lunar orbits (1,900-2,600 km from the Moon's centre,
    circular about the Moon, random planes), as geocentric states at one
    epoch from the synthetic Moon path."""
    rng = np.random.default_rng(seed)
    fns = body_functions()
    h = 1e-3
    moon = fns["moon"](epoch)
    moon_v = (fns["moon"](epoch + h) - fns["moon"](epoch - h)) / (2 * h * SECONDS_PER_DAY)
    gm_moon = 4902.800192171393
    states = np.zeros((n, 6))
    for i in range(n):
        r = rng.uniform(1900.0, 2600.0)
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        w = np.cross(u, rng.normal(size=3))
        w /= np.linalg.norm(w)
        states[i, :3] = moon + r * u
        states[i, 3:] = moon_v + math.sqrt(gm_moon / r) * np.cross(w, u)
    ids = np.arange(1, n + 1)
    return Population(ids, np.full(n, epoch), states, rng.uniform(500.0, 2000.0, n), rng.uniform(2.0, 10.0, n),
                      rng.uniform(2.0, 10.0, n), np.full(n, 2.2), np.full(n, 1.3), seed=seed,
                      note="low lunar orbits, geocentric states")


def population_mixed(n=1000000, seed=3):
    """Uneven population: 70% LEO (30 s), 20% MEO (120 s), 10% GEO/GTO (300 s);
    epochs U(-10,+10) d around MJD2000 4035; durations log-uniform 1 h - 7 d."""
    rng = np.random.default_rng(seed)
    kind = rng.choice(3, size=n, p=[0.7, 0.2, 0.1])
    a = np.empty(n); e = np.empty(n); step = np.empty(n)
    m0 = kind == 0; m1 = kind == 1; m2 = kind == 2
    a[m0] = R_EARTH + rng.uniform(300.0, 2000.0, m0.sum()); e[m0] = rng.uniform(0, 0.02, m0.sum()); step[m0] = 30.0
    a[m1] = rng.uniform(20000.0, 27000.0, m1.sum()); e[m1] = rng.uniform(0, 0.05, m1.sum()); step[m1] = 120.0
    a[m2] = rng.uniform(24000.0, 42164.0, m2.sum()); e[m2] = rng.uniform(0, 0.7, m2.sum()); step[m2] = 300.0
    # perigee above 250 km for every orbit class
    e = np.minimum(e, np.maximum(0.0, 1.0 - (R_EARTH + 250.0) / a))
    inc = np.radians(rng.uniform(0.0, 180.0, n))
    raan, argp, M = (np.radians(rng.uniform(0.0, 360.0, n)) for _ in range(3))
    st = kepler_to_state(a, e, inc, raan, argp, M)
    mass = _loguniform(rng, 100.0, 8000.0, n)
    ad = _loguniform(rng, 1.0, 50.0, n)
    asrp = _loguniform(rng, 1.0, 50.0, n)
    epochs = EPOCH0 + rng.uniform(-10.0, 10.0, n)
    dur = _loguniform(rng, 3600.0, 7 * 86400.0, n)
    mass, ad, asrp = _screen_decay(rng, a, e, mass, ad, asrp, np.full(n, 2.2), dur)
    return Population(np.arange(1, n + 1), epochs, st, mass, ad, asrp, np.full(n, 2.2), np.full(n, 1.3),
                      duration=dur, step=step, seed=seed,
                      note=f"mixed LEO/MEO/GEO population, n={n}, seed={seed}")


# --------------------------------------------------------------------------
# Environment
# --------------------------------------------------------------------------
@dataclass
class EnvSpec:
    degree: int = 70
    seed: int = 7
    start_mjd: float = 4016.0     # coverage, MJD2000 TDB
    end_mjd: float = 4064.0
    gm_tab: float = 398600.4415   # GGM03C header values
    r_tab: float = 6378.1363
    zonal_only: bool = False      # J2-J6 zonal field for the light serving requests
    force: str = "full"           # "full" | "central" | "sh" | "zonal"
    bodies: list = field(default_factory=lambda: ["Sun", "Moon", "JupiterBarycenter"])
    tides: bool = True
    relativity: bool = True
    drag: bool = True
    srp: bool = True
    ephemeris_type: int = 2       # 2: Chebyshev positions; 3: positions and velocities (6 blocks)
    ephemeris_chain: str = "direct"  # "direct": Earth, Sun, Jupiter -> SSB, Moon -> Earth; "emb": DE440's
                                     # Earth and Moon -> Earth-Moon barycenter (3) -> SSB
    brie_layout: int = 1          # CBOR layout of bodies.brie and earth.brot2 (1: unit list; 2: member arrays)
    ephemeris_files: int = 1      # 2: Sun, Earth and Moon in bodies.brie; Jupiter and a displaced duplicate
                                  # Moon unit (which the first file's unit must shadow) in bodies2.brie
    earth_frame: str = "iers"     # earth.brot2 holds: "iers" the IERS2000 model unit (3001), "itrf93" a binary
                                  # Chebyshev Euler-angle unit (3000, ECLIPJ2000-based), "both" the two, "iau"
                                  # an IAU body model (399) with barycentric nutation-precession terms
    moon_frame: bool = False      # earth.brot2 also holds an IAU body model of the Moon (301)
    moon_field: int = 0           # degree of a synthetic lunar field written to moon.tab (0: none)


def kaula_field(degree, seed, zonal_only=False):
    """Normalized Cnm/Snm: C20 = -4.841695e-4, others N(0,(1e-5/n^2)^2)."""
    rng = np.random.default_rng(seed)
    C = np.zeros((degree + 1, degree + 1)); S = np.zeros((degree + 1, degree + 1))
    for n in range(2, degree + 1):
        sig = 1e-5 / n ** 2
        C[n, :n + 1] = rng.normal(0.0, sig, n + 1)
        S[n, 1:n + 1] = rng.normal(0.0, sig, n)
    C[2, 0] = -4.841695e-4
    if zonal_only:
        C[:, 1:] = 0.0
        S[:] = 0.0
        # J2..J6-like zonals
        C[2, 0] = -4.841695e-4; C[3, 0] = 9.57e-7; C[4, 0] = 5.40e-7; C[5, 0] = 6.87e-8; C[6, 0] = -1.50e-7
    return C, S


def write_tab(path, C, S, gm, r, degree):
    with open(path, "w") as f:
        f.write(f"{r:.10f}, {gm:.10f}, 0.0, {degree}, {degree}, 1, 0, 0\n")
        for n in range(1, degree + 1):
            for m in range(n + 1):
                f.write(f"{n}, {m}, {C[n, m]:.17e}, {S[n, m]:.17e}, 0.0, 0.0\n")


def _rot_x(a):
    c, s = math.cos(a), math.sin(a)
    return np.array([[1, 0, 0], [0, c, -s], [0, s, c]])


def _rot_z(a):
    c, s = math.cos(a), math.sin(a)
    return np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])


def circular_orbit(t_days, radius, period_days, inc, raan, phase0):
    """Position (km) on a circular orbit, inertial frame."""
    th = phase0 + 2 * math.pi * np.asarray(t_days) / period_days
    p = np.stack([radius * np.cos(th), radius * np.sin(th), np.zeros_like(th)], -1)
    R = _rot_z(raan) @ _rot_x(inc)
    return p @ R.T


OBLIQUITY = math.radians(23.439291)


def body_functions():
    """Barycentric / geocentric two-body paths (t in days from MJD2000 0)."""
    ecl = _rot_x(OBLIQUITY)

    def earth_ssb(t):     # Earth around the SSB: 1 AU, 365.25 d, ecliptic
        return circular_orbit(t, AU_KM, 365.25, 0.0, 0.0, 1.75) @ ecl.T

    def sun_ssb(t):       # small reflex motion of the Sun about the SSB
        return circular_orbit(t, 7.4e5, 4332.59, 0.0, 0.0, 0.3) @ ecl.T

    def moon_earth(t):    # Moon about the Earth: 384400 km, 27.32 d, i = 5.1 deg to the ecliptic
        return circular_orbit(t, 384400.0, 27.32, math.radians(5.1), 2.1, 0.4) @ ecl.T

    def jupiter_ssb(t):   # Jupiter barycenter: 5.2 AU, 4332.59 d
        return circular_orbit(t, 5.2 * AU_KM, 4332.59, math.radians(1.3), 1.75, 3.4) @ ecl.T

    return {"earth": earth_ssb, "sun": sun_ssb, "moon": moon_earth, "jupiter": jupiter_ssb}


def cheb_unit(fn, target, center, start_mjd, end_mjd, seg_days, pdeg=13, dtype=2):
    """Fit a Chebyshev unit to ``fn`` over [start, end): Type 2 holds the
    position coefficients (X, Y, Z blocks); Type 3 adds velocity blocks (VX,
    VY, VZ: the time derivative of the position fit, km/s, padded to the same
    degree), as ``brie/core/Type3BodyUnit.h`` reads them."""
    nint = int(math.ceil((end_mjd - start_mjd) / seg_days))
    radius = seg_days * SECONDS_PER_DAY / 2.0
    starts = [mjd2000_to_et(start_mjd + k * seg_days) for k in range(nint)]
    npts = pdeg + 1
    xk = np.cos(np.pi * (np.arange(npts) + 0.5) / npts)  # Chebyshev nodes in [-1,1]
    coef = np.zeros((3, pdeg + 1, nint))
    for k in range(nint):
        mid = start_mjd + (k + 0.5) * seg_days
        t = mid + xk * seg_days / 2.0
        P = fn(t)
        for d in range(3):
            coef[d, :, k] = np.polynomial.chebyshev.chebfit(xk, P[:, d], pdeg)
    data = [radius] + starts
    for d in range(3):
        data += coef[d].reshape(-1).tolist()  # index k + j*n
    if dtype == 3:
        for d in range(3):
            vel = np.zeros((pdeg + 1, nint))
            for k in range(nint):
                vel[:pdeg, k] = np.polynomial.chebyshev.chebder(coef[d, :, k]) / radius
            data += vel.reshape(-1).tolist()
    meta = {"frame": 1, "dtype": dtype, "target": target, "center": center, "nintervals": nint,
            "pdeg": pdeg, "startEpoch": starts[0], "finalEpoch": starts[0] + nint * 2 * radius}
    return {"metadata": meta, "data": data}


STATE_INT_KEYS = ("frame", "dtype", "target", "center", "nintervals", "pdeg")
ORIENTATION_INT_KEYS = {4: ("unit_type", "target", "model_id", "interp_id", "n_nodes_nut", "n_nodes_erp",
                            "lag_order_nut", "lag_order_erp", None, None),
                        3: ("unit_type", "frameClassID", "inertialFrame", "dtype", "nintervals", "pdeg",
                            None, None, None, None),
                        1: ("unit_type", "target", "pdeg_ra", "pdeg_dec", "pdeg_pm", "num_dims_radii",
                            "barycenter", "num_np_terms_ra", "num_np_terms_dec", "num_np_terms_pm"),
                        2: ("unit_type", "target", "pdeg_np", "num_np_angles", None, None, None, None, None, None)}


def brie_layout2(units, int_keys) -> dict:
    """Layout-2 form of a unit list: the reader's member arrays written out
    member-major (member k of unit i at k * n + i), each unit's data offset
    and size as the last two integer members, then the start and final
    epochs as the real members, over one concatenated data array."""
    n = len(units)
    width = len(next(iter(int_keys.values()))) if isinstance(int_keys, dict) else len(int_keys)
    cols = [[] for _ in range(width + 2)]
    data = []
    for u in units:
        keys = int_keys[u["metadata"]["unit_type"]] if isinstance(int_keys, dict) else int_keys
        for q, k in enumerate(keys):
            cols[q].append(int(u["metadata"][k]) if k else 0)
        cols[-2].append(len(data))
        cols[-1].append(len(u["data"]))
        data += [float(x) for x in u["data"]]
    return {"layout": 2, "core": {"metadata": {
        "nBodyUnits": n, "intMetadata": [v for c in cols for v in c],
        "doubleMetadata": [float(u["metadata"]["startEpoch"]) for u in units]
        + [float(u["metadata"]["finalEpoch"]) for u in units]}, "data": data}}


def write_brie_split(path1, path2, start_mjd, end_mjd):
    """The direct-chain units over two files: Sun, Earth and Moon in the
    first; Jupiter and a Moon unit displaced by 20,000 km in the second, which
    a reader that keeps the first file's unit for a body ignores."""
    f = body_functions()
    first = [cheb_unit(f["sun"], 10, 0, start_mjd, end_mjd, 8.0), cheb_unit(f["earth"], 399, 0, start_mjd, end_mjd, 8.0),
             cheb_unit(f["moon"], 301, 399, start_mjd, end_mjd, 4.0)]
    second = [cheb_unit(f["jupiter"], 5, 0, start_mjd, end_mjd, 32.0),
              cheb_unit(lambda t: f["moon"](t) + 20000.0, 301, 399, start_mjd, end_mjd, 4.0)]
    for path, units in ((path1, first), (path2, second)):
        with open(path, "wb") as fh:
            fh.write(cbor_dumps({"layout": 1, "core": units}))


def write_brie(path, start_mjd, end_mjd, dtype=2, chain="direct", layout=1):
    f = body_functions()
    if chain == "emb":
        # DE440's layout: the Earth-Moon barycenter about the SSB, the Earth
        # and the Moon about the barycenter (mass ratio from the constants)
        k = 4902.800192171393 / (398600.4415 + 4902.800192171393)
        units = [
            cheb_unit(f["sun"], 10, 0, start_mjd, end_mjd, 8.0, dtype=dtype),
            cheb_unit(lambda t: f["earth"](t) + k * f["moon"](t), 3, 0, start_mjd, end_mjd, 8.0, dtype=dtype),
            cheb_unit(lambda t: -k * f["moon"](t), 399, 3, start_mjd, end_mjd, 4.0, dtype=dtype),
            cheb_unit(lambda t: (1.0 - k) * f["moon"](t), 301, 3, start_mjd, end_mjd, 4.0, dtype=dtype),
            cheb_unit(f["jupiter"], 5, 0, start_mjd, end_mjd, 32.0, dtype=dtype),
        ]
    else:
        units = [
            cheb_unit(f["sun"], 10, 0, start_mjd, end_mjd, 8.0, dtype=dtype),
            cheb_unit(f["earth"], 399, 0, start_mjd, end_mjd, 8.0, dtype=dtype),
            cheb_unit(f["moon"], 301, 399, start_mjd, end_mjd, 4.0, dtype=dtype),
            cheb_unit(f["jupiter"], 5, 0, start_mjd, end_mjd, 32.0, dtype=dtype),
        ]
    with open(path, "wb") as fh:
        fh.write(cbor_dumps(brie_layout2(units, STATE_INT_KEYS) if layout == 2 else {"layout": 1, "core": units}))


def itrf93_unit(start_mjd, end_mjd, seg_days=8.0, pdeg=13):
    """Binary orientation unit for ITRF93 (target 3000) relative to
    ECLIPJ2000: Chebyshev series of the three Euler angles v0 = pi/2 + RA,
    v1 = pi/2 - Dec, v2 = W of the pole and prime meridian in ecliptic
    coordinates — the ICRF pole (RA pi/2, Dec pi/2 - obliquity) with small
    slow pole and rate perturbations, W the Earth rotation angle."""
    eps = math.radians(84381.448 / 3600.0)

    def angles(t):  # t in days from MJD2000 0 (TDB)
        v0 = math.pi + 1.0e-4 * np.sin(2.0 * math.pi * t / 6798.4) + 2.0e-7 * t
        v1 = eps + 4.0e-5 * np.cos(2.0 * math.pi * t / 6798.4)
        w = 2.0 * math.pi * (0.7790572732640 + 1.00273781191135448 * (t - 0.5)) + 3.0e-6 * np.sin(2.0 * math.pi * t)
        return np.stack([v0, v1, w], -1)

    u = cheb_unit(angles, 3000, 0, start_mjd, end_mjd, seg_days, pdeg)
    md = u["metadata"]
    u["metadata"] = {"unit_type": 3, "frameClassID": 3000, "inertialFrame": 17, "dtype": 2,
                     "nintervals": md["nintervals"], "pdeg": md["pdeg"], "startEpoch": md["startEpoch"],
                     "finalEpoch": md["finalEpoch"]}
    return u


def iau_earth_units(start_mjd, end_mjd):
    """IAU body model of the Earth (RA = -0.641 T, Dec = 90 - 0.557 T,
    W = 190.147 + 360.9856235 d, degrees; T in centuries, d in days) with two
    small nutation-precession terms on the angles of an Earth-Moon barycenter
    unit (3), so that both series are exercised."""
    t0, t1 = mjd2000_to_et(start_mjd), mjd2000_to_et(end_mjd)
    body = {"metadata": {"unit_type": 1, "target": 399, "pdeg_ra": 1, "pdeg_dec": 1, "pdeg_pm": 1,
                         "num_dims_radii": 0, "barycenter": 3, "num_np_terms_ra": 2, "num_np_terms_dec": 2,
                         "num_np_terms_pm": 2, "startEpoch": t0, "finalEpoch": t1},
            "data": [0.0, -0.641, 90.0, -0.557, 190.147, 360.9856235,
                     -3.6e-3, 5.0e-4, 1.3e-3, -2.0e-4, 2.1e-3, -3.0e-4]}
    bary = {"metadata": {"unit_type": 2, "target": 3, "pdeg_np": 1, "num_np_angles": 2,
                         "startEpoch": t0, "finalEpoch": t1},
            "data": [125.045, -1935.5364525, 250.089, -3871.0729]}
    return [body, bary]


def iau_moon_unit(start_mjd, end_mjd):
    """IAU body model of the Moon (RA = 269.9949 + 0.0031 T, Dec = 66.5392 +
    0.0130 T, W = 38.3213 + 13.17635815 d, degrees; the IAU WG's leading
    terms) without nutation-precession terms."""
    t0, t1 = mjd2000_to_et(start_mjd), mjd2000_to_et(end_mjd)
    return {"metadata": {"unit_type": 1, "target": 301, "pdeg_ra": 1, "pdeg_dec": 1, "pdeg_pm": 1,
                         "num_dims_radii": 0, "barycenter": 3, "num_np_terms_ra": 0, "num_np_terms_dec": 0,
                         "num_np_terms_pm": 0, "startEpoch": t0, "finalEpoch": t1},
            "data": [269.9949, 0.0031, 66.5392, 0.0130, 38.3213, 13.17635815]}


def write_brot2(path, start_mjd, end_mjd, layout=1, frame="iers", moon=False):
    """IERS2000 unit: X, Y, s (rad) on a 1-day TT grid, ERP on daily keys.
    Constant EOP: xp = yp = 0, UT1-UTC = 0.3 s, TAI-UTC = 34 s."""
    t0 = start_mjd - 3.0
    n_nut = int(end_mjd - start_mjd) + 7
    tn = t0 + np.arange(n_nut)
    T = tn / 36525.0
    # smooth CIP coordinates (non-zero: X = Y = 0 makes the model's omega 0/0)
    X = 1.1e-3 + 9.7e-3 * T + 4.0e-8 * np.sin(2 * np.pi * tn / 13.66)
    Y = -3.0e-5 + 1.0e-6 * T + 3.0e-8 * np.cos(2 * np.pi * tn / 13.66)
    s = -1.0e-8 - 5.0e-10 * T
    keys = tn.copy()
    n_erp = len(keys)
    dut1 = np.full(n_erp, (0.3 - 32.184 - TAI_UTC_2011) / SECONDS_PER_DAY)
    zeros = np.zeros(n_erp)
    data = (X.tolist() + Y.tolist() + s.tolist() + zeros.tolist() + zeros.tolist() + dut1.tolist()
            + zeros.tolist() + zeros.tolist() + [float(tn[0]), 1.0, float(keys[0]), 1.0] + keys.tolist())
    meta = {"unit_type": 4, "target": 3001, "model_id": 0, "interp_id": 1,
            "n_nodes_nut": n_nut, "n_nodes_erp": n_erp, "lag_order_nut": 5, "lag_order_erp": 3,
            "startEpoch": mjd2000_to_et(start_mjd - 1.0), "finalEpoch": mjd2000_to_et(end_mjd + 1.0)}
    with open(path, "wb") as fh:
        units = []
        if frame in ("iers", "both"):
            units.append({"metadata": meta, "data": data})
        if frame in ("itrf93", "both"):
            units.append(itrf93_unit(start_mjd - 2.0, end_mjd + 2.0))
        if frame == "iau":
            units += iau_earth_units(start_mjd - 2.0, end_mjd + 2.0)
        if moon:
            units.append(iau_moon_unit(start_mjd - 2.0, end_mjd + 2.0))
        fh.write(cbor_dumps(brie_layout2(units, ORIENTATION_INT_KEYS) if layout == 2
                            else {"layout": 1, "core": units}))


def write_space_weather(path, start_mjd, end_mjd, f107=150.0, ap=15):
    """Constant CelesTrak SW-All rows over [start-6, end+3] (MJD, UTC days)."""
    first = int(math.floor(start_mjd + 51544.0)) - 6
    last = int(math.floor(end_mjd + 51544.0)) + 3
    with open(path, "w") as f:
        for mjd in range(first, last + 1):
            y, m, d = calendar(mjd)
            kp = " ".join(["20"] * 8)
            aps = " ".join([str(ap)] * 8)
            f.write(f"{y} {m:2d} {d:2d} 2400 1 {kp} 160 {aps} {ap} 0.8 4 50 "
                    f"{f107:.1f} 0 {f107:.1f} {f107:.1f} {f107:.1f} {f107:.1f} {f107:.1f}\n")


def write_eop(path, start_mjd, end_mjd, ut1_utc=0.3, tai_utc=TAI_UTC_2011):
    first = int(math.floor(start_mjd + 51544.0)) - 3
    last = int(math.floor(end_mjd + 51544.0)) + 3
    with open(path, "w") as f:
        for mjd in range(first, last + 1):
            y, m, d = calendar(mjd)
            f.write(f"{y} {m:2d} {d:2d} {mjd} 0.000000 0.000000 {ut1_utc:.7f} 0.0000000 "
                    f"0.000000 0.000000 0.000000 0.000000 {tai_utc:.0f}\n")


CONSTANTS = [
    {"CONSTANTS": "synthetic set (values of the HPOP / GGM03C / DE440 compatible set)",
     "AU": 149597870.7, "CLIGHT": 299792.458, "EMRAT": 81.30056822149722, "PS": 4.559821181358739e-09},
    {"NAME": "Sun", "NAIFID": 10, "GM": 132712440041.27942, "SOI": 10000000000.0, "R": 696000.0,
     "A_MEAN": 0.0, "J2": 0.0},
    {"NAME": "Moon", "NAIFID": 301, "MAIN_BODY": "Earth", "GM": 4902.800192171393, "SOIOld": 66194.3772804927,
     "R": 1738.0, "A_MEAN": 384466.5276989999, "J2": 0.00020343},
    {"NAME": "Earth", "NAIFID": 399, "MAIN_BODY": "Sun", "GM": 398600.4415, "SOIOld": 924646.788599425,
     "R": 6378.137, "A_MEAN": 149597870.7, "J2": 0.0010826355254902923},
]


def write_environment(directory, spec: EnvSpec = EnvSpec()) -> Path:
    """Write every environment file for ``spec`` into ``directory``; returns it."""
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    C, S = kaula_field(spec.degree, spec.seed, spec.zonal_only)
    write_tab(d / "gravity.tab", C, S, spec.gm_tab, spec.r_tab, spec.degree)
    if spec.moon_field:
        Cm, Sm = kaula_field(spec.moon_field, spec.seed + 101)
        Cm[2, 0] = -9.0881e-5  # the Moon's C20 (normalized), its other terms the Kaula-like draw
        write_tab(d / "moon.tab", Cm, Sm, 4902.800192171393, 1738.0, spec.moon_field)
    if spec.ephemeris_files == 2:
        write_brie_split(d / "bodies.brie", d / "bodies2.brie", spec.start_mjd, spec.end_mjd)
    else:
        write_brie(d / "bodies.brie", spec.start_mjd, spec.end_mjd, spec.ephemeris_type, spec.ephemeris_chain,
                   spec.brie_layout)
    write_brot2(d / "earth.brot2", spec.start_mjd, spec.end_mjd, spec.brie_layout, spec.earth_frame,
                spec.moon_frame)
    write_space_weather(d / "SW-All.txt", spec.start_mjd, spec.end_mjd)
    write_eop(d / "EOP-All.txt", spec.start_mjd, spec.end_mjd)
    (d / "constants.json").write_text(json.dumps(CONSTANTS, indent=2) + "\n")
    return d


# Exponential atmosphere bands (rho0 in kg/km^3 = SI x 1e9, heights in km):
# textbook base densities and scale heights of a static exponential model.
EXPONENTIAL_BANDS = [
    {"rho0": 2.418e-2, "h0": 300.0, "scaleHeight": 53.628, "hCutoff": 500.0},
    {"rho0": 6.967e-4, "h0": 500.0, "scaleHeight": 63.822, "hCutoff": 700.0},
    {"rho0": 3.614e-5, "h0": 700.0, "scaleHeight": 88.667, "hCutoff": 1000.0},
]


def make_config(env_dir, duration, step, max_steps=1000000, threads=1, force="full",
                degree=70, bodies=("Sun", "Moon", "JupiterBarycenter"), tides=True,
                relativity=True, drag=True, srp=True, start_mjd=4016.0, end_mjd=4064.0,
                gravity="shape", atmosphere="nrlmsise00", tide_system="zero_tide",
                occulting=("Earth",), earth_orientation=None, ephemeris=("bodies.brie",),
                moon_gravity="point", moon_degree=8, moon_atmosphere=False) -> dict:
    """Run configuration in the reference schema (``example/config/envisat_full.json``).
    Paths are relative to ``env_dir`` (where the config file is written).
    ``gravity``: "shape" (the spherical-harmonic file) or "oblateness" (the
    J2 model from the constants file); ``atmosphere``: "nrlmsise00",
    "exponential" (one band) or "piecewise" (three bands); ``moon_gravity``:
    "point", "oblateness" (the Moon's J2 model in its IAU frame) or "shape"
    (the lunar field of moon.tab, degree ``moon_degree``, in the same frame);
    ``moon_atmosphere``: an exponential atmosphere on the Moon (a test of
    drag about a body other than the Earth, not a lunar model)."""
    earth: dict = {}
    if force == "central":
        earth = {"gravity": True}
    else:
        if gravity == "oblateness":
            grav = {"oblateness": True}
        else:
            grav = {"shape": {"body": "Earth", "file": "gravity.tab", "delimiter": ",",
                              "headerLines": 0, "degree": degree, "order": degree}}
        earth = {"occulting": "Earth" in occulting, "flattening": 0.0033528106647474805, "gravity": grav}
        if earth_orientation:
            earth["orientation"] = earth_orientation
        if drag and force == "full":
            if atmosphere == "exponential":
                earth["atmosphere"] = {"exponential": {"rho0": 3.725e-3, "h0": 400.0, "scaleHeight": 58.515,
                                                       "hCutoff": 1000.0}}
            elif atmosphere == "piecewise":
                earth["atmosphere"] = {"exponential": [dict(b) for b in EXPONENTIAL_BANDS[::-1]]}
            else:
                earth["atmosphere"] = {"nrlmsise00": {
                    "spaceWeatherFile": "SW-All.txt", "coverageStartMjdUtc": start_mjd + 51544.0 - 1.0,
                    "coverageEndMjdUtc": end_mjd + 51544.0 + 1.0, "hCutoff": 1000.0, "densityScale": 1.0}}
    bodies_cfg = {"Earth": earth}
    if force == "full":
        for b in bodies:
            if b == "Sun":
                bodies_cfg["Sun"] = {"gravity": True, "radiation": bool(srp)}
            elif b == "Moon":
                grav_m = {"oblateness": True} if moon_gravity == "oblateness" else True
                if moon_gravity == "shape":
                    grav_m = {"shape": {"file": "moon.tab", "delimiter": ",", "headerLines": 0,
                                        "degree": moon_degree, "order": moon_degree}}
                bodies_cfg["Moon"] = ({"gravity": grav_m, "occulting": True} if "Moon" in occulting
                                      else {"gravity": grav_m})
                if moon_atmosphere:
                    bodies_cfg["Moon"]["flattening"] = 0.0012
                    bodies_cfg["Moon"]["atmosphere"] = {"exponential": {"rho0": 0.05, "h0": 100.0,
                                                                        "scaleHeight": 120.0, "hCutoff": 1200.0}}
            elif b == "JupiterBarycenter":
                bodies_cfg["JupiterBarycenter"] = {"gm": 126712764.1, "gravity": True}
    env = {"bodies": bodies_cfg, "ephemeris": list(ephemeris), "constants": "constants.json", "preferSSB": True}
    if force != "central":
        env["orientations"] = ["earth.brot2"]
    if force == "full" and (tides or relativity):
        env["earthCorrections"] = {"model": "iers2010_fes2004", "tideSystem": tide_system,
                                   "solidEarthTides": bool(tides), "oceanTides": bool(tides),
                                   "relativity": bool(relativity), "eopFile": "EOP-All.txt"}
    return {"run": {"duration_seconds": float(duration)},
            "execution": {"maxThreads": int(threads),
                          "integration": {"initialStepSize": float(step), "maxNumSteps": int(max_steps)}},
            "model": {"environment": env}}


def write_case(directory, population: Population, duration, step, **cfg) -> tuple[Path, Path]:
    """Write ``config.json`` and ``targets.json`` into ``directory`` (which must
    already hold the environment files); returns their paths."""
    d = Path(directory)
    cfgd = make_config(d, duration, step, **cfg)
    (d / "config.json").write_text(json.dumps(cfgd, indent=2) + "\n")
    (d / "targets.json").write_text(json.dumps(population.targets_json()) + "\n")
    return d / "config.json", d / "targets.json"
