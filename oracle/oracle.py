"""CPU oracle driver: loads a ParaHPOP run configuration and its environment
files with independent Python readers, and propagates targets with the C++
restatement in ``phop_oracle.cpp``.  TEST INFRASTRUCTURE ONLY - used by the
tests, the smoke check and the benchmark's CPU-baseline leg as the checker.

Readers follow the reference loaders:
  config + targets    src/common/driver.cpp:72-123
  .tab                src/common/engine/interface/config/model/sphericalharmonics/Coefficients.h:241-362
  .brie (layout 1)    third_party/brie/brie/states/metadata/EphUnit.h:55-86, states/EphUnit.h:223-238
  .brot2 (type 4)     third_party/brie/brie/orientations/metadata/EphUnit.cpp:148-167
  SW-All              src/common/engine/paraHPOP/model/environment/atmosphere/Nrlmsise00Atmosphere.h:168-235
  EOP-All             src/common/engine/paraHPOP/model/environment/earthcorrections/EarthCorrections.h:142-177
  bodies              src/common/engine/interface/config/model/environment/Bodies.h:105-120 (NAIF-id order)
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
import struct
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "lib" / "liboracle.so"

NAIF = {"Sun": 10, "Moon": 301, "Earth": 399, "MercuryBarycenter": 1, "VenusBarycenter": 2, "MarsBarycenter": 4,
        "JupiterBarycenter": 5, "SaturnBarycenter": 6, "UranusBarycenter": 7, "NeptuneBarycenter": 8,
        "PlutoBarycenter": 9}
F_GRAVITY, F_SHAPE, F_RADIATION, F_ATMOSPHERE, F_OCCULTING, F_OBLATENESS = 1, 2, 4, 8, 16, 32


REF_MODELS = HERE / "_ref" / "ref_models.o"


def build(force=False):
    """Compile the oracle library (g++, OpenMP), linked with the reference's
    NRLMSISE-00 and tide sources compiled into oracle/_ref/ref_models.o by
    ``make -f oracle/Makefile.ref models REF=<reference tree>``."""
    src = HERE / "phop_oracle.cpp"
    if not REF_MODELS.exists():
        raise RuntimeError(f"{REF_MODELS} is missing: build it from the reference sources with "
                           "`make -f oracle/Makefile.ref models REF=<reference tree>`")
    deps = [src, REF_MODELS]
    if LIB.exists() and not force and all(LIB.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return LIB
    LIB.parent.mkdir(parents=True, exist_ok=True)
    cmd = ["g++", "-O3", "-march=x86-64-v3", "-std=c++17", "-fopenmp", "-shared", "-fPIC", "-w",
           str(src), str(REF_MODELS), "-o", str(LIB)]
    subprocess.run(cmd, check=True)
    return LIB


# ---------------------------------------------------------------------------
# CBOR (RFC 8949) decoder, the subset the .brie/.brot files use
# ---------------------------------------------------------------------------
def cbor_loads(buf: bytes):
    pos = 0

    def head():
        nonlocal pos
        b = buf[pos]; pos += 1
        major, info = b >> 5, b & 31
        if info < 24:
            return major, info
        n = {24: 1, 25: 2, 26: 4, 27: 8}[info]
        v = int.from_bytes(buf[pos:pos + n], "big"); pos += n
        if major == 7:
            return major, (info, v)
        return major, v

    def item():
        nonlocal pos
        major, v = head()
        if major == 0:
            return v
        if major == 1:
            return -1 - v
        if major == 2:
            out = buf[pos:pos + v]; pos += v; return out
        if major == 3:
            out = buf[pos:pos + v].decode(); pos += v; return out
        if major == 4:
            return [item() for _ in range(v)]
        if major == 5:
            d = {}
            for _ in range(v):
                k = item(); d[k] = item()
            return d
        if major == 6:
            return item()
        if major == 7:
            if isinstance(v, tuple):
                info, raw = v
                if info == 27:
                    return struct.unpack(">d", raw.to_bytes(8, "big"))[0]
                if info == 26:
                    return struct.unpack(">f", raw.to_bytes(4, "big"))[0]
                if info == 25:
                    return float(np.frombuffer(raw.to_bytes(2, "big"), dtype=">f2")[0])
            return {20: False, 21: True, 22: None}.get(v)
        raise ValueError("bad CBOR")

    return item()


# ---------------------------------------------------------------------------
class _Env(C.Structure):
    _fields_ = [
        ("sh_degree", C.c_int), ("sh_order", C.c_int), ("sh_normalized", C.c_int),
        ("sh_R", C.c_double), ("sh_GM", C.c_double),
        ("sh_C", C.POINTER(C.c_double)), ("sh_S", C.POINTER(C.c_double)),
        ("nbodies", C.c_int), ("body_id", C.POINTER(C.c_int)), ("body_gm", C.POINTER(C.c_double)),
        ("body_radius", C.POINTER(C.c_double)), ("body_flags", C.POINTER(C.c_int)),
        ("flattening", C.c_double), ("au", C.c_double),
        ("neph", C.c_int), ("eph_target", C.POINTER(C.c_int)), ("eph_center", C.POINTER(C.c_int)),
        ("eph_nint", C.POINTER(C.c_int)), ("eph_pdeg", C.POINTER(C.c_int)), ("eph_offset", C.POINTER(C.c_int64)),
        ("eph_data", C.POINTER(C.c_double)),
        ("has_rot", C.c_int), ("rot_nnut", C.c_int), ("rot_nerp", C.c_int), ("rot_data", C.POINTER(C.c_double)),
        ("has_nrl", C.c_int), ("nrl_ndays", C.c_int), ("nrl_start_mjd", C.c_double), ("nrl_hcutoff", C.c_double),
        ("nrl_density_scale", C.c_double), ("nrl_weather", C.POINTER(C.c_double)),
        ("solid", C.c_int), ("ocean", C.c_int), ("relativity", C.c_int), ("zero_tide", C.c_int),
        ("eop_n", C.c_int), ("eop_first_mjd", C.c_double), ("eop", C.POINTER(C.c_double)),
        ("body_j2", C.POINTER(C.c_double)), ("body_gm_const", C.POINTER(C.c_double)),
        ("body_soi", C.POINTER(C.c_double)), ("n_exp", C.c_int), ("exp_seg", C.POINTER(C.c_double)),
        ("rot_kind", C.c_int), ("rot_nint", C.c_int), ("rot_pdeg", C.c_int), ("rot_ecliptic", C.c_int),
        ("iau_deg", C.c_int * 3), ("iau_np", C.c_int * 3), ("iau_bary_offset", C.c_int), ("iau_np_deg", C.c_int),
        ("iau_np_angles", C.c_int),
        ("frame_data", C.POINTER(C.c_double) * 12), ("frame_deg", (C.c_int * 3) * 12),
        ("frame_np", (C.c_int * 3) * 12), ("frame_bary_offset", C.c_int * 12), ("frame_np_deg", C.c_int * 12),
        ("body_flattening", C.c_double * 12),
    ]


STATE_INT_KEYS = ["frame", "dtype", "target", "center", "nintervals", "pdeg", "@offset", "@size"]
ORIENTATION_INT_KEYS = ["unit_type", "@m1", "@m2", "@m3", "@m4", "@m5", "@m6", "@m7", "@m8", "@m9", "@offset",
                        "@size"]
# names of the positional members per orientation unit type (Layout.h)
ORIENTATION_FIELDS = {4: {"target": "@m1", "model_id": "@m2", "interp_id": "@m3", "n_nodes_nut": "@m4",
                          "n_nodes_erp": "@m5", "lag_order_nut": "@m6", "lag_order_erp": "@m7"},
                      3: {"frameClassID": "@m1", "inertialFrame": "@m2", "dtype": "@m3", "nintervals": "@m4",
                          "pdeg": "@m5"},
                      1: {"target": "@m1", "pdeg_ra": "@m2", "pdeg_dec": "@m3", "pdeg_pm": "@m4",
                          "num_dims_radii": "@m5", "barycenter": "@m6", "num_np_terms_ra": "@m7",
                          "num_np_terms_dec": "@m8", "num_np_terms_pm": "@m9"},
                      2: {"target": "@m1", "pdeg_np": "@m2", "num_np_angles": "@m3"}}


def brie_units(j, int_keys):
    """Units of a BRIE file in layout 1 (a list of {metadata, data}) or layout
    2 (member-major metadata arrays over one data array; brie/util/cbor.cpp
    211-379 and the readers' member enums)."""
    while isinstance(j, list) and len(j) == 1:
        j = j[0]
    if j["layout"] == 1:
        return j["core"]
    assert j["layout"] == 2, "unknown BRIE layout"
    md, data = j["core"]["metadata"], j["core"]["data"]
    n, im, dm = md["nBodyUnits"], md["intMetadata"], md.get("doubleMetadata")
    assert len(im) == len(int_keys) * n
    units = []
    for i in range(n):
        meta = {k: im[q * n + i] for q, k in enumerate(int_keys) if k}
        if dm is not None:
            meta["startEpoch"], meta["finalEpoch"] = dm[i], dm[n + i]
        units.append({"metadata": meta, "data": data[meta["@offset"]:meta["@offset"] + meta["@size"]]})
    return units


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def calendar_mjd(y, m, d):
    a = (14 - m) // 12
    yy = y + 4800 - a
    mm = m + 12 * a - 3
    jdn = d + (153 * mm + 2) // 5 + 365 * yy + yy // 4 - yy // 100 + yy // 400 - 32045
    return float(jdn) - 2400001.0


@dataclass
class Environment:
    cfg: dict
    keep: list
    env: _Env
    duration: float
    step: float
    max_steps: int
    threads: int


def load_environment(config_path) -> Environment:
    config_path = Path(config_path).resolve()
    cfg = json.loads(config_path.read_text())
    base = config_path.parent
    envc = cfg["model"]["environment"]
    P = lambda p: (base / p).resolve()
    keep = []
    e = _Env()

    def hold(a):
        keep.append(a); return a

    # constants
    consts = json.loads(P(envc["constants"]).read_text())
    au = next(c["AU"] for c in consts if "AU" in c)
    byid = {c["NAIFID"]: c for c in consts if "NAIFID" in c}
    e.au = au
    # bodies (sorted by NAIF id, Bodies.h:105-120)
    rows = []
    flattening = 0.0
    earth_orientation = None
    shape = None
    atm = None
    exp_segments = []
    for name, bc in envc["bodies"].items():
        nid = NAIF[name]
        flags = 0
        g = bc.get("gravity", False)
        if g:
            flags |= F_GRAVITY
            if isinstance(g, dict) and "shape" in g:
                flags |= F_SHAPE
                shape = g["shape"]
            if (isinstance(g, dict) and g.get("oblateness")) or (isinstance(g, list) and "oblateness" in g):
                flags |= F_OBLATENESS
        if bc.get("radiation"):
            flags |= F_RADIATION
        if "atmosphere" in bc:
            flags |= F_ATMOSPHERE
            model = {k.lower(): v for k, v in bc["atmosphere"].items()}
            if "nrlmsise00" in model or "nrlmsise-00" in model:
                atm = model.get("nrlmsise00", model.get("nrlmsise-00"))
            else:
                blocks = model["exponential"]
                blocks = blocks if isinstance(blocks, list) else [blocks]
                segs = []
                for b in blocks:
                    b = {k.lower(): v for k, v in b.items()}
                    segs.append((b["h0"], b["rho0"], b["scaleheight"], b["hcutoff"]))
                segs.sort()
                exp_segments = segs
        if bc.get("occulting"):
            flags |= F_OCCULTING
        if name == "Earth":
            flattening = bc.get("flattening", 0.0)
            earth_orientation = bc.get("orientation")
        cst = byid.get(nid, {})
        gm = bc.get("gm", cst.get("GM", 0.0))
        radius = cst.get("R", 0.0)
        soi = cst.get("SOIOld", cst.get("SOI", 1e20))
        rows.append((nid, gm, radius, flags, cst.get("J2", 0.0), cst.get("GM", 0.0), soi, bc.get("flattening", 0.0)))
    rows.sort()
    e.nbodies = len(rows)
    e.body_id = _ip(hold(np.array([r[0] for r in rows], dtype=np.int32)))
    e.body_gm = _dp(hold(np.array([r[1] for r in rows], dtype=np.float64)))
    e.body_radius = _dp(hold(np.array([r[2] for r in rows], dtype=np.float64)))
    e.body_flags = _ip(hold(np.array([r[3] for r in rows], dtype=np.int32)))
    e.body_j2 = _dp(hold(np.array([r[4] for r in rows], dtype=np.float64)))
    e.body_gm_const = _dp(hold(np.array([r[5] for r in rows], dtype=np.float64)))
    e.body_soi = _dp(hold(np.array([r[6] for r in rows], dtype=np.float64)))
    e.n_exp = len(exp_segments)
    if exp_segments:
        # component-major: rho0, h0, scaleHeight, hCutoff
        seg = np.array([[s[1] for s in exp_segments], [s[0] for s in exp_segments],
                        [s[2] for s in exp_segments], [s[3] for s in exp_segments]], dtype=np.float64)
        e.exp_seg = _dp(hold(np.ascontiguousarray(seg.reshape(-1))))
    e.flattening = flattening
    # geopotential
    if shape is not None:
        lines = [l for l in P(shape["file"]).read_text().splitlines() if l.strip()]
        hdr = [float(x) for x in lines[0].split(",")]
        N = int(shape.get("degree", hdr[3]))
        M = int(shape.get("order", hdr[4]))
        half = (N + 2) * (N + 3) // 2  # storage for maxDeg+1 as the loader allocates
        Cc = np.zeros(half); Ss = np.zeros(half)
        for l in lines[1:]:
            v = [float(x) for x in l.split(",")]
            n, m = int(v[0]), int(v[1])
            if n > N or m > M:
                continue
            Cc[n * (n + 1) // 2 + m] = v[2]
            if m > 0:
                Ss[n * (n + 1) // 2 + m] = v[3]
        e.sh_degree, e.sh_order, e.sh_normalized = N, M, int(hdr[5])
        e.sh_R, e.sh_GM = hdr[0], hdr[1]
        e.sh_C = _dp(hold(Cc)); e.sh_S = _dp(hold(Ss))
    # ephemeris
    units = []
    for f in envc.get("ephemeris", []):
        units += brie_units(cbor_loads(P(f).read_bytes()), STATE_INT_KEYS)
    off = np.zeros(len(units), dtype=np.int64)
    data = []
    o = 0
    for k, u in enumerate(units):
        off[k] = o
        data += list(u["data"])
        o += len(u["data"])
    e.neph = len(units)
    e.eph_target = _ip(hold(np.array([u["metadata"]["target"] for u in units], dtype=np.int32)))
    e.eph_center = _ip(hold(np.array([u["metadata"]["center"] for u in units], dtype=np.int32)))
    e.eph_nint = _ip(hold(np.array([u["metadata"]["nintervals"] for u in units], dtype=np.int32)))
    e.eph_pdeg = _ip(hold(np.array([u["metadata"]["pdeg"] for u in units], dtype=np.int32)))
    e.eph_offset = hold(off).ctypes.data_as(C.POINTER(C.c_int64))
    e.eph_data = _dp(hold(np.array(data, dtype=np.float64)))
    # orientation
    # Earth frames: ITRF93 (binary Chebyshev angles, target 3000) and the
    # IERS2000 model unit (3001); bodies.Earth.orientation picks one, else
    # the unique loaded one (interface naming/orientations Resolver.h)
    frames, barys, other_iau = {}, {}, {}
    for f in envc.get("orientations", []):
        for u in brie_units(cbor_loads(P(f).read_bytes()), ORIENTATION_INT_KEYS):
            md = u["metadata"]
            kind = md["unit_type"]
            if kind not in ORIENTATION_FIELDS:
                continue
            for name, member in ORIENTATION_FIELDS[kind].items():
                md.setdefault(name, md.get(member))
            if kind == 2:
                barys[md["target"]] = (md, u["data"])
                continue
            target = md["frameClassID"] if kind == 3 else md["target"]
            if target in (3000, 3001, 399):
                frames[target] = (kind, md, u["data"])
            elif kind == 1:
                other_iau.setdefault(target, (md, u["data"]))
    want = {"ITRF93": 3000, "ITRF": 3000, "EARTH_FIXED": 3000, "ITRF_IERS2000": 3001, "ITRF_IPF": 3001,
            "ITRF_NATIVE": 3001, "EARTH_BODY_FIXED": 399, "IAU_EARTH": 399}.get(
                str(earth_orientation).upper()) if earth_orientation else None
    binary = {k: v for k, v in frames.items() if k != 399}
    if want is None and len(binary) > 1:
        raise ValueError("Body 399 has more than one loaded high-precision orientation frame")
    if want is None:
        want = next(iter(binary)) if binary else 399
    sel = frames.get(want)
    if sel is not None:
        kind, md, data = sel
        e.has_rot = 1
        e.rot_kind = kind
        e.rot_data = _dp(hold(np.array(data, dtype=np.float64)))
        if kind == 4:
            e.rot_nnut, e.rot_nerp = md["n_nodes_nut"], md["n_nodes_erp"]
        elif kind == 3:
            e.rot_nint, e.rot_pdeg = md["nintervals"], md["pdeg"]
            e.rot_ecliptic = 1 if md["inertialFrame"] == 17 else 0
        else:
            for k, name in enumerate(("ra", "dec", "pm")):
                e.iau_deg[k] = md["pdeg_" + name] + 1
                e.iau_np[k] = md["num_np_terms_" + name]
            e.iau_bary_offset = -1
            if md["barycenter"] in barys:
                bmd, bdata = barys[md["barycenter"]]
                e.iau_bary_offset = len(data)
                e.iau_np_deg, e.iau_np_angles = bmd["pdeg_np"] + 1, bmd["num_np_angles"]
                e.rot_data = _dp(hold(np.array(list(data) + list(bdata), dtype=np.float64)))
    # bodies other than the Earth with the J2 model or the field: their IAU body models
    for bi, r in enumerate(rows):
        e.frame_bary_offset[bi] = -1
        e.body_flattening[bi] = r[7]
        if r[0] == 399 or not (r[3] & (F_OBLATENESS | F_SHAPE | F_ATMOSPHERE)) or r[0] not in other_iau:
            continue
        md, data = other_iau[r[0]]
        vals = list(data)
        for k, name in enumerate(("ra", "dec", "pm")):
            e.frame_deg[bi][k] = md["pdeg_" + name] + 1
            e.frame_np[bi][k] = md["num_np_terms_" + name]
        if max(md["num_np_terms_" + n] for n in ("ra", "dec", "pm")) > 0 and md["barycenter"] in barys:
            bmd, bdata = barys[md["barycenter"]]
            e.frame_bary_offset[bi] = len(vals)
            e.frame_np_deg[bi] = bmd["pdeg_np"] + 1
            vals += list(bdata)
        e.frame_data[bi] = _dp(hold(np.array(vals, dtype=np.float64)))
    # atmosphere
    if atm is not None:
        recs = []
        for line in P(atm["spaceWeatherFile"]).read_text().splitlines():
            t = line.split()
            if len(t) < 33:
                continue
            try:
                y, mo, d = int(t[0]), int(t[1]), int(t[2])
                ap = [int(x) for x in t[14:22]]
                avg = int(t[22])
                adj, adjc, obs, obsc = float(t[26]), float(t[28]), float(t[30]), float(t[31])
            except ValueError:
                continue
            recs.append((calendar_mjd(y, mo, d), obs, obsc, adj, adjc, avg, ap))
        s0 = atm.get("coverageStartMjdUtc", -1.0)
        s1 = atm.get("coverageEndMjdUtc", -1.0)
        ks = math.floor(s0) - 4.0 if s0 >= 0 else recs[0][0]
        ke = math.floor(s1) + 1.0 if s1 >= 0 else recs[-1][0]
        sel = [r for r in recs if ks <= r[0] <= ke]
        W = np.zeros((13, len(sel)))
        for i, r in enumerate(sel):
            W[0, i], W[1, i], W[2, i], W[3, i], W[4, i] = r[1], r[2], r[3], r[4], r[5]
            W[5:13, i] = r[6]
        e.has_nrl = 1
        e.nrl_ndays = len(sel)
        e.nrl_start_mjd = sel[0][0]
        e.nrl_hcutoff = atm.get("hCutoff", 1000.0)
        e.nrl_density_scale = atm.get("densityScale", 1.0)
        e.nrl_weather = _dp(hold(np.ascontiguousarray(W.reshape(-1))))
    # Earth corrections
    ec = envc.get("earthCorrections")
    if ec:
        e.solid = int(bool(ec.get("solidEarthTides", False)))
        e.ocean = int(bool(ec.get("oceanTides", False)))
        e.relativity = int(bool(ec.get("relativity", False)))
        e.zero_tide = int(ec.get("tideSystem", "zero_tide") == "zero_tide")
        if e.solid or e.ocean:
            rows = []
            for line in P(ec["eopFile"]).read_text().splitlines():
                t = line.split()
                if len(t) < 13:
                    continue
                rows.append((float(t[3]), float(t[4]), float(t[5]), float(t[6]), float(t[12])))
            E = np.array(rows)
            e.eop_n = len(rows)
            e.eop_first_mjd = E[0, 0]
            e.eop = _dp(hold(np.ascontiguousarray(E[:, 1:].T.reshape(-1))))
    ex = cfg["execution"]
    return Environment(cfg, keep, e, float(cfg["run"]["duration_seconds"]),
                       float(ex["integration"]["initialStepSize"]), int(ex["integration"]["maxNumSteps"]),
                       int(ex.get("maxThreads", 1)))


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(str(build()))
        _lib.oracle_propagate.restype = C.c_int
        _lib.oracle_propagate.argtypes = [C.POINTER(_Env), C.c_int64] + [C.POINTER(C.c_double)] * 9 + \
            [C.c_int64, C.POINTER(C.c_double), C.c_int]
        _lib.oracle_nrl_density.restype = C.c_double
        _lib.oracle_nrl_density.argtypes = [C.c_int] + [C.c_double] * 8 + [C.POINTER(C.c_double)]
    return _lib


def propagate(environment: Environment, targets: dict, duration=None, step=None, threads=None, max_steps=None):
    """Propagate every target of a reference-schema targets document; returns
    (ids, final_epochs_mjd2000, final_states (n, 6)).  Per-target
    ``duration_seconds`` / ``step_seconds`` override the run values."""
    t = targets["targets"]
    n = len(t)
    ids = np.array([x["id"] for x in t])
    ep = np.array([x["epoch_mjd2000_tdb"] for x in t], dtype=np.float64)
    st = np.ascontiguousarray(np.array([x["state_km_km_s"] for x in t], dtype=np.float64))
    g = lambda k: np.array([x[k] for x in t], dtype=np.float64)
    mass, ad, asrp, cd, cr = g("mass_kg"), g("drag_area_m2"), g("srp_area_m2"), g("cd"), g("cr")
    dur0 = environment.duration if duration is None else duration
    stp0 = environment.step if step is None else step
    dur = np.array([x.get("duration_seconds", dur0) for x in t], dtype=np.float64)
    stp = np.array([x.get("step_seconds", stp0) for x in t], dtype=np.float64)
    out_ep = np.zeros(n)
    ms = environment.max_steps if max_steps is None else max_steps
    th = threads if threads is not None else (os.cpu_count() or 1)
    rc = lib().oracle_propagate(C.byref(environment.env), n, _dp(ep), _dp(st), _dp(mass), _dp(ad), _dp(asrp),
                                _dp(cd), _dp(cr), _dp(dur), _dp(stp), ms, _dp(out_ep), th)
    if rc:
        raise RuntimeError("A target stopped without reaching the requested end of simulation.")
    return ids, out_ep, st


def nrl_density(doy, sec, alt, glat, glong, lst, f107A, f107, ap, ap_a):
    a = np.ascontiguousarray(np.asarray(ap_a, dtype=np.float64))
    return lib().oracle_nrl_density(int(doy), sec, alt, glat, glong, lst, f107A, f107, ap, _dp(a))


def read_final_states(directory):
    """Parse a final_states.csv written by the reference or by this package."""
    import csv
    with open(Path(directory) / "final_states.csv") as fh:
        rows = list(csv.DictReader(fh))
    ids = np.array([int(r["id"]) for r in rows])
    ep = np.array([float(r["epoch_mjd2000_tdb"]) for r in rows])
    st = np.array([[float(r[k]) for k in ("x_km", "y_km", "z_km", "vx_km_s", "vy_km_s", "vz_km_s")] for r in rows])
    return ids, ep, st
