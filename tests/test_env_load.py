"""Host environment loading (phop_load_environment; no device needed).

The loader reads every environment file on a thread of its own and parses
CBOR float64 arrays packed; these tests hold it to what a sequential load
gives:

* the same files in CBOR layout 1 or 2, Type-2 or Type-3 units, and text
  files with CRLF line ends or lines the readers skip (headers, truncated
  rows, trailing fields) load to the same digest;
* repeated loads agree (no order dependence between the file threads);
* with several broken files, the error reported is the one a sequential load
  meets first (field table, ephemerides, orientations, space weather, EOP,
  in the order parahpop_gpu/driver.cpp:52-84 reads the environment).
"""
import json
import shutil

import numpy as np
import pytest

from parahpop_b200 import api, synthetic as S


def _env(tmp_path, name, spec=None, **cfg):
    d = tmp_path / name
    d.mkdir()
    S.write_environment(d, spec or S.EnvSpec())
    (d / "config.json").write_text(json.dumps(S.make_config(d, 3600.0, 60.0, **cfg)))
    return d


def _variant(src, dst, transforms):
    shutil.copytree(src, dst)
    for name, f in transforms.items():
        p = dst / name
        p.write_bytes(f(p.read_bytes()))
    # make_config writes paths relative to the configuration's directory
    return dst / "config.json"


def _digest(d):
    return api.load_environment(d if str(d).endswith(".json") else d / "config.json")[0]


def _crlf(b):
    return b.replace(b"\n", b"\r\n")


def _skipped_lines(b):
    out = [b"# header", b"", b"   ", b"DATATYPE 123 abc"]
    for i, line in enumerate(b.split(b"\n")):
        if i % 9 == 4 and line.strip():
            line += b"  1e  extra +"       # fields after the last one read are ignored
        out.append(line)
        if i % 50 == 7:
            out.append(line[: len(line) // 2])  # a truncated row is skipped
    out.append(b"END")
    return b"\n".join(out)


def _tab_spacing(b):
    out = []
    for i, line in enumerate(b.split(b"\n")):
        if i % 5 == 1:
            line = b"  " + line.replace(b",", b" , ") + b","
        if i % 7 == 2:
            line += b"\r"
        out.append(line)
    out.insert(3, b"")
    out.insert(5, b" , ,")
    return b"\n".join(out) + b"\n\n"


def test_equivalent_files_load_alike(tmp_path):
    base = _env(tmp_path, "base")
    ref = _digest(base)
    assert _digest(_env(tmp_path, "layout2", S.EnvSpec(brie_layout=2))) == ref
    assert _digest(_env(tmp_path, "type3", S.EnvSpec(ephemeris_type=3))) == ref
    assert _digest(_variant(base, tmp_path / "crlf", {"SW-All.txt": _crlf, "EOP-All.txt": _crlf,
                                                       "gravity.tab": _crlf})) == ref
    assert _digest(_variant(base, tmp_path / "junk", {"SW-All.txt": _skipped_lines,
                                                       "EOP-All.txt": _skipped_lines})) == ref
    assert _digest(_variant(base, tmp_path / "tab", {"gravity.tab": _tab_spacing})) == ref
    # and a changed value is seen
    sw = (base / "SW-All.txt").read_bytes()
    changed = _variant(base, tmp_path / "changed", {})
    lines = sw.split(b"\n")
    k = next(i for i, line in enumerate(lines) if line.split()[:3] == [b"2011", b"1", b"10"])
    fields = lines[k].split()
    fields[14] = b"%d" % (int(fields[14]) + 12)  # the day's first 3-hour ap
    lines[k] = b" ".join(fields)
    (changed.parent / "SW-All.txt").write_bytes(b"\n".join(lines))
    assert _digest(changed) != ref


def test_repeated_loads_agree(tmp_path):
    d = _env(tmp_path, "both", S.EnvSpec(earth_frame="both", brie_layout=2, ephemeris_files=2),
             earth_orientation="ITRF93", ephemeris=["bodies.brie", "bodies2.brie"])
    first = _digest(d)
    assert all(_digest(d) == first for _ in range(10))
    assert first != _digest(_env(tmp_path, "iers"))


# Files that exist (paths are checked up front, in configuration order) but
# do not parse; each loader names its file in its message.
BROKEN = {"bad.tab": b"", "bad.brie": b"\xa0", "bad.brot2": b"\xa0", "bad_sw.txt": b"", "bad_eop.txt": b""}

ERROR_CASES = {
    # broken entries -> the message of the first one a sequential load reaches
    "field_and_ephemeris": ({"shape": "bad.tab", "ephemeris": ["bad.brie"]}, "No coefficients found in file"),
    "field_and_later_option": ({"shape": "bad.tab", "sun_option": True}, "No coefficients found in file"),
    "field_and_orientation": ({"shape": "bad.tab", "orientations": ["bad.brot2"]}, "No coefficients found in file"),
    "ephemeris_and_orientation": ({"ephemeris": ["bad.brie"], "orientations": ["bad.brot2"]},
                                  "Unknown BRIE layout type: .*bad.brie"),
    "second_ephemeris_and_weather": ({"ephemeris": ["bodies.brie", "bad.brie"], "sw": "bad_sw.txt"},
                                     "Unknown BRIE layout type: .*bad.brie"),
    "orientation_and_weather": ({"orientations": ["bad.brot2"], "sw": "bad_sw.txt"},
                                "Unknown BRIE layout type: .*bad.brot2"),
    "weather_and_eop": ({"sw": "bad_sw.txt", "eop": "bad_eop.txt"}, "No CelesTrak SW-All records found in"),
    "eop_alone": ({"eop": "bad_eop.txt"}, "Earth tides require at least two HPOP EOP-All records in"),
    "later_option_alone": ({"sun_option": True}, "Unsupported body option for Sun: bogus"),
}


@pytest.mark.parametrize("case", sorted(ERROR_CASES))
def test_error_is_the_first_a_sequential_load_meets(tmp_path, case):
    d = _env(tmp_path, "e")
    for name, data in BROKEN.items():
        (d / name).write_bytes(data)
    cfg = json.loads((d / "config.json").read_text())
    env = cfg["model"]["environment"]
    change, expect = ERROR_CASES[case]
    if "shape" in change:
        env["bodies"]["Earth"]["gravity"]["shape"]["file"] = change["shape"]
    if "ephemeris" in change:
        env["ephemeris"] = change["ephemeris"]
    if "orientations" in change:
        env["orientations"] = change["orientations"]
    if "sw" in change:
        env["bodies"]["Earth"]["atmosphere"]["nrlmsise00"]["spaceWeatherFile"] = change["sw"]
    if "eop" in change:
        env["earthCorrections"]["eopFile"] = change["eop"]
    if "sun_option" in change:
        env["bodies"]["Sun"]["bogus"] = 1
    (d / "bad.json").write_text(json.dumps(cfg))
    for _ in range(3):  # whichever file thread finishes first
        with pytest.raises(api.PhopError, match=expect):
            api.load_environment(d / "bad.json")


def _encoder(floats):
    """A CBOR writer like synthetic.cbor_dumps whose arrays of reals are
    written another legal way: `floats` maps one real to its item bytes,
    and a None result writes the array with indefinite length."""
    import struct
    scalar = S.cbor_dumps  # the module's own writer, for everything but arrays

    def enc(obj):
        if isinstance(obj, np.ndarray):
            obj = obj.tolist()
        if isinstance(obj, (list, tuple)) and obj and all(isinstance(x, float) for x in obj):
            items = [floats(x) for x in obj]
            if items[0] is None:
                return b"\x9f" + b"".join(b"\xfb" + struct.pack(">d", x) for x in obj) + b"\xff"
            return S._cbor_head(4, len(obj)) + b"".join(items)
        if isinstance(obj, (list, tuple)):
            return S._cbor_head(4, len(obj)) + b"".join(enc(x) for x in obj)
        if isinstance(obj, dict):
            return S._cbor_head(5, len(obj)) + b"".join(enc(k) + enc(v) for k, v in obj.items())
        return scalar(obj)
    return enc


def _compact(x):
    import struct
    if x == int(x) and abs(x) < 2 ** 53:
        v = int(x)
        return S._cbor_head(0, v) if v >= 0 else S._cbor_head(1, -1 - v)
    f32 = struct.pack(">f", x)
    if struct.unpack(">f", f32)[0] == x:
        return b"\xfa" + f32
    return b"\xfb" + struct.pack(">d", x)


@pytest.mark.parametrize("form", ["indefinite", "mixed"])
def test_other_cbor_encodings_of_the_same_reals(tmp_path, monkeypatch, form):
    """Ephemeris data arrays that are not all float64 items (indefinite
    length; integers, single and double floats mixed) take the reader's
    general path and load to the same values as the packed one."""
    base = _env(tmp_path, "base")
    ref = _digest(base)
    other = _variant(base, tmp_path / form, {})
    spec = S.EnvSpec()
    monkeypatch.setattr(S, "cbor_dumps", _encoder((lambda x: None) if form == "indefinite" else _compact))
    S.write_brie(other.parent / "bodies.brie", spec.start_mjd, spec.end_mjd)
    monkeypatch.undo()
    assert (other.parent / "bodies.brie").read_bytes() != (base / "bodies.brie").read_bytes()
    assert _digest(other) == ref


def test_refusal_while_file_jobs_run(tmp_path):
    """A synchronous step that refuses the configuration (two high-precision
    Earth frames loaded, none named) while the ephemeris files are still
    being read on their own threads: every load ends with the refusal and no
    job writes into the loader's freed per-file parts."""
    d = S.write_environment(tmp_path / "both", S.EnvSpec(earth_frame="both"))
    (d / "config.json").write_text(json.dumps(S.make_config(d, 600.0, 60.0, max_steps=1000)))
    for _ in range(40):
        with pytest.raises(api.PhopError, match="more than one loaded high-precision orientation frame"):
            api.load_environment(d / "config.json")


def _moon_config(d, **kw):
    cfg = S.make_config(d, 7200.0, 60.0, **kw)
    p = d / f"moon_{len(list(d.glob('moon_*.json')))}.json"
    p.write_text(json.dumps(cfg))
    return p


def test_other_bodies_frames_and_refusals(tmp_path):
    """The J2 model and the field of a body other than the Earth take the
    body's IAU body model from the orientations; without it, or with a
    second field, the load is refused with the reason."""
    with_frame = S.write_environment(tmp_path / "a", S.EnvSpec(moon_frame=True, moon_field=8))
    without = S.write_environment(tmp_path / "b", S.EnvSpec(moon_field=8))
    point, _ = api.load_environment(_moon_config(with_frame))
    j2, _ = api.load_environment(_moon_config(with_frame, moon_gravity="oblateness"))
    field, _ = api.load_environment(_moon_config(with_frame, moon_gravity="shape", gravity="oblateness"))
    assert len({point, j2, field}) == 3
    for kw, what in (({"moon_gravity": "oblateness"}, "The oblateness (J2) model of Moon"),
                     ({"moon_gravity": "shape", "gravity": "oblateness"}, "The spherical-harmonic field of Moon")):
        with pytest.raises(api.PhopError) as e:
            api.load_environment(_moon_config(without, **kw))
        assert str(e.value).startswith(what + " needs its body-fixed orientation: an IAU body model unit for "
                                       "NAIF id 301")
    with pytest.raises(api.PhopError) as e:
        api.load_environment(_moon_config(with_frame, moon_gravity="shape"))
    assert "one spherical-harmonic field per configuration" in str(e.value)


def test_atmosphere_of_another_body(tmp_path):
    """An exponential atmosphere on a body other than the Earth takes the
    body's IAU frame; NRLMSISE-00 stays on the Earth, and a configuration
    holds one atmosphere."""
    with_frame = S.write_environment(tmp_path / "a", S.EnvSpec(moon_frame=True))
    without = S.write_environment(tmp_path / "b", S.EnvSpec())
    # the Earth without drag, the Moon with an exponential atmosphere
    cfg = S.make_config(with_frame, 7200.0, 60.0, drag=False, moon_atmosphere=True)
    p = with_frame / "moon_air.json"
    p.write_text(json.dumps(cfg))
    api.load_environment(p)
    cfg = S.make_config(without, 7200.0, 60.0, drag=False, moon_atmosphere=True)
    p = without / "moon_air.json"
    p.write_text(json.dumps(cfg))
    with pytest.raises(api.PhopError) as e:
        api.load_environment(p)
    assert str(e.value).startswith("The atmosphere of Moon needs its body-fixed orientation")
    # the Earth's NRLMSISE-00 beside the Moon's exponential atmosphere loads;
    # two exponential atmospheres do not
    cfg = S.make_config(with_frame, 7200.0, 60.0, moon_atmosphere=True)
    p = with_frame / "two_air.json"
    p.write_text(json.dumps(cfg))
    api.load_environment(p)
    cfg = S.make_config(with_frame, 7200.0, 60.0, atmosphere="exponential", moon_atmosphere=True)
    p = with_frame / "two_exp.json"
    p.write_text(json.dumps(cfg))
    with pytest.raises(api.PhopError) as e:
        api.load_environment(p)
    assert "one exponential atmosphere per configuration" in str(e.value)
    cfg = S.make_config(with_frame, 7200.0, 60.0, drag=False)
    cfg["model"]["environment"]["bodies"]["Moon"]["atmosphere"] = {"nrlmsise00": {
        "spaceWeatherFile": "SW-All.txt", "coverageStartMjdUtc": 55559.0, "coverageEndMjdUtc": 55610.0}}
    p = with_frame / "moon_nrl.json"
    p.write_text(json.dumps(cfg))
    with pytest.raises(api.PhopError) as e:
        api.load_environment(p)
    assert "NRLMSISE-00 may only be configured on Earth." in str(e.value)
