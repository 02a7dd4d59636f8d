"""Regenerate the empirical-model data tables used by the kernels and the oracle.

Reads the published model data that the reference carries and writes them,
as plain numbers in this package's own layout, to
``parahpop_b200/csrc/tables/``:

* ``nrlmsise00_coeffs.inc`` - NRLMSISE-00 coefficient blocks (Picone, Hedin
  and Drob; public-domain C release 20041227).  Reference copy:
  ``src/common/engine/paraHPOP/model/environment/atmosphere/detail/Nrlmsise00Data.inl``.
* ``tide_tables.inc`` - IERS 2010 Table 6.5a/b/c frequency-dependent Love
  number corrections and the FES2004 Stokes amplitudes (18 waves, 402 terms).
  Reference copies: ``src/common/engine/paraHPOP/model/accelerations/hpop_compat/
  HpopFrequencyTerms.inc`` and ``Fes2004Terms.inc``.

The numbers must be identical to the reference's (they are the physical
model), so they are extracted rather than retyped.  Run here, where the
reference tree is available; the output is committed:

    python oracle/gen_model_tables.py <reference tree>
"""
import re
import sys
from pathlib import Path

NUM = r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?"


def block(text, name):
    m = re.search(r"\b" + re.escape(name) + r"\b[^=;{]*=\s*\{", text)
    if not m:
        raise SystemExit(f"table {name} not found")
    i = m.end()
    depth = 1
    j = i
    while depth:
        c = text[j]
        if c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
        j += 1
    body = text[i:j - 1]
    body = re.sub(r"/\*.*?\*/", " ", body, flags=re.S)
    body = re.sub(r"//[^\n]*", " ", body)
    return body


def numbers(body):
    return [float(x) for x in re.findall(NUM, body)]


def fmt(vals, per_line=4):
    lines = []
    for k in range(0, len(vals), per_line):
        lines.append("    " + ", ".join(repr(v) if v != 0.0 else "0.0" for v in vals[k:k + per_line]) + ",")
    return "\n".join(lines)


def main(ref):
    ref = Path(ref)
    out = Path(__file__).resolve().parents[1] / "parahpop_b200" / "csrc" / "tables"
    out.mkdir(parents=True, exist_ok=True)

    nrl = (ref / "src/common/engine/paraHPOP/model/environment/atmosphere/detail/Nrlmsise00Data.inl").read_text()
    spec = [("pt", 150), ("pd", 9 * 150), ("ps", 150), ("pdl", 2 * 25), ("ptm", 10), ("pdm", 8 * 10),
            ("ptl", 4 * 100), ("pma", 10 * 100), ("sam", 100), ("pavgm", 10)]
    parts = ["// NRLMSISE-00 empirical atmosphere coefficients (Picone, Hedin, Drob;",
             "// public-domain C release 20041227).  Generated by oracle/gen_model_tables.py;",
             "// numbers only, flat row-major blocks.  Instantiate with",
             "// PHOP_NRL_TABLE(name, count) defined as the storage declaration.", ""]
    for name, count in spec:
        vals = numbers(block(nrl, name))
        if len(vals) != count:
            raise SystemExit(f"{name}: expected {count}, got {len(vals)}")
        parts.append(f"PHOP_NRL_TABLE(nrl_{name}, {count}) = {{\n{fmt(vals)}\n}};")
    (out / "nrlmsise00_coeffs.inc").write_text("\n".join(parts) + "\n")

    hp = ref / "src/common/engine/paraHPOP/model/accelerations/hpop_compat"
    freq = (hp / "HpopFrequencyTerms.inc").read_text()
    fes = (hp / "Fes2004Terms.inc").read_text()
    parts = ["// IERS Conventions 2010 Tables 6.5a-c (frequency-dependent solid-tide",
             "// corrections, units 1e-12) and FES2004 ocean-tide Stokes amplitudes",
             "// (dimensionless, source values * 1e-11), degree/order <= 6.",
             "// Generated by oracle/gen_model_tables.py; numbers only.",
             "// PHOP_TIDE_TABLE(type, name, count) is the storage declaration.", ""]
    for order, name, count in ((0, "terms20", 21), (1, "terms21", 48), (2, "terms22", 2)):
        vals = numbers(block(freq, name))
        if len(vals) != 7 * count:
            raise SystemExit(f"{name}: expected {7 * count}, got {len(vals)}")
        rows = []
        for k in range(count):
            r = vals[7 * k:7 * k + 7]
            rows.append("    {{%d,%d,%d,%d,%d}, %r, %r}," % (tuple(int(x) for x in r[:5]) + (r[5], r[6])))
        parts.append(f"PHOP_TIDE_TABLE(PhopFreqTerm, tide_freq{order}, {count}) = {{\n" + "\n".join(rows) + "\n};")
    waves = numbers(block(fes, "waves"))
    if len(waves) != 18 * 8:
        raise SystemExit("FES waves")
    rows = []
    for k in range(18):
        r = [int(x) for x in waves[8 * k:8 * k + 8]]
        rows.append("    {{%d,%d,%d,%d,%d,%d}, %d, %d}," % tuple(r))
    parts.append("PHOP_TIDE_TABLE(PhopOceanWave, tide_fes_waves, 18) = {\n" + "\n".join(rows) + "\n};")
    terms = numbers(block(fes, "terms"))
    if len(terms) != 402 * 6:
        raise SystemExit(f"FES terms {len(terms)}")
    rows = []
    for k in range(402):
        r = terms[6 * k:6 * k + 6]
        rows.append("    {%d, %d, %r, %r, %r, %r}," % (int(r[0]), int(r[1]), r[2], r[3], r[4], r[5]))
    parts.append("PHOP_TIDE_TABLE(PhopOceanTerm, tide_fes_terms, 402) = {\n" + "\n".join(rows) + "\n};")
    (out / "tide_tables.inc").write_text("\n".join(parts) + "\n")
    print("wrote", out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python oracle/gen_model_tables.py <reference tree>")
    main(sys.argv[1])
