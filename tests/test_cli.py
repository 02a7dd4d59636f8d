"""Command-line driver: usage and the reference's refusal cases
(scripts/validate.py:107-128, src/common/driver.cpp:59-129).  Every case here
fails during validation, before any device work."""
import json
import shutil

import pytest

from parahpop_b200 import api


def run(case, config=None, targets=None, out=None):
    cfg = config if config is not None else case.config_path
    tg = targets if targets is not None else case.targets_path
    return api.run_cli(cfg, tg, out if out is not None else case.dir / "out")


def test_help():
    r = api.run_cli("--help", "", "")
    r = __import__("subprocess").run([str(api.CLI_PATH), "--help"], capture_output=True, text=True)
    assert r.returncode == 0
    assert "CONFIG.json TARGETS.json OUTPUT_DIRECTORY" in r.stdout
    assert "Backend: device; integrator: RKF78 fixed step" in r.stdout


def test_wrong_argument_count():
    r = __import__("subprocess").run([str(api.CLI_PATH), "a"], capture_output=True, text=True)
    assert r.returncode == 1
    assert r.stderr.startswith("ParaHPOP: Expected CONFIG.json TARGETS.json OUTPUT_DIRECTORY")


def _mutate_config(case, fn, name="c2.json"):
    cfg = json.loads(case.config_path.read_text())
    fn(cfg)
    p = case.dir / name
    p.write_text(json.dumps(cfg))
    return p


def _mutate_targets(case, fn, name="t2.json"):
    tg = json.loads(case.targets_path.read_text())
    fn(tg)
    p = case.dir / name
    p.write_text(json.dumps(tg))
    return p


@pytest.mark.parametrize("mutation,message", [
    (lambda c: c["execution"]["integration"].__setitem__("maxNumSteps", 0), "maxNumSteps and maxThreads must be positive integers."),
    (lambda c: c["execution"].__setitem__("maxThreads", -1), "maxNumSteps and maxThreads must be positive integers."),
    (lambda c: c["execution"]["integration"].__setitem__("absTol", 1e-9), "Unsupported integration option: absTol"),
    (lambda c: c["execution"]["integration"].__setitem__("maxStepSize", 60), "Unsupported integration option: maxStepSize"),
    (lambda c: c["run"].__setitem__("duration_seconds", -5.0), "duration_seconds must be finite and positive."),
    (lambda c: c["execution"]["integration"].__setitem__("initialStepSize", 0.0), "initialStepSize must be finite and positive."),
    (lambda c: c["model"]["environment"].__setitem__("constants", "missing.json"), "Required data file not found"),
])
def test_config_refusals(golden, mutation, message):
    case = golden("full_600s")
    r = run(case, config=_mutate_config(case, mutation))
    assert r.returncode == 1
    assert r.stderr.startswith("ParaHPOP: ") and message in r.stderr


@pytest.mark.parametrize("mutation,message", [
    (lambda t: t["targets"][1].__setitem__("id", t["targets"][0]["id"]), "Target IDs must be unique."),
    (lambda t: t["targets"][0].__setitem__("mass_kg", 0.0), "Invalid target epoch or physical parameter."),
    (lambda t: t["targets"][0].__setitem__("drag_area_m2", -1.0), "Invalid target epoch or physical parameter."),
    (lambda t: t["targets"][0].__setitem__("cr", -0.1), "Invalid target epoch or physical parameter."),
    (lambda t: t.__setitem__("targets", []), "targets must be a nonempty array."),
])
def test_target_refusals(golden, mutation, message):
    case = golden("full_600s")
    r = run(case, targets=_mutate_targets(case, mutation))
    assert r.returncode == 1
    assert message in r.stderr


def test_nonfinite_state_refused(golden):
    case = golden("full_600s")
    tg = json.loads(case.targets_path.read_text())
    tg["targets"][0]["state_km_km_s"][2] = 12345.5
    p = case.dir / "t_inf.json"
    p.write_text(json.dumps(tg).replace("12345.5", "1e999"))  # overflows to +inf when parsed
    r = run(case, targets=p)
    assert r.returncode == 1
    assert "State contains a nonfinite value." in r.stderr


def test_refuses_to_overwrite_outputs(golden):
    case = golden("full_600s")
    out = case.dir / "existing"
    out.mkdir()
    (out / "summary.json").write_text("{}")
    r = run(case, out=out)
    assert r.returncode == 1
    assert "Output exists; use a new directory" in r.stderr
