"""CPU: how hsolve_b200.solve turns its keyword arguments and config document into the solver
configuration, following hsolve's rules (python/hsolve/__init__.py:231-275: keywords override the
document, lower/upper select the interval target, sigma the nearest one, unknown keys and non-finite
numbers are rejected) and the mapping onto the C struct of include/hsg_solve.h.
"""
import json

import numpy as np
import pytest

from hsolve_b200 import api
from hsolve_b200.errors import HsolveIOError, InvalidInputError

D = api._Default


def merge(config=None, sigma=None, k=D(6), mode=D("nearest"), lower=None, upper=None, tol=D(1e-10), threads=D(0)):
    return api.merge_config(config, sigma, k, mode, lower, upper, tol, threads)


def test_target_selection():
    assert merge(sigma=2.0)["target"] == {"mode": "nearest", "sigma": 2.0}
    assert merge(lower=1.0, upper=3.0)["target"] == {"mode": "interval", "lower": 1.0, "upper": 3.0}
    assert merge(sigma=1.0, k=4, mode="nearest")["target"] == {"mode": "nearest", "sigma": 1.0, "k": 4}
    assert merge(mode="smallest", k=3)["target"] == {"mode": "smallest", "k": 3}
    with pytest.raises(InvalidInputError):
        merge(sigma=1.0, lower=0.0, upper=2.0)      # ambiguous without mode=
    assert merge(sigma=1.0, lower=0.0, upper=2.0, mode="interval")["target"]["mode"] == "interval"


def test_keywords_override_the_document():
    doc = {"target": {"mode": "nearest", "sigma": 5.0, "k": 2}, "tol": 1e-8, "threads": 2, "seed": 7}
    cfg = merge(doc, sigma=6.0, k=9, tol=1e-9, threads=4)
    assert cfg["target"] == {"mode": "nearest", "sigma": 6.0, "k": 9}
    assert cfg["tol"] == 1e-9 and cfg["threads"] == 4 and cfg["seed"] == 7
    assert doc["target"]["sigma"] == 5.0             # the caller's document is not modified
    cfg = merge(doc)
    assert cfg["target"]["sigma"] == 5.0 and cfg["tol"] == 1e-8


def test_numpy_scalars_are_accepted():
    cfg = merge({"seed": np.int64(3), "tol": np.float64(1e-9)}, sigma=np.float32(1.5), k=np.int32(2))
    assert cfg["seed"] == 3 and cfg["tol"] == 1e-9 and cfg["target"]["sigma"] == 1.5 and cfg["target"]["k"] == 2
    assert merge(sigma=np.array(2.5))["target"]["sigma"] == 2.5


@pytest.mark.parametrize("bad, exc", [
    (dict(config={"no_such_key": 1}), InvalidInputError),
    (dict(config={"target": [1, 2]}), InvalidInputError),
    (dict(mode="closest"), InvalidInputError),
    (dict(mode=3), TypeError),
    (dict(sigma="1.0"), TypeError),
    (dict(sigma=True), TypeError),
    (dict(sigma=1.0, k=True), TypeError),
    (dict(sigma=1.0, k=2.5), TypeError),
    (dict(sigma=np.inf), InvalidInputError),
    (dict(lower=0.0, upper=np.nan), InvalidInputError),
    (dict(config={"tol": float("inf")}), InvalidInputError),
    (dict(config=42), TypeError),
])
def test_rejections(bad, exc):
    with pytest.raises(exc):
        merge(**bad)


def test_config_file(tmp_path):
    good = tmp_path / "config.json"
    good.write_text(json.dumps({"target": {"mode": "interval", "lower": 1.0, "upper": 2.0}, "ncv": 40}))
    cfg = merge(str(good))
    assert cfg["target"]["mode"] == "interval" and cfg["ncv"] == 40
    bad = tmp_path / "bad.json"
    bad.write_text("{not json")
    with pytest.raises(InvalidInputError):
        merge(str(bad))
    arr = tmp_path / "arr.json"
    arr.write_text("[1, 2]")
    with pytest.raises(InvalidInputError):
        merge(str(arr))
    with pytest.raises(HsolveIOError):
        merge(str(tmp_path / "missing.json"))


def test_c_struct_mapping():
    cfg = merge({"ncv": 48, "block_size": 4, "seed": 11, "certificate": "off", "factor_precision": "single",
                 "batch_shifts": False, "problem": "generalized_definite"}, lower=1.0, upper=9.0, tol=1e-9)
    c = api._struct_from(cfg, verbose=1)
    assert c.mode == api._MODES.index("interval") and c.lower == 1.0 and c.upper == 9.0
    assert c.tol == 1e-9 and c.ncv == 48 and c.block_size == 4 and c.seed == 11
    assert c.certificate == 3 and c.factor_precision == 1 and c.batch_shifts == 0 and c.verbose == 1
    assert c.problem == api._PROBLEMS.index("generalized_definite")
    d = api._struct_from(merge(sigma=2.0), verbose=0)
    assert d.mode == 0 and d.sigma == 2.0 and d.k == 6 and d.tol == 1e-10 and d.batch_shifts == 1
    for key, val in [("factor_precision", "half"), ("certificate", "maybe"), ("problem", "weird"), ("tol", 2.0)]:
        with pytest.raises(InvalidInputError):
            api._struct_from(merge({key: val}, sigma=1.0), verbose=0)
