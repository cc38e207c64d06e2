"""The autotuner picks among launch variants that must give identical results.

Processes are forced (through PM7_AUTOTUNE_CACHE files, or PM7_AUTOTUNE_FORCE key prefixes)
onto different variants of the SP2 squaring tile shape and of the Fock near-pair and atom
launch shapes (lanes per pair or atom, threads per block), single-molecule and batched; their
results must agree bit for bit, and a run without a cache must time the variants and record
a choice.
"""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent

SCRIPT = r"""
import json, sys
sys.path.insert(0, %r)
from pm7b200 import api, geometry as G
z, x = G.water_cluster(60, seed=2)   # nao 360: SP2 purification, near pairs
r = api.run_pm7(z, x, want_matrices=0)
print(json.dumps({"dhf": r["heat_of_formation_kcal"], "q": list(r["charges"]), "eps": list(r["mo_energies"]),
                  "tune": api.autotune_report()}))
"""


BATCH_SCRIPT = r"""
import json, sys
sys.path.insert(0, %r)
from pm7b200 import api, geometry as G
mols = G.batch(24, seed=3)
res = api.run_batch(mols, want_matrices=0)
print(json.dumps({"dhf": [r["heat_of_formation_kcal"] for r in res], "q": [list(r["charges"]) for r in res],
                  "tune": api.autotune_report()}))
"""


def _run(tmp_path, name, cache, force=None, script=SCRIPT):
    env = dict(os.environ)
    env.pop("PM7_AUTOTUNE_FORCE", None)
    if force is not None:
        env["PM7_AUTOTUNE_FORCE"] = force
    if cache is None:
        env.pop("PM7_AUTOTUNE_CACHE", None)
    else:
        path = tmp_path / f"{name}.json"
        path.write_text(json.dumps(cache))
        env["PM7_AUTOTUNE_CACHE"] = str(path)
    out = subprocess.run([sys.executable, "-c", script % str(ROOT / "pm7-rs_b200")], env=env, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return json.loads(out.stdout.strip().splitlines()[-1])


def _device_name():
    out = subprocess.run(["nvidia-smi", "--query-gpu=name", "--format=csv,noheader", "-i", "0"], capture_output=True,
                         text=True)
    return out.stdout.strip().splitlines()[0]


def test_forced_variants_give_identical_results(tmp_path):
    dev = _device_name()
    first = _run(tmp_path, "free", None)
    assert any("sp2_square|n512" in k for k in first["tune"]), first["tune"]
    near_key = next(k.split("|", 1)[1] for k in first["tune"] if "|fock_near|" in k)
    a = _run(tmp_path, "a", {f"{dev}|sp2_square|n512": {"choice": 0}, f"{dev}|{near_key}": {"choice": 0}})
    b = _run(tmp_path, "b", {f"{dev}|sp2_square|n512": {"choice": 1}, f"{dev}|{near_key}": {"choice": 4}})
    assert a["tune"][f"{dev}|sp2_square|n512"] == 0 and b["tune"][f"{dev}|sp2_square|n512"] == 1
    for r in (a, b):
        assert r["dhf"] == first["dhf"]
        assert r["q"] == first["q"]
        assert r["eps"] == first["eps"]


# (SP2 square tile, near-pair shape, atom shape): whole warps, 8-, 4- and 1-lane groups
FORCED = [(0, 0, 0), (1, 1, 1), (0, 2, 1), (1, 3, 2), (0, 4, 2)]


def test_forced_fock_shapes_single(tmp_path):
    runs = [_run(tmp_path, f"s{i}", None, force=f"sp2_square={s},fock_near={n},fock_atom={a}")
            for i, (s, n, a) in enumerate(FORCED)]
    for (s, n, a), r in zip(FORCED, runs):
        atom = [v for k, v in r["tune"].items() if "|fock_atom|" in k]
        near = [v for k, v in r["tune"].items() if "|fock_near|" in k]
        assert atom and near, r["tune"]
        assert set(atom) == {a} and set(near) == {n}
        assert r["dhf"] == runs[0]["dhf"] and r["q"] == runs[0]["q"] and r["eps"] == runs[0]["eps"]


def test_forced_fock_shapes_batched(tmp_path):
    runs = [_run(tmp_path, f"b{i}", None, force=f"b_fock_near={n},b_fock_atom={a}", script=BATCH_SCRIPT)
            for i, (_, n, a) in enumerate(FORCED)]
    for (_, n, a), r in zip(FORCED, runs):
        near = {k: v for k, v in r["tune"].items() if "|b_fock_near|" in k}
        atom = {k: v for k, v in r["tune"].items() if "|b_fock_atom|" in k}
        assert near and atom, r["tune"]
        assert set(near.values()) == {n} and set(atom.values()) == {a}
        assert r["dhf"] == runs[0]["dhf"] and r["q"] == runs[0]["q"]
