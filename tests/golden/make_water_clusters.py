"""Generate tests/golden/water_clusters.json: the oracle's results on the seeded water
clusters the benchmark uses (334 H2O = 1,002 atoms, 1,000 H2O = 3,000 atoms; seed 0),
at the default SCF tolerances.

The oracle (oracle/, the C++ restatement of pm7-rs `run_pm7`) takes seconds on the first
cluster and tens of minutes on the second, too long for a test run, so the GPU parity
tests read these recorded values. Fields: heat of formation, energies, iterations,
charges, HOMO/LUMO and dipole. Run from the repository root after `make -C oracle`:

    python tests/golden/make_water_clusters.py [334 1000]
"""
import json
import platform
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "pm7-rs_b200"))

from oracle import harness  # noqa: E402
from pm7b200 import geometry  # noqa: E402


def main():
    sizes = [int(a) for a in sys.argv[1:]] or [334, 1000]
    path = Path(__file__).with_name("water_clusters.json")
    out = json.loads(path.read_text()) if path.exists() else {}
    for k in sizes:
        z, x = geometry.water_cluster(k, seed=0)
        t0 = time.time()
        r = harness.run(z, x, want_matrices=0)
        out[f"water{k}"] = {
            "waters": k, "seed": 0, "n_atoms": int(r["n_atoms"]), "nao": int(r["nao"]),
            "iterations": int(r["iterations"]),
            "heat_of_formation_kcal": r["heat_of_formation_kcal"], "total_ev": r["total_ev"],
            "electronic_ev": r["electronic_ev"], "core_ev": r["core_ev"], "correction_kcal": r["correction_kcal"],
            "homo_ev": r["homo_ev"], "lumo_ev": r["lumo_ev"],
            "dipole_debye": [float(v) for v in r["dipole_debye"]],
            "charges": [float(v) for v in r["charges"]],
            "oracle_seconds": round(time.time() - t0, 1), "host": platform.processor() or platform.machine(),
        }
        print(f"water{k}: dHf {r['heat_of_formation_kcal']:.9f} kcal/mol, {r['iterations']} iterations, "
              f"{time.time() - t0:.0f} s", flush=True)
        path.write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    main()
