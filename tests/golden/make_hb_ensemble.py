"""Reference heatbath ensemble for the statistical parity of the GPU heatbath.

Runs the unmodified reference (oracle/_ref/lgf_ref heatbath, seeds 1..9 via
oracle/seed_shim.h) for 200 x (Cabibbo-Marinari + 5 OR) sweeps at beta 6.0 on
8^4, one configuration per seed, and records per configuration the average
plaquette and E, Q after flowing to t = 1.0 (oracle flow, eps 0.01; the
oracle's flow is byte-identical to the reference's).  Writes
hb8_ensemble.json beside this script.

    python tests/golden/make_hb_ensemble.py
"""
import json
import os
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
from oracle import oracle as O  # noqa: E402

# The reference checkout this script reads (override with LGF_REFERENCE).
REFERENCE_LGF = os.environ.get("LGF_REFERENCE", "/root/reference/LGF")
SHAPE = (8, 8, 8, 8)
SEEDS = list(range(1, 10))


def plaquette(U, shape):
    """Average plaquette ReTr(U_mu U_nu U_mu^dag U_nu^dag)/3 over sites and planes."""
    V = int(np.prod(shape))
    M = (U.reshape(V, 4, 18)[:, :, 0::2] + 1j * U.reshape(V, 4, 18)[:, :, 1::2]).reshape(V, 4, 3, 3)
    idx = np.arange(V).reshape(shape)
    tot = 0.0
    for mu in range(4):
        for nu in range(mu + 1, 4):
            xpm = np.roll(idx, -1, axis=mu).reshape(-1)
            xpn = np.roll(idx, -1, axis=nu).reshape(-1)
            P = M[:, mu] @ M[xpm, nu] @ np.conj(np.transpose(M[xpn, mu], (0, 2, 1))) @ np.conj(
                np.transpose(M[:, nu], (0, 2, 1)))
            tot += np.trace(P, axis1=1, axis2=2).real.sum()
    return tot / (3 * 6 * V)


def one(seed, tmp):
    d = Path(tmp) / f"s{seed}"
    O.run_reference(["heatbath", str(d) + "/", "6.0", *SHAPE, 200, 5], env={"LGF_REF_SEED": str(seed)},
                    timeout=3600)
    U = np.fromfile(d / "ensembles/su3/beta6_000000/8X8X8X8/Heatbath_5_ORperHB/torus_extdof4_0.bin")
    _, E, Q, _ = O.flow(U, SHAPE, 0.01, 100, 100)
    return {"seed": seed, "plaquette": plaquette(U, SHAPE), "E_t1": float(E[-1]), "Q_t1": float(Q[-1])}


def main():
    O.build(REFERENCE_LGF)
    if not O.reference_available():
        sys.exit("reference harness not built: the reference tree is needed")
    with tempfile.TemporaryDirectory() as tmp, ThreadPoolExecutor(max_workers=len(SEEDS)) as ex:
        rows = list(ex.map(lambda s: one(s, tmp), SEEDS))
    rec = {"shape": list(SHAPE), "beta": 6.0, "sweeps": "200 x (CM heatbath + 5 OR), hot start", "flow": "eps 0.01 to t = 1.0",
           "configs": rows, "generator": "oracle/_ref/lgf_ref heatbath (unmodified LGF sources), seeds 1..9, "
                                         "via tests/golden/make_hb_ensemble.py"}
    (HERE / "hb8_ensemble.json").write_text(json.dumps(rec, indent=1))
    print(json.dumps(rec, indent=1))


if __name__ == "__main__":
    main()
