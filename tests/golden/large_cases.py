"""Golden cases at the production shape (r = 64), regenerated from seeds.

The data of these cases is too large to commit (up to 262,144 observations),
so each fixture directory holds only

  spec.json         the seeded generator call and SHA-256 digests of the
                    generated locations, prediction points and values
  golden.json       d and the log-likelihood of the reference's own sources
                    compiled here (oracle/_ref/mra_ref_ext), with its timings
  pred_golden.npz   the reference's posterior predictive mean and variance, in
                    the order of its prediction dump

and ``generate`` rebuilds the inputs bit for bit (the digests prove it).

Cases:
  r64_c2s_nu12   65,536 locations, 70% in 16 clusters + 30% uniform, M=7,
                 J=4, r=64, nu=1/2, 4,096 prediction points
  r64_c2s_nu32   the same layout with nu=3/2 (another seed)
  r64_c2         the full clustered configuration: 262,144 locations, M=8,
                 J=4, r=64, nu=1/2, 16,384 prediction points

Locations, prediction points and the field coefficients come from
synth.locations / synth.true_theta; the observation values from
synth.smooth_values (a random Fourier-feature field scaled by sigma(s) plus
nugget noise), because a draw from the MRA prior at these sizes would take the
numpy oracle minutes per case.
"""
from __future__ import annotations

import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from nonstationary_mra_b200 import refio, synth  # noqa: E402

SPECS = {
    "r64_c2s_nu12": synth.Config("r64_c2s_nu12", 65536, 7, 4, 64, 1, 4096, "mix70", 0.3, 41),
    "r64_c2s_nu32": synth.Config("r64_c2s_nu32", 65536, 7, 4, 64, 3, 4096, "mix70", 0.3, 42),
    "r64_c2": synth.Config("r64_c2", 262144, 8, 4, 64, 1, 16384, "mix70", 0.3, 2),
}


def names():
    return [n for n in SPECS if os.path.exists(os.path.join(HERE, n, "golden.json"))]


def generate(name: str):
    """(cfg, xy, pred, theta, y) of a case, from its seeds."""
    cfg = SPECS[name]
    rng = np.random.Generator(np.random.PCG64(cfg.seed))
    xy, pred = synth.locations(cfg, rng)
    theta = synth.true_theta(cfg, rng)
    y = synth.smooth_values(xy, theta, cfg.seed + 500)
    return cfg, xy, pred, theta, y


def digests(xy, pred, y) -> dict:
    return {"locations": synth.digest(xy), "predictions": synth.digest(pred), "values": synth.digest(y)}


def write_inputs(case_dir: str, name: str, mode: str = "likelihood") -> dict:
    """Writes the case in the reference's formats into ``case_dir``; returns its digests."""
    cfg, xy, pred, theta, y = generate(name)
    synth.write_case(case_dir, cfg, xy, y, pred, theta, mode=mode)
    return digests(xy, pred, y)


def load(name: str, mode: str = "prediction"):
    """(Structure, Model, spec) of a case, read back through the reference's file
    formats exactly as the reference's main() reads them.  Raises if the
    regenerated inputs differ from the ones the golden outputs were made from."""
    spec = json.load(open(os.path.join(HERE, name, "spec.json")))
    with tempfile.TemporaryDirectory() as tmp:
        got = write_inputs(tmp, name, mode)
        if got != spec["digests"]:
            raise RuntimeError(f"{name}: regenerated inputs differ from the golden ones: {got} vs {spec['digests']}")
        st, md, _ = refio.load_case(tmp, mode=mode)
    return st, md, spec


def golden(name: str) -> dict:
    return json.load(open(os.path.join(HERE, name, "golden.json")))


def golden_prediction(name: str):
    z = np.load(os.path.join(HERE, name, "pred_golden.npz"))
    return z["mean"], z["var"]
