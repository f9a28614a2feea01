"""Generates the golden fixtures that pin the CPU oracle to the reference.

Runs the UNMODIFIED reference library (compiled from its own sources into
oracle/_ref/ by oracle/Makefile) on a GPU, on seeded inputs from the oracle's
generators, and stores for every output: the values at 512 sampled entries
(complex128) plus two whole-array checksums (sum |v|^2 and sum w_i v_i with
w_i = cos(0.37 i)). Needs a GPU and oracle/_ref/libqcu_ref.so:

    python tests/golden/make_golden.py            # writes tests/golden/ref_8x8x8x8.npz

Cases (lattice 8^3x8, the smallest whose half volume the reference accepts):
  * gauge "random:2024:0.3" (SU(3) exp(0.3 i H)), spinor seed 11:
    dslashQcu both parities, fullDslashQcu both dagger flags,
    invertCloverDslash, preCloverDslash, newFullCloverDslashOneRound and
    cloverDslashOneRound both flags, MmV_one_round;
  * gauge "pure:7" (a random gauge transform of the unit field, where the
    reference CG converges): cg_inverter solution and iteration count.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref_runner  # noqa: E402

L = (8, 8, 8, 8)
NSAMPLE = 512


def weights(n: int) -> np.ndarray:
    return np.cos(0.37 * np.arange(n))


def digest(name: str, arr: np.ndarray, out: dict) -> None:
    v = np.ascontiguousarray(arr).reshape(-1)
    rng = np.random.default_rng(12345)
    idx = np.sort(rng.choice(v.size, size=min(NSAMPLE, v.size), replace=False))
    out[f"{name}__idx"] = idx.astype(np.int64)
    out[f"{name}__val"] = v[idx]
    out[f"{name}__norm2"] = np.array(np.vdot(v, v).real)
    out[f"{name}__wsum"] = np.array(np.sum(weights(v.size) * v))


def main():
    out = {"lattice": np.array(L)}
    d, _ = ref_runner.run(L, "random:2024:0.3", ["dslash", "full", "invert", "pre", "newfull", "round", "mmv"], 11)
    for k in ("dslash_p0", "dslash_p1", "full_d0", "full_d1", "invert", "pre", "newfull_d0", "newfull_d1",
              "round_d0", "round_d1", "mmv"):
        digest(k, d[k], out)
    d, stdout = ref_runner.run(L, "pure:7", ["cg"], 11)
    digest("cg_x", d["cg_x"], out)
    out["cg_iterations"] = d["cg_iterations"]
    out["cg_converged"] = d["cg_converged"]
    path = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_8x8x8x8.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, "cg iterations", int(d["cg_iterations"]), "converged", bool(d["cg_converged"]))


if __name__ == "__main__":
    main()
