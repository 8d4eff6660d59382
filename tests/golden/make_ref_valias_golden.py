"""Run the reference's own Vose alias resampler (resampling-valias.cl, built as
CUDA into oracle/_ref/libref_valias.so by oracle/build_ref_valias.sh) on
seeded weights and uniforms and store inputs and outputs in ref_valias.npz
(beside this script, or in the directory given as the first argument).  Needs
a GPU.  The CPU tests check the oracle's normalisation and draw rule against
them bit for bit, and its tables' selection probabilities within FP32
rounding (the reference fills its work lists with atomics, so the tables'
order is the hardware's, not a fixed one)."""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent / "oracle"))
import ref_kernels as R  # noqa: E402


def inputs(m, seed):
    """8 sub-filters: exponential weights with zeros, all zero (the uniform
    fallback), one dominant weight, equal weights, a heavy tail, and three
    more exponential ones; 2 uniforms in [0,1) per particle, exact in FP32."""
    rng = np.random.default_rng(seed)
    nsub = 8
    w = rng.exponential(1.0, (nsub, m)).astype(np.float32)
    w[0, rng.random(m) < 0.3] = 0.0
    w[1] = 0.0
    w[2] = 1e-3
    w[2, m // 3] = 50.0
    w[3] = 0.25
    w[4] = (rng.pareto(1.2, m) + 1e-6).astype(np.float32)
    u2 = (rng.integers(0, 1 << 23, 2 * nsub * m) / float(1 << 23)).astype(np.float32)
    return w.reshape(-1), u2


def main():
    out_dir = Path(sys.argv[1]) if len(sys.argv) > 1 else HERE
    out = {}
    for m in (32, 64, 256, 512, 1024):
        w, u2 = inputs(m, 900 + m)
        scaled, prob, alias, sel = R.valias(w, u2, m)
        out["w_%d" % m], out["u2_%d" % m] = w, u2
        out["scaled_%d" % m], out["prob_%d" % m], out["alias_%d" % m], out["sel_%d" % m] = scaled, prob, alias, sel
    np.savez_compressed(out_dir / "ref_valias.npz", **out)
    print("wrote", out_dir / "ref_valias.npz", sorted(out))


if __name__ == "__main__":
    main()
